"""Regenerate the bundled physical tables in this folder from an IRSounderLBL.jl checkout.

Usage:  python extract_tables.py <path of an IRSounderLBL.jl checkout>

What it writes (next to this script):

* ``tips2024_q.csv``      TIPS-2024 v1.2 Q(T), T = 70..400 K at 1 K, one row per
                          (mol, iso).  Parsed from ``src/HITRAN/tips2024_data.jl``
                          (the Julia Dict literal) -- data only, no code.
* ``afgl_<name>_50lev.csv``  the six AFGL 50-level profiles, copied verbatim.
* ``mt_ckd43_h2o_coeffs.csv``, ``mt_ckd_co2_coeffs.csv``  MT-CKD tables, verbatim.

The provenance and licence terms of each table are in ``SOURCES.md``.
"""
import re
import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
AFGL = ("us_standard", "tropical", "midlatitude_summer", "midlatitude_winter",
        "subarctic_summer", "subarctic_winter")


def parse_tips(jl_text: str):
    """Return {(mol, iso): [q70 .. q400]} from the tips2024_data.jl Dict literal."""
    tmin = int(re.search(r"const TIPS_T_MIN\s*=\s*(\d+)", jl_text).group(1))
    tmax = int(re.search(r"const TIPS_T_MAX\s*=\s*(\d+)", jl_text).group(1))
    out = {}
    for m in re.finditer(r"\((\d+),\s*(\d+)\)\s*=>\s*\[([^\]]*)\]", jl_text):
        vals = [float(v) for v in m.group(3).replace("\n", " ").split(",") if v.strip()]
        assert len(vals) == tmax - tmin + 1, (m.group(1), m.group(2), len(vals))
        out[(int(m.group(1)), int(m.group(2)))] = vals
    return tmin, tmax, out


def main(ref: Path):
    tmin, tmax, tips = parse_tips((ref / "src/HITRAN/tips2024_data.jl").read_text())
    with open(HERE / "tips2024_q.csv", "w") as f:
        f.write(f"# TIPS-2024 v1.2 Q(T), T={tmin}..{tmax} K step 1; columns mol,iso,Q(T_min)..Q(T_max)\n")
        for (mol, iso) in sorted(tips):
            f.write(f"{mol},{iso}," + ",".join(repr(v) for v in tips[(mol, iso)]) + "\n")
    for name in AFGL:
        shutil.copyfile(ref / "data" / f"afgl_{name}_50lev.csv", HERE / f"afgl_{name}_50lev.csv")
    shutil.copyfile(ref / "data/mt_ckd_h2o/mt_ckd43_h2o_coeffs.csv", HERE / "mt_ckd43_h2o_coeffs.csv")
    shutil.copyfile(ref / "data/mt_ckd_co2/mt_ckd_co2_coeffs.csv", HERE / "mt_ckd_co2_coeffs.csv")
    print(f"wrote {len(tips)} TIPS tables, {len(AFGL)} profiles, 2 MT-CKD tables to {HERE}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python extract_tables.py <path of an IRSounderLBL.jl checkout>")
    main(Path(sys.argv[1]))
