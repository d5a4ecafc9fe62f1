"""bench.py --impl reference on the host cores: the one JSON line that the ratio against
our arm is computed from.  It must carry our arm's metric string, unit, direction and
workload config (a ratio is only formed between lines that agree on them), a
cpu_baseline block describing the sample it timed, and an e2e block with no
host<->device bytes (the reference path has no device)."""
import json
import re
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_json_contract():
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "3"],
                       capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.strip().splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    d = json.loads(lines[0])
    sys.path.insert(0, str(ROOT))
    import bench
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC
    assert d["unit"] == "spectra/s" and d["higher_is_better"] is True
    assert d["config"] == bench.workload_config()
    assert d["steps"] == 1 and d["warmup"] == 3 and d["n_gpus"] == 1
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and "scaled by grid points" in cb["sample"]
    # spectra/s = (sampled grid points / all grid points) / seconds per step
    m = re.search(r"\((\d+) internal grid points of (\d+)\)", cb["sample"])
    assert m, cb["sample"]
    frac = int(m.group(1)) / int(m.group(2))
    assert 0 < frac < 1 and d["value"] > 0
    assert abs(d["value"] * d["ms_per_step"] / 1e3 - frac) <= 1e-9 * frac
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
