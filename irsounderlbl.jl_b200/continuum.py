"""HITRAN collision-induced absorption tables (src/CrossSections/continuum.jl:104-165).

Host-side reader of the .cia format, as the reference's: a block starts at a header
line whose first character is a letter ("pair  nu_min  nu_max  N  T  ..."), followed by
"nu sigma" lines; sigma is clamped at 0 and each block's knots are put in ascending
order.  The tables are handed to the library with B200Context.set_cia and evaluated on
the GPU inside the RTE kernels (block selection, linear interpolation in nu and T).
"""
from __future__ import annotations

from typing import List, Optional, Tuple

import numpy as np

CIA_PAIRS = {"co2_cia": 1, "n2": 2, "o2": 3}  # continua names -> irs_set_cia pair ids


def load_cia_table(path: str) -> Optional[List[Tuple[float, np.ndarray, np.ndarray]]]:
    """_load_cia_table (continuum.jl:116-159) -> [(T, nu[], sigma[])] or None when empty."""
    blocks = []
    cur_T, cur_nu, cur_sg = float("nan"), [], []

    def flush():
        if cur_nu:
            nu = np.array(cur_nu)
            sg = np.array(cur_sg)
            if np.any(np.diff(nu) < 0):
                order = np.argsort(nu, kind="stable")
                nu, sg = nu[order], sg[order]
            blocks.append((cur_T, nu, sg))

    with open(path) as fh:
        for line in fh:
            st = line.strip()
            if not st:
                continue
            if st[0].isalpha():
                flush()
                cur_nu, cur_sg = [], []
                cur_T = float(st.split()[4])
            else:
                parts = st.split()
                cur_nu.append(float(parts[0]))
                cur_sg.append(max(0.0, float(parts[1])))
    flush()
    return blocks or None
