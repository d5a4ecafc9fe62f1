"""The allocation-free cross-section entry point against the regular one.

irs_cross_sections_noalloc serves callers that cannot allocate device memory (hosts
whose own allocator owns the device, or that forbid allocation after start-up).  It
must give the same cross sections as irs_cross_sections, within the FP64 tolerance
the other parity tests use (1e-12 of the peak), on consecutive calls that reuse its
shared scratch array, for every Voigt method, for a list that mixes isotopologues
(each line on its own TIPS table), and with no TIPS tables (Q proportional to T, the
reference's fallback, checked against the oracle); it must reject line counts and
table counts beyond its fixed capacity.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu


def _call(lib, d_lines, n, d_q, keys, n_tips, d_grid, n_nu, T, p, method, d_sigma, stream):
    kp = keys.ctypes.data_as(C.POINTER(C.c_int32)) if keys is not None else None
    return lib.irs_cross_sections_noalloc(d_lines, n, d_q, kp, n_tips, 70, 331, d_grid, n_nu, T, p, 0.0, 25.0,
                                          method, 122.0, d_sigma, stream)


def test_noalloc_matches_regular_entry_point(oracle):
    import torch
    pkg = load_package()
    from irs_b200 import _lib
    lib = _lib.load()
    ctx = pkg.B200Context()
    try:
        dev = torch.device("cuda", 0)
        ll = pkg.synthetic.lists_5k_co2()[2]
        # the same list with every other line on the second CO2 isotopologue
        mixed = ll.lines.copy()
        mixed["iso_id"][1::2] = 2
        ll2 = pkg.HITRANLinelist(mixed)
        grid = np.array([(251600 + i) / 400 for i in range(34801)])  # 629:0.0025:716
        tips = pkg._read_tips()
        keys = np.ascontiguousarray(np.array(sorted(tips), dtype=np.int32).reshape(-1, 2))
        q_all = np.ascontiguousarray(np.concatenate([tips[tuple(k)] for k in keys]))
        assert len(keys) <= 64 and all(len(tips[tuple(k)]) == 331 for k in keys)
        d_q = torch.from_numpy(q_all).to(dev)
        d_grid = torch.from_numpy(grid).to(dev)
        d_sigma = torch.empty(len(grid), dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream().cuda_stream
        # consecutive calls with different lists, states and methods: no call may see
        # what the one before it left in the shared scratch
        for lst, T, p, method in ((ll, 230.0, 0.2, 3), (ll2, 296.0, 1.0, 3), (ll, 250.0, 0.05, 1),
                                  (ll2, 215.0, 0.3, 2), (ll2, 260.0, 0.6, 1)):
            d_lines = torch.from_numpy(lst.lines.view(np.uint8).copy()).to(dev)
            ref = pkg.compute_voigt_cross_sections(grid, lst, T, p, backend=ctx, method=pkg.VoigtMethod(method))
            pkg.check(_call(lib, d_lines.data_ptr(), len(lst), d_q.data_ptr(), keys, len(keys), d_grid.data_ptr(),
                            len(grid), T, p, method, d_sigma.data_ptr(), stream))
            torch.cuda.synchronize()
            got = d_sigma.cpu().numpy()
            assert np.max(np.abs(got - ref)) <= 1e-12 * ref.max(), (T, p, method)
        # no TIPS tables: Q proportional to T for every line, as the oracle does for a
        # (mol, iso) without a table (CO2 iso 14 has none)
        assert (2, 14) not in tips
        no_tab = ll.lines.copy()
        no_tab["iso_id"] = 14
        d_lines = torch.from_numpy(ll.lines.view(np.uint8).copy()).to(dev)
        for method, mname in ((3, "FullFaddeeva"), (2, "PseudoVoigt")):
            ref = oracle.voigt_xsec(no_tab, grid, 240.0, 0.4, method=mname)
            pkg.check(_call(lib, d_lines.data_ptr(), len(ll), 0, None, 0, d_grid.data_ptr(), len(grid), 240.0, 0.4,
                            method, d_sigma.data_ptr(), stream))
            torch.cuda.synchronize()
            got = d_sigma.cpu().numpy()
            assert np.max(np.abs(got - ref)) <= 1e-12 * ref.max(), mname
        # capacity: lines, then tables
        rc = _call(lib, d_lines.data_ptr(), 131073, d_q.data_ptr(), keys, len(keys), d_grid.data_ptr(), len(grid),
                   250.0, 0.5, 3, d_sigma.data_ptr(), stream)
        assert rc == -1 and b"131072" in lib.irs_last_error()
        many = np.zeros((65, 2), dtype=np.int32)
        rc = _call(lib, d_lines.data_ptr(), len(ll), d_q.data_ptr(), many, 65, d_grid.data_ptr(), len(grid),
                   250.0, 0.5, 3, d_sigma.data_ptr(), stream)
        assert rc == -1 and b"64" in lib.irs_last_error()
    finally:
        ctx.close()
