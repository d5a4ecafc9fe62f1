"""The allocation-free cross-section entry point against the regular one.

irs_cross_sections_noalloc serves callers that cannot allocate device memory (hosts
whose own allocator owns the device, or that forbid allocation after start-up).  It
must give the same cross sections as irs_cross_sections, within the FP64 tolerance
the other parity tests use (1e-12 of the peak), on consecutive calls that reuse its
shared scratch array, and must reject line counts beyond its fixed capacity.
"""
import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu


def test_noalloc_matches_regular_entry_point():
    import torch
    pkg = load_package()
    from irs_b200 import _lib
    lib = _lib.load()
    ctx = pkg.B200Context()
    try:
        dev = torch.device("cuda", 0)
        ll = pkg.synthetic.lists_5k_co2()[2]
        grid = np.array([(251600 + i) / 400 for i in range(34801)])  # 629:0.0025:716
        q = np.ascontiguousarray(pkg._read_tips()[(2, 1)])
        d_lines = torch.from_numpy(ll.lines.view(np.uint8).copy()).to(dev)
        d_q = torch.from_numpy(q).to(dev)
        d_grid = torch.from_numpy(grid).to(dev)
        d_sigma = torch.empty(len(grid), dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream()
        # two calls in a row with different states: the second must not see the first
        for T, p, method in ((230.0, 0.2, 3), (296.0, 1.0, 3), (250.0, 0.05, 1)):
            ref = pkg.compute_voigt_cross_sections(grid, ll, T, p, backend=ctx,
                                                   method=pkg.VoigtMethod(method))
            rc = lib.irs_cross_sections_noalloc(d_lines.data_ptr(), len(ll), d_q.data_ptr(), 70, len(q),
                                                d_grid.data_ptr(), len(grid), T, p, 0.0, 25.0, method,
                                                122.0, d_sigma.data_ptr(), stream.cuda_stream)
            pkg.check(rc)
            torch.cuda.synchronize()
            got = d_sigma.cpu().numpy()
            assert np.max(np.abs(got - ref)) <= 1e-12 * ref.max(), (T, p, method)
        rc = lib.irs_cross_sections_noalloc(d_lines.data_ptr(), 131073, d_q.data_ptr(), 70, len(q),
                                            d_grid.data_ptr(), len(grid), 250.0, 0.5, 0.0, 25.0, 3, 122.0,
                                            d_sigma.data_ptr(), stream.cuda_stream)
        assert rc == -1 and b"131072" in lib.irs_last_error()
    finally:
        ctx.close()
