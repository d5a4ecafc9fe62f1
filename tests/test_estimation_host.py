"""Host logic of the estimation interface: state layout, labels, packing, reduced VMR
bases and FD steps (src/Estimation/state_vector.jl:40-403, jacobian_fd.jl:76-92).
No GPU: these are argument-marshalling functions."""
import numpy as np
import pytest

from conftest import load_package


@pytest.fixture(scope="module")
def pkg():
    return load_package()


def prof(pkg, n=5):
    p = np.linspace(1000.0, 100.0, n)
    return pkg.AtmosphericProfile(p, np.linspace(290.0, 220.0, n), np.zeros(n),
                                  {1: np.linspace(1e-2, 1e-5, n), 2: np.full(n, 4e-4), 3: np.zeros(n)})


def test_layout_and_labels(pkg):  # state_vector.jl:268-342
    s = pkg.StateVectorSpec(5, [pkg.H2O, pkg.ColumnScale(pkg.O3)])
    assert s.n == 5 + 5 + 1 + 2
    assert list(s.temp_range) == list(range(5))
    assert list(pkg.vmr_range(s, pkg.H2O)) == list(range(5, 10))
    assert list(pkg.vmr_range(s, pkg.O3)) == [10]
    assert (s.tsfc_index, s.emis_index) == (11, 12)
    lab = pkg.state_labels(s)
    assert lab[0] == "T[1]" and lab[5] == "logVMR_H₂O[1]" and lab[10] == "logVMRscale_O₃"
    assert lab[-2:] == ["T_sfc", "emissivity"]
    s2 = pkg.StateVectorSpec(5, [pkg.CO2], include_temperature=False, include_tsfc=False, log_vmr=False)
    assert s2.n == 6 and pkg.state_labels(s2)[0] == "VMR_CO₂[1]" and s2.tsfc_index == -1
    with pytest.raises(pkg.IRSError):
        pkg.vmr_range(s2, pkg.O3)
    with pytest.raises(pkg.IRSError):
        pkg.StateVectorSpec(0, [])


def test_pack_unpack_round_trip(pkg):  # state_vector.jl:350-403
    pr = prof(pkg)
    s = pkg.StateVectorSpec(5, [pkg.H2O, pkg.O3, pkg.PartialColumns(pkg.CO2, np.ones((5, 1)))])
    x = pkg.pack_state(s, pr, T_sfc=293.0, eps_sfc=0.97)
    assert x[s.tsfc_index] == 293.0 and x[s.emis_index] == 0.97
    assert np.all(x[10:15] == np.log(1e-30))  # zero VMR clamped at the floor
    assert np.all(x[15:16] == 0.0)             # reduced block packs theta = 0
    p2, Ts, e = pkg.unpack_state(s, x, pr)
    assert Ts == 293.0 and e == 0.97
    assert np.allclose(p2.vmr[1], pr.vmr[1], rtol=1e-15)
    assert np.array_equal(p2.vmr[2], pr.vmr[2])
    x[15] = np.log(2.0)
    p3, _, _ = pkg.unpack_state(s, x, pr)
    assert np.allclose(p3.vmr[2], 2 * pr.vmr[2], rtol=1e-15)
    assert pkg.pack_state(pkg.StateVectorSpec(5, [], include_tsfc=True), pr)[5] == pr.temperature[0]
    with pytest.raises(pkg.IRSError):
        pkg.pack_state(pkg.StateVectorSpec(6, []), pr)
    with pytest.raises(pkg.IRSError):
        pkg.unpack_state(s, x[:-1], pr)
    with pytest.raises(pkg.IRSError):
        pkg.pack_state(pkg.StateVectorSpec(5, [pkg.CH4]), pr)


def test_partial_column_bases(pkg):  # state_vector.jl:122-227
    B = pkg.partial_column_basis(np.linspace(1000, 100, 10), n_blocks=3)
    assert B.shape == (10, 3) and np.allclose(B.sum(axis=1), 1.0)
    assert [int(B[:, m].sum()) for m in range(3)] == [3, 4, 3]  # round(0:10/3:10) = 0,3,7,10
    Be = pkg.partial_column_basis(np.linspace(1000, 100, 10), edges_hPa=[500.0])
    assert Be.shape == (10, 2) and Be[:, 0].sum() == 6  # levels with p > 500 hPa
    Bt = pkg.partial_column_basis(10, [range(0, 4), range(4, 10)], taper="tent")
    assert np.allclose(Bt.sum(axis=1), 1.0) and 0 < Bt[4, 0] < 1
    with pytest.raises(pkg.IRSError):
        pkg.partial_column_basis(10, [range(0, 4), range(5, 10)])
    with pytest.raises(pkg.IRSError):
        pkg.partial_column_basis(np.linspace(1000, 100, 10))
    blocks = pkg.dfs_partition([0.4, 0.4, 0.4, 0.1, 0.9, 0.2], target_dfs=1.0)
    assert [list(b) for b in blocks] == [[0, 1, 2], [3, 4], [5]]
    with pytest.raises(pkg.IRSError):
        pkg.dfs_partition([1.0], target_dfs=0.0)


def test_default_fd_steps(pkg):  # jacobian_fd.jl:76-92
    s = pkg.StateVectorSpec(3, [pkg.H2O, pkg.ColumnScale(pkg.O3)], log_vmr=False)
    st = pkg.default_fd_steps(s)
    assert list(st) == [0.5] * 3 + [1e-9] * 3 + [1e-3] + [0.5, 1e-3]
