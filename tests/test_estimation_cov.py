"""a-priori and measurement covariances (sa_builder.jl:101-153, covariance.jl:106-117)."""
import numpy as np
import pytest

from conftest import load_package


@pytest.fixture(scope="module")
def pkg():
    return load_package()


def test_build_sa(pkg):
    p = np.array([1000.0, 800.0, 500.0, 200.0])
    prof = pkg.AtmosphericProfile(p, np.full(4, 250.0), np.zeros(4), {1: np.full(4, 1e-3)})
    s = pkg.StateVectorSpec(4, [pkg.H2O])
    Sa = pkg.build_sa(s, prof, sigma_T=0.5, L_T=1.0, sigma_vmr=0.3, L_vmr=2.0)
    assert Sa.shape == (10, 10) and np.allclose(Sa, Sa.T)
    assert np.all(np.linalg.eigvalsh(Sa) > 0)
    r = abs(np.log(1000.0 / 800.0)) / 1.0
    c = (1 + np.sqrt(5) * r + 5 * r * r / 3) * np.exp(-np.sqrt(5) * r)
    assert np.isclose(Sa[0, 1], 0.25 * c)
    assert np.isclose(Sa[4, 4], 0.09) and Sa[0, 4] == 0.0
    assert Sa[8, 8] == 4.0 and np.isclose(Sa[9, 9], 0.02 ** 2)
    Se = pkg.build_sa(s, prof, kernel="exponential", sigma_T=[1, 2, 3, 4])
    assert np.isclose(Se[1, 2], 2 * 3 * np.exp(-abs(np.log(800 / 500))))
    with pytest.raises(pkg.IRSError):
        pkg.build_sa(s, prof, kernel="gauss")
    with pytest.raises(pkg.IRSError):
        pkg.build_sa(s, prof, sigma_vmr={2: 0.3})


def test_scene_nedt_and_mask(pkg):
    nu = np.array([700.0, 1000.0, 2400.0])
    assert np.allclose(pkg.scene_nedt(nu, np.full(3, 280.0), nedt_280K=0.2), 0.2)
    cold = pkg.scene_nedt(nu, np.full(3, 220.0), nedt_280K=0.2)
    assert np.all(cold > 0.2) and cold[2] > cold[0]
    keep = pkg.exclude_channels(nu, (650.0, 800.0), (2300.0, 2500.0))
    assert keep.tolist() == [False, True, False]
