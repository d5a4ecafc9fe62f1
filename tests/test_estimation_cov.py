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


def test_apodized_measurement_covariance(pkg):  # runtests.jl:1614-1636
    nu = 645.0 + 0.25 * np.arange(21)
    Se = pkg.apodized_measurement_covariance(nu, 0.2)
    assert np.array_equal(Se, Se.T) and np.all(np.linalg.eigvalsh(Se) > 0)
    assert np.allclose(np.diag(Se), 0.04)
    s2 = 0.04
    assert abs(Se[0, 1] / s2 - 0.705) < 0.02 and abs(Se[0, 2] / s2 - 0.250) < 0.02
    assert abs(Se[0, 3] / s2 - 0.044) < 0.01 and Se[0, 4] / s2 < 0.006 and Se[0, 5] == 0.0
    Ssp = pkg.apodized_measurement_covariance([645.0, 647.0, 649.0], 0.2)
    assert Ssp[0, 1] == 0.0 and Ssp[0, 2] == 0.0
    sv = np.array([0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7])
    Sv = pkg.apodized_measurement_covariance(645.0 + 0.25 * np.arange(7), sv)
    assert np.allclose(np.diag(Sv), sv ** 2)
    Sd = pkg.apodized_measurement_covariance(nu, 0.2, fwhm_gauss=0.0)
    assert Sd[0, 1] == 0.0 and np.allclose(np.diag(Sd), 0.04)
    nuv = 660.0 + 0.25 * np.arange(5)
    Tb = np.full(5, 230.0)
    S = pkg.scene_measurement_covariance(nuv, Tb, nedt_280K=0.25)
    assert np.array_equal(S, S.T) and np.all(np.linalg.eigvalsh(S) > 0)
    assert abs(np.sqrt(S[0, 0]) - pkg.scene_nedt(nuv, Tb, nedt_280K=0.25)[0]) <= 1e-12 * np.sqrt(S[0, 0])
