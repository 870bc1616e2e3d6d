"""Effective sample size of a series (integrated autocorrelation time with
Sokal's automatic window) on processes whose tau_int is known in closed form."""
import numpy as np

from parellel_mc_mpi_for_liquidcrystalsystems_b200 import da


def ar1(phi, n, seed):
    rng = np.random.default_rng(seed)
    e = rng.normal(size=n)
    x = np.empty(n)
    x[0] = e[0] / np.sqrt(1 - phi * phi)
    for i in range(1, n):
        x[i] = phi * x[i - 1] + e[i]
    return x


def test_ar1_tau_matches_closed_form():
    # AR(1): rho(t) = phi^t, tau_int = (1 + phi) / (2 (1 - phi))
    for phi in (0.5, 0.8, 0.95):
        x = ar1(phi, 200_000, int(phi * 100))
        want = (1 + phi) / (2 * (1 - phi))
        got = da.integrated_autocorrelation_time(x)
        assert abs(got / want - 1) < 0.1, (phi, got, want)
        assert abs(da.ess(x) / (len(x) / (2 * want)) - 1) < 0.1


def test_white_noise_and_degenerate_series():
    x = np.random.default_rng(1).normal(size=50_000)
    assert abs(da.integrated_autocorrelation_time(x) - 0.5) < 0.05
    assert da.integrated_autocorrelation_time(np.ones(100)) == 0.5
    assert da.integrated_autocorrelation_time([1.0, 2.0]) == 0.5
