"""Ensemble averages against the reference's own Monte Carlo chain.

tests/golden/ensemble_golden.npz holds <U/N> and <P2> (block-averaged, with
standard errors from the spread of twelve independent chains) of runs of the reference's attempt_monte_carlo_move
(MCnptColloid.c:2445-2604, random particle per attempt) on N = 1728 rods at
rho* = 0.10, T* = 2.0, step 0.5 and rotation 0.3, with a colloid of radius 2
(made by tests/golden/make_ensemble_golden.py).  The checkerboard sweeps here sample
the same Boltzmann distribution with a different move schedule; 16 replicas
from the same lattice start, each with its own seed, give means whose
standard error comes from the spread of the replica means.  Both must agree
within 3 combined standard errors, for the FP32 kernel (the production path)
and the FP64 kernel.  The lattice start relaxes slowly: means over blocks of
1000 sweeps from sweep 200 on (16 replicas, both kernels) run -0.777, -0.750,
-0.746 and then stay within 0.001 of -0.7452, so the production sweeps start
after a burn-in of 5000.
"""
import numpy as np
import pytest

import parellel_mc_mpi_for_liquidcrystalsystems_b200 as lcmc
from parellel_mc_mpi_for_liquidcrystalsystems_b200 import da

pytestmark = pytest.mark.gpu

REPLICAS, BURN, SWEEPS = 16, 5000, 4000


@pytest.mark.parametrize("precision", [1, 0])
def test_ensemble_matches_reference_chain(golden, precision):
    g = golden("ensemble_golden.npz")
    n = int(g["n"])
    common = dict(num_particles=n, system_density=float(g["rho"]), system_temperature=float(g["T"]),
                  colloid_wall_option=1, colloid_radius=float(g["colloid_R"]), gb_kappa=3.0, gb_kappa_prime=5.0,
                  gb_mu_exponent=2.0, gb_nu_exponent=1.0, cutoff_radius=4.0,
                  max_displacement=float(g["dmax"]), max_rotation=float(g["rot"]), precision_mode=precision,
                  cell_capacity=64)  # the gas's ~27 rods per cell: the largest FP32 class, chosen explicitly
    start, box = lcmc.lattice(lcmc.default_params(rng_seed=int(g["seed"]), **common))
    ps = [lcmc.default_params(rng_seed=9000 + 17 * r, **common) for r in range(REPLICAS)]
    with lcmc.GBSystem(ps) as s:
        for r in range(REPLICAS):
            s.upload(*start, box, replica=r)
        s.sweep(BURN)
        # the lattice start relaxes from overlap energies of ~1e10: restart the
        # running energies from an FP64 recompute before the production sweeps
        for r in range(REPLICAS):
            s.tot_ene(r)
        s.record_history(SWEEPS)
        s.sweep(SWEEPS)
        u = np.array([da.p2_series(s, r)[2].mean() / n for r in range(REPLICAS)])
        p2 = np.array([da.p2_series(s, r)[1].mean() for r in range(REPLICAS)])
        drift = max(abs(s.stats(r)["energy"] - s.tot_ene(r)) / n for r in range(REPLICAS))
    # running energy after the production sweeps vs an FP64 recompute, per
    # particle: FP32 pair terms leave ~4e-5 kT of rounding in each dE, which
    # adds up as a random walk over the ~3e6 accepted moves of a replica
    assert drift < (1e-4 if precision == 1 else 1e-9), drift
    for name, gpu, ref_m, ref_se in (("U/N", u, float(g["u_mean"]), float(g["u_se"])),
                                     ("P2", p2, float(g["p2_mean"]), float(g["p2_se"]))):
        m, se = gpu.mean(), gpu.std(ddof=1) / np.sqrt(len(gpu))
        assert abs(m - ref_m) <= 3.0 * np.hypot(se, ref_se), (name, m, se, ref_m, ref_se)


def test_dense_liquid_matches_reference_chain(golden):
    """The CPU-runnable configuration's state point (N = 1000, rho* = 0.30,
    T* = 1.0, d = 0.1, rotation 0.1) with a colloid of radius 2, against the
    reference's own chain from the same compressed start
    (tests/golden/ensemble_dense_golden.npz, made by make_ensemble_golden.py
    dense): 16 FP64 replicas, <U/N> and <P2> within 3 combined standard
    errors."""
    g = golden("ensemble_dense_golden.npz")
    n = int(g["n"])
    common = dict(num_particles=n, system_density=float(g["rho"]), system_temperature=float(g["T"]),
                  colloid_wall_option=1, colloid_radius=float(g["colloid_R"]), gb_kappa=3.0, gb_kappa_prime=5.0,
                  gb_mu_exponent=2.0, gb_nu_exponent=1.0, cutoff_radius=4.0, max_displacement=float(g["dmax"]),
                  max_rotation=float(g["rot"]), precision_mode=0)
    start = [np.ascontiguousarray(g["start_" + k]) for k in ("px", "py", "pz", "ox", "oy", "oz")]
    box = np.ascontiguousarray(g["start_box"])
    ps = [lcmc.default_params(rng_seed=7100 + 13 * r, **common) for r in range(REPLICAS)]
    with lcmc.GBSystem(ps) as s:
        for r in range(REPLICAS):
            s.upload(*start, box, replica=r)
        s.sweep(int(g["burn"]))  # the reference chain's burn-in from the same start
        s.record_history(2500)
        s.sweep(2500)
        u = np.array([da.p2_series(s, r)[2].mean() / n for r in range(REPLICAS)])
        p2 = np.array([da.p2_series(s, r)[1].mean() for r in range(REPLICAS)])
    for name, gpu, ref_m, ref_se in (("U/N", u, float(g["u_mean"]), float(g["u_se"])),
                                     ("P2", p2, float(g["p2_mean"]), float(g["p2_se"]))):
        m, se = gpu.mean(), gpu.std(ddof=1) / np.sqrt(len(gpu))
        assert abs(m - ref_m) <= 3.0 * np.hypot(se, ref_se), (name, m, se, ref_m, ref_se)
