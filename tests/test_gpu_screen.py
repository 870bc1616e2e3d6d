"""Delayed-acceptance volume moves with the FP32-pair screen.

* the screen's energy change is within ~1e-3 kT of the exact one and stage 1
  uses the plain move's draw, so from one state and seed a screened chain
  makes the same decisions as the plain chain (every particle outcome, every
  box bit for bit) while the exact FP64 recompute runs only for moves that
  passed stage 1;
* independent screened chains sample the plain chains' volume distribution
  (mean volume within 4.5 standard errors of the spread of chain means).
"""
import numpy as np
import pytest

import parellel_mc_mpi_for_liquidcrystalsystems_b200 as lcmc
from parellel_mc_mpi_for_liquidcrystalsystems_b200 import da

pytestmark = pytest.mark.gpu

NPT = dict(gb_kappa=3.0, gb_kappa_prime=5.0, gb_mu_exponent=2.0, gb_nu_exponent=1.0, cutoff_radius=4.0,
           max_displacement=0.1, max_rotation=0.1, mc_ensemble_type=2, system_pressure=1.0,
           system_temperature=1.2, precision_mode=1, colloid_wall_option=1, colloid_radius=3.0)


def dilute_start(n, rho0, R, seed):
    """Simple-cubic sites at density rho0, none within R + 2.5 of the colloid
    centre (a lattice site right outside R leaves a rod inside the colloid's
    flat overlap clamp, which no move leaves), uniform orientations."""
    rng = np.random.default_rng(seed)
    L = (n / rho0 + 4.0 * np.pi * R ** 3 / 3.0) ** (1.0 / 3.0)
    ns = int(np.ceil((1.3 * n) ** (1.0 / 3.0)))
    g = (np.arange(ns) + 0.5) * (L / ns)
    pos = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pos = pos[np.linalg.norm(pos - 0.5 * L, axis=1) > R + 2.5]
    pos = pos[rng.permutation(len(pos))[:n]]
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    return [np.ascontiguousarray(a) for a in (*pos.T, *u.T)], np.array([L, L, L])


def compressed(n=6000, seed=8):
    """A dilute start compressed by the volume moves (FP32 kernel)."""
    p = lcmc.default_params(num_particles=n, system_density=0.10, rng_seed=seed, npt_max_dlnV=0.05,
                            cell_capacity=64, **NPT)
    with lcmc.GBSystem(p) as s:
        st, box = dilute_start(n, 0.08, NPT["colloid_radius"], seed)
        s.upload(*st, box)
        s.sweep(600)
        state, box = s.download()
        assert s.stats()["energy"] / n < 5.0
    return state, box


def params(n, seed):
    return lcmc.default_params(num_particles=n, system_density=0.10, rng_seed=seed, npt_max_dlnV=0.01,
                               cell_capacity=64, **NPT)


def test_screened_chain_decides_as_the_plain_chain():
    state, box = compressed()
    runs = []
    for screen in (False, True):
        with lcmc.GBSystem(params(6000, 77)) as s:
            s.upload(*state, box)
            s.set_fp32_screen(screen)
            outs, boxes = [], []
            for _ in range(40):
                s.sweep(1)
                outs.append(s.outcomes())
                boxes.append(np.array(s.stats()["box"]))
            runs.append((outs, boxes, s.stats()))
    (o0, b0, st0), (o1, b1, st1) = runs
    assert st1["kernel"] == 1
    for k in range(40):
        assert np.array_equal(o0[k], o1[k]), k
        assert np.array_equal(b0[k].view(np.uint64), b1[k].view(np.uint64)), k
    assert st0["volume_accepted"] == st1["volume_accepted"] > 0
    assert st1["volume_attempted"] == 40 and st0["volume_stage1_rejected"] == 0
    # the screen spared the FP64 recompute of every move it rejected
    assert st1["volume_stage1_rejected"] >= 40 - 2 * st1["volume_accepted"] - 10


def test_screened_chains_keep_the_volume_distribution():
    state, box = compressed()
    means = []
    for screen in (False, True):
        ps = [params(6000, 500 + r + 50 * screen) for r in range(12)]
        with lcmc.GBSystem(ps) as s:
            for r in range(12):
                s.upload(*state, box, replica=r)
            s.set_fp32_screen(screen)
            s.sweep(200)
            s.record_history(1500)
            s.sweep(1500)
            means.append(np.array([da.p2_series(s, r)[3].mean() for r in range(12)]))
            if screen:
                assert sum(s.stats(r)["volume_stage1_rejected"] for r in range(12)) > 0
    plain, screened = means
    se = np.hypot(plain.std(ddof=1), screened.std(ddof=1)) / np.sqrt(len(plain))
    assert abs(plain.mean() - screened.mean()) < 4.5 * se, (plain.mean(), screened.mean(), se)
