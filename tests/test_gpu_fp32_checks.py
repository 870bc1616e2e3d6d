"""FP32 production kernel against the FP64 kernel at the large-system state
point (rho* = 0.32, T* = 0.8, orientations within 20 degrees of z), the FP64
hand-over of overlapping or over-full cells, and the periodic FP64 energy
check (EnergyCheck, MCnptColloid.c:1343-1362).

Lockstep: an FP32-kernel system and an FP64-kernel system start every sweep
from the same FP64 state with the same seed and sweep counter, so they draw
the same trial moves and the same Metropolis numbers; their decisions are
compared particle by particle, and every attempt's energy change dE is
compared with the FP64 kernel's.  FP32 pair terms carry at most 1.9e-4
relative error (max(|phi|, 1)); terms above 100 eps0 are evaluated in FP64, so
an attempt's FP32 dE differs from FP64 by about one worst-case FP32 term
(0.02) at most (measured: 0.004 over 36 sweeps of 32,768 attempts) or by
FP64 rounding where overlaps make it huge, and decisions differ only where
beta dE is within that difference of ln u.
"""
import numpy as np
import pytest

import parellel_mc_mpi_for_liquidcrystalsystems_b200 as lcmc
from parellel_mc_mpi_for_liquidcrystalsystems_b200 import _lib

pytestmark = pytest.mark.gpu

T = 0.8


def params(n, lattice, seed=7, precision=1, **kw):
    return lcmc.default_params(num_particles=n, system_density=0.32, system_temperature=T, gb_kappa=3.0,
                               gb_kappa_prime=5.0, gb_mu_exponent=2.0, gb_nu_exponent=1.0, cutoff_radius=4.0,
                               max_displacement=0.1, max_rotation=0.1, init_orientation_cone_deg=20.0,
                               precision_mode=precision, rng_seed=seed, init_lattice=lattice, **kw)


def lockstep(n, lattice, sweeps, relax=0):
    """Per sweep: (outcomes32, outcomes64, dE32, dE64, ln u, fp64 cells so far)."""
    p = params(n, lattice)
    st, box = lcmc.lattice(p)
    rows = []
    with lcmc.GBSystem(p) as a, lcmc.GBSystem(p) as b:
        b.set_kernel(0)
        b.upload(*st, box)
        if relax:
            b.sweep(relax)
        a.record_moves(True)
        b.record_moves(True)
        for _ in range(sweeps):
            x, bx = b.download()
            a.upload(*x, bx)
            _lib.check(_lib.lib().lcmc_set_sweep_counter(a._h, 0, b.stats()["sweeps"]))
            a.sweep(1)
            b.sweep(1)
            ea, _ = a.move_records()
            eb, lu = b.move_records()
            rows.append((a.outcomes(), b.outcomes(), ea, eb, lu, a.stats()["fp64_cells"]))
    return rows


@pytest.mark.parametrize("lattice,relax", [(0, 0), (1, 40)], ids=["jammed-sc-lattice", "relaxed-bct"])
def test_fp32_decisions_match_fp64_at_rho032(lattice, relax):
    """50 lockstep sweeps of N = 32,768: from the simple-cubic lattice start
    (spacing 1.46 for rods of length 3: overlaps up to the 1e9 clamp and
    terms of 1e36 beside it) and from a relaxed state."""
    n = 32768
    rows = lockstep(n, lattice, 50, relax)
    dd_all = []
    for o32, o64, e32, e64, lu, _ in rows:
        assert np.array_equal(o32 == 2, o64 == 2)  # hard-core rejects need no energy
        soft = o64 != 2
        agree = np.mean(o32[soft] == o64[soft])
        assert agree >= 0.999, agree
        dd = np.abs(e32 - e64)
        # a decision differs only where the FP32 error crosses the acceptance threshold
        for i in np.nonzero(o32 != o64)[0]:
            # accepted iff ln u + beta dE <= 0
            assert abs(e64[i] / T + lu[i]) <= abs(e32[i] - e64[i]) / T + 1e-12
        if np.array_equal(o32, o64):
            # FP32 error of an attempt: within one worst-case FP32 term (1.9e-4 of
            # the 100 eps0 largest FP32 term) where |dE| is O(1), and relative
            # 1e-5 where FP64 carried the large terms.  (After a differing
            # decision, later partners in that cell add the other pair difference,
            # so sweeps with a mismatch are left out of this bound.)
            assert np.all(dd[soft] <= 0.02 + 1e-5 * np.abs(e64[soft])), dd[soft].max()
        dd_all.append(dd[soft] / (1.0 + 1e-3 * np.abs(e64[soft])))
    assert np.quantile(np.concatenate(dd_all), 0.999) <= 0.02
    if lattice == 0:
        assert rows[-1][5] > 0  # the overlapping start went through the FP64 hand-over


def test_overfull_cells_run_in_fp64():
    """cell_capacity = 8 at 22 particles per cell: every cell is above the
    FP32 kernel's capacity and is attempted in FP64 (fail-safe, counted),
    with the FP64 kernel's decisions."""
    n = 32768
    p = params(n, 1, cell_capacity=8)
    st, box = lcmc.lattice(p)
    with lcmc.GBSystem(p) as a, lcmc.GBSystem(params(n, 1)) as b:
        b.set_kernel(0)
        for s in (a, b):
            s.upload(*st, box)
        same = True
        for _ in range(3):
            a.sweep(1)
            b.sweep(1)
            oa, ob = a.outcomes(), b.outcomes()
            assert np.mean(oa == ob) >= 0.9999
            same = same and np.array_equal(oa, ob)
        sa = a.stats()
        assert sa["error_flags"] == 0 and sa["kernel"] == 1
        assert sa["overcap_cells"] == sa["fp64_cells"] > 0
        if same:  # identical decisions: the same states up to the pair term's last bits
            ea, eb = a.tot_ene(), b.tot_ene()
            assert abs(ea - eb) <= 1e-9 * abs(eb)


def test_periodic_energy_check_passes_and_resets():
    """energy_check_interval = 5: four checks in 20 sweeps, none out of
    tolerance, the running energy equal to the FP64 recompute after each."""
    n = 32768
    p = params(n, 1, energy_check_interval=5)
    with lcmc.GBSystem(p) as s:
        s.get_initial_config()
        s.sweep(20)
        st = s.stats()
        assert st["energy_checks"] == 4 and st["drift_breaches"] == 0
        assert abs(st["drift"]) <= st["drift_bound"]
        assert st["drift_bound"] > 0.0
        assert st["energy"] == st["last_recompute"]
        e = s.tot_ene()
        assert abs(st["energy"] - e) <= 1e-9 * abs(e)


def test_energy_check_flags_a_planted_drift():
    """A caller that hands over a wrong running energy (the in/out energy of
    attempt_monte_carlo_move) is caught by the next check: LCMC_EDRIFT, the
    breach counted, the running energy reset to the recompute; after the
    caller clears the flags the run goes on."""
    n = 8192
    p = params(n, 1, energy_check_interval=2)
    with lcmc.GBSystem(p) as s:
        s.get_initial_config()
        s.sweep(20)  # relax the lattice start (its overlaps carry large |dE| into the tolerance)
        state, box = s.download()
        e_true = s.tot_ene()
        s.upload(*state, box, energy=e_true + 1.0e4)
        s.sweep(1)  # no check due yet
        with pytest.raises(lcmc.LcmcError) as ex:
            s.sweep(1)
        assert ex.value.code == _lib.EDRIFT
        st = s.stats()
        assert st["drift_breaches"] == 1 and st["error_flags"] & _lib.F_DRIFT
        assert abs(st["drift"] - 1.0e4) < 1.0 and st["drift_bound"] < 100.0
        assert st["energy"] == st["last_recompute"]
        s.clear_error_flags()
        s.sweep(4)
        assert s.stats()["drift_breaches"] == 1
        # the explicit check agrees
        s.energy_check()
        assert s.stats()["drift_breaches"] == 1


def test_npt_running_energy_tracks_the_recompute():
    """NPT: the volume move's exact U(V) is compared with the running energy
    every sweep (after the colour phases' dE is added), so the running
    energy equals the FP64 recompute within FP32 rounding."""
    n = 8192
    p = lcmc.default_params(num_particles=n, system_density=0.30, system_temperature=0.9, system_pressure=2.0,
                            mc_ensemble_type=2, npt_max_dlnV=0.01, rng_seed=3, precision_mode=1,
                            init_orientation_cone_deg=20.0, init_lattice=1, gb_kappa=3.0, gb_kappa_prime=5.0,
                            gb_mu_exponent=2.0, gb_nu_exponent=1.0, cutoff_radius=4.0, max_displacement=0.1,
                            max_rotation=0.1)
    with lcmc.GBSystem(p) as s:
        s.get_initial_config()
        s.sweep(30)
        st = s.stats()
        assert st["drift_breaches"] == 0 and st["energy_checks"] == 30
        e = s.tot_ene()
        assert abs(st["energy"] - e) <= 1e-6 * (abs(e) + n)


def _batch_params(precision=1):
    """Small boxes on the fine cell grid (odd counts allowed): 5, 6 and 7 cells
    of about 4.7 per axis instead of 4, 6 and 6 cells up to 5.9 wide, so each
    replica keeps the FP32 kernel; NVT, NPT and a colloid replica."""
    common = dict(gb_kappa=3.0, gb_kappa_prime=5.0, gb_mu_exponent=2.0, gb_nu_exponent=1.0, cutoff_radius=4.0,
                  max_displacement=0.1, max_rotation=0.1, precision_mode=precision, cell_grid=1,
                  init_orientation_cone_deg=20.0, init_lattice=1)
    return [
        lcmc.default_params(num_particles=4096, system_density=0.32, system_temperature=0.8, rng_seed=201, **common),
        lcmc.default_params(num_particles=6000, system_density=0.32, system_temperature=1.2, rng_seed=202,
                            mc_ensemble_type=2, system_pressure=2.0, **common),
        lcmc.default_params(num_particles=8192, system_density=0.30, system_temperature=0.9, rng_seed=203,
                            colloid_radius=3.0, colloid_wall_option=1, **common),
    ]


@pytest.mark.parametrize("precision", [1, 0])
def test_fine_grid_batch_matches_single_runs(precision):
    """Replicas of a batch on the fine grid (27 colour phases, of which the
    6-cell replica uses 8) reproduce their single runs bit for bit, on the FP32
    and on the FP64 kernel."""
    ps = _batch_params(precision)
    singles = []
    for p in ps:
        with lcmc.GBSystem(p) as s:
            s.get_initial_config()
            s.sweep(4)
            st = s.stats()
            assert st["kernel"] == precision, st
            singles.append((s.download(), st))
    with lcmc.GBSystem(ps) as b:
        for r in range(len(ps)):
            b.get_initial_config(r)
        b.sweep(4)
        for r, (want, wst) in enumerate(singles):
            got = b.download(r)
            for x, y in zip(got[0], want[0]):
                assert np.array_equal(x.view(np.uint64), y.view(np.uint64))
            assert np.array_equal(got[1].view(np.uint64), want[1].view(np.uint64))
            st = b.stats(r)
            assert st["accepted"] == wst["accepted"] and st["energy"] == wst["energy"] and st["kernel"] == precision


def test_fine_grid_fp32_decisions_match_fp64():
    """Lockstep on a small box (N = 4096, 5 cells per axis, 3 colours on each
    axis = 27 phases): FP32 against FP64 kernel decisions."""
    p = _batch_params()[0]
    st0, box = lcmc.lattice(p)
    with lcmc.GBSystem(p) as a, lcmc.GBSystem(p) as b:
        b.set_kernel(0)
        b.upload(*st0, box)
        b.sweep(20)
        a.record_moves(True)
        b.record_moves(True)
        for _ in range(30):
            x, bx = b.download()
            a.upload(*x, bx)
            _lib.check(_lib.lib().lcmc_set_sweep_counter(a._h, 0, b.stats()["sweeps"]))
            a.sweep(1)
            b.sweep(1)
            oa, ob = a.outcomes(), b.outcomes()
            ea, _ = a.move_records()
            eb, _ = b.move_records()
            soft = ob != 2
            assert np.mean(oa[soft] == ob[soft]) >= 0.999
            if np.array_equal(oa, ob):
                assert np.all(np.abs(ea - eb)[soft] <= 0.02 + 1e-5 * np.abs(eb[soft]))
        assert a.stats()["kernel"] == 1 and b.stats()["kernel"] == 0


def test_fp32_npt_ensemble_matches_fp64():
    """The reference never moves the volume, so the FP32 kernel's NPT ensemble
    is checked against the FP64 kernel's at a colloid NPT state point
    (N = 32,768, P* = 2, T* = 0.9, colloid R = 5, GB(3, 5, 2, 1)): 12
    independent chains per kernel from one compressed start, 300 sweeps of
    burn-in and 2000 recorded; <rho>, <U/N> and <P2> agree within 3.5 standard
    errors of the spread of the chain means (12 chains: a t-distribution with
    11 degrees of freedom)."""
    from parellel_mc_mpi_for_liquidcrystalsystems_b200 import da
    from test_gpu_screen import dilute_start
    n, R = 32768, 5.0
    base = dict(gb_kappa=3.0, gb_kappa_prime=5.0, gb_mu_exponent=2.0, gb_nu_exponent=1.0, cutoff_radius=4.0,
                max_displacement=0.1, max_rotation=0.1, mc_ensemble_type=2, system_pressure=2.0,
                system_temperature=0.9, colloid_wall_option=1, colloid_radius=R, num_particles=n,
                system_density=0.06, cell_capacity=64)
    with lcmc.GBSystem(lcmc.default_params(rng_seed=41, precision_mode=1, npt_max_dlnV=0.05, **base)) as s:
        st, box = dilute_start(n, 0.06, R, 41)
        s.upload(*st, box)
        s.sweep(1000)
        state, box = s.download()
    res = {}
    for prec in (0, 1):
        ps = [lcmc.default_params(rng_seed=700 + r + 50 * prec, precision_mode=prec, npt_max_dlnV=0.01, **base)
              for r in range(12)]
        with lcmc.GBSystem(ps) as s:
            for r in range(12):
                s.upload(*state, box, replica=r)
            s.sweep(300)
            s.record_history(2000)
            s.sweep(2000)
            rho = np.array([np.mean(n / da.p2_series(s, r)[3]) for r in range(12)])
            u = np.array([da.p2_series(s, r)[2].mean() / n for r in range(12)])
            p2 = np.array([da.p2_series(s, r)[1].mean() for r in range(12)])
            assert all(s.stats(r)["kernel"] == prec for r in range(12))
        res[prec] = (rho, u, p2)
    for i, name in enumerate(("rho", "U/N", "P2")):
        a, b = res[0][i], res[1][i]
        se = np.hypot(a.std(ddof=1), b.std(ddof=1)) / np.sqrt(len(a))
        assert abs(a.mean() - b.mean()) < 3.5 * se, (name, a.mean(), b.mean(), se)
