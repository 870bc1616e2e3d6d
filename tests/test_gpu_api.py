"""Host-boundary behaviour of the C ABI on the GPU.

* a rejected upload (particle outside the box, inside the colloid, zero
  orientation) returns its error and leaves the replica's state unchanged;
* lcmc_upload_with_energy takes the caller's running energy in place of the
  FP64 recompute and makes the same decisions as lcmc_upload;
* download into caller-owned arrays.
"""
import numpy as np
import pytest

import parellel_mc_mpi_for_liquidcrystalsystems_b200 as lcmc
from parellel_mc_mpi_for_liquidcrystalsystems_b200 import _lib

pytestmark = pytest.mark.gpu

COMMON = dict(gb_kappa=3.0, gb_kappa_prime=5.0, gb_mu_exponent=2.0, gb_nu_exponent=1.0, cutoff_radius=4.0,
              max_displacement=0.1, max_rotation=0.1)


def bits(a):
    return np.asarray(a, dtype=np.float64).view(np.uint64)


def test_rejected_upload_keeps_the_state():
    p = lcmc.default_params(num_particles=2000, system_density=0.30, rng_seed=3, colloid_wall_option=1,
                            colloid_radius=3.0, **COMMON)
    with lcmc.GBSystem(p) as s:
        s.get_initial_config()
        s.sweep(2)
        (a, box) = s.download()
        e = s.stats()["energy"]
        cases = []
        bad = [x.copy() for x in a]
        bad[0][5] = -1.0
        cases.append((bad, _lib.EINVAL))
        bad = [x.copy() for x in a]
        bad[0][7], bad[1][7], bad[2][7] = 0.5 * box[0], 0.5 * box[1], 0.5 * box[2] + 1.0
        cases.append((bad, _lib.EOVERLAP))
        bad = [x.copy() for x in a]
        bad[3][9] = bad[4][9] = bad[5][9] = 0.0
        cases.append((bad, _lib.EINVAL))
        bad = [x.copy() for x in a]
        bad[4][11] = np.nan
        cases.append((bad, _lib.EINVAL))
        for arrs, code in cases:
            with pytest.raises(lcmc.LcmcError) as ei:
                s.upload(*arrs, box)
            assert ei.value.code == code
            (b, box2) = s.download()
            for u, v in zip(a, b):
                assert np.array_equal(bits(u), bits(v))
            assert np.array_equal(box, box2)
            assert s.stats()["energy"] == e
        s.sweep(1)  # the context still works


def test_upload_with_energy_matches_upload():
    p = lcmc.default_params(num_particles=4000, system_density=0.30, rng_seed=9, **COMMON)
    a, box = lcmc.lattice(p)
    with lcmc.GBSystem(p) as s1, lcmc.GBSystem(p) as s2:
        s1.upload(*a, box)
        e0 = s1.stats()["energy"]
        s2.upload(*a, box, energy=e0 + 100.0)
        assert s2.stats()["energy"] == e0 + 100.0
        for _ in range(3):
            s1.sweep(1)
            s2.sweep(1)
            assert np.array_equal(s1.outcomes(), s2.outcomes())
        d1, d2 = s1.stats()["energy"], s2.stats()["energy"]
        assert abs((d2 - d1) - 100.0) <= 1e-9 * max(1.0, abs(d1))
        with pytest.raises(lcmc.LcmcError):
            s2.upload(*a, box, energy=float("inf"))


def test_download_into_caller_arrays():
    p = lcmc.default_params(num_particles=1000, system_density=0.30, rng_seed=4, **COMMON)
    with lcmc.GBSystem(p) as s:
        s.get_initial_config()
        s.sweep(1)
        want, box = s.download()
        out = [np.full(1000, -7.0) for _ in range(6)]
        got, box2 = s.download(out=out)
        assert all(g is o for g, o in zip(got, out))
        for u, v in zip(want, out):
            assert np.array_equal(bits(u), bits(v))
        with pytest.raises(ValueError):
            s.download(out=[np.zeros(999)] * 6)


def test_restart_resumes_exactly(tmp_path):
    """A run saved after 3 sweeps and resumed in a new context makes the same
    decisions and reaches the same bits as 6 uninterrupted sweeps; a plain
    fortSphere.1 (no sidecar) loads as the reference's restart would."""
    p = lcmc.default_params(num_particles=4000, system_density=0.30, rng_seed=12, precision_mode=1, **COMMON)
    with lcmc.GBSystem(p) as s:
        s.get_initial_config()
        s.sweep(3)
        s.save_restart(tmp_path / "fortSphere.1")
        saved, _ = s.download()
        outs = []
        for _ in range(3):
            s.sweep(1)
            outs.append(s.outcomes())
        want, wbox = s.download()
    with lcmc.GBSystem(p) as t:
        t.load_restart(tmp_path / "fortSphere.1")
        assert t.stats()["sweeps"] == 3
        for k in range(3):
            t.sweep(1)
            assert np.array_equal(t.outcomes(), outs[k]), k
        got, gbox = t.download()
    for a, b in zip(want, got):
        assert np.array_equal(bits(a), bits(b))
    assert np.array_equal(wbox, gbox)
    (tmp_path / "fortSphere.1.lcmc").unlink()
    with lcmc.GBSystem(p) as u:
        u.load_restart(tmp_path / "fortSphere.1")  # text only: 8 decimals
        a, _ = u.download()
        assert u.stats()["sweeps"] == 0
        assert max(np.max(np.abs(x - y)) for x, y in zip(a, saved)) <= 5e-9


def test_adaptive_step_follows_the_reference_rule():
    """The step after every sweep equals a host replay of MCnptColloid.c:987-1031
    (blocks of >= 10,000 attempts, +-5 %, resets at 1e-4 / 1.5 sigma_ss) with the
    cap at the creation value; switched off, it stays put."""
    # 6 cells per axis of width 4.45 (>= rc + d): about 28 rods per cell
    kw = dict(COMMON, max_displacement=0.4, max_rotation=0.6)
    n = 6070
    p = lcmc.default_params(num_particles=n, system_density=0.32, rng_seed=5, precision_mode=1, **kw)
    with lcmc.GBSystem(p) as s:
        s.get_initial_config()
        s.sweep(30)
        s.set_adaptive_step(True)
        d, a = s.step()
        cap = d
        assert d == float(np.float32(0.4)) and a == float(np.float32(0.6))
        att = acc = 0
        for _ in range(15):
            before = s.stats()["accepted"]
            s.sweep(1)
            att += n
            acc += s.stats()["accepted"] - before
            if att >= 10000:
                ratio = acc / att
                att = acc = 0
                if ratio < 0.3:
                    d -= d * 0.05
                    if d < 0.0001 * 1.0:
                        d = 0.01
                        if a > 0.000001:
                            a -= 0.5 * a
                elif ratio > 0.55:
                    d += d * 0.05
                    if d > 1.5:
                        d = 0.75
                        if a < 0.7:
                            a += 0.5 * a
                d = min(d, cap)
            assert s.step() == (d, a)
        assert d < cap  # the dense start accepts < 30 %: the step shrank
        s.set_adaptive_step(False)
        s.sweep(5)
        assert s.step() == (d, a)


def test_autotune_keeps_the_chain(tmp_path):
    """lcmc_autotune times the three phase-kernel capacity classes (11,000 rods,
    8 cells per axis, ~22 per cell) and restores everything after each trial: the
    chain continues bit for bit as an untuned run's.  A second context with the
    same workload takes the choice from the cache file without timing."""
    p = lcmc.default_params(num_particles=11000, system_density=0.30, rng_seed=17, precision_mode=1, **COMMON)
    cache = tmp_path / "tune.tsv"
    with lcmc.GBSystem(p) as s:
        s.get_initial_config()
        s.sweep(3)
        before, _ = s.download()
        t = s.autotune(2, cache)
        assert t["trials"] == 3 and not t["from_cache"] and t["ms_per_sweep"] > 0.0
        assert t["capacity"] in (48, 56, 64)
        after, _ = s.download()
        for u, v in zip(before, after):
            assert np.array_equal(bits(u), bits(v))
        assert s.stats()["sweeps"] == 3
        s.sweep(3)
        tuned, box1 = s.download()
        st1 = s.stats()
    with lcmc.GBSystem(p) as s:
        s.get_initial_config()
        s.sweep(6)
        plain, box2 = s.download()
        st2 = s.stats()
    for u, v in zip(tuned, plain):
        assert np.array_equal(bits(u), bits(v))
    assert st1["attempted"] == st2["attempted"] == 6 * 11000
    assert st1["accepted"] == st2["accepted"] and st1["energy"] == st2["energy"]
    with lcmc.GBSystem(p) as s:
        s.get_initial_config()
        t2 = s.autotune(2, cache)
        assert t2["from_cache"] and t2["trials"] == 0 and t2["capacity"] == t["capacity"]
        s.sweep(1)


def test_autotune_npt_volume_kernels():
    """For an NPT system with >= 4 cells per axis both kernels for the volume
    move's energies are timed with each capacity class that holds the
    system's cells (48, 56 and 64 particles); state and statistics are
    untouched."""
    p = lcmc.default_params(num_particles=11000, system_density=0.30, rng_seed=23, precision_mode=1,
                            mc_ensemble_type=2, system_pressure=2.0, system_temperature=1.2, npt_max_dlnV=0.01,
                            **COMMON)
    with lcmc.GBSystem(p) as s:
        s.get_initial_config()
        s.sweep(2)
        before, box0 = s.download()
        st0 = s.stats()
        t = s.autotune(1)
        assert t["trials"] == 6 and t["capacity"] in (48, 56, 64)
        after, box1 = s.download()
        for u, v in zip(before, after):
            assert np.array_equal(bits(u), bits(v))
        assert np.array_equal(bits(box0), bits(box1))
        st1 = s.stats()
        assert (st1["sweeps"], st1["volume_attempted"], st1["energy"]) == (st0["sweeps"], st0["volume_attempted"],
                                                                          st0["energy"])
        s.sweep(2)
        assert s.stats()["volume_attempted"] == st0["volume_attempted"] + 2


@pytest.mark.parametrize("bad,code", [
    (dict(num_particles=0), _lib.EINVAL),
    (dict(system_density=-0.3), _lib.EINVAL),
    (dict(system_temperature=0.0), _lib.EINVAL),
    (dict(num_particles=8), _lib.EBOX),  # L = 3 < 2 rc
])
def test_create_rejects_bad_parameters(bad, code):
    """Invalid sizes come back as status codes (the reference exits or runs on),
    for a single system and for a batch holding one bad replica; a good
    context still works afterwards."""
    good = lcmc.default_params(num_particles=2000, system_density=0.30, rng_seed=1, **COMMON)
    kw = dict(COMMON, num_particles=2000, system_density=0.30, rng_seed=1)
    kw.update(bad)
    p = lcmc.default_params(**kw)
    for arg in (p, [good, p]):
        with pytest.raises(lcmc.LcmcError) as ei:
            lcmc.GBSystem(arg)
        assert ei.value.code == code
    with lcmc.GBSystem(good) as s:
        s.get_initial_config()
        s.sweep(1)
        assert s.stats()["attempted"] == 2000


def test_sweep_before_upload_and_bad_replica_index():
    p = lcmc.default_params(num_particles=2000, system_density=0.30, rng_seed=2, **COMMON)
    with lcmc.GBSystem([p, p]) as s:
        s.get_initial_config(0)
        with pytest.raises(lcmc.LcmcError) as ei:
            s.sweep(1)  # replica 1 holds no configuration
        assert ei.value.code == _lib.EINVAL
        with pytest.raises(lcmc.LcmcError) as ei:
            s.stats(2)
        assert ei.value.code == _lib.EINVAL
        s.get_initial_config(1)
        s.sweep(1)
        assert s.stats(1)["attempted"] == 2000
