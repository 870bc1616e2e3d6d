"""GPU parity tests: the CUDA library (through its C ABI) against the CPU oracle.

* FP64 kernel: accept/reject outcome of every attempt and the final
  coordinates bit-identical to the oracle's canonical checkerboard sweep
  (same grid shifts, colour orders and Philox streams);
* FP64 total energy within 1e-12 relative of the oracle;
* NPT volume moves: same decisions and boxes;
* FP32 kernel: same decisions as the FP64 kernel for all but a few attempts,
  energies within the FP32 tolerance stated below;
* batched replicas reproduce their single-system runs bit for bit.
"""
import numpy as np
import pytest

import oracle_ctypes as oc
import parellel_mc_mpi_for_liquidcrystalsystems_b200 as lcmc

pytestmark = pytest.mark.gpu

COMMON = dict(gb_kappa=3.0, gb_kappa_prime=5.0, gb_mu_exponent=2.0, gb_nu_exponent=1.0, cutoff_radius=4.0,
              max_displacement=0.1, max_rotation=0.1)


def params_pair(n, rho, seed, **kw):
    d = dict(COMMON)
    d.update(num_particles=n, system_density=rho, rng_seed=seed)
    d.update(kw)
    return lcmc.default_params(**d), oc.params(**d)


def bits(a):
    return np.asarray(a, dtype=np.float64).view(np.uint64)


def oracle_sweeps(op, state, box, n_sweeps, start=0, npt=False, fine=False):
    c = oc.consts(op, oc.ARITH_CANONICAL)
    k = oc.key(op.rng_seed)
    outs, vols = [], []
    n = len(state[0])
    for s in range(start, start + n_sweeps):
        st, b, order = oc.sweep(c, k, s, state, box, record=True, fine=fine)
        o = np.zeros(n, dtype=np.uint8)
        o[order] = b
        outs.append(o)
        if npt:
            r, info = oc.volume_move(c, k, s, op.system_pressure, op.npt_max_dlnV, state, box)
            vols.append((r, info.delta, info.U_old, info.U_new))
    return outs, vols


def gpu_sweeps(sys_, n_sweeps):
    outs = []
    for _ in range(n_sweeps):
        sys_.sweep(1)
        outs.append(sys_.outcomes())
    return outs


def start_state(p):
    a, box = lcmc.lattice(p)
    return [np.ascontiguousarray(x) for x in a], np.ascontiguousarray(box)


@pytest.mark.parametrize("case", ["lattice", "relaxed", "colloid"])
def test_fp64_sweeps_bitwise_vs_oracle(golden, case):
    if case == "relaxed":
        g = golden("totene_golden.npz")
        lp, op = params_pair(1000, 0.30, 11, precision_mode=0)
        state = [np.ascontiguousarray(g["plain_" + k]) for k in ("px", "py", "pz", "ox", "oy", "oz")]
        box = np.ascontiguousarray(g["plain_box"])
    elif case == "colloid":
        lp, op = params_pair(1000, 0.30, 12, precision_mode=0, colloid_radius=3.0, colloid_wall_option=1)
        state, box = start_state(lp)
    else:
        lp, op = params_pair(1000, 0.30, 13, precision_mode=0)
        state, box = start_state(lp)
    with lcmc.GBSystem(lp) as s:
        s.set_kernel(0)
        s.upload(*state, box)
        e0 = s.stats()["energy"]
        got = gpu_sweeps(s, 4)
        (gx, gy, gz, gox, goy, goz), gbox = s.download()
        st = s.stats()
    ostate = [x.copy() for x in state]
    obox = box.copy()
    want, _ = oracle_sweeps(op, ostate, obox, 4)
    for i, (a, b) in enumerate(zip(got, want)):
        assert np.array_equal(a, b), f"sweep {i}: {np.sum(a != b)} outcomes differ"
    for a, b in zip((gx, gy, gz, gox, goy, goz), ostate):
        assert np.array_equal(bits(a), bits(b))
    assert st["attempted"] == 4 * 1000
    assert st["accepted"] == sum(int(np.sum(o == 1)) for o in want)
    c = oc.consts(op, oc.ARITH_CANONICAL)
    e_or = oc.total_energy(c, ostate, obox)
    # running energy = initial FP64 recompute + accepted dE
    assert abs(st["energy"] - e_or) <= 1e-9 * max(abs(e_or), abs(e0), 1.0)
    if case == "colloid":
        assert sum(int(np.sum(o == 2)) for o in want) >= 0


def test_fp64_sweeps_bitwise_general_grid():
    """8 cells per axis: the 27-cell stencil without duplicates, many active cells per colour."""
    lp, op = params_pair(11000, 0.30, 21, precision_mode=0)
    state, box = start_state(lp)
    with lcmc.GBSystem(lp) as s:
        s.set_kernel(0)
        s.upload(*state, box)
        got = gpu_sweeps(s, 2)
        g, _ = s.download()
    want, _ = oracle_sweeps(op, state, box, 2)
    for a, b in zip(got, want):
        assert np.array_equal(a, b)
    for a, b in zip(g, state):
        assert np.array_equal(bits(a), bits(b))


@pytest.mark.parametrize("n,rho,R", [(4096, 0.32, 0.0), (8000, 0.30, 3.0)])
def test_fp64_sweeps_bitwise_fine_grid(n, rho, R):
    """Fine cell grid (cell_grid 1): an odd cell count per axis (5 and 7 here)
    takes three colours on that axis, 27 colour phases per sweep; the FP64
    kernel reproduces the oracle's fine-grid sweeps bit for bit (outcomes and
    coordinates)."""
    kw = dict(colloid_radius=R, colloid_wall_option=1) if R > 0 else {}
    lp, op = params_pair(n, rho, 31, precision_mode=0, **kw)
    lp.cell_grid = 1
    state, box = start_state(lp)
    with lcmc.GBSystem(lp) as s:
        s.set_kernel(0)
        s.upload(*state, box)
        got = gpu_sweeps(s, 3)
        g, _ = s.download()
    want, _ = oracle_sweeps(op, state, box, 3, fine=True)
    for i, (a, b) in enumerate(zip(got, want)):
        assert np.array_equal(a, b), f"sweep {i}: {np.sum(a != b)} outcomes differ"
    for a, b in zip(g, state):
        assert np.array_equal(bits(a), bits(b))


@pytest.mark.parametrize("n,R", [(1000, 0.0), (6000, 4.0)])
def test_total_energy_vs_oracle(golden, n, R):
    lp, op = params_pair(n, 0.30, 5, colloid_radius=R, colloid_wall_option=1 if R > 0 else 0)
    g = golden("totene_golden.npz")
    if n == 1000:
        state = [np.ascontiguousarray(g["plain_" + k]) for k in ("px", "py", "pz", "ox", "oy", "oz")]
        box = np.ascontiguousarray(g["plain_box"])
    else:
        state, box = start_state(lp)
    with lcmc.GBSystem(lp) as s:
        s.upload(*state, box)
        e = s.tot_ene()
    c = oc.consts(op, oc.ARITH_CANONICAL)
    want = oc.total_energy(c, state, box)
    assert abs(e - want) <= 1e-12 * abs(want)
    if n == 1000:  # and the reference's own tot_ene on this state (golden)
        assert abs(e - float(g["plain_E"])) <= 1e-12 * abs(float(g["plain_E"]))


@pytest.mark.parametrize("n,sweeps,dmax", [(1000, 4, 0.1), (11000, 2, 0.1), (11000, 2, 1.0)])
def test_npt_volume_moves_vs_oracle(n, sweeps, dmax):
    """N = 1000: 3 cells per axis (per-particle volume-energy kernel); N = 11000:
    8 cells per axis (cell kernel for the volume move's energies); with
    max_displacement 1.0 the cells are 5.5 wide (~51 particles) and a cell's 13
    forward neighbours exceed one staging chunk (576 particles)."""
    lp, op = params_pair(n, 0.30, 31, precision_mode=0, mc_ensemble_type=2, system_pressure=2.0,
                         system_temperature=0.9, npt_max_dlnV=0.01, max_displacement=dmax)
    g_state, box = start_state(lp)
    with lcmc.GBSystem(lp) as s:
        s.set_kernel(0)
        s.upload(*g_state, box)
        got = gpu_sweeps(s, sweeps)
        st = s.stats()
        (gx, gy, gz, gox, goy, goz), gbox = s.download()
    state = [x.copy() for x in g_state]
    obox = box.copy()
    want, vols = oracle_sweeps(op, state, obox, sweeps, npt=True)
    for a, b in zip(got, want):
        assert np.array_equal(a, b)
    assert st["volume_attempted"] == sweeps
    assert st["volume_accepted"] == sum(1 for v in vols if v[0] == 1)
    # the last sweep's U(V) (volume kernel) against the oracle's, same configuration
    assert abs(st["last_recompute"] - vols[-1][2]) <= 1e-12 * abs(vols[-1][2])
    assert np.array_equal(bits(gbox), bits(obox))
    for a, b in zip((gx, gy, gz, gox, goy, goz), state):
        assert np.array_equal(bits(a), bits(b))


def test_fp32_kernel_agrees_with_fp64():
    """From the same state, one FP32 sweep and one FP64 sweep make the same
    decisions except where dE is within FP32 rounding of the Metropolis
    threshold; the FP32 running energy (FP32 pair terms, FP64 sums) stays
    within 2e-6 relative of the FP64 recompute."""
    lp, _ = params_pair(11000, 0.08, 41, precision_mode=0)
    state, box = start_state(lp)
    with lcmc.GBSystem(lp) as s:
        s.set_kernel(0)
        s.upload(*state, box)
        s.sweep(100)  # relax the lattice with the FP64 kernel
        relaxed, rbox = s.download()
        e_relaxed = s.tot_ene() / 11000
    assert e_relaxed < 0.0  # no overlapping pairs left
    res = {}
    for kern in (0, 1):
        with lcmc.GBSystem(lp) as s:
            s.set_kernel(kern)
            s.upload(*relaxed, rbox)
            s.sweep(1)
            st = s.stats()
            res[kern] = (s.outcomes(), st, s.tot_ene())
            if kern == 1:
                assert st["kernel"] == 1
    o64, o32 = res[0][0], res[1][0]
    agree = np.mean(o64 == o32)
    print(f"relaxed E/N {e_relaxed:.4g}; outcome agreement {agree:.5f}; "
          f"acceptance fp64 {np.mean(o64 == 1):.4f} fp32 {np.mean(o32 == 1):.4f}")
    assert agree >= 0.995, agree
    st32, e32 = res[1][1], res[1][2]
    assert abs(st32["energy"] - e32) <= 2e-6 * abs(e32) + 1e-3
    assert st32["pairs_in_cutoff"] > 0 and st32["stencil_candidates"] > st32["pairs_in_cutoff"] // 2


def test_pair_terms_fp64_bitwise_and_fp32_error():
    """Pair term on the GPU: the FP64 kernel's arithmetic equals the oracle's
    canonical pij_GB bit for bit.  FP32 error relative to max(|phi|, 1),
    measured on B200 over 1.8e5 random in-cutoff pairs: median 1.8e-8, p99
    2.2e-5, max 1.9e-4 (the largest errors sit on the repulsive wall, where
    phi ~ R^12 amplifies the rounding of r - sigma + sigma0)."""
    import ctypes as C
    from parellel_mc_mpi_for_liquidcrystalsystems_b200 import _lib
    rng = np.random.default_rng(77)
    M = 200000
    lp, op = params_pair(1000, 0.30, 1)
    ei = rng.normal(size=(M, 3))
    ej = rng.normal(size=(M, 3))
    ei /= np.linalg.norm(ei, axis=1, keepdims=True)
    ej /= np.linalg.norm(ej, axis=1, keepdims=True)
    d = rng.normal(size=(M, 3))
    d *= (rng.uniform(0.8, 4.2, size=M) / np.linalg.norm(d, axis=1))[:, None]
    d, ei, ej = (np.ascontiguousarray(x) for x in (d, ei, ej))
    o32 = np.zeros(M)
    o64 = np.zeros(M)
    _lib.check(_lib.lib().lcmc_pair_terms(C.byref(lp), M, d.ctypes.data_as(_lib.DP), ei.ctypes.data_as(_lib.DP),
                                          ej.ctypes.data_as(_lib.DP), o32.ctypes.data_as(_lib.DP),
                                          o64.ctypes.data_as(_lib.DP)))
    c = oc.consts(op, oc.ARITH_CANONICAL)
    big = np.array([1e9, 1e9, 1e9])
    zero = np.zeros(3)
    want = np.empty(2000)
    for m in range(2000):
        inc = C.c_int()
        want[m] = oc.lib().lco_pair(C.byref(c), oc.ptr(zero), oc.ptr(np.ascontiguousarray(ei[m])),
                                    oc.ptr(np.ascontiguousarray(d[m])), oc.ptr(np.ascontiguousarray(ej[m])),
                                    oc.ptr(big), C.byref(inc))
    assert np.array_equal(bits(o64[:2000]), bits(want))
    inc = (np.sum(d * d, axis=1) < 16.0) & (o64 < 1e8)
    err = np.abs(o32 - o64)[inc] / np.maximum(np.abs(o64[inc]), 1.0)
    print(f"FP32 pair error over {inc.sum()} pairs: median {np.median(err):.2e}, p99 {np.quantile(err, 0.99):.2e}, "
          f"max {err.max():.2e}")
    assert np.median(err) < 1e-6
    assert np.quantile(err, 0.99) < 1e-4
    assert err.max() < 1e-3


def test_fp32_runs_are_deterministic():
    lp, _ = params_pair(11000, 0.30, 42, precision_mode=1)
    outs = []
    for _ in range(2):
        with lcmc.GBSystem(lp) as s:
            s.get_initial_config()
            s.sweep(3)
            outs.append(s.download())
            ms = s.last_sweep_timing()  # event nodes inside the sweep graph
            assert ms[0] > 0 and ms[1] > 0 and ms[3] >= 0 and s.kernels_per_sweep() == 27
    for a, b in zip(outs[0][0], outs[1][0]):
        assert np.array_equal(bits(a), bits(b))


def test_batched_replicas_match_single_runs():
    ps = [
        lcmc.default_params(num_particles=1000, system_density=0.30, rng_seed=101, precision_mode=0, **COMMON),
        lcmc.default_params(num_particles=1500, system_density=0.32, rng_seed=102, precision_mode=0,
                            mc_ensemble_type=2, system_pressure=2.0, system_temperature=1.2, **COMMON),
        lcmc.default_params(num_particles=2000, system_density=0.30, rng_seed=103, precision_mode=0,
                            colloid_radius=3.0, colloid_wall_option=1, system_temperature=0.8, **COMMON),
    ]
    singles = []
    for p in ps:
        with lcmc.GBSystem(p) as s:
            s.get_initial_config()
            s.sweep(3)
            singles.append((s.download(), s.stats()))
    with lcmc.GBSystem(ps) as b:
        for r in range(len(ps)):
            b.get_initial_config(r)
        b.sweep(3)
        for r, (want, wst) in enumerate(singles):
            got = b.download(r)
            for x, y in zip(got[0], want[0]):
                assert np.array_equal(bits(x), bits(y))
            assert np.array_equal(bits(got[1]), bits(want[1]))
            assert b.stats(r)["accepted"] == wst["accepted"]


def test_replica_groups_match_single_runs():
    """A batch of nine replicas (FP64 and FP32 kernels, NVT and NPT, with and
    without a colloid) runs its colour phases as replica groups on their own
    streams; every replica still reproduces its single run bit for bit."""
    ps = []
    for r in range(9):
        kw = dict(COMMON, num_particles=1000 + 250 * r, system_density=0.30, rng_seed=300 + r,
                  precision_mode=r % 2, system_temperature=0.9 + 0.05 * r)
        if r % 3 == 1:
            kw.update(mc_ensemble_type=2, system_pressure=2.0)
        if r % 3 == 2:
            kw.update(colloid_radius=3.0, colloid_wall_option=1)
        ps.append(lcmc.default_params(**kw))
    singles = []
    for p in ps:
        with lcmc.GBSystem(p) as s:
            s.get_initial_config()
            s.sweep(3)
            singles.append((s.download(), s.stats()))
    with lcmc.GBSystem(ps) as b:
        for r in range(len(ps)):
            b.get_initial_config(r)
        b.sweep(3)
        for r, (want, wst) in enumerate(singles):
            got = b.download(r)
            for x, y in zip(got[0], want[0]):
                assert np.array_equal(bits(x), bits(y)), r
            assert np.array_equal(bits(got[1]), bits(want[1])), r
            assert b.stats(r)["accepted"] == wst["accepted"] and b.stats(r)["energy"] == wst["energy"], r


def test_order_parameter_vs_oracle():
    lp, _ = params_pair(4096, 0.32, 7, init_orientation_cone_deg=20.0)
    state, box = start_state(lp)
    with lcmc.GBSystem(lp) as s:
        s.upload(*state, box)
        Q, P2, d = s.compute_liquid_crystal_order_parameters()
    Qo, P2o, do = oc.order_parameter(state[3], state[4], state[5])
    assert np.allclose(Q, Qo, rtol=0, atol=1e-13)
    assert abs(P2 - P2o) < 1e-12
    assert abs(abs(np.dot(d, do)) - 1.0) < 1e-10
    assert P2 > 0.8


def test_fp64_configs0_full_run_bitwise_vs_oracle():
    """The CPU-runnable configuration in full: N = 1000, rho* = 0.30, T* = 1.0,
    GB(3, 5, 2, 1), rc = 4, d = 0.1, rotation 0.1, seeded simple-cubic start
    with orientations uniform on the sphere, 1000 sweeps.  Every sweep's
    accept/reject outcomes and the final coordinates and energy equal the
    oracle's canonical checkerboard run bit for bit (about 35 s of oracle)."""
    lp, op = params_pair(1000, 0.30, 2024, precision_mode=0, system_temperature=1.0)
    state, box = start_state(lp)
    c = oc.consts(op, oc.ARITH_CANONICAL)
    k = oc.key(op.rng_seed)
    ostate = [x.copy() for x in state]
    obox = box.copy()
    n = 1000
    with lcmc.GBSystem(lp) as s:
        s.set_kernel(0)
        s.upload(*state, box)
        for sw in range(1000):
            s.sweep(1)
            _, b, order = oc.sweep(c, k, sw, ostate, obox, record=True)
            want = np.zeros(n, dtype=np.uint8)
            want[order] = b
            got = s.outcomes()
            assert np.array_equal(got, want), f"sweep {sw}: {int(np.sum(got != want))} outcomes differ"
        (gx, gy, gz, gox, goy, goz), gbox = s.download()
        e = s.tot_ene()
    for a, b in zip((gx, gy, gz, gox, goy, goz), ostate):
        assert np.array_equal(bits(a), bits(b))
    want_e = oc.total_energy(c, ostate, obox)
    assert abs(e - want_e) <= 1e-12 * abs(want_e)
