#!/usr/bin/env python3
"""Ensemble averages from the reference's OWN Monte Carlo chain.

Runs in a container where the reference source is available: loads
oracle/_ref/libmcref_serial.so (MCnptColloid.c built by oracle/build_ref.sh)
and runs attempt_monte_carlo_move (MCnptColloid.c:2445-2604, random particle
per attempt, libc rand()) from the seeded lattice of the oracle, with the
Verlet list rebuilt every N/2 attempts (refdrv_run_attempts_periodic;
the 2.5 skin is far more than a rod travels in that time).  After a
burn-in it records U/N (the reference's running energy) and P2 (largest
eigenvalue of the Q tensor, in numpy) after every N attempts, and stores the
means with block-averaged standard errors in ensemble_golden.npz.

System: N = 1728 Gay-Berne rods GB(3, 5, 2, 1), rho* = 0.10, T* = 2.0,
r_c = 4.0, r_v = 6.5, d = 0.5, rotation 0.3, NVT, colloid of radius 2 at the
box centre (colloid_wall_option 1, so the reference's ungated colloid term in
moves and ours agree).  An isotropic fluid; the large steps let it forget the
lattice within the burn-in (with d = 0.1 the energy still drifted by 6 % over
10^4 sweeps).  The script prints the means of the two halves of the
production run as a stationarity check.

`make_ensemble_golden.py part K` runs the gas chain with seed SEED + K into
ensemble_part_K.npz (independent chains can run on separate cores), and
`make_ensemble_golden.py combine K1 K2 ...` merges those parts with the main
chain into ensemble_golden.npz: the mean of the chain means, with the
standard error from their spread (ensemble_golden.npz holds 12 chains:
combine 1 2 ... 11).

`make_ensemble_golden.py dense` writes ensemble_dense_golden.npz instead: the
dense liquid of the CPU-runnable configuration (N = 1000, rho* = 0.30,
T* = 1.0, d = 0.1, rotation 0.1, r_v = 4.8) with a colloid of radius 2 (for
the same colloid-term reason).  A lattice at this density holds rods in the
flat 1e9 overlap clamp, which no move leaves, so the start is relaxed first:
a dilute lattice (rho* = 0.06, no site within R + 2.5 of the colloid, where a
rod could sit in the colloid term's flat 1e8 clamp) compressed by the oracle's checkerboard sweeps
with ln V moves at P* = 4 until rho* >= 0.30, scaled to 0.30 exactly and
stored with the averages, so the GPU test starts from the same state.
"""
import ctypes as C
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(HERE))
REF_SO = os.path.join(REPO, "oracle", "_ref", "libmcref_serial.so")

N, RHO, T, R_COLL, SEED = 1728, 0.10, 2.0, 2.0, 4242
DMAX, ROT = 0.5, 0.3
BURN, SWEEPS, BLOCKS = 2000, 10000, 20

PARAM_TEXT = f"""# written by tests/golden/make_ensemble_golden.py
mc_ensemble_type 1
num_particles {N}
system_density {RHO}
system_temperature {T}
system_pressure 1.0
gb_sigma_sidetoside 1.0
gb_epsilon0 1.0
gb_kappa 3.0
gb_kappa_prime 5.0
gb_mu_exponent 2.0
gb_nu_exponent 1.0
max_displacement {DMAX}
max_rotation {ROT}
initial_configuration_type 2
cutoff_radius 4.0
verlet_radius 6.5
total_mc_cycles 1000
configuration_save_interval 100
statistics_print_interval 100
colloid_wall_option 1
colloid_interaction_epsilon 15
colloid_interaction_amplitude 1.5
colloid_radius {R_COLL}
"""

D, DP, IP = C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_int)


def p2_of(ox, oy, oz):
    u = np.stack([ox, oy, oz], 1)
    u = u / np.linalg.norm(u, axis=1)[:, None]
    Q = 1.5 * (u.T @ u) / len(u) - 0.5 * np.eye(3)
    return float(np.linalg.eigvalsh(Q)[-1])


def block_mean_se(x, blocks):
    b = np.array_split(np.asarray(x), blocks)
    m = np.array([v.mean() for v in b])
    return float(m.mean()), float(m.std(ddof=1) / np.sqrt(blocks))


def compressed_start(oc, n, rho, T, R, seed):
    """Dilute lattice compressed to rho by the oracle (checkerboard sweeps and
    ln V moves at P* = 4), then scaled to rho exactly."""
    p = oc.params(num_particles=n, system_density=0.06, system_temperature=T, colloid_radius=R,
                  colloid_wall_option=1, rng_seed=seed, max_displacement=0.1, max_rotation=0.1)
    c = oc.consts(p, oc.ARITH_CANONICAL)
    k = oc.key(seed)
    # no site within R + 2.5 of the colloid: a rod closer to its wall can sit in
    # the colloid term's flat 1e8 clamp, which no move leaves
    px, py, pz, ox, oy, oz, box = oc.init_lattice(n=n, rho=0.06, R=R + 2.5, seed=seed)
    state = [np.ascontiguousarray(a, dtype=np.float64) for a in (px, py, pz, ox, oy, oz)]
    box = np.ascontiguousarray(box, dtype=np.float64)
    vcol = 4.0 * np.pi * R ** 3 / 3.0
    sweep = 0
    while n / (np.prod(box) - vcol) < rho:
        oc.sweep(c, k, sweep, state, box)
        oc.volume_move(c, k, sweep, 4.0, 0.05, state, box)
        sweep += 1
        if sweep > 20000:
            raise RuntimeError("compression did not reach the density")
    for _ in range(200):  # settle at the compressed box
        oc.sweep(c, k, sweep, state, box)
        sweep += 1
    L = (n / rho + vcol) ** (1.0 / 3.0)
    lam = L / box[0]
    for a in state[:3]:
        a *= lam
    box[:] = L
    print(f"compressed to rho {n / (np.prod(box) - vcol):.4f} in {sweep} oracle sweeps (scale {lam:.5f})")
    return state, box


def combine(parts):
    """The main chain (ensemble_golden.npz, its u/p2 series every 10 sweeps)
    plus independent chains ensemble_part_K.npz: the golden mean is the mean
    of the chain means and its standard error their spread over the square
    root of the number of chains (P2 in particular drifts slowly, so blocks
    inside one chain are not independent enough to give the error)."""
    main_f = os.path.join(HERE, "ensemble_golden.npz")
    files = [main_f] + [os.path.join(HERE, f"ensemble_part_{k}.npz") for k in parts]
    cu, cp = [], []
    for f in files:
        g = np.load(f)
        cu.append(float(np.mean(g["u_series"])))
        cp.append(float(np.mean(g["p2_series"])))
    g = dict(np.load(main_f))
    n = len(files)
    g["u_mean"], g["u_se"] = float(np.mean(cu)), float(np.std(cu, ddof=1) / np.sqrt(n))
    g["p2_mean"], g["p2_se"] = float(np.mean(cp)), float(np.std(cp, ddof=1) / np.sqrt(n))
    g["chains"] = n
    g["chain_u"], g["chain_p2"] = np.array(cu), np.array(cp)
    np.savez(main_f, **g)
    print(f"{n} chains: U/N = {g['u_mean']:.6f} +- {g['u_se']:.6f}  P2 = {g['p2_mean']:.6f} +- "
          f"{g['p2_se']:.6f} -> {main_f}")


def main():
    import oracle_ctypes as oc
    global N, RHO, T, R_COLL, SEED, DMAX, ROT, BURN, SWEEPS, PARAM_TEXT
    if len(sys.argv) > 1 and sys.argv[1] == "combine":
        return combine([int(k) for k in sys.argv[2:]])
    dense = len(sys.argv) > 1 and sys.argv[1] == "dense"
    part = int(sys.argv[2]) if len(sys.argv) > 2 and sys.argv[1] == "part" else None
    if part is not None:
        SEED = SEED + part
    if dense:
        N, RHO, T, R_COLL, SEED, DMAX, ROT, BURN, SWEEPS = 1000, 0.30, 1.0, 2.0, 4343, 0.1, 0.1, 2000, 10000
        PARAM_TEXT = (PARAM_TEXT.replace("num_particles 1728", f"num_particles {N}")
                      .replace("system_density 0.1", f"system_density {RHO}")
                      .replace("system_temperature 2.0", f"system_temperature {T}")
                      .replace("max_displacement 0.5", f"max_displacement {DMAX}")
                      .replace("max_rotation 0.3", f"max_rotation {ROT}")
                      .replace("verlet_radius 6.5", "verlet_radius 4.8"))
    ref = C.CDLL(REF_SO)
    ref.load_initial_conditions.argtypes = [C.c_char_p]
    ref.refdrv_set_box.argtypes = [C.c_int, DP]
    ref.refdrv_run_attempts_periodic.argtypes = [C.c_long, C.c_long, DP, DP, DP, DP, DP, DP, IP, IP, C.c_long, DP,
                                                 C.POINTER(C.c_long)]
    ref.refdrv_run_attempts_periodic.restype = D
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        f.write(PARAM_TEXT)
        path = f.name
    ref.load_initial_conditions(path.encode())
    os.unlink(path)
    if dense:
        state, box = compressed_start(oc, N, RHO, T, R_COLL, SEED)
        start = [a.copy() for a in state]
    else:
        px, py, pz, ox, oy, oz, box = oc.init_lattice(n=N, rho=RHO, R=R_COLL, seed=SEED)
        state = [np.ascontiguousarray(a, dtype=np.float64) for a in (px, py, pz, ox, oy, oz)]
        box = np.ascontiguousarray(box, dtype=np.float64)
    start_box = box.copy()
    ref.refdrv_set_box(N, box.ctypes.data_as(DP))
    C.CDLL("libc.so.6").srand(SEED)
    ref.refdrv_fill_rotation_table()
    ptrs = [a.ctypes.data_as(DP) for a in state]
    cap = 400 * N
    cnt = np.zeros(N, dtype=np.int32)
    lst = np.zeros(cap, dtype=np.int32)
    E = D(0.0)
    acc = C.c_long(0)
    t0 = time.time()
    args = (*ptrs, cnt.ctypes.data_as(IP), lst.ctypes.data_as(IP), cap, C.byref(E), C.byref(acc))
    ref.refdrv_run_attempts_periodic(BURN * N, N // 2 if not dense else N // 4, *args)
    acc.value = 0
    u, p2 = np.empty(SWEEPS), np.empty(SWEEPS)
    for s in range(SWEEPS):
        ref.refdrv_run_attempts_periodic(N, N // 2 if not dense else N // 4, *args)
        u[s] = E.value / N
        p2[s] = p2_of(state[3], state[4], state[5])
    mu, su = block_mean_se(u, BLOCKS)
    mp, sp = block_mean_se(p2, BLOCKS)
    h = SWEEPS // 2
    print(f"halves: U/N {u[:h].mean():.5f} {u[h:].mean():.5f}  P2 {p2[:h].mean():.5f} {p2[h:].mean():.5f}")
    out = os.path.join(HERE, "ensemble_dense_golden.npz" if dense else "ensemble_golden.npz")
    if part is not None:
        out = os.path.join(HERE, f"ensemble_part_{part}.npz")
    extra = {}
    if dense:
        extra = dict(start_px=start[0], start_py=start[1], start_pz=start[2], start_ox=start[3], start_oy=start[4],
                     start_oz=start[5], start_box=start_box)
    np.savez(out, n=N, rho=RHO, T=T, colloid_R=R_COLL, seed=SEED, dmax=DMAX, rot=ROT, burn=BURN, sweeps=SWEEPS,
             blocks=BLOCKS,
             u_mean=mu, u_se=su, p2_mean=mp, p2_se=sp, acceptance=acc.value / (SWEEPS * N),
             u_series=u[::10], p2_series=p2[::10], **extra)
    print(f"U/N = {mu:.6f} +- {su:.6f}  P2 = {mp:.6f} +- {sp:.6f}  acceptance {acc.value / (SWEEPS * N):.3f}  "
          f"in {time.time() - t0:.0f} s -> {out}")


if __name__ == "__main__":
    main()
