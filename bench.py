#!/usr/bin/env python3
"""Attempted Gay-Berne Monte Carlo moves per second on B200 (and the CPU reference).

Workload (one system per GPU, weak scaling over GPUs): GB(kappa=3, kappa'=5,
mu=2, nu=1), N = 1,048,576 ellipsoids, rho* = 0.32, T* = 0.8, cutoff 4.0,
max displacement 0.1, max rotation 0.1, NVT, seeded lattice start with
orientations within 20 degrees of z: a body-centred tetragonal lattice with
layers 1.05 sigma_ee apart along z (no pair in the 1e9 overlap clamp; tilted
neighbours overlap mildly and relax in a few sweeps); FP32 pair terms,
FP64 state and sums.  A step is one checkerboard sweep (N trial moves).  The
line's `jammed_start` sub-object times the same system from the simple-cubic
lattice (spacing 1.46 for rods of length 3: pairs in the 1e9 overlap clamp
and terms up to 1e36 beside it, attempted in FP64 by the hand-over kernel).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints one JSON line (rank 0).  `value` times K sweeps with the state resident
in HBM (CUDA events on the library's stream, max over ranks, L2 flushed
between sweeps); `e2e` times the public C ABI with host arrays in pinned
memory: upload + sweep + download every step.  `--impl reference` times the
reference's own attempt_monte_carlo_move (MCnptColloid.c, built in
oracle/_ref with its OpenMP pragmas) on the host cores.

The line also carries `npt_da`: effective samples per second of the P2 (and
volume) series of NPT sweeps at N = 262,144 with a colloid (R = 8), plain
volume moves against delayed acceptance with the learned surrogate and with
the FP32-pair screen (`--da-sweeps` per arm, 0 skips it).
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "GB attempted moves/s"
UNIT = "moves/s"
N_PART = 1048576
WORKLOAD = {
    "workload": "Gay-Berne NVT sweep, N=1048576, rho*=0.32, T*=0.8, GB(3,5,2,1), rc=4.0, d=0.1, rot=0.1, "
                "lattice start (body-centred tetragonal, layers 1.05 sigma_ee apart along z) with orientations "
                "within 20 deg of z",
    "n_particles": N_PART,
    # timing hygiene of the GPU arm (both arms print this same config)
    "l2": "GPU arm: L2 flushed between timed sweeps (256 MiB memset)",
}


def gb_params(lcmc, seed, lattice=1):
    """lattice 1: body-centred tetragonal start (the headline); 0: the
    reference's simple-cubic lattice (jammed at this density)."""
    return lcmc.default_params(
        mc_ensemble_type=1, num_particles=N_PART, system_density=0.32, system_temperature=0.8,
        gb_sigma_sidetoside=1.0, gb_epsilon0=1.0, gb_kappa=3.0, gb_kappa_prime=5.0, gb_mu_exponent=2.0,
        gb_nu_exponent=1.0, max_displacement=0.1, max_rotation=0.1, cutoff_radius=4.0, verlet_radius=4.8,
        colloid_wall_option=0, colloid_radius=0.0, init_orientation_cone_deg=20.0, precision_mode=1,
        rng_seed=seed, init_lattice=lattice)


def bct_lattice(n, rho, seed, cone_deg, kappa=3.0):
    """The workload's start for the CPU arms (which load none of this
    library): the library's body-centred tetragonal sites (layers
    c = L / floor(L / (1.05 kappa)) apart along z, square sites a = L / n_a
    apart, the smallest n_a holding n, surplus sites left empty evenly),
    orientations uniform on the cap within cone_deg of z from numpy's
    generator (same distribution, other draws)."""
    import numpy as np
    L = (n / rho) ** (1.0 / 3.0)
    nz = max(1, int(np.floor(L / (1.05 * kappa))))
    c = L / nz
    na = 1
    while 2 * na * na * nz < n:
        na += 1
    a = L / na
    S = 2 * na * na * nz
    s = np.arange(S)
    keep = ((s + 1) * n) // S > (s * n) // S
    s = s[keep]
    b, q = s & 1, s >> 1
    ix, iy, iz = q % na, (q // na) % na, q // (na * na)
    x = (ix + 0.5 * b) * a
    y = (iy + 0.5 * b) * a
    z = (iz + 0.5 * b) * c
    rng = np.random.default_rng(seed)
    ct = 1.0 - rng.random(n) * (1.0 - np.cos(np.radians(cone_deg)))
    st = np.sqrt(1.0 - ct * ct)
    ph = 2.0 * np.pi * rng.random(n)
    return [np.ascontiguousarray(v) for v in (x, y, z, st * np.cos(ph), st * np.sin(ph), ct)], np.array([L, L, L])


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.first = 0

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the sampler's first line marks it running; later lines fall in the timed region
            t0 = time.perf_counter()
            while not self.lines and time.perf_counter() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.01)
            self.first = len(self.lines)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.lines[self.first:] or self.lines
        for l in lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU reference (oracle/_ref/libmcref_omp.so: the reference's own functions)
# ---------------------------------------------------------------------------
def reference_cpu(n_part, seconds=12.0, threads=None, steps=1, warmup=0):
    """Time the reference's attempt_monte_carlo_move on the workload: `warmup`
    untimed and `steps` timed steps, each a bounded sample of the same number
    of consecutive attempts, sized so that the timed steps take about
    `seconds` together.  The Verlet list (r_v = 4.8) is built once with the
    same content as the reference's build_neighbor_lists (its O(N^2) double
    loop is infeasible at N = 1M) and not rebuilt inside the sample, which
    favours the reference."""
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import numpy as np

    import oracle_ctypes as oc
    so = os.path.join(REPO, "oracle", "_ref", "libmcref_omp.so")
    if not os.path.exists(so):
        return None, "oracle/_ref/libmcref_omp.so not built (needs the reference source at build time)"
    threads = threads or os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    ref = C.CDLL(so)
    D, DP, IP = C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_int)
    ref.refdrv_set_box.argtypes = [C.c_int, DP]
    ref.load_initial_conditions.argtypes = [C.c_char_p]
    ref.refdrv_build_verlet_cells.argtypes = [DP, DP, DP, IP, IP, C.c_long]
    ref.refdrv_build_verlet_cells.restype = C.c_long
    ref.refdrv_run_attempts.argtypes = [C.c_long, C.c_int, DP, DP, DP, DP, DP, DP, IP, IP, C.c_long, DP,
                                        C.POINTER(C.c_long), C.POINTER(C.c_long)]
    ref.refdrv_run_attempts.restype = D
    text = (f"mc_ensemble_type 1\nnum_particles {n_part}\nsystem_density 0.32\nsystem_temperature 0.8\n"
            "system_pressure 2.0\ngb_sigma_sidetoside 1.0\ngb_epsilon0 1.0\ngb_kappa 3.0\ngb_kappa_prime 5.0\n"
            "gb_mu_exponent 2.0\ngb_nu_exponent 1.0\nmax_displacement 0.1\nmax_rotation 0.1\n"
            "initial_configuration_type 2\ncutoff_radius 4.0\nverlet_radius 4.8\ntotal_mc_cycles 1000\n"
            "configuration_save_interval 100\nstatistics_print_interval 100\ncolloid_wall_option 0\n"
            "colloid_interaction_epsilon 15\ncolloid_interaction_amplitude 1.5\ncolloid_radius 0.0\n")
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        f.write(text)
        path = f.name
    ref.load_initial_conditions(path.encode())
    os.unlink(path)
    (px, py, pz, ox, oy, oz), box = bct_lattice(n_part, 0.32, 1234, 20.0)
    ref.refdrv_set_box(n_part, box.ctypes.data_as(DP))
    libc = C.CDLL("libc.so.6")
    libc.srand(1234)
    ref.refdrv_fill_rotation_table()
    arrs = [np.ascontiguousarray(a) for a in (px, py, pz, ox, oy, oz)]
    ptrs = [a.ctypes.data_as(DP) for a in arrs]
    cap = 200 * n_part
    cnt = np.zeros(n_part, dtype=np.int32)
    lst = np.zeros(cap, dtype=np.int32)
    t0 = time.perf_counter()
    if ref.refdrv_build_verlet_cells(*ptrs[:3], cnt.ctypes.data_as(IP), lst.ctypes.data_as(IP), cap) < 0:
        return None, "Verlet list capacity"
    t_list = time.perf_counter() - t0
    E = D(0.0)
    acc, nreb = C.c_long(0), C.c_long(0)
    def run(k):
        return ref.refdrv_run_attempts(k, 0, *ptrs, cnt.ctypes.data_as(IP), lst.ctypes.data_as(IP), cap,
                                       C.byref(E), C.byref(acc), C.byref(nreb))

    # calibrate, then `warmup` + `steps` steps of n_step attempts each
    n_try = 20
    dt = run(n_try)
    steps = max(1, steps)
    n_step = max(10, int(n_try * seconds / steps / max(dt, 1e-6)))
    for _ in range(warmup):
        run(n_step)
    step_s = [run(n_step) for _ in range(steps)]
    dt = sum(step_s)
    n_att = n_step * steps
    return {"value": n_att / dt, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"{steps} timed steps of {n_step} consecutive attempt_monte_carlo_move calls "
                      f"(MCnptColloid.c:2445) at N={n_part}, {n_att} attempts in {dt:.1f} s after {warmup} untimed "
                      f"steps, OpenMP threads={threads}, Verlet list (r_v=4.8) built once in {t_list:.1f} s and "
                      "not rebuilt",
            "seconds": dt, "attempts_per_step": n_step, "ms_per_step": 1e3 * dt / steps}, None


# ---------------------------------------------------------------------------
# FP32 peak (for the roofline denominator): cuBLAS SGEMM, TF32 off
# ---------------------------------------------------------------------------
def fp32_peak_tflops(torch):
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192
    a = torch.randn(n, n, device="cuda", dtype=torch.float32)
    b = torch.randn(n, n, device="cuda", dtype=torch.float32)
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(6):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        a @ b
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def measured_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def kernel_traffic():
    """DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one
    k_phase_fast launch on this workload and where the figure comes from: a
    fixed ncu capture (ncu cannot run inside the timed process), so it is
    the same in every run and is refreshed when the kernel changes."""
    return 45.368576e6 + 1.271808e6, ("fixed, from one ncu --set full capture of k_phase_fast launches 265-266 "
                                      "of `bench.py --steps 3 --warmup 3 --e2e-steps 1 --cpu-seconds 2 "
                                      "--port-seconds 0 --da-sweeps 0 --jammed-steps 0 --batch-steps 0` (45.4 MB "
                                      "read + 1.3 MB written per launch); not measured in this run")


# ---------------------------------------------------------------------------
# NPT P2 ESS/s: delayed-acceptance volume moves vs plain
# ---------------------------------------------------------------------------
GB_NPT = dict(gb_kappa=3.0, gb_kappa_prime=5.0, gb_mu_exponent=2.0, gb_nu_exponent=1.0, cutoff_radius=4.0,
              max_displacement=0.1, max_rotation=0.1)


def dilute_start(n, rho0, R, seed):
    """Simple-cubic start at density rho0 with uniform orientations, no site
    within R + 2.5 of the colloid centre.  At rho0 = 0.06 the spacing (2.4)
    leaves no pair inside the reference's flat 1e9 overlap clamp (distreal <
    0.001) and no rod inside the colloid's 1e8 clamp; a lattice at rho = 0.3
    with random orientations does, and such rods never leave the clamp."""
    import numpy as np
    rng = np.random.default_rng(seed)
    L = (n / rho0 + 4.0 * np.pi * R ** 3 / 3.0) ** (1.0 / 3.0)
    ns = int(np.ceil((1.3 * n) ** (1.0 / 3.0)))
    while True:
        g = (np.arange(ns) + 0.5) * (L / ns)
        X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
        pos = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
        ok = np.linalg.norm(pos - 0.5 * L, axis=1) > R + 2.5
        if ok.sum() >= n:
            break
        ns += 1
    pos = pos[ok][rng.permutation(int(ok.sum()))[:n]]
    u = rng.normal(size=(n, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    return [np.ascontiguousarray(a) for a in (pos[:, 0], pos[:, 1], pos[:, 2], u[:, 0], u[:, 1], u[:, 2])], \
        np.array([L, L, L])


def npt_params(lcmc, n, T, P, R, seed, dlnv, cap=64):
    """cap: active-cell capacity of the FP32 kernel (64: the large class, room
    for the training replicas' compression to P* = 4; the library's own NPT
    default is 56; 48, the small class, is enough at the density P* = 2
    compresses these systems to)."""
    return lcmc.default_params(num_particles=n, system_density=0.06, system_temperature=T, system_pressure=P,
                               mc_ensemble_type=2, npt_max_dlnV=dlnv, colloid_wall_option=1, colloid_radius=R,
                               rng_seed=seed, precision_mode=1, cell_capacity=cap, **GB_NPT)


def timed_sweeps(torch, s, k):
    ext = torch.cuda.ExternalStream(s.stream_handle())
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(ext)
    s.sweep(k)
    b.record(ext)
    b.synchronize()
    return a.elapsed_time(b) * 1e-3


def npt_da(lcmc, torch, sweeps, train_sweeps):
    """P2 (and volume) effective samples per second of NPT sweeps at N = 262,144
    with a colloid of R = 8 (T* = 0.85, P* = 2, dlnV_max = 0.01), plain volume
    moves vs delayed acceptance with the surrogate trained on N = 32,768
    systems (R = 5, T* = 0.9)."""
    import numpy as np

    from parellel_mc_mpi_for_liquidcrystalsystems_b200 import da
    t_start = time.perf_counter()
    # training samples: 16 replicas, compressed from dilute starts, pressures 2..4
    nr, n1 = 16, 32768
    pres = [2.0 + 2.0 * r / (nr - 1) for r in range(nr)]
    with lcmc.GBSystem([npt_params(lcmc, n1, 0.9, pres[r], 5.0, 200 + r, 0.05) for r in range(nr)]) as s:
        for r in range(nr):
            st, box = dilute_start(n1, 0.06, 5.0, 300 + r)
            s.upload(*st, box, replica=r)
        s.sweep(600)
        states = [s.download(r) for r in range(nr)]
    with lcmc.GBSystem([npt_params(lcmc, n1, 0.9, pres[r], 5.0, 400 + r, 0.01) for r in range(nr)]) as s:
        for r in range(nr):
            s.upload(*states[r][0], states[r][1], replica=r)
        s.sweep(100)
        x, y = da.collect_samples(s, train_sweeps)
        rho = [n1 / np.prod(s.stats(r)["box"]) for r in range(nr)]
    sur = da.Surrogate(max_batch=512, seed=1)
    t0 = time.perf_counter()
    sur.fit(x, y, epochs=20, batch=256, lr=1e-3)
    t_train = time.perf_counter() - t0
    keep = np.abs(y) < 1000.0
    k = min(4000, int(keep.sum()))
    corr = float(np.corrcoef(sur.predict(x[keep][:k]), y[keep][:k])[0, 1])

    # the N = 262,144 system: compress from a dilute start, settle at dlnV_max
    # 0.01, then every arm from that one state with one seed
    n = 262144
    with lcmc.GBSystem(npt_params(lcmc, n, 0.85, 2.0, 8.0, 11, 0.05, 48)) as s:
        st, box = dilute_start(n, 0.06, 8.0, 12)
        s.upload(*st, box)
        s.sweep(1000)
        st4, box4 = s.download()
    with lcmc.GBSystem(npt_params(lcmc, n, 0.85, 2.0, 8.0, 13, 0.01, 48)) as s:
        s.upload(*st4, box4)
        s.sweep(1000)
        st4, box4 = s.download()
    arms = {}
    for name in ("plain", "learned", "fp32_screen"):
        with lcmc.GBSystem(npt_params(lcmc, n, 0.85, 2.0, 8.0, 21, 0.01, 48)) as s:
            s.upload(*st4, box4)
            if name == "learned":
                s.set_surrogate(sur)
            elif name == "fp32_screen":
                s.set_fp32_screen(True)
            s.sweep(100)
            st0 = s.stats()
            s.record_history(sweeps)
            secs = timed_sweeps(torch, s, sweeps)
            st1 = s.stats()
            _, p2, E, V = da.p2_series(s)
            tp, tv = da.integrated_autocorrelation_time(p2), da.integrated_autocorrelation_time(V)
            arms[name] = {
                "sweeps": sweeps, "seconds": secs, "ms_per_sweep": 1e3 * secs / sweeps,
                "p2_mean": float(p2.mean()), "p2_tau_sweeps": tp, "p2_ess": sweeps / (2 * tp),
                "p2_ess_per_s": sweeps / (2 * tp) / secs, "volume_tau_sweeps": tv,
                "volume_ess_per_s": sweeps / (2 * tv) / secs, "rho_mean": float(np.mean(n / V)),
                "volume_accepted": st1["volume_accepted"] - st0["volume_accepted"],
                "volume_stage1_rejected": st1["volume_stage1_rejected"] - st0["volume_stage1_rejected"],
                "exact_volume_energies": (st1["volume_attempted"] - st0["volume_attempted"])
                                         - (st1["volume_stage1_rejected"] - st0["volume_stage1_rejected"]),
                "sweep_ms_parts": [round(float(t), 4) for t in s.last_sweep_timing()]}
            if name == "plain":
                p2_plain = p2
            elif name == "fp32_screen":
                arms[name]["p2_series_equals_plain"] = bool(np.array_equal(p2, p2_plain))
    sur.close()
    pl, le, sc = arms["plain"], arms["learned"], arms["fp32_screen"]
    return {
        "metric": "NPT P2 ESS/s, delayed-accept vs plain",
        "workload": "NPT N=262144, colloid R=8, T*=0.85, P*=2.0, dlnV_max=0.01 (one move per sweep), GB(3,5,2,1), "
                    "FP32 sweeps, FP64 volume energies; compressed for 1000 sweeps (dlnV_max 0.05) from a dilute "
                    "lattice (rho 0.06), 1000 sweeps at dlnV_max 0.01, then 100 sweeps before each timed arm; "
                    "every arm from the same state and seed",
        "training": {"samples": int(len(y)), "used": int(keep.sum()), "replicas": nr, "n": n1, "colloid_R": 5.0,
                     "T": 0.9, "pressures": [pres[0], pres[-1]], "rho_range": [float(min(rho)), float(max(rho))],
                     "train_seconds": t_train, "final_loss": sur.history[-1] if sur.history else None,
                     "pred_corr": corr},
        "plain": pl, "learned": le, "fp32_screen": sc,
        "p2_ess_per_s_ratio": {"learned": le["p2_ess_per_s"] / pl["p2_ess_per_s"],
                               "fp32_screen": sc["p2_ess_per_s"] / pl["p2_ess_per_s"]},
        "volume_ess_per_s_ratio": {"learned": le["volume_ess_per_s"] / pl["volume_ess_per_s"],
                                   "fp32_screen": sc["volume_ess_per_s"] / pl["volume_ess_per_s"]},
        "sweeps_per_s_ratio": {"learned": pl["ms_per_sweep"] / le["ms_per_sweep"],
                               "fp32_screen": pl["ms_per_sweep"] / sc["ms_per_sweep"]},
        "ess_note": "tau_int by Sokal's automatic window (c=5); with tau of a few hundred sweeps the ESS of one "
                    "arm has a relative error of tens of percent, except that the fp32_screen arm repeats the "
                    "plain arm's decisions (p2_series_equals_plain), so its ratio is exactly the sweep-rate ratio",
        "seconds_total": time.perf_counter() - t_start}


def npt_workload(lcmc, torch, n, steps, warmup, screen=False):
    """NPT sweeps of one system (colloid R = 8, T* = 0.85, P* = 2): a dilute
    start compressed for 700 sweeps (dlnV_max 0.05), `warmup` sweeps at
    dlnV_max = 0.01, then `steps` timed sweeps; device time per sweep by part."""
    import numpy as np
    with lcmc.GBSystem(npt_params(lcmc, n, 0.85, 2.0, 8.0, 11, 0.05, 48)) as s:
        st, box = dilute_start(n, 0.06, 8.0, 12)
        s.upload(*st, box)
        s.sweep(700)
        st, box = s.download()
    with lcmc.GBSystem(npt_params(lcmc, n, 0.85, 2.0, 8.0, 21, 0.01, 48)) as s:
        s.upload(*st, box)
        s.set_fp32_screen(screen)
        s.sweep(max(3, warmup))
        parts, total = [], 0.0
        for _ in range(steps):
            total += timed_sweeps(torch, s, 1)
            parts.append(s.last_sweep_timing())
        stt = s.stats()
        parts = np.median(np.array(parts), axis=0)
        return {"workload": f"NPT sweeps, N={n}, colloid R=8, T*=0.85, P*=2.0, dlnV_max=0.01, GB(3,5,2,1), FP32 "
                            "sweep kernel, FP64 volume energies, compressed from a dilute lattice",
                "steps": steps, "ms_per_sweep": 1e3 * total / steps,
                "ms_parts_median": {"rebin": parts[0], "colour_phases": parts[1], "volume_move": parts[2],
                                    "finalize": parts[3]},
                "fp32_screen": screen, "volume_accepted": stt["volume_accepted"],
                "volume_stage1_rejected": stt["volume_stage1_rejected"],
                "rho": n / float(np.prod(stt["box"])), "energy_per_particle": stt["energy"] / n,
                "kernels_per_sweep": s.kernels_per_sweep()}


def port_cpu(n_part, seconds=8.0, threads=None):
    """The same checkerboard algorithm on the host cores: the oracle's FP64
    cell-list sweep (oracle/lcmc_oracle.c, lco_sweep_parallel) with each
    colour's active cells shared among OpenMP threads, on the workload's own
    lattice start, whole sweeps until `seconds` have passed (at least one)."""
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import numpy as np

    import oracle_ctypes as oc
    threads = threads or os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(threads)
    try:
        oc.omp_lib()
    except OSError as e:
        return None, f"oracle OpenMP build not loadable: {e}"
    state, box = bct_lattice(n_part, 0.32, 1234, 20.0)
    p = oc.params(num_particles=n_part, system_density=0.32, system_temperature=0.8, max_displacement=0.1,
                  max_rotation=0.1, cutoff_radius=4.0, rng_seed=1234, init_orientation_cone_deg=20.0)
    consts = oc.Consts()
    oc.omp_lib().lco_consts_from_params(C.byref(p), oc.ARITH_CANONICAL, C.byref(consts))
    key = (C.c_uint32 * 2)()
    oc.omp_lib().lco_key(1234, 0, key)
    t0 = time.perf_counter()
    done = 0
    while True:
        oc.sweep_parallel(consts, key, done, state, box)
        done += 1
        dt = time.perf_counter() - t0
        if dt >= seconds:
            break
    return {"value": n_part * done / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{done} sweep(s) of the oracle's FP64 checkerboard (cell lists, lco_sweep_parallel) at "
                      f"N={n_part} from the workload's lattice start in {dt:.1f} s, OpenMP threads={threads}",
            "seconds": dt}, None


# ---------------------------------------------------------------------------
# FP64 energy check of the running energy (EnergyCheck, MCnptColloid.c:1343-1362)
# ---------------------------------------------------------------------------
def energy_check_record(lcmc, s, sweeps):
    """Run the library's FP64 energy check on system s (outside any timed
    region) and describe it; ok = False when the running energy was outside
    the check's tolerance."""
    try:
        s.energy_check()
        ok = True
    except lcmc.LcmcError:
        ok = False
    st = s.stats()
    n = s.params[0].num_particles
    return {"ok": ok, "running_energy_per_particle": (st["last_recompute"] + st["drift"]) / n,
            "recomputed_energy_per_particle": st["last_recompute"] / n, "drift": st["drift"],
            "tolerance": st["drift_bound"], "breaches": st["drift_breaches"],
            "fp64_cells_per_sweep": st["fp64_cells"] / max(1, sweeps),
            "overcap_cells": st["overcap_cells"]}


def jammed_start(lcmc, torch, steps, warmup):
    """The same system from the reference's simple-cubic lattice (spacing 1.46
    for rods of length 3 within 20 deg of z): overlapping pairs in the 1e9
    clamp and terms up to 1e36 beside it, attempted in FP64 by the hand-over
    kernel.  Device time per sweep, L2 flushed between sweeps."""
    s = lcmc.GBSystem(gb_params(lcmc, 4321, lattice=0))
    s.get_initial_config()
    e0 = s.stats()["energy"] / N_PART
    ext = torch.cuda.ExternalStream(s.stream_handle())
    s.sweep(max(3, warmup))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    st0 = s.stats()
    ms = []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(ext)
        s.sweep(1)
        b.record(ext)
        b.synchronize()
        ms.append(a.elapsed_time(b))
    st1 = s.stats()
    chk = energy_check_record(lcmc, s, max(3, warmup) + steps)
    chk["fp64_cells_per_sweep_timed"] = (st1["fp64_cells"] - st0["fp64_cells"]) / steps
    s.close()
    return {"workload": "as the headline, from the simple-cubic lattice (spacing L/102 = 1.46)",
            "start_energy_per_particle": e0, "steps": steps, "warmup": max(3, warmup),
            "ms_per_step": statistics.mean(ms), "value": N_PART * steps / (sum(ms) * 1e-3), "unit": UNIT,
            "acceptance": (st1["accepted"] - st0["accepted"]) / max(1, st1["attempted"] - st0["attempted"]),
            "energy_check": chk}


# ---------------------------------------------------------------------------
# batched replicas (64 independent systems of uneven N, T, P, colloid)
# ---------------------------------------------------------------------------
def batch_replica_params(lcmc, n_rep=64, seed=2024):
    """The batch workload: N log-uniform in [4096, 65536], T* uniform on
    [0.6, 1.4]; even replicas NVT at rho* 0.30-0.34, odd ones NPT at P*
    1.5-2.5; every third replica with a colloid of R uniform in [3, 6];
    GB(3, 5, 2, 1), rc = 4, FP32 kernel, fine cell grid (odd cell counts
    allowed, so small boxes keep cells about one cutoff wide), body-centred
    lattice starts with orientations within 20 degrees of z."""
    import numpy as np
    rng = np.random.default_rng(seed)
    ps = []
    for r in range(n_rep):
        n = int(round(float(np.exp(rng.uniform(np.log(4096), np.log(65536))))))
        T = float(rng.uniform(0.6, 1.4))
        rho = float(rng.uniform(0.30, 0.34))
        npt = r % 2 == 1
        P = float(rng.uniform(1.5, 2.5))
        R = float(rng.uniform(3.0, 6.0)) if r % 3 == 0 else 0.0
        ps.append(lcmc.default_params(
            num_particles=n, system_density=rho, system_temperature=T, system_pressure=P,
            mc_ensemble_type=2 if npt else 1, npt_max_dlnV=0.01, colloid_radius=R, colloid_wall_option=1 if R else 0,
            gb_kappa=3.0, gb_kappa_prime=5.0, gb_mu_exponent=2.0, gb_nu_exponent=1.0, cutoff_radius=4.0,
            max_displacement=0.1, max_rotation=0.1, precision_mode=1, cell_grid=1, init_lattice=1,
            init_orientation_cone_deg=20.0, rng_seed=seed * 1000 + r))
    return ps


def lpt_split(costs, world):
    """Longest-processing-time placement of independent replicas on `world`
    ranks: replicas in decreasing cost (ties: lower index first), each to the
    rank with the least total cost so far (ties: lower rank).  Returns each
    rank's replica indices in ascending order; every rank computes the same
    split from the same costs, so no exchange is needed."""
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += costs[i]
        parts[r].append(i)
    return [sorted(p) for p in parts]


def batch_workload(lcmc, torch, steps, warmup, single_rate=None, dist=None, rank=0, world=1, relax=30):
    """Moves/s of the 64-replica batch in one graph-launched sweep per rank
    (device time per sweep, L2 flushed between sweeps), with the autotuner's
    choice.  With N ranks the replicas are split by longest-processing-time
    on N x sweeps (every replica runs the same sweeps); the job's time is the
    slowest rank's, and value counts every replica's moves."""
    import numpy as np
    ps_all = batch_replica_params(lcmc)
    ntot = sum(p.num_particles for p in ps_all)
    share = lpt_split([float(p.num_particles) for p in ps_all], world)[rank]
    ps = [ps_all[i] for i in share]
    s = lcmc.GBSystem(ps)
    for r in range(len(ps)):
        s.get_initial_config(r)
    # NPT replicas screen their volume moves with the FP32-pair energy change:
    # the plain move's decisions, with the FP64 recompute only where stage 1 passes
    s.set_fp32_screen(True)
    breaches = 0

    def sweep1(k):
        """k sweeps; an energy-check breach (LCMC_EDRIFT) is counted, its sticky
        flag cleared, and the run goes on (the chain is unchanged by it)."""
        nonlocal breaches
        try:
            s.sweep(k)
        except lcmc.LcmcError as e:
            if e.code != -12:
                raise
            breaches += 1
            s.clear_error_flags()

    sweep1(max(1, relax))  # untimed: the lattice starts relax their overlaps
    tune = s.autotune(sweeps=2)
    sweep1(max(3, warmup))
    ext = torch.cuda.ExternalStream(s.stream_handle())
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    st0 = [s.stats(r) for r in range(len(ps))]
    ms, parts = [], []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(ext)
        sweep1(1)
        b.record(ext)
        b.synchronize()
        ms.append(a.elapsed_time(b))
        parts.append(s.last_sweep_timing())
    st1 = [s.stats(r) for r in range(len(ps))]
    parts = np.median(np.array(parts), axis=0)
    fp64_cells = sum(b_["fp64_cells"] - a_["fp64_cells"] for a_, b_ in zip(st0, st1))
    try:
        s.energy_check()
        check_ok = True
    except lcmc.LcmcError:
        check_ok = False
    worst = max(abs(s.stats(r)["drift"]) / max(s.stats(r)["drift_bound"], 1e-300) for r in range(len(ps)))
    kps = s.kernels_per_sweep()
    s.close()
    total_ms = max_over_ranks(dist, sum(ms))
    value = ntot * steps / (total_ms * 1e-3)
    out = {"workload": "64 replicas, N log-uniform in [4096, 65536], T* U[0.6, 1.4], half NVT at rho* 0.30-0.34, "
                       "half NPT at P* 1.5-2.5 (volume moves screened by the FP32-pair energy change), a third "
                       "with a colloid R U[3, 6]; FP32 kernel, fine cell grid, one CUDA graph per sweep over the "
                       "replica table",
           "replicas": len(ps_all), "n_total": ntot, "n_min": min(p.num_particles for p in ps_all),
           "n_max": max(p.num_particles for p in ps_all), "steps": steps, "warmup": max(3, warmup),
           "relax_sweeps": max(1, relax),
           "ms_per_step": total_ms / steps, "value": value, "unit": UNIT,
           "placement": {"ranks": world, "rank0_replicas": len(ps),
                         "rank0_particles": sum(p.num_particles for p in ps)},
           "replicas_on_fp32_kernel": int(sum(st["kernel"] for st in st1)),
           "fp64_cells_per_sweep": fp64_cells / steps,
           "ms_parts_median": {"rebin": parts[0], "colour_phases": parts[1], "stats_and_volume": parts[2],
                               "advance": parts[3]},
           "kernels_per_sweep": kps, "autotune": tune,
           "energy_check": {"ok": check_ok and breaches == 0, "max_drift_over_tolerance": worst,
                            "breaches_during_sweeps": breaches}}
    if single_rate:
        out["per_move_rate_vs_single_system"] = value / single_rate
    return out


# ---------------------------------------------------------------------------
# ranks: the job's time is the slowest rank's; value = all ranks' units / that
# ---------------------------------------------------------------------------
def max_over_ranks(dist, x, device="cuda"):
    """Largest of the ranks' values of x, on every rank (x itself without a
    process group)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, world, seconds):
    """Whole-job throughput of a weak-scaling run: every rank processed
    units_per_rank in a job that took `seconds` (the max over ranks)."""
    return units_per_rank * world / seconds


# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--port-seconds", type=float, default=8.0,
                    help="host time for the checkerboard port baseline (0 skips it)")
    ap.add_argument("--da-sweeps", type=int, default=4000,
                    help="sweeps per arm of the NPT delayed-acceptance measurement (0 skips it)")
    ap.add_argument("--da-train-sweeps", type=int, default=400)
    ap.add_argument("--workload", default="moves", choices=["moves", "npt"],
                    help="npt: time NPT sweeps of one compressed system (per-part device times) instead")
    ap.add_argument("--npt-n", type=int, default=262144)
    ap.add_argument("--npt-screen", action="store_true", help="npt workload with the FP32-pair volume screen")
    ap.add_argument("--jammed-steps", type=int, default=5,
                    help="timed sweeps of the simple-cubic (jammed) start sub-measurement (0 skips it)")
    ap.add_argument("--relax-sweeps", type=int, default=30,
                    help="untimed sweeps from the lattice start before the warm-up (the start relaxes its overlaps; "
                         "the timed window is then sweeps relax+warmup+1 .. of the run)")
    ap.add_argument("--batch-steps", type=int, default=10,
                    help="timed sweeps of the 64-replica batch sub-measurement (0 skips it)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        steps = max(1, args.steps)
        res, why = reference_cpu(N_PART, seconds=max(2.0, args.cpu_seconds), steps=steps, warmup=args.warmup)
        if res is None:
            print(json.dumps({"impl": "reference", "unavailable": why}))
            return 0
        line = {"impl": "reference", "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": args.gpus,
                "steps": steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded body-centred lattice, the GPU arm's start)",
                "config": dict(WORKLOAD),
                "arm": {"parallelism": "cpu openmp", "precision": "fp64 (the reference's own code)",
                        "step": f"a bounded sample of {res['attempts_per_step']} consecutive attempts of the "
                                f"N={N_PART} system (a sweep is {N_PART} attempts)"},
                "cpu_baseline": {k: res[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import numpy as np
    import torch

    import parellel_mc_mpi_for_liquidcrystalsystems_b200 as lcmc

    torch.cuda.set_device(local)
    if args.workload == "npt":
        if rank == 0:
            print(json.dumps(npt_workload(lcmc, torch, args.npt_n, args.steps, args.warmup, args.npt_screen)))
        return 0
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    params = gb_params(lcmc, 1234 + rank)
    s = lcmc.GBSystem(params)
    s.get_initial_config()
    ext = torch.cuda.ExternalStream(s.stream_handle())
    if args.relax_sweeps > 0:
        s.sweep(args.relax_sweeps)
    for _ in range(max(3, args.warmup)):
        s.sweep(1)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    st0 = s.stats()
    step_ms, phase_ms = [], []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.zero_()  # evict the state from L2 between sweeps
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(ext)
            s.sweep(1)
            b.record(ext)
            b.synchronize()
            step_ms.append(a.elapsed_time(b))
            phase_ms.append(s.last_sweep_timing()[1])
    torch.cuda.synchronize()
    total_ms = max_over_ranks(dist, sum(step_ms))
    if dist:
        dist.barrier()
    st1 = s.stats()
    check = energy_check_record(lcmc, s, args.relax_sweeps + max(3, args.warmup) + args.steps)
    attempted = st1["attempted"] - st0["attempted"]
    value = job_rate(N_PART * args.steps, world, total_ms * 1e-3)

    # roofline of the colour-phase kernel: algorithmic flops per attempt
    # 2 (8 C + 61 P): C = 27-cell stencil candidates, P = in-cutoff pairs per state
    C_att = (st1["stencil_candidates"] - st0["stencil_candidates"]) / attempted
    P2_att = (st1["pairs_in_cutoff"] - st0["pairs_in_cutoff"]) / attempted  # old + new states
    flop_att = 16.0 * C_att + 61.0 * P2_att
    launches_phase = 8
    avg_launch_ms = statistics.mean(phase_ms) / launches_phase
    flop_launch = flop_att * N_PART / launches_phase
    achieved = flop_launch / (avg_launch_ms * 1e-3) / 1e12

    # e2e through the C ABI: the caller's state in pinned host arrays; every
    # step uploads it with the caller's running energy (the in/out energy of
    # attempt_monte_carlo_move), sweeps, downloads it and reads the energy back
    pinned = [torch.empty(N_PART, dtype=torch.float64, pin_memory=True) for _ in range(6)]
    hv = [p.numpy() for p in pinned]
    _, box = s.download(out=hv)
    energy = s.stats()["energy"]
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        s.upload(*hv, box, energy=energy)
        s.sweep(1)
        _, box = s.download(out=hv)
        energy = s.stats()["energy"]
    e2e_s = max_over_ranks(dist, time.perf_counter() - t0)
    e2e = job_rate(N_PART * args.e2e_steps, world, e2e_s)
    kps = s.kernels_per_sweep()
    st = s.stats()
    e_exact = s.tot_ene()  # FP64 recompute of the final state (outside the timed region)
    s.close()
    jam = None
    if args.jammed_steps > 0 and world == 1:
        jam = jammed_start(lcmc, torch, args.jammed_steps, args.warmup)
    batch = None
    if args.batch_steps > 0:  # every rank takes part (its share of the replicas)
        batch = batch_workload(lcmc, torch, args.batch_steps, args.warmup, single_rate=value, dist=dist, rank=rank,
                               world=world, relax=args.relax_sweeps)

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0

    peaks = measured_peaks()
    sgemm = fp32_peak_tflops(torch)
    nominal = 148 * 128 * 2 * peaks.get("sm_max_mhz", 1965.0) * 1e6 / 1e12
    cpu, why = reference_cpu(N_PART, seconds=args.cpu_seconds) if world == 1 else (None, "rank 0 of N>1")
    port, port_why = port_cpu(N_PART, seconds=args.port_seconds) if world == 1 and args.port_seconds > 0 \
        else (None, "not run")
    clocks = clk.summary()
    traffic = kernel_traffic()
    npt = None
    if args.da_sweeps > 0 and world == 1:
        try:
            npt = npt_da(lcmc, torch, args.da_sweeps, args.da_train_sweeps)
        except lcmc.LcmcError as e:  # keep the headline line if the side measurement fails
            npt = {"unavailable": str(e)}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded lattice, relaxing from the lattice start)",
        "config": dict(WORKLOAD),
        "arm": {"parallelism": f"replicas x{world}" if world > 1 else "single system",
                "precision": "fp32 pair terms, fp64 state and sums",
                "timed_window": f"sweeps {args.relax_sweeps + max(3, args.warmup) + 1}-"
                                f"{args.relax_sweeps + max(3, args.warmup) + args.steps} of the run from the "
                                "lattice start"},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 6 * 8 * N_PART + 24 + 8,
                "d2h_bytes_per_step": 6 * 8 * N_PART + 24 + 8,
                "step": "lcmc_upload_with_energy (pinned host SoA, caller-carried energy) + lcmc_sweep + "
                        "lcmc_download (into the pinned arrays) + lcmc_get_stats"},
        "gpu_launches": kps * args.steps,
        "roofline": {"bound": "fp32", "kernel": "k_phase_fast", "achieved": achieved, "peak": sgemm,
                     "unit": "TFLOP/s", "frac": achieved / sgemm,
                     "peak_source": "cuBLAS FP32 SGEMM (TF32 off) measured in this run; nominal FP32 "
                                    f"{nominal:.1f} TFLOP/s at max clock",
                     "traffic": traffic[0], "traffic_source": traffic[1], "flop_per_attempt": flop_att, "stencil_candidates_per_attempt": C_att,
                     "in_cutoff_pairs_per_attempt_old_plus_new": P2_att, "avg_launch_ms": avg_launch_ms,
                     "phase_share_of_step": statistics.mean(phase_ms) / (total_ms / args.steps)},
        "cpu_baseline": cpu if cpu else {"unavailable": why},
        "cpu_port": port if port else {"unavailable": port_why},
        "acceptance": (st["accepted"] / max(st["attempted"], 1)),
        # FP64 energy check after the timed sweeps (running vs recomputed, tolerance)
        "energy_check": check,
        # after the e2e steps: running energy carried through the C ABI vs an FP64 recompute
        "energy_per_particle": e_exact / N_PART,
        "running_energy_per_particle": st["energy"] / N_PART,
    }
    if jam:
        line["jammed_start"] = jam
    if batch:
        line["batch"] = batch
    if clocks:
        line["clocks"] = clocks
    if peaks:
        line["measured_peaks"] = {k: peaks.get(k) for k in ("hbm_gbs", "bf16_tflops", "sm_max_mhz")}
    if npt:
        line["npt_da"] = npt
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()
    if not check["ok"]:
        sys.stderr.write("bench: the running energy failed the FP64 energy check\n")
        return 3
    return 0


if __name__ == "__main__":
    sys.exit(main())
