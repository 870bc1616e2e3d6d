"""Python host mirror of the reference's Monte Carlo interface over liblcmc.so.

Function names follow MCnptColloid.c (load_initial_conditions,
get_initial_config, tot_ene, compute_liquid_crystal_order_parameters) so that
driver code and tests read like the reference; every call goes through the C
ABI of include/lcmc.h and runs on the GPU.  Errors raise LcmcError (the
reference calls exit(1)).
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import LcmcError, Params, Stats, check, lib


def default_params(**overrides):
    """lcmc_params with the library defaults, then `overrides` applied."""
    p = Params()
    check(lib().lcmc_params_defaults(C.byref(p)))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def load_initial_conditions(path, **overrides):
    """Read a parametersFile.txt (MCnptColloid.c:3933-4133): the 23 keys of the
    reference are required; added keys are optional."""
    p = default_params()
    rc = lib().lcmc_params_load(str(path).encode(), C.byref(p))
    if rc != _lib.OK:
        raise LcmcError(rc, f"{_lib.last_error()} (missing mask 0x{p.missing_mask:x})")
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def lattice(params, replica=0):
    """Seeded lattice start (initialize_cubic_lattice_positions,
    MCnptColloid.c:2920-3033: simple cubic; init_lattice = 1: body-centred
    tetragonal along z) computed on the host; returns (6 arrays, box)."""
    n = params.num_particles
    a = [np.zeros(n) for _ in range(6)]
    box = np.zeros(3)
    check(lib().lcmc_lattice(C.byref(params), replica, *[x.ctypes.data_as(_lib.DP) for x in a],
                             box.ctypes.data_as(_lib.DP)))
    return a, box


def _dp(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_lib.DP)


class GBSystem:
    """One system or a batch of independent replicas on the GPU."""

    def __init__(self, params):
        if isinstance(params, Params):
            params = [params]
        arr = (Params * len(params))(*params)
        h = C.c_void_p()
        check(lib().lcmc_create_batch(arr, len(params), C.byref(h)))
        self._h = h
        self.params = list(params)
        self.n_replicas = len(params)

    # -- lifetime --
    def close(self):
        if self._h:
            lib().lcmc_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        return check(rc, self._h)

    # -- configuration --
    def get_initial_config(self, replica=0):
        """get_initial_config (MCnptColloid.c:4215-4235), lattice type: seeded
        lattice uploaded to the device, FP64 total energy computed."""
        self._check(lib().lcmc_init_config(self._h, replica))

    def upload(self, px, py, pz, ox, oy, oz, box, replica=0, energy=None):
        """Copy a configuration to the device; the total energy is recomputed
        in FP64, or taken from `energy` (the caller's running energy, as the
        reference's attempt_monte_carlo_move carries it)."""
        arrs = [_dp(x) for x in (px, py, pz, ox, oy, oz)]
        b, bp = _dp(box)
        n = len(arrs[0][0])
        if energy is None:
            self._check(lib().lcmc_upload(self._h, replica, *[p for _, p in arrs], n, bp))
        else:
            self._check(lib().lcmc_upload_with_energy(self._h, replica, *[p for _, p in arrs], n, bp, float(energy)))

    def download(self, replica=0, out=None):
        """(6 arrays in id order, box); `out` = 6 float64 arrays to fill (for
        example pinned host buffers) instead of new ones."""
        n = self.params[replica].num_particles
        if out is None:
            out = [np.empty(n) for _ in range(6)]
        elif len(out) != 6 or any(a.dtype != np.float64 or a.shape != (n,) or not a.flags.c_contiguous for a in out):
            raise ValueError("out must be 6 contiguous float64 arrays of num_particles")
        box = np.zeros(3)
        self._check(lib().lcmc_download(self._h, replica, *[x.ctypes.data_as(_lib.DP) for x in out], n,
                                        box.ctypes.data_as(_lib.DP)))
        return out, box

    # -- Monte Carlo --
    def sweep(self, n_sweeps=1):
        """n_sweeps checkerboard sweeps (N attempts each) on every replica."""
        self._check(lib().lcmc_sweep(self._h, n_sweeps))

    def set_adaptive_step(self, on=True):
        """Adaptive max displacement/rotation (MCnptColloid.c:987-1031), for
        equilibration only."""
        self._check(lib().lcmc_set_adaptive_step(self._h, int(bool(on))))

    def step(self, replica=0):
        """Current (max displacement, max rotation)."""
        d, a = C.c_double(), C.c_double()
        self._check(lib().lcmc_get_step(self._h, replica, C.byref(d), C.byref(a)))
        return d.value, a.value

    def set_kernel(self, kernel):
        """-1 automatic, 0 the FP64 kernel, 1 the FP32 kernel."""
        self._check(lib().lcmc_set_kernel(self._h, kernel))

    def energy_check(self):
        """EnergyCheck (MCnptColloid.c:1343-1362) now: FP64 recompute of every
        replica, drift recorded, running energy reset; raises LcmcError
        (EDRIFT) when a replica's drift is beyond its tolerance."""
        self._check(lib().lcmc_energy_check(self._h))

    def clear_error_flags(self):
        """Clear the sticky error flags (after handling an error)."""
        self._check(lib().lcmc_clear_error_flags(self._h))

    def record_moves(self, on=True):
        """Record every attempt's dE and ln u (per particle id) from now on."""
        self._check(lib().lcmc_record_moves(self._h, int(bool(on))))

    def move_records(self, replica=0):
        """(dE, ln u) of the last sweep's attempts, by particle id."""
        n = self.params[replica].num_particles
        dE, lu = np.zeros(n), np.zeros(n)
        self._check(lib().lcmc_get_move_records(self._h, replica, dE.ctypes.data_as(_lib.DP),
                                                lu.ctypes.data_as(_lib.DP), n))
        return dE, lu

    def stats(self, replica=0):
        s = Stats()
        self._check(lib().lcmc_get_stats(self._h, replica, C.byref(s)))
        d = {k: getattr(s, k) for k, _ in Stats._fields_}
        d["box"] = list(s.box)
        return d

    def autotune(self, sweeps=3, cache=None):
        """Time every candidate kernel configuration over `sweeps` sweeps and
        keep the fastest (lcmc_autotune); the chain continues as if it had not
        run.  `cache`: file of earlier choices, read and appended."""
        t = _lib.Tuning()
        self._check(lib().lcmc_autotune(self._h, int(sweeps), str(cache).encode() if cache else None, C.byref(t)))
        return {"capacity": t.capacity, "volume_by_cell": bool(t.volume_by_cell), "ms_per_sweep": t.ms_per_sweep,
                "from_cache": bool(t.from_cache), "trials": t.trials}

    def tot_ene(self, replica=0):
        """tot_ene (MCnptColloid.c:1598-1622): FP64 recompute of the total energy."""
        e = C.c_double()
        self._check(lib().lcmc_total_energy(self._h, replica, 0, C.byref(e)))
        return e.value

    def compute_liquid_crystal_order_parameters(self, replica=0):
        """Q tensor (xx, xy, xz, yy, yz, zz), P2 and director (MCnptColloid.c:2117-2218)."""
        Q = np.zeros(6)
        P2 = C.c_double()
        d = np.zeros(3)
        self._check(lib().lcmc_order_parameter(self._h, replica, Q.ctypes.data_as(_lib.DP), C.byref(P2),
                                               d.ctypes.data_as(_lib.DP)))
        return Q, P2.value, d

    # -- NPT volume moves: learned screen, recordings --
    def set_surrogate(self, surrogate):
        """Delayed-acceptance volume moves with a trained da.Surrogate (None: plain)."""
        if surrogate is None:
            self._check(lib().lcmc_set_surrogate(self._h, None, 1.0))
            self._surrogate = None
        else:
            self._check(lib().lcmc_set_surrogate(self._h, surrogate.handle, surrogate.scale))
            self._surrogate = surrogate  # keep it alive while set

    def set_fp32_screen(self, on=True):
        """Delayed-acceptance volume moves screened by the FP32-pair energy
        change (NPT replicas on the FP32 kernel); clears a surrogate."""
        self._check(lib().lcmc_set_fp32_screen(self._h, int(bool(on))))
        self._surrogate = None

    def record_volume_samples(self, capacity):
        """Record (features, exact dU / (N delta)) of the next `capacity` exactly
        evaluated volume moves (0 stops and frees)."""
        self._check(lib().lcmc_record_volume_samples(self._h, capacity))
        self.samples_capacity = capacity

    def get_volume_samples(self):
        """Recorded samples: features (n, 4097) float32 and dU / (N delta) (n,)."""
        cap = getattr(self, "samples_capacity", 0)
        x = np.zeros((max(cap, 1), _lib.N_FEATURES), dtype=np.float32)
        y = np.zeros(max(cap, 1), dtype=np.float32)
        n = lib().lcmc_get_volume_samples(self._h, x.ctypes.data_as(_lib.FP), y.ctypes.data_as(_lib.FP), cap)
        if n < 0:
            self._check(n)
        return x[:n], y[:n].astype(np.float64)

    def record_history(self, capacity):
        """Keep a per-sweep row (sweep, Q sums, energy, volume) of the last
        `capacity` sweeps of every replica (0 stops and frees)."""
        self._check(lib().lcmc_record_history(self._h, capacity))
        self.history_capacity = capacity

    def get_history(self, replica=0):
        """Recorded rows in sweep order, shape (n, 9)."""
        cap = getattr(self, "history_capacity", 0)
        rows = np.zeros((max(cap, 1), 9))
        n = lib().lcmc_get_history(self._h, replica, rows.ctypes.data_as(_lib.DP), cap)
        if n < 0:
            self._check(n)
        return rows[:n]

    # -- files (the reference's formats) --
    def esc_fort1(self, path="fortSphere.1", replica=0):
        """Write fortSphere.1 as esc_fort1 (MCnptColloid.c:3193-3212) does."""
        (a, box) = self.download(replica)
        self._check(lib().lcmc_write_fort1(str(path).encode(), len(a[0]), *[x.ctypes.data_as(_lib.DP) for x in a],
                                           box.ctypes.data_as(_lib.DP), float(self.params[replica].colloid_radius)))

    def print_Trayectoria(self, path="Configuraciones.dat", append=True, replica=0):
        """Append (or start) a snapshot as print_Trayectoria (3081-3107) does."""
        (a, box) = self.download(replica)
        self._check(lib().lcmc_write_trajectory(str(path).encode(), int(append), len(a[0]),
                                                *[x.ctypes.data_as(_lib.DP) for x in a], box.ctypes.data_as(_lib.DP)))

    def print_Qmga(self, path="qmga_mcnvtGB.cnf", append=False, replica=0):
        """Write a QMGA snapshot as print_Qmga (3110-3158) does."""
        (a, box) = self.download(replica)
        self._check(lib().lcmc_write_qmga(str(path).encode(), int(append), len(a[0]),
                                          *[x.ctypes.data_as(_lib.DP) for x in a], box.ctypes.data_as(_lib.DP)))

    def save_restart(self, path="fortSphere.1", replica=0):
        """fortSphere.1 plus the exact sidecar (path + '.lcmc')."""
        self._check(lib().lcmc_save_restart(self._h, replica, str(path).encode()))

    def load_restart(self, path="fortSphere.1", replica=0):
        """Resume from save_restart's files (exactly, with the sidecar), or
        start from a plain fortSphere.1 (read_initial_configuration)."""
        self._check(lib().lcmc_load_restart(self._h, replica, str(path).encode()))

    # -- measurement --
    def stream_handle(self):
        """cudaStream_t of this context (as an integer) for event timing."""
        s = C.c_void_p()
        self._check(lib().lcmc_get_stream(self._h, C.byref(s)))
        return s.value or 0

    def kernels_per_sweep(self):
        return lib().lcmc_kernels_per_sweep(self._h)

    def last_sweep_timing(self):
        """Device ms of the last sweep by part: (rebin, colour phases, volume move, finalize)."""
        ms = np.zeros(4)
        self._check(lib().lcmc_last_sweep_timing(self._h, ms.ctypes.data_as(_lib.DP)))
        return ms

    def outcomes(self, replica=0):
        """Per particle id, outcome of the last sweep: 0 reject, 1 accept, 2 hard-core reject."""
        n = self.params[replica].num_particles
        out = np.zeros(n, dtype=np.uint8)
        self._check(lib().lcmc_last_outcomes(self._h, replica, out.ctypes.data_as(C.POINTER(C.c_ubyte)), n))
        return out


def run(params, n_sweeps, stats_interval=10, callback=None):
    """Mirror of the reference's cycle loop (MCnptColloid.c:887-1061) at sweep
    granularity: sweeps, running averages of E/N, rho and P2 every
    `stats_interval` sweeps (update_running_averages, 2225-2260)."""
    sums = {"E": 0.0, "rho": 0.0, "P2": 0.0, "n": 0}
    with GBSystem(params) as s:
        s.get_initial_config()
        done = 0
        while done < n_sweeps:
            k = min(stats_interval, n_sweeps - done)
            s.sweep(k)
            done += k
            st = s.stats()
            _, P2, _ = s.compute_liquid_crystal_order_parameters()
            V = st["box"][0] * st["box"][1] * st["box"][2]
            rec = {"sweep": done, "E_per_N": st["energy"] / params.num_particles,
                   "rho": params.num_particles / V, "P2": P2,
                   "acceptance": st["accepted"] / max(st["attempted"], 1)}
            sums["E"] += rec["E_per_N"]
            sums["rho"] += rec["rho"]
            sums["P2"] += rec["P2"]
            sums["n"] += 1
            if callback:
                callback(rec)
        n = max(sums["n"], 1)
        return {"E_per_N": sums["E"] / n, "rho": sums["rho"] / n, "P2": sums["P2"] / n, "stats": s.stats()}


def run_simulation(params, out_dir=".", adaptive=False, histogram=True, log=None):
    """The reference's main cycle loop (MCnptColloid.c:887-1061) over this
    library, at sweep granularity: one sweep is num_particles attempts, where a
    reference cycle is a single attempt, so intervals given in cycles become
    ceil(interval / N) sweeps, and the run lasts total_mc_sweeps sweeps (or
    ceil(total_mc_cycles / N) when that key is 0).

    * start: initial_configuration_type 0 reads out_dir/fortSphere.1
      (read_initial_configuration; exactly, when its .lcmc sidecar is there),
      2 the lattice; 1 (random placement) is not provided;
    * every configuration_save_interval: a status line to `log`
      (print_intermedio), a snapshot appended to Configuraciones.dat
      (print_Trayectoria) and fortSphere.1 rewritten (backup_restart_file, with
      the exact sidecar);
    * every statistics_print_interval: P2 and the running averages of E/N, rho
      and P2 (compute_liquid_crystal_order_parameters, update_running_averages);
    * `adaptive`: the step-size controller (the reference always runs it; here
      it is for equilibration and off by default);
    * at the end: qmga_mcnvtGB.cnf (print_Qmga), Histograma_Movimientos.dat
      (accepted moves per particle id) and fortSphere.1 (esc_fort1).

    `params`: lcmc_params or the path of a parametersFile.txt.  Returns the
    averages and the final statistics."""
    import math
    import os
    if not isinstance(params, Params):
        params = load_initial_conditions(params)
    n = params.num_particles
    sweeps = params.total_mc_sweeps if params.total_mc_sweeps > 0 else math.ceil(params.total_mc_cycles / n)
    save_every = max(1, math.ceil(params.configuration_save_interval / n))
    stats_every = max(1, math.ceil(params.statistics_print_interval / n))
    os.makedirs(out_dir, exist_ok=True)
    path = lambda name: os.path.join(out_dir, name)  # noqa: E731
    avg = {"E": 0.0, "rho": 0.0, "P2": 0.0, "n": 0}
    hist = np.zeros(n, dtype=np.int64)
    with GBSystem(params) as s:
        if params.initial_configuration_type == 0:
            s.load_restart(path("fortSphere.1"))
        elif params.initial_configuration_type == 2:
            s.get_initial_config()
        else:
            raise LcmcError(_lib.EPARAM, "initial_configuration_type 1 (random placement) is not provided")
        if adaptive:
            s.set_adaptive_step(True)
        first = True
        P2 = 0.0
        for sweep in range(1, sweeps + 1):
            s.sweep(1)
            if histogram:
                hist += s.outcomes() == 1
            if sweep % stats_every == 0:
                st = s.stats()
                _, P2, _ = s.compute_liquid_crystal_order_parameters()
                V = st["box"][0] * st["box"][1] * st["box"][2]
                avg["E"] += st["energy"] / n
                avg["rho"] += n / V
                avg["P2"] += P2
                avg["n"] += 1
            if sweep % save_every == 0:
                st = s.stats()
                if log:
                    k = max(avg["n"], 1)
                    log(f"sweep {sweep}: E/N {st['energy'] / n:.6f} <E/N> {avg['E'] / k:.6f} P2 {P2:.4f} "
                        f"<P2> {avg['P2'] / k:.4f} <rho> {avg['rho'] / k:.5f} "
                        f"acceptance {st['accepted'] / max(st['attempted'], 1):.4f}")
                s.print_Trayectoria(path("Configuraciones.dat"), append=not first)
                first = False
                s.save_restart(path("fortSphere.1"))
        s.print_Qmga(path("qmga_mcnvtGB.cnf"))
        if histogram:
            with open(path("Histograma_Movimientos.dat"), "w") as f:
                for i, h in enumerate(hist):
                    f.write(f"{i}       {h}\n")
        s.save_restart(path("fortSphere.1"))
        k = max(avg["n"], 1)
        return {"sweeps": sweeps, "E_per_N": avg["E"] / k, "rho": avg["rho"] / k, "P2": avg["P2"] / k,
                "stats": s.stats()}
