"""ctypes bindings for the CPU oracle (oracle/lcmc_oracle.c).

Test infrastructure: the oracle is the checker for the CUDA library; nothing in
the product imports this module.  The oracle library is built on first use
(``make -C oracle``) if it is missing.
"""
import ctypes as C
import os
import subprocess

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(REPO, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "_build", "liblcmc_oracle.so")

D = C.c_double
DP = C.POINTER(C.c_double)
IP = C.POINTER(C.c_int)
U32P = C.POINTER(C.c_uint32)

ARITH_REFERENCE = 0
ARITH_CANONICAL = 1


class Params(C.Structure):
    _fields_ = [
        ("mc_ensemble_type", C.c_int), ("num_particles", C.c_int), ("system_density", D),
        ("system_temperature", D), ("system_pressure", D), ("gb_sigma_sidetoside", D), ("gb_epsilon0", D),
        ("gb_kappa", D), ("gb_kappa_prime", D), ("gb_mu_exponent", D), ("gb_nu_exponent", D),
        ("max_displacement", C.c_float), ("max_rotation", C.c_float), ("initial_configuration_type", C.c_int),
        ("cutoff_radius", D), ("verlet_radius", D), ("total_mc_cycles", C.c_int),
        ("configuration_save_interval", C.c_int), ("statistics_print_interval", C.c_int),
        ("colloid_wall_option", C.c_int), ("colloid_interaction_epsilon", D), ("colloid_interaction_amplitude", D),
        ("colloid_radius", D), ("rng_seed", C.c_uint64), ("total_mc_sweeps", C.c_int), ("cell_capacity", C.c_int),
        ("npt_max_dlnV", D), ("volume_moves_per_sweep", C.c_int), ("precision_mode", C.c_int),
        ("init_orientation_cone_deg", D), ("n_read", C.c_int), ("missing_mask", C.c_int),
    ]


class Consts(C.Structure):
    _fields_ = [(n, D) for n in ("beta", "four_eps0", "rc", "rc2", "sigma0", "sigma_ee", "kappa_sq", "chi",
                                 "chi_sq", "chi_prime", "k_imu", "mu", "nu", "kappa_prime", "coll_R",
                                 "coll_cutoff")] + [("coll_on", C.c_int), ("max_disp", D), ("max_rot", D),
                                                     ("wmin", D), ("arith", C.c_int)]


class SweepStats(C.Structure):
    _fields_ = [("attempted", C.c_long), ("accepted", C.c_long), ("hardcore_rejected", C.c_long), ("dE_sum", D)]


class VolumeInfo(C.Structure):
    _fields_ = [("delta", D), ("lam", D), ("U_old", D), ("U_new", D), ("dV", D), ("lnA", D), ("accepted", C.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            subprocess.check_call(["make", "-s", "-C", ORACLE_DIR])
        L = C.CDLL(ORACLE_SO)
        L.lco_params_defaults.argtypes = [C.POINTER(Params)]
        L.lco_params_load.argtypes = [C.c_char_p, C.POINTER(Params)]
        L.lco_consts_from_params.argtypes = [C.POINTER(Params), C.c_int, C.POINTER(Consts)]
        L.lco_pij_gb.restype = D
        L.lco_pij_gb.argtypes = [C.POINTER(Consts), DP, DP, D, D, D, D, D, DP]
        L.lco_pair.restype = D
        L.lco_pair.argtypes = [C.POINTER(Consts), DP, DP, DP, DP, DP, IP]
        L.lco_colloid_rod.restype = D
        L.lco_colloid_rod.argtypes = [C.POINTER(Consts), DP, DP, DP]
        L.lco_tot_ene.restype = D
        L.lco_tot_ene.argtypes = [C.POINTER(Consts), C.c_int, DP, DP, DP, DP, DP, DP, DP]
        L.lco_total_energy_cells.restype = D
        L.lco_total_energy_cells.argtypes = [C.POINTER(Consts), C.c_int, DP, DP, DP, DP, DP, DP, DP]
        L.lco_move_refsem.argtypes = [C.POINTER(Consts), C.c_int, DP, DP, DP, DP, DP, DP, DP, IP, IP,
                                      C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float), IP,
                                      C.c_int, IP, DP, C.POINTER(C.c_long), DP, C.c_int]
        L.lco_ref_table_index.argtypes = [C.c_int]
        L.lco_ref_table_index.restype = C.c_int
        L.lco_philox.argtypes = [U32P, U32P, U32P]
        L.lco_u01.restype = D
        L.lco_u01.argtypes = [C.c_uint32]
        L.lco_log.restype = D
        L.lco_log.argtypes = [D]
        L.lco_expm1.restype = D
        L.lco_expm1.argtypes = [D]
        L.lco_key.argtypes = [C.c_uint64, C.c_int, U32P]
        L.lco_sphere_point.argtypes = [U32P, C.c_uint32, C.c_uint64, DP]
        L.lco_init_lattice.argtypes = [C.POINTER(Params), C.c_int, DP, DP, DP, DP, DP, DP, DP]
        L.lco_grid_dims.argtypes = [D, D, IP]
        L.lco_sweep_shift.argtypes = [U32P, C.c_uint64, IP, DP, DP]
        L.lco_colour_order.argtypes = [U32P, C.c_uint64, IP]
        L.lco_sweep.argtypes = [C.POINTER(Consts), U32P, C.c_uint64, C.c_int, DP, DP, DP, DP, DP, DP, DP,
                                C.POINTER(SweepStats), C.POINTER(C.c_ubyte), IP]
        L.lco_sweep_grid.argtypes = [C.POINTER(Consts), U32P, C.c_uint64, C.c_int, C.c_int, DP, DP, DP, DP, DP, DP, DP,
                                C.POINTER(SweepStats), C.POINTER(C.c_ubyte), IP]
        L.lco_volume_move.argtypes = [C.POINTER(Consts), U32P, C.c_uint64, D, D, C.c_int, DP, DP, DP, DP, DP, DP,
                                      DP, C.POINTER(VolumeInfo)]
        L.lco_order_parameter.argtypes = [C.c_int, DP, DP, DP, DP, DP, DP]
        _lib = L
    return _lib


def ptr(a, t=D):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(t))


def params(**kw):
    p = Params()
    lib().lco_params_defaults(C.byref(p))
    base = dict(mc_ensemble_type=1, num_particles=1000, system_density=0.30, system_temperature=1.0,
                system_pressure=2.0, gb_sigma_sidetoside=1.0, gb_epsilon0=1.0, gb_kappa=3.0, gb_kappa_prime=5.0,
                gb_mu_exponent=2.0, gb_nu_exponent=1.0, max_displacement=0.1, max_rotation=0.1,
                initial_configuration_type=2, cutoff_radius=4.0, verlet_radius=4.8, total_mc_cycles=1000,
                configuration_save_interval=100, statistics_print_interval=100, colloid_wall_option=0,
                colloid_interaction_epsilon=15.0, colloid_interaction_amplitude=1.5, colloid_radius=0.0,
                rng_seed=12345, init_orientation_cone_deg=180.0)
    base.update(kw)
    for k, v in base.items():
        setattr(p, k, v)
    return p


def consts(p, arith=ARITH_CANONICAL):
    c = Consts()
    lib().lco_consts_from_params(C.byref(p), arith, C.byref(c))
    return c


def key(seed, replica=0):
    k = (C.c_uint32 * 2)()
    lib().lco_key(seed, replica, k)
    return k


def philox(ctr, k):
    c = (C.c_uint32 * 4)(*ctr)
    kk = (C.c_uint32 * 2)(*k)
    o = (C.c_uint32 * 4)()
    lib().lco_philox(c, kk, o)
    return list(o)


def init_lattice(n=1000, rho=0.30, R=0.0, seed=12345, cone=180.0, replica=0, **kw):
    p = params(num_particles=n, system_density=rho, colloid_radius=R, rng_seed=seed, init_orientation_cone_deg=cone,
               **kw)
    a = [np.zeros(n) for _ in range(6)]
    box = np.zeros(3)
    rc = lib().lco_init_lattice(C.byref(p), replica, *[ptr(x) for x in a], ptr(box))
    if rc != 0:
        raise RuntimeError("lattice init failed")
    return (*a, box)


def sweep(c, k, sweep_index, state, box, record=False, fine=False):
    """One canonical checkerboard sweep on `state` (list of 6 arrays, updated in
    place); fine: on the fine cell grid (cell_grid 1)."""
    n = len(state[0])
    st = SweepStats()
    bits = np.zeros(n, dtype=np.uint8) if record else None
    order = np.zeros(n, dtype=np.int32) if record else None
    lib().lco_sweep_grid(C.byref(c), k, sweep_index, int(fine), n, *[ptr(x) for x in state], ptr(box), C.byref(st),
                         ptr(bits, C.c_ubyte) if record else None, ptr(order, C.c_int) if record else None)
    return st, bits, order


_omp = None


def omp_lib():
    """The OpenMP build of the oracle (lco_sweep_parallel's threads)."""
    global _omp
    if _omp is None:
        so = os.path.join(ORACLE_DIR, "_build", "liblcmc_oracle_omp.so")
        if not os.path.exists(so):
            subprocess.check_call(["make", "-s", "-C", ORACLE_DIR])
        L = C.CDLL(so)
        L.lco_consts_from_params.argtypes = [C.POINTER(Params), C.c_int, C.POINTER(Consts)]
        L.lco_key.argtypes = [C.c_uint64, C.c_int, U32P]
        L.lco_sweep_parallel.argtypes = [C.POINTER(Consts), U32P, C.c_uint64, C.c_int, DP, DP, DP, DP, DP, DP, DP,
                                         C.POINTER(SweepStats)]
        _omp = L
    return _omp


def sweep_parallel(c, k, sweep_index, state, box):
    """lco_sweep_parallel (OpenMP over each colour's cells) on `state`, in place."""
    st = SweepStats()
    omp_lib().lco_sweep_parallel(C.byref(c), k, sweep_index, len(state[0]), *[ptr(x) for x in state], ptr(box),
                                 C.byref(st))
    return st


def total_energy(c, state, box, allpairs=False):
    n = len(state[0])
    f = lib().lco_tot_ene if allpairs else lib().lco_total_energy_cells
    return f(C.byref(c), n, *[ptr(x) for x in state], ptr(box))


def volume_move(c, k, sweep_index, pressure, dlnv, state, box):
    info = VolumeInfo()
    n = len(state[0])
    r = lib().lco_volume_move(C.byref(c), k, sweep_index, pressure, dlnv, n, *[ptr(x) for x in state], ptr(box),
                              C.byref(info))
    return r, info


def order_parameter(ox, oy, oz):
    Q = np.zeros(6)
    P2 = C.c_double()
    d = np.zeros(3)
    lib().lco_order_parameter(len(ox), ptr(ox), ptr(oy), ptr(oz), ptr(Q), C.byref(P2), ptr(d))
    return Q, P2.value, d
