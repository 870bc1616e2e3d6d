"""ctypes binding of liblcmc.so (the C ABI in include/lcmc.h).

The library is loaded from this package directory (built in-tree by
``build.py``).  There is no Python or CPU fallback: if the shared library is
missing, :func:`lib` raises.
"""
import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "liblcmc.so")

OK = 0
EINVAL, ENOFILE, EPARAM, ECUDA, ENOMEM, ECELLCAP, ENUMERIC, EBOX, ENODEV, EOVERLAP, ETIMEOUT, EDRIFT = range(-1, -13, -1)
F_DRIFT = 32
PREC_FP64, PREC_FP32 = 0, 1
NVT, NPT = 1, 2

D = C.c_double
DP = C.POINTER(C.c_double)
FP = C.POINTER(C.c_float)
N_FEATURES = 4097


class Params(C.Structure):
    """lcmc_params: the 23 parametersFile.txt keys plus the added ones."""
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
        ("energy_check_interval", C.c_int), ("energy_check_tolerance", D), ("init_lattice", C.c_int),
        ("cell_grid", C.c_int),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Stats(C.Structure):
    _fields_ = [
        ("sweeps", C.c_int64), ("attempted", C.c_int64), ("accepted", C.c_int64), ("hardcore_rejected", C.c_int64),
        ("volume_attempted", C.c_int64), ("volume_accepted", C.c_int64), ("energy", D), ("box", D * 3),
        ("last_recompute", D), ("drift", D), ("pairs_in_cutoff", C.c_int64), ("stencil_candidates", C.c_int64),
        ("error_flags", C.c_int), ("kernel", C.c_int), ("volume_stage1_rejected", C.c_int64),
        ("fp64_cells", C.c_int64), ("overcap_cells", C.c_int64), ("energy_checks", C.c_int64),
        ("drift_breaches", C.c_int64), ("drift_bound", D), ("abs_dE_since_check", D),
    ]


class LcmcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"lcmc error {code}: {msg}")
        self.code = code


_lib = None

class Tuning(C.Structure):
    """lcmc_tuning."""
    _fields_ = [("capacity", C.c_int), ("volume_by_cell", C.c_int), ("ms_per_sweep", C.c_double),
                ("from_cache", C.c_int), ("trials", C.c_int)]


EXPORTS = {
    "lcmc_params_defaults": ([C.POINTER(Params)], C.c_int),
    "lcmc_params_load": ([C.c_char_p, C.POINTER(Params)], C.c_int),
    "lcmc_create": ([C.POINTER(Params), C.POINTER(C.c_void_p)], C.c_int),
    "lcmc_create_batch": ([C.POINTER(Params), C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "lcmc_destroy": ([C.c_void_p], C.c_int),
    "lcmc_num_replicas": ([C.c_void_p], C.c_int),
    "lcmc_init_config": ([C.c_void_p, C.c_int], C.c_int),
    "lcmc_lattice": ([C.POINTER(Params), C.c_int, DP, DP, DP, DP, DP, DP, DP], C.c_int),
    "lcmc_upload": ([C.c_void_p, C.c_int, DP, DP, DP, DP, DP, DP, C.c_int, DP], C.c_int),
    "lcmc_upload_with_energy": ([C.c_void_p, C.c_int, DP, DP, DP, DP, DP, DP, C.c_int, DP, C.c_double], C.c_int),
    "lcmc_download": ([C.c_void_p, C.c_int, DP, DP, DP, DP, DP, DP, C.c_int, DP], C.c_int),
    "lcmc_sweep": ([C.c_void_p, C.c_int], C.c_int),
    "lcmc_get_stats": ([C.c_void_p, C.c_int, C.POINTER(Stats)], C.c_int),
    "lcmc_total_energy": ([C.c_void_p, C.c_int, C.c_int, DP], C.c_int),
    "lcmc_order_parameter": ([C.c_void_p, C.c_int, DP, DP, DP], C.c_int),
    "lcmc_last_outcomes": ([C.c_void_p, C.c_int, C.POINTER(C.c_ubyte), C.c_int], C.c_int),
    "lcmc_set_kernel": ([C.c_void_p, C.c_int], C.c_int),
    "lcmc_clear_error_flags": ([C.c_void_p], C.c_int),
    "lcmc_energy_check": ([C.c_void_p], C.c_int),
    "lcmc_record_moves": ([C.c_void_p, C.c_int], C.c_int),
    "lcmc_get_move_records": ([C.c_void_p, C.c_int, DP, DP, C.c_int], C.c_int),
    "lcmc_strerror": ([C.c_int], C.c_char_p),
    "lcmc_last_error": ([C.c_void_p, C.c_char_p, C.c_size_t], C.c_int),
    "lcmc_abi_version": ([], C.c_int),
    "lcmc_get_stream": ([C.c_void_p, C.POINTER(C.c_void_p)], C.c_int),
    "lcmc_kernels_per_sweep": ([C.c_void_p], C.c_int),
    "lcmc_last_sweep_timing": ([C.c_void_p, DP], C.c_int),
    "lcmc_pair_terms": ([C.POINTER(Params), C.c_int, DP, DP, DP, DP, DP], C.c_int),
    "lcmc_total_energy_noalloc": ([C.POINTER(Params), C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, DP, C.c_void_p, C.c_void_p], C.c_int),
    "lcmc_mlp_create": ([C.c_int, C.c_int, C.c_int, C.c_uint64, C.POINTER(C.c_void_p)], C.c_int),
    "lcmc_mlp_destroy": ([C.c_void_p], C.c_int),
    "lcmc_mlp_train": ([C.c_void_p, FP, FP, C.c_int, C.c_int, C.c_int, C.c_float, C.c_uint64, FP], C.c_int),
    "lcmc_mlp_predict": ([C.c_void_p, FP, C.c_int, FP], C.c_int),
    "lcmc_mlp_num_params": ([C.c_void_p], C.c_int),
    "lcmc_mlp_gradients": ([C.c_void_p, FP, FP, C.c_int, FP, FP], C.c_int),
    "lcmc_mlp_get_params": ([C.c_void_p, FP], C.c_int),
    "lcmc_mlp_set_params": ([C.c_void_p, FP], C.c_int),
    "lcmc_gemm_bf16": ([FP, FP, FP, C.c_int, C.c_int, C.c_int], C.c_int),
    "lcmc_set_wait_limit": ([C.c_uint], C.c_int),
    "lcmc_set_surrogate": ([C.c_void_p, C.c_void_p, C.c_double], C.c_int),
    "lcmc_set_fp32_screen": ([C.c_void_p, C.c_int], C.c_int),
    "lcmc_get_params": ([C.c_void_p, C.c_int, C.POINTER(Params)], C.c_int),
    "lcmc_set_adaptive_step": ([C.c_void_p, C.c_int], C.c_int),
    "lcmc_get_step": ([C.c_void_p, C.c_int, DP, DP], C.c_int),
    "lcmc_set_sweep_counter": ([C.c_void_p, C.c_int, C.c_int64], C.c_int),
    "lcmc_autotune": ([C.c_void_p, C.c_int, C.c_char_p, C.POINTER(Tuning)], C.c_int),
    "lcmc_cell_capacity": ([C.POINTER(Params), C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
    "lcmc_write_fort1": ([C.c_char_p, C.c_int, DP, DP, DP, DP, DP, DP, DP, C.c_double], C.c_int),
    "lcmc_read_fort1": ([C.c_char_p, C.c_int, DP, DP, DP, DP, DP, DP, DP, DP, C.POINTER(C.c_int)], C.c_int),
    "lcmc_write_trajectory": ([C.c_char_p, C.c_int, C.c_int, DP, DP, DP, DP, DP, DP, DP], C.c_int),
    "lcmc_write_qmga": ([C.c_char_p, C.c_int, C.c_int, DP, DP, DP, DP, DP, DP, DP], C.c_int),
    "lcmc_save_restart": ([C.c_void_p, C.c_int, C.c_char_p], C.c_int),
    "lcmc_load_restart": ([C.c_void_p, C.c_int, C.c_char_p], C.c_int),
    "lcmc_record_volume_samples": ([C.c_void_p, C.c_int], C.c_int),
    "lcmc_get_volume_samples": ([C.c_void_p, FP, FP, C.c_int], C.c_int),
    "lcmc_record_history": ([C.c_void_p, C.c_int], C.c_int),
    "lcmc_get_history": ([C.c_void_p, C.c_int, DP, C.c_int], C.c_int),
}


def lib():
    """Load liblcmc.so from this package (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with "
                              "`python -m parellel_mc_mpi_for_liquidcrystalsystems_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in EXPORTS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def last_error(ctx=None):
    buf = C.create_string_buffer(512)
    lib().lcmc_last_error(ctx, buf, 512)
    return buf.value.decode(errors="replace")


def check(code, ctx=None):
    if code != OK:
        raise LcmcError(code, f"{lib().lcmc_strerror(code).decode()}: {last_error(ctx)}")
    return code
