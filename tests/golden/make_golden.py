#!/usr/bin/env python3
"""Generate golden vectors from the reference's OWN functions.

Runs in a container where the reference source is available: it loads
oracle/_ref/libmcref_serial.so (built from MCnptColloid.c by
oracle/build_ref.sh, -O2 -ffp-contract=off, no OpenMP) through ctypes, calls the
reference's functions on seeded inputs and stores inputs and outputs as
``*.npz`` beside this script.  The committed fixtures are what the CPU tests
check the oracle against; nothing at test time needs the reference itself.

Fixtures:
  params_golden.npz  load_initial_conditions on a parameter file written here
  consts_golden.npz  get_system_const (first call shows the chi ordering bug)
  pair_golden.npz    pij_GB on direct inputs; GBij_PosMod on 2-particle systems
  colloid_golden.npz GBCollRod
  totene_golden.npz  tot_ene on a seeded lattice (N=1000, rho=0.30)
  move_golden.npz    a sequence of attempt_monte_carlo_move calls with the libc
                     rand() values they consumed
  order_golden.npz   compute_liquid_crystal_order_parameters
"""
import ctypes as C
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF_SO = os.path.join(REPO, "oracle", "_ref", "libmcref_serial.so")
ORACLE_SO = os.path.join(REPO, "oracle", "_build", "liblcmc_oracle.so")

D = C.c_double
DP = C.POINTER(C.c_double)
IP = C.POINTER(C.c_int)

PARAM_TEXT = """# parameter file written by tests/golden/make_golden.py
mc_ensemble_type 1          # NVT
num_particles 216
system_density 0.30
system_temperature 1.0
system_pressure 2.0
gb_sigma_sidetoside 1.0
gb_epsilon0 1.0
gb_kappa 3.0
gb_kappa_prime 5.0
gb_mu_exponent 2.0
gb_nu_exponent 1.0
max_displacement 0.1
max_rotation 0.1
initial_configuration_type 2
cutoff_radius 4.0
verlet_radius 4.8
total_mc_cycles 1000
configuration_save_interval 100
statistics_print_interval 100
colloid_wall_option 1
colloid_interaction_epsilon 15
colloid_interaction_amplitude 1.5
colloid_radius 1.5
rng_seed 777
"""


def arr(a, t=D):
    return np.ascontiguousarray(a).ctypes.data_as(C.POINTER(t))


def load():
    ref = C.CDLL(REF_SO)
    ref.pij_GB.restype = D
    ref.pij_GB.argtypes = [DP, DP, D, D, D, D, D, DP]
    ref.GBCollRod.restype = D
    ref.GBCollRod.argtypes = [C.c_int, DP, DP, DP]
    ref.GBij_PosMod.restype = D
    ref.GBij_PosMod.argtypes = [C.c_int, DP, DP, DP, DP, DP, DP, DP, DP]
    ref.tot_ene.restype = D
    ref.tot_ene.argtypes = [DP] * 6
    ref.refdrv_set_box.argtypes = [C.c_int, DP]
    ref.load_initial_conditions.argtypes = [C.c_char_p]
    ref.attempt_monte_carlo_move.argtypes = [DP, DP, DP, DP, DP, DP, C.c_float, DP, IP, IP,
                                             C.POINTER(C.c_long), DP, C.POINTER(C.c_size_t)]
    ref.build_neighbor_lists.argtypes = [C.c_int, DP, DP, DP, DP, DP, DP, IP, IP]
    ref.refdrv_table_index.argtypes = [C.c_int]
    ref.refdrv_table_index.restype = C.c_int
    ref.compute_liquid_crystal_order_parameters.argtypes = [C.c_int, DP, DP, DP, C.POINTER(C.c_float),
                                                            C.POINTER(C.c_float), C.POINTER(C.c_float),
                                                            C.POINTER(C.c_float)]
    return ref


def g(ref, name, t=D):
    return t.in_dll(ref, name)


def set_params(ref, kappa, kprime, mu, nu, T=1.0, rc=4.0, R=0.0, option=0, eps0=1.0, sigma0=1.0,
               rv=4.8, maxd=0.1, maxr=0.1):
    g(ref, "gb_kappa").value = kappa
    g(ref, "gb_kappa_prime").value = kprime
    g(ref, "gb_mu_exponent").value = mu
    g(ref, "gb_nu_exponent").value = nu
    g(ref, "system_temperature").value = T
    g(ref, "cutoff_radius").value = rc
    g(ref, "verlet_radius").value = rv
    g(ref, "colloid_radius").value = R
    g(ref, "colloid_wall_option", C.c_int).value = option
    g(ref, "gb_epsilon0").value = eps0
    g(ref, "gb_sigma_sidetoside").value = sigma0
    g(ref, "gb_sigma_endtoend").value = sigma0 * kappa
    g(ref, "max_displacement", C.c_float).value = maxd
    g(ref, "max_rotation", C.c_float).value = maxr


GB_SETS = [  # kappa, kappa', mu, nu
    (3.0, 5.0, 2.0, 1.0),
    (4.4, 20.0, 1.0, 1.0),
    (3.0, 5.0, 1.0, 2.0),
]


def gen_params(ref):
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        f.write(PARAM_TEXT)
        path = f.name
    ref.load_initial_conditions(path.encode())
    os.unlink(path)
    out = {"text": np.frombuffer(PARAM_TEXT.encode(), dtype=np.uint8)}
    for k in ["system_density", "system_temperature", "system_pressure", "gb_sigma_sidetoside", "gb_epsilon0",
              "gb_kappa", "gb_kappa_prime", "gb_mu_exponent", "gb_nu_exponent", "cutoff_radius", "verlet_radius",
              "colloid_interaction_epsilon", "colloid_interaction_amplitude", "colloid_radius",
              "gb_sigma_endtoend"]:
        out[k] = np.float64(g(ref, k).value)
    for k in ["mc_ensemble_type", "num_particles", "initial_configuration_type", "total_mc_cycles",
              "configuration_save_interval", "statistics_print_interval", "colloid_wall_option"]:
        out[k] = np.int64(g(ref, k, C.c_int).value)
    for k in ["max_displacement", "max_rotation"]:
        out[k] = np.float32(g(ref, k, C.c_float).value)
    np.savez(os.path.join(HERE, "params_golden.npz"), **out)


def gen_consts(ref):
    rows = []
    for (kap, kp, mu, nu) in GB_SETS:
        set_params(ref, kap, kp, mu, nu, T=0.9, rc=4.0)
        g(ref, "gb_kappa_sq").value = 0.0  # fresh process state: kappa^2 not yet assigned
        box = np.array([20.0, 20.0, 20.0])
        g(ref, "num_particles", C.c_int).value = 10
        ref.get_system_const()
        first_chi = g(ref, "gb_chi").value
        ref.get_system_const()
        rows.append([kap, kp, mu, nu, first_chi, g(ref, "gb_chi").value, g(ref, "gb_chi_sq").value,
                     g(ref, "gb_chi_prime").value, g(ref, "gb_k_imu").value, g(ref, "gb_beta").value,
                     g(ref, "gb_4eps0").value, g(ref, "cutoff_radius_sq").value, g(ref, "colloid_rod_cutoff").value])
        del box
    np.savez(os.path.join(HERE, "consts_golden.npz"), rows=np.array(rows),
             cols=np.array(["kappa", "kappa_prime", "mu", "nu", "chi_first_call", "chi", "chi_sq", "chi_prime",
                            "k_imu", "beta", "four_eps0", "rc2", "colloid_cutoff"]))


def gen_pair(ref):
    rng = np.random.default_rng(2024)
    out = {}
    for si, (kap, kp, mu, nu) in enumerate(GB_SETS):
        set_params(ref, kap, kp, mu, nu, rc=4.0)
        ref.refdrv_set_box(2, arr(np.array([30.0, 30.0, 30.0])))
        # direct pij_GB inputs
        M = 1200
        ei = rng.normal(size=(M, 3)) * rng.uniform(0.9, 1.1, size=(M, 1))
        ej = rng.normal(size=(M, 3)) * rng.uniform(0.9, 1.1, size=(M, 1))
        ei /= np.linalg.norm(ei, axis=1, keepdims=True)
        ej /= np.linalg.norm(ej, axis=1, keepdims=True)
        ei *= rng.uniform(0.95, 1.05, size=(M, 1))
        dr = rng.normal(size=(M, 3))
        dr /= np.linalg.norm(dr, axis=1, keepdims=True)
        rij = rng.uniform(0.3, 4.2, size=M)
        dr *= rij[:, None]
        irij = 1.0 / rij
        iei = 1.0 / np.linalg.norm(ei, axis=1)
        iej = 1.0 / np.linalg.norm(ej, axis=1)
        eiej = iei * iej * np.einsum("ij,ij->i", ei, ej)
        res = np.empty(M)
        for m in range(M):
            a, b, d = ei[m].copy(), ej[m].copy(), dr[m].copy()
            res[m] = ref.pij_GB(arr(a), arr(b), rij[m], irij[m], iei[m], iej[m], eiej[m], arr(d))
        out[f"s{si}_ei"], out[f"s{si}_ej"], out[f"s{si}_dr"] = ei, ej, dr
        out[f"s{si}_scal"] = np.stack([rij, irij, iei, iej, eiej], axis=1)
        out[f"s{si}_pij"] = res
        # GBij_PosMod on 2-particle systems: full per-pair preamble incl. minimum image
        L = 12.0
        ref.refdrv_set_box(2, arr(np.array([L, L, L])))
        M2 = 800
        ri = rng.uniform(0, L, size=(M2, 3))
        rj = np.mod(ri + rng.normal(size=(M2, 3)) * 2.5, L)
        oi = rng.normal(size=(M2, 3))
        oj = rng.normal(size=(M2, 3))
        oi /= np.linalg.norm(oi, axis=1, keepdims=True)
        oj /= np.linalg.norm(oj, axis=1, keepdims=True)
        res2 = np.empty(M2)
        for m in range(M2):
            px = np.array([ri[m, 0], rj[m, 0]]); py = np.array([ri[m, 1], rj[m, 1]])
            pz = np.array([ri[m, 2], rj[m, 2]])
            ox = np.array([oi[m, 0], oj[m, 0]]); oy = np.array([oi[m, 1], oj[m, 1]])
            oz = np.array([oi[m, 2], oj[m, 2]])
            r0 = ri[m].copy(); e0 = oi[m].copy()
            res2[m] = ref.GBij_PosMod(0, arr(r0), arr(e0), arr(px), arr(py), arr(pz), arr(ox), arr(oy), arr(oz))
        out[f"s{si}_ri"], out[f"s{si}_rj"], out[f"s{si}_oi"], out[f"s{si}_oj"] = ri, rj, oi, oj
        out[f"s{si}_box"] = np.array([L, L, L])
        out[f"s{si}_posmod"] = res2
    out["sets"] = np.array(GB_SETS)
    np.savez(os.path.join(HERE, "pair_golden.npz"), **out)


def gen_colloid(ref):
    rng = np.random.default_rng(99)
    out = {}
    for si, (kap, kp, mu, nu) in enumerate(GB_SETS):
        for R in (0.0, 3.0, 5.0):
            set_params(ref, kap, kp, mu, nu, R=R, option=1)
            L = 30.0
            ref.refdrv_set_box(1, arr(np.array([L, L, L])))
            M = 500
            C0 = np.array([L / 2] * 3)
            dirs = rng.normal(size=(M, 3))
            dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
            dist = rng.uniform(max(R - 0.5, 0.0), R + 14.0, size=M)
            ri = C0 + dirs * dist[:, None]
            ei = rng.normal(size=(M, 3))
            ei /= np.linalg.norm(ei, axis=1, keepdims=True)
            res = np.empty(M)
            cc = C0.copy()
            for m in range(M):
                a, b = ri[m].copy(), ei[m].copy()
                res[m] = ref.GBCollRod(m, arr(a), arr(b), arr(cc))
            key = f"s{si}_R{int(R)}"
            out[key + "_ri"], out[key + "_ei"], out[key + "_U"] = ri, ei, res
    out["sets"] = np.array(GB_SETS)
    np.savez(os.path.join(HERE, "colloid_golden.npz"), **out)


def oracle_lattice(n, rho, R, seed, cone=180.0):
    """Seeded lattice from the oracle (positions and orientations as inputs)."""
    sys.path.insert(0, os.path.join(REPO, "tests"))
    import oracle_ctypes as oc  # noqa: E402
    return oc.init_lattice(n=n, rho=rho, R=R, seed=seed, cone=cone)


def relax(ref, px, py, pz, ox, oy, oz, box, n_att, seed):
    """Relax an overlapped lattice with the reference's own moves (all-pairs list)."""
    n = len(px)
    cnt = np.zeros(n, dtype=np.int32)
    lst = np.zeros(n * n, dtype=np.int32)
    rx, ry, rz = px.copy(), py.copy(), pz.copy()
    g(ref, "verlet_radius").value = 1e9  # every pair in the list: no stale lists during the relaxation
    ref.get_system_const()
    ref.build_neighbor_lists(n * n, arr(px), arr(py), arr(pz), arr(rx), arr(ry), arr(rz), arr(cnt, C.c_int),
                             arr(lst, C.c_int))
    libc = C.CDLL("libc.so.6")
    libc.srand(seed)
    ref.refdrv_fill_rotation_table()
    e = D(ref.tot_ene(arr(px), arr(py), arr(pz), arr(ox), arr(oy), arr(oz)))
    acc = C.c_long(0)
    tr = D(0.0)
    hist = np.zeros(n, dtype=np.uint64)
    for _ in range(n_att):
        ref.attempt_monte_carlo_move(arr(px), arr(py), arr(pz), arr(ox), arr(oy), arr(oz), C.c_float(0.1),
                                     C.byref(e), arr(cnt, C.c_int), arr(lst, C.c_int), C.byref(acc), C.byref(tr),
                                     arr(hist, C.c_size_t))


def gen_totene(ref):
    out = {}
    for tag, R, option in (("plain", 0.0, 0), ("colloid", 3.0, 1)):
        set_params(ref, 3.0, 5.0, 2.0, 1.0, T=1.0, rc=4.0, R=R, option=option)
        px, py, pz, ox, oy, oz, box = oracle_lattice(1000, 0.30, R, 4242)
        ref.refdrv_set_box(1000, arr(box))
        E0 = ref.tot_ene(arr(px), arr(py), arr(pz), arr(ox), arr(oy), arr(oz))
        relax(ref, px, py, pz, ox, oy, oz, box, 20000, 5)
        E1 = ref.tot_ene(arr(px), arr(py), arr(pz), arr(ox), arr(oy), arr(oz))
        for k, v in dict(px=px, py=py, pz=pz, ox=ox, oy=oy, oz=oz, box=box).items():
            out[f"{tag}_{k}"] = v
        out[f"{tag}_E_lattice"] = np.float64(E0)
        out[f"{tag}_E"] = np.float64(E1)
        out[f"{tag}_R"] = np.float64(R)
        out[f"{tag}_option"] = np.int64(option)
    np.savez(os.path.join(HERE, "totene_golden.npz"), **out)


def gen_moves(ref):
    """A run of attempt_monte_carlo_move with every libc rand() value it consumed."""
    out = {}
    libc = C.CDLL("libc.so.6")
    tot = np.load(os.path.join(HERE, "totene_golden.npz"))
    for tag, R, option in (("plain", 0.0, 0), ("colloid", 3.0, 1), ("ungated", 3.0, 2)):
        src = "plain" if tag == "plain" else "colloid"
        set_params(ref, 3.0, 5.0, 2.0, 1.0, T=1.0, rc=4.0, R=R, option=option, rv=4.8)
        px, py, pz = (tot[f"{src}_{k}"].copy() for k in ("px", "py", "pz"))
        ox, oy, oz = (tot[f"{src}_{k}"].copy() for k in ("ox", "oy", "oz"))
        box = tot[f"{src}_box"].copy()
        n = len(px)
        ref.refdrv_set_box(n, arr(box))
        libc.srand(31337)
        ref.refdrv_fill_rotation_table()
        rvx = np.ctypeslib.as_array((C.c_float * 1000000).in_dll(ref, "rot_vec_x"))
        rvy = np.ctypeslib.as_array((C.c_float * 1000000).in_dll(ref, "rot_vec_y"))
        rvz = np.ctypeslib.as_array((C.c_float * 1000000).in_dll(ref, "rot_vec_z"))
        maxn = 400
        cnt = np.zeros(n, dtype=np.int32)
        lst = np.zeros(n * maxn, dtype=np.int32)
        rx, ry, rz = px.copy(), py.copy(), pz.copy()
        ref.build_neighbor_lists(n * maxn, arr(px), arr(py), arr(pz), arr(rx), arr(ry), arr(rz),
                                 arr(cnt, C.c_int), arr(lst, C.c_int))
        E = D(ref.tot_ene(arr(px), arr(py), arr(pz), arr(ox), arr(oy), arr(oz)))
        seed = 4321 + len(tag)
        libc.srand(seed)
        K = 6000
        rands = np.array([libc.rand() for _ in range(K)], dtype=np.int32)
        libc.srand(seed)
        start = dict(px=px.copy(), py=py.copy(), pz=pz.copy(), ox=ox.copy(), oy=oy.copy(), oz=oz.copy(), E=E.value)
        acc = C.c_long(0)
        tr = D(0.0)
        hist = np.zeros(n, dtype=np.uint64)
        n_moves = 800
        for _ in range(n_moves):
            ref.attempt_monte_carlo_move(arr(px), arr(py), arr(pz), arr(ox), arr(oy), arr(oz), C.c_float(0.1),
                                         C.byref(E), arr(cnt, C.c_int), arr(lst, C.c_int), C.byref(acc),
                                         C.byref(tr), arr(hist, C.c_size_t))
        # rand() values actually consumed: count by the state of libc's generator
        probe = libc.rand()
        used = int(np.where(rands == probe)[0][0])
        idx = sorted({ref.refdrv_table_index(int(r)) for r in rands[:used]})
        idx = np.array(idx, dtype=np.int64)
        pre = f"{tag}_"
        out.update({pre + k: v for k, v in start.items()})
        out.update({pre + "box": box, pre + "nb_count": cnt, pre + "nb_list": lst[:cnt[-1]],
                    pre + "rands": rands[:used], pre + "tab_idx": idx,
                    pre + "tab": np.stack([rvx[idx], rvy[idx], rvz[idx]], axis=1).astype(np.float32),
                    pre + "n_moves": np.int64(n_moves), pre + "R": np.float64(R), pre + "option": np.int64(option),
                    pre + "end_px": px, pre + "end_py": py, pre + "end_pz": pz, pre + "end_ox": ox,
                    pre + "end_oy": oy, pre + "end_oz": oz, pre + "end_E": np.float64(E.value),
                    pre + "end_acc": np.int64(acc.value), pre + "end_tracker": np.float64(tr.value),
                    pre + "hist": hist.astype(np.int64)})
    np.savez_compressed(os.path.join(HERE, "move_golden.npz"), **out)


def gen_order(ref):
    rng = np.random.default_rng(7)
    rows = []
    ors = []
    for case in range(40):
        n = 200
        if case % 3 == 0:
            u = rng.normal(size=(n, 3))
        else:
            axis = rng.normal(size=3)
            axis /= np.linalg.norm(axis)
            u = axis[None, :] * rng.uniform(1.0, 4.0) + rng.normal(size=(n, 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        dx, dy, dz, p2 = C.c_float(), C.c_float(), C.c_float(), C.c_float()
        ox, oy, oz = (np.ascontiguousarray(u[:, k]) for k in range(3))
        ref.compute_liquid_crystal_order_parameters(n, arr(ox), arr(oy), arr(oz), C.byref(dx), C.byref(dy),
                                                    C.byref(dz), C.byref(p2))
        rows.append([p2.value, dx.value, dy.value, dz.value])
        ors.append(u)
    np.savez_compressed(os.path.join(HERE, "order_golden.npz"), u=np.array(ors), out=np.array(rows))


def main():
    if not os.path.exists(REF_SO):
        sys.exit("build oracle/_ref first (oracle/build_ref.sh)")
    ref = load()
    gen_params(ref)
    gen_consts(ref)
    gen_pair(ref)
    gen_colloid(ref)
    gen_totene(ref)
    gen_moves(ref)
    gen_order(ref)
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
