"""Pin the CPU oracle against the reference's own functions.

The golden vectors in tests/golden/ were produced by running the reference's
functions (MCnptColloid.c, built by oracle/build_ref.sh) on seeded inputs; see
tests/golden/make_golden.py.  In reference arithmetic the oracle must agree bit
for bit; in canonical arithmetic (the one the GPU FP64 kernel reproduces) it may
differ by an ulp where glibc's pow(x, 2.0) differs from x*x.
"""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

import oracle_ctypes as oc


def bits(a):
    return np.asarray(a, dtype=np.float64).view(np.uint64)


def consts_for(kap, kp, mu, nu, arith, **kw):
    p = oc.params(gb_kappa=kap, gb_kappa_prime=kp, gb_mu_exponent=mu, gb_nu_exponent=nu, **kw)
    return oc.consts(p, arith)


def test_params_load_matches_reference(golden):
    g = golden("params_golden.npz")
    text = bytes(g["text"]).decode()
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        f.write(text + "unknown_key 5\n")
        path = f.name
    try:
        p = oc.Params()
        oc.lib().lco_params_defaults(C.byref(p))
        assert oc.lib().lco_params_load(path.encode(), C.byref(p)) == 0
    finally:
        os.unlink(path)
    for k in ["system_density", "system_temperature", "system_pressure", "gb_sigma_sidetoside", "gb_epsilon0",
              "gb_kappa", "gb_kappa_prime", "gb_mu_exponent", "gb_nu_exponent", "cutoff_radius", "verlet_radius",
              "colloid_interaction_epsilon", "colloid_interaction_amplitude", "colloid_radius"]:
        assert getattr(p, k) == float(g[k]), k
    for k in ["mc_ensemble_type", "num_particles", "initial_configuration_type", "total_mc_cycles",
              "configuration_save_interval", "statistics_print_interval", "colloid_wall_option"]:
        assert getattr(p, k) == int(g[k]), k
    for k in ["max_displacement", "max_rotation"]:
        assert np.float32(getattr(p, k)) == g[k], k
    assert p.gb_sigma_sidetoside * p.gb_kappa == float(g["gb_sigma_endtoend"])
    assert p.rng_seed == 777
    assert p.n_read == 23


def test_params_missing_key_is_an_error(golden):
    text = bytes(golden("params_golden.npz")["text"]).decode()
    text = "\n".join(l for l in text.splitlines() if not l.startswith("gb_kappa "))
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        f.write(text)
        path = f.name
    try:
        p = oc.Params()
        oc.lib().lco_params_defaults(C.byref(p))
        assert oc.lib().lco_params_load(path.encode(), C.byref(p)) == -2
        assert p.missing_mask == 1 << 7
    finally:
        os.unlink(path)


def test_constants_match_reference(golden):
    g = golden("consts_golden.npz")
    cols = list(g["cols"])
    for row in g["rows"]:
        r = dict(zip(cols, row))
        c = consts_for(r["kappa"], r["kappa_prime"], r["mu"], r["nu"], oc.ARITH_REFERENCE, system_temperature=0.9)
        assert r["chi_first_call"] == -1.0  # the reference's ordering bug on its first call
        for name, attr in [("chi", "chi"), ("chi_sq", "chi_sq"), ("chi_prime", "chi_prime"), ("k_imu", "k_imu"),
                           ("beta", "beta"), ("four_eps0", "four_eps0"), ("rc2", "rc2"),
                           ("colloid_cutoff", "coll_cutoff")]:
            assert getattr(c, attr) == r[name], name


@pytest.mark.parametrize("si", [0, 1, 2])
def test_pij_gb_bitwise(golden, si):
    g = golden("pair_golden.npz")
    kap, kp, mu, nu = g["sets"][si]
    c_ref = consts_for(kap, kp, mu, nu, oc.ARITH_REFERENCE)
    c_can = consts_for(kap, kp, mu, nu, oc.ARITH_CANONICAL)
    ei, ej, dr, sc, want = (g[f"s{si}_{k}"] for k in ("ei", "ej", "dr", "scal", "pij"))
    got_ref = np.empty(len(want))
    got_can = np.empty(len(want))
    for m in range(len(want)):
        a, b, d = (np.ascontiguousarray(x[m]) for x in (ei, ej, dr))
        args = (oc.ptr(a), oc.ptr(b), *sc[m], oc.ptr(d))
        got_ref[m] = oc.lib().lco_pij_gb(C.byref(c_ref), *args)
        got_can[m] = oc.lib().lco_pij_gb(C.byref(c_can), *args)
    assert np.array_equal(bits(got_ref), bits(want))
    # canonical arithmetic: integer exponents as products, within an ulp or two of the reference
    np.testing.assert_allclose(got_can, want, rtol=4e-16 * 8, atol=0)


@pytest.mark.parametrize("si", [0, 1, 2])
def test_pair_with_minimum_image_bitwise(golden, si):
    g = golden("pair_golden.npz")
    kap, kp, mu, nu = g["sets"][si]
    c = consts_for(kap, kp, mu, nu, oc.ARITH_REFERENCE)
    ri, rj, oi, oj, box, want = (g[f"s{si}_{k}"] for k in ("ri", "rj", "oi", "oj", "box", "posmod"))
    box = np.ascontiguousarray(box)
    got = np.empty(len(want))
    n_in = 0
    for m in range(len(want)):
        a, b, e, f = (np.ascontiguousarray(x[m]) for x in (ri, oi, rj, oj))
        inc = C.c_int()
        got[m] = oc.lib().lco_pair(C.byref(c), oc.ptr(a), oc.ptr(b), oc.ptr(e), oc.ptr(f), oc.ptr(box),
                                   C.byref(inc))
        n_in += inc.value
    assert n_in > len(want) // 4
    assert np.array_equal(bits(got), bits(want))


@pytest.mark.parametrize("si", [0, 1, 2])
@pytest.mark.parametrize("R", [0, 3, 5])
def test_colloid_rod_bitwise(golden, si, R):
    g = golden("colloid_golden.npz")
    kap, kp, mu, nu = g["sets"][si]
    c = consts_for(kap, kp, mu, nu, oc.ARITH_REFERENCE, colloid_radius=float(R), colloid_wall_option=1)
    key = f"s{si}_R{R}"
    ri, ei, want = g[key + "_ri"], g[key + "_ei"], g[key + "_U"]
    box = np.array([30.0, 30.0, 30.0])
    got = np.array([oc.lib().lco_colloid_rod(C.byref(c), oc.ptr(np.ascontiguousarray(ri[m])),
                                             oc.ptr(np.ascontiguousarray(ei[m])), oc.ptr(box))
                    for m in range(len(want))])
    assert np.array_equal(bits(got), bits(want))
    assert np.any(got != 0.0)


@pytest.mark.parametrize("tag", ["plain", "colloid"])
def test_tot_ene_bitwise_and_cells(golden, tag):
    g = golden("totene_golden.npz")
    R, option = float(g[f"{tag}_R"]), int(g[f"{tag}_option"])
    c = consts_for(3.0, 5.0, 2.0, 1.0, oc.ARITH_REFERENCE, colloid_radius=R, colloid_wall_option=option)
    state = [np.ascontiguousarray(g[f"{tag}_{k}"]) for k in ("px", "py", "pz", "ox", "oy", "oz")]
    box = np.ascontiguousarray(g[f"{tag}_box"])
    e_all = oc.total_energy(c, state, box, allpairs=True)
    assert bits(e_all) == bits(g[f"{tag}_E"])
    e_cells = oc.total_energy(c, state, box)
    assert abs(e_cells - e_all) <= 1e-12 * abs(e_all)
    # the lattice start is heavily overlapped (E/N ~ 1e11 and beyond)
    lat = [np.ascontiguousarray(x) for x in oc.init_lattice(n=1000, rho=0.30, R=R, seed=4242)[:6]]
    assert bits(oc.total_energy(c, lat, box, allpairs=True)) == bits(g[f"{tag}_E_lattice"])


@pytest.mark.parametrize("tag", ["plain", "colloid", "ungated"])
def test_move_sequence_replays_bitwise(golden, tag):
    """attempt_monte_carlo_move adds GBCollRod in both energies whatever
    colloid_wall_option says (MCnptColloid.c:2495, 2560); with R = 0 that is a
    point colloid at the box centre.  The replay keeps that (gate = 0)."""
    gate = 0
    g = golden("move_golden.npz")
    pre = tag + "_"
    R, option = float(g[pre + "R"]), int(g[pre + "option"])
    c = consts_for(3.0, 5.0, 2.0, 1.0, oc.ARITH_REFERENCE, colloid_radius=R, colloid_wall_option=option,
                   verlet_radius=4.8)
    st = [np.ascontiguousarray(g[pre + k]).copy() for k in ("px", "py", "pz", "ox", "oy", "oz")]
    box = np.ascontiguousarray(g[pre + "box"])
    n = len(st[0])
    cnt = np.ascontiguousarray(g[pre + "nb_count"]).astype(np.int32)
    lst = np.ascontiguousarray(g[pre + "nb_list"]).astype(np.int32)
    tab = np.zeros((3, 1000000), dtype=np.float32)
    tab[:, g[pre + "tab_idx"]] = g[pre + "tab"].T
    rvx, rvy, rvz = (np.ascontiguousarray(tab[k]) for k in range(3))
    rands = np.ascontiguousarray(g[pre + "rands"]).astype(np.int32)
    pos = C.c_int(0)
    E = C.c_double(float(g[pre + "E"]))
    acc = C.c_long(0)
    tr = C.c_double(0.0)
    outcomes = []
    for _ in range(int(g[pre + "n_moves"])):
        r = oc.lib().lco_move_refsem(C.byref(c), n, *[oc.ptr(x) for x in st], oc.ptr(box), oc.ptr(cnt, C.c_int),
                                     oc.ptr(lst, C.c_int), oc.ptr(rvx, C.c_float), oc.ptr(rvy, C.c_float),
                                     oc.ptr(rvz, C.c_float), oc.ptr(rands, C.c_int), len(rands), C.byref(pos),
                                     C.byref(E), C.byref(acc), C.byref(tr), gate)
        assert r >= 0
        outcomes.append(r)
    assert pos.value == len(rands)  # consumed exactly the reference's rand() values
    for k, arr in zip(("px", "py", "pz", "ox", "oy", "oz"), st):
        assert np.array_equal(bits(arr), bits(g[pre + "end_" + k])), k
    assert bits(E.value) == bits(g[pre + "end_E"])
    assert acc.value == int(g[pre + "end_acc"])
    assert bits(tr.value) == bits(g[pre + "end_tracker"])
    assert 0 < acc.value < len(outcomes)


def test_order_parameter_vs_reference(golden):
    """P2 from the reference's float Jacobi agrees with the oracle's double one,
    except where the reference's largest-eigenvalue search (ip = 1 start,
    MCnptColloid.c:1890) returns the wrong eigenvalue."""
    g = golden("order_golden.npz")
    n_ok = n_bug = 0
    for u, (p2_ref, *_dir) in zip(g["u"], g["out"]):
        ox, oy, oz = (np.ascontiguousarray(u[:, k]) for k in range(3))
        Q, p2, d = oc.order_parameter(ox, oy, oz)
        M = np.array([[Q[0], Q[1], Q[2]], [Q[1], Q[3], Q[4]], [Q[2], Q[4], Q[5]]])
        ev = np.linalg.eigvalsh(M)
        assert abs(p2 - 1.5 * ev[-1]) < 1e-12
        assert abs(np.linalg.norm(d) - 1.0) < 1e-12
        assert np.allclose(M @ d, ev[-1] * d, atol=1e-10)
        if abs(p2_ref - p2) < 2e-5:
            n_ok += 1
        else:
            assert np.min(np.abs(1.5 * ev[:2] - p2_ref)) < 2e-5  # one of the other eigenvalues
            n_bug += 1
    assert n_ok > 0
    assert n_ok + n_bug == len(g["u"])
