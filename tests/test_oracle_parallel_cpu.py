"""The OpenMP checkerboard port (lco_sweep_parallel, the CPU baseline's
implementation) ends each sweep in the state the canonical oracle sweep
reaches, bit for bit: same-colour cells never interact, so sharing them among
threads changes nothing but the order of the dE sum."""
import os

import numpy as np

import oracle_ctypes as oc


def test_parallel_sweeps_equal_the_oracle(monkeypatch):
    monkeypatch.setenv("OMP_NUM_THREADS", "4")
    px, py, pz, ox, oy, oz, box = oc.init_lattice(n=3000, rho=0.30, R=3.0, seed=71)
    p = oc.params(num_particles=3000, system_density=0.30, colloid_radius=3.0, colloid_wall_option=1, rng_seed=71)
    c = oc.consts(p, oc.ARITH_CANONICAL)
    k = oc.key(71)
    a = [np.ascontiguousarray(x.copy()) for x in (px, py, pz, ox, oy, oz)]
    b = [np.ascontiguousarray(x.copy()) for x in (px, py, pz, ox, oy, oz)]
    for s in range(3):
        st_a, _, _ = oc.sweep(c, k, s, a, box)
        st_b = oc.sweep_parallel(c, k, s, b, box)
        assert (st_a.attempted, st_a.accepted, st_a.hardcore_rejected) == (st_b.attempted, st_b.accepted,
                                                                            st_b.hardcore_rejected)
        assert abs(st_a.dE_sum - st_b.dE_sum) <= 1e-9 * max(1.0, abs(st_a.dE_sum))
        for u, v in zip(a, b):
            assert np.array_equal(u.view(np.uint64), v.view(np.uint64))
    assert os.environ["OMP_NUM_THREADS"] == "4"


def test_fine_grid_sweep_schedule():
    """The oracle's fine-grid sweep (lco_sweep_grid, fine = 1): with an even cell
    count it is the even-grid sweep bit for bit (same colours, draws and cell
    order); with an odd count (5 cells per axis, 27 colours) it attempts every
    particle exactly once."""
    import ctypes as C
    # even: 6 cells per axis at N = 6000, rho* = 0.3 (L = 27.1)
    px, py, pz, ox, oy, oz, box = oc.init_lattice(n=6000, rho=0.30, seed=72)
    p = oc.params(num_particles=6000, system_density=0.30, rng_seed=72)
    c = oc.consts(p, oc.ARITH_CANONICAL)
    k = oc.key(72)
    nc = C.c_int()
    oc.lib().lco_grid_dims_fine.argtypes = [C.c_double, C.c_double, C.c_int, C.POINTER(C.c_int)]
    oc.lib().lco_grid_dims_fine(box[0], c.wmin, 1, C.byref(nc))
    assert nc.value % 2 == 0
    a = [np.ascontiguousarray(x.copy()) for x in (px, py, pz, ox, oy, oz)]
    b = [np.ascontiguousarray(x.copy()) for x in (px, py, pz, ox, oy, oz)]
    for s in range(2):
        _, ba, oa = oc.sweep(c, k, s, a, box, record=True)
        _, bb, ob = oc.sweep(c, k, s, b, box, record=True, fine=True)
        assert np.array_equal(oa, ob) and np.array_equal(ba, bb)
    for u, v in zip(a, b):
        assert np.array_equal(u.view(np.uint64), v.view(np.uint64))
    # odd: 5 cells per axis at N = 4096, rho* = 0.32
    px, py, pz, ox, oy, oz, box = oc.init_lattice(n=4096, rho=0.32, seed=73)
    p = oc.params(num_particles=4096, system_density=0.32, rng_seed=73)
    c = oc.consts(p, oc.ARITH_CANONICAL)
    oc.lib().lco_grid_dims_fine(box[0], c.wmin, 1, C.byref(nc))
    assert nc.value == 5
    st = [np.ascontiguousarray(x.copy()) for x in (px, py, pz, ox, oy, oz)]
    s0, _, order = oc.sweep(c, oc.key(73), 0, st, box, record=True, fine=True)
    assert s0.attempted == 4096 and sorted(order.tolist()) == list(range(4096))
