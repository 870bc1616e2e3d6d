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
