"""Allocation-free total energy (lcmc_total_energy_noalloc).

For callers that cannot let this library allocate device memory (their own
pool owns the GPU, or their time step cannot take the device-wide
synchronisation of cudaMalloc/cudaFree): the energy of a configuration the
caller holds in device memory, computed with a fixed scratch area inside
liblcmc.so.  Checked here through the C ABI against the CPU oracle's FP64
total energy (canonical arithmetic) and against the allocating entry point
(lcmc_total_energy), within the 1e-12 relative tolerance of the other energy
tests, on two calls in a row, plus the size limit.

This file is collected last on purpose, so that a run stopping at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import oracle_ctypes as oc
import pytest

import parellel_mc_mpi_for_liquidcrystalsystems_b200 as lcmc
from parellel_mc_mpi_for_liquidcrystalsystems_b200 import _lib

pytestmark = pytest.mark.gpu

COMMON = dict(gb_kappa=3.0, gb_kappa_prime=5.0, gb_mu_exponent=2.0, gb_nu_exponent=1.0, cutoff_radius=4.0,
              max_displacement=0.1, max_rotation=0.1)


def _config(n, rho, seed, sweeps, **kw):
    p = lcmc.default_params(num_particles=n, system_density=rho, rng_seed=seed, precision_mode=0, **COMMON, **kw)
    with lcmc.GBSystem(p) as s:
        s.get_initial_config()
        if sweeps:
            s.sweep(sweeps)
        state, box = s.download()
        want = s.tot_ene()
    return p, state, box, want


def _noalloc(torch, p, state, box, out, stream):
    dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in state]
    b = np.ascontiguousarray(box, dtype=np.float64)
    rc = _lib.lib().lcmc_total_energy_noalloc(C.byref(p), len(state[0]), *[C.c_void_p(t.data_ptr()) for t in dev],
                                               b.ctypes.data_as(_lib.DP), C.c_void_p(out.data_ptr()),
                                               C.c_void_p(stream))
    return rc, dev


def test_noalloc_total_energy_matches_allocating_entry_point():
    torch = pytest.importorskip("torch")
    cases = [_config(1000, 0.30, 5, 3),
             _config(20000, 0.30, 6, 2, colloid_radius=4.0, colloid_wall_option=1)]
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    # two calls in a row (the second reuses the scratch the first one left behind)
    for p, state, box, want in cases:
        rc, keep = _noalloc(torch, p, state, box, out, stream)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        got = float(out.item())
        assert abs(got - want) <= 1e-12 * abs(want), (got, want)
        del keep
    # repeating the first case gives the same bits
    p, state, box, want = cases[0]
    rc, _ = _noalloc(torch, p, state, box, out, stream)
    assert rc == 0
    torch.cuda.synchronize()
    first = float(out.item())
    rc, _ = _noalloc(torch, p, state, box, out, stream)
    torch.cuda.synchronize()
    assert float(out.item()) == first


@pytest.mark.parametrize("n,R", [(1000, 0.0), (6000, 3.0)])
def test_noalloc_total_energy_matches_oracle(n, R):
    """The allocation-free energy against the oracle's FP64 cell-list total of
    the same state (tot_ene, MCnptColloid.c:1598-1622, canonical arithmetic)."""
    torch = pytest.importorskip("torch")
    kw = dict(colloid_radius=R, colloid_wall_option=1) if R > 0 else {}
    p, state, box, _ = _config(n, 0.30, 9, 2, **kw)
    op = oc.params(num_particles=n, system_density=0.30, rng_seed=9, **COMMON, **kw)
    want = oc.total_energy(oc.consts(op, oc.ARITH_CANONICAL), [np.ascontiguousarray(a) for a in state],
                           np.ascontiguousarray(box, dtype=np.float64))
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc, _ = _noalloc(torch, p, state, box, out, torch.cuda.current_stream().cuda_stream)
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    got = float(out.item())
    assert abs(got - want) <= 1e-12 * abs(want), (got, want)


def test_noalloc_rejects_sizes_beyond_its_limit():
    torch = pytest.importorskip("torch")
    n = lcmc_max = 65536 + 1
    p = lcmc.default_params(num_particles=n, system_density=0.3, **COMMON)
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    box = np.array([60.0, 60.0, 60.0])
    rc = _lib.lib().lcmc_total_energy_noalloc(C.byref(p), lcmc_max, *[C.c_void_p(dummy.data_ptr())] * 6,
                                               box.ctypes.data_as(_lib.DP), C.c_void_p(dummy.data_ptr()), None)
    assert rc == _lib.EINVAL
    assert "limit" in _lib.last_error()


def _call_with_box(torch, n, box):
    p = lcmc.default_params(num_particles=max(n, 1), system_density=0.3, **COMMON)
    dummy = torch.zeros(16, dtype=torch.float64, device="cuda")
    b = np.ascontiguousarray(box, dtype=np.float64)
    return _lib.lib().lcmc_total_energy_noalloc(C.byref(p), n, *[C.c_void_p(dummy.data_ptr())] * 6,
                                                 b.ctypes.data_as(_lib.DP), C.c_void_p(dummy.data_ptr()), None)


def test_noalloc_rejects_cell_grids_beyond_its_limit_before_launching():
    """Every size check runs on the host before the first launch, so these
    calls return an error and enqueue nothing (the dummy device arrays are
    never read)."""
    torch = pytest.importorskip("torch")
    # 33 x 33 x 33 cells = 35,937 > 32,768
    assert _call_with_box(torch, 10, [33 * 4.0 + 1.0] * 3) == _lib.EINVAL
    assert "limit" in _lib.last_error()
    # 1300^3 cells: the product overflows a 32-bit int (2.197e9 wraps negative)
    assert _call_with_box(torch, 10, [5200.0] * 3) == _lib.EINVAL
    # one axis alone past the limit
    assert _call_with_box(torch, 10, [4.0 * 40000, 8.0, 8.0]) == _lib.EINVAL
    # non-finite edges
    assert _call_with_box(torch, 10, [np.inf, 20.0, 20.0]) == _lib.EINVAL
    assert _call_with_box(torch, 10, [np.nan, 20.0, 20.0]) == _lib.EINVAL
    # shorter than twice the cutoff
    assert _call_with_box(torch, 10, [7.9, 20.0, 20.0]) == _lib.EBOX
    torch.cuda.synchronize()


def test_noalloc_empty_configuration_has_zero_energy():
    torch = pytest.importorskip("torch")
    p = lcmc.default_params(num_particles=1, system_density=0.3, **COMMON)
    out = torch.full((1,), 123.0, dtype=torch.float64, device="cuda")
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    box = np.array([20.0, 20.0, 20.0])
    for _ in range(2):
        rc = _lib.lib().lcmc_total_energy_noalloc(C.byref(p), 0, *[C.c_void_p(dummy.data_ptr())] * 6,
                                                   box.ctypes.data_as(_lib.DP), C.c_void_p(out.data_ptr()), None)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        assert float(out.item()) == 0.0
