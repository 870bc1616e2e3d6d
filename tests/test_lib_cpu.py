"""CPU-side checks of the C ABI library (no GPU needed).

* liblcmc.so loads and exports every function declared in include/lcmc.h;
* the host-side parameter parser and lattice initialiser agree with the
  oracle bit for bit;
* without a GPU every device call fails loudly with LCMC_ENODEV (no CPU
  fallback).
"""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import oracle_ctypes as oc
import parellel_mc_mpi_for_liquidcrystalsystems_b200 as lcmc
from parellel_mc_mpi_for_liquidcrystalsystems_b200 import _lib

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def header_functions():
    text = open(os.path.join(REPO, "include", "lcmc.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lcmc_\w+)\s*\(", text)))


def test_library_exports_every_header_symbol():
    lib = _lib.lib()
    names = header_functions()
    assert len(names) >= 18
    for name in names:
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (lcmc_\w+)", out))
    assert set(names) <= exported
    assert lib.lcmc_abi_version() == 2


def test_params_parser_matches_oracle(golden):
    text = bytes(golden("params_golden.npz")["text"]).decode()
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        f.write(text + "precision_mode fp64\nnpt_max_dlnV 0.02\nsomething_else 3\n")
        path = f.name
    try:
        p = lcmc.load_initial_conditions(path)
        q = oc.Params()
        oc.lib().lco_params_defaults(C.byref(q))
        assert oc.lib().lco_params_load(path.encode(), C.byref(q)) == 0
    finally:
        os.unlink(path)
    for name, _ in oc.Params._fields_:
        assert getattr(p, name) == getattr(q, name), name
    assert p.precision_mode == 0 and p.npt_max_dlnV == 0.02


def test_params_missing_key_raises(golden):
    text = bytes(golden("params_golden.npz")["text"]).decode()
    text = "\n".join(l for l in text.splitlines() if not l.startswith("cutoff_radius"))
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        f.write(text)
        path = f.name
    try:
        with pytest.raises(lcmc.LcmcError) as e:
            lcmc.load_initial_conditions(path)
        assert e.value.code == _lib.EPARAM
    finally:
        os.unlink(path)
    with pytest.raises(lcmc.LcmcError):
        lcmc.load_initial_conditions("/nonexistent/parametersFile.txt")


@pytest.mark.parametrize("n,rho,R,cone,seed", [
    (1000, 0.30, 0.0, 180.0, 1), (4096, 0.32, 0.0, 20.0, 2), (3000, 0.30, 5.0, 180.0, 3), (777, 0.05, 2.0, 45.0, 4)])
def test_lattice_matches_oracle_bitwise(n, rho, R, cone, seed):
    p = lcmc.default_params(num_particles=n, system_density=rho, colloid_radius=R, init_orientation_cone_deg=cone,
                            rng_seed=seed)
    a, box = lcmc.lattice(p)
    b = oc.init_lattice(n=n, rho=rho, R=R, cone=cone, seed=seed)
    for x, y in zip(a, b[:6]):
        assert np.array_equal(x, y)
    assert np.array_equal(box, b[6])
    # orientations are unit vectors, positions inside the box, none inside the colloid
    assert np.allclose(a[3] ** 2 + a[4] ** 2 + a[5] ** 2, 1.0, atol=1e-14)
    assert np.all((a[0] >= 0) & (a[0] < box[0]))
    if R > 0:
        d2 = sum((a[k] - box[k] / 2) ** 2 for k in range(3))
        assert np.all(d2 > R * R)
    if cone < 180:
        assert np.all(a[5] >= np.cos(np.radians(cone)) - 1e-12)


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU error path")
def test_no_gpu_is_a_loud_error():
    p = lcmc.default_params(num_particles=1000)
    with pytest.raises(lcmc.LcmcError) as e:
        lcmc.GBSystem(p)
    assert e.value.code == _lib.ENODEV


@pytest.mark.parametrize("kw,lo,cls", [
    # the NVT bench system: ~22.5 rods per 4.13-wide cell of a dense liquid
    (dict(num_particles=1048576, system_density=0.32, init_orientation_cone_deg=20.0), 35, 48),
    # a gas (rho* = 0.1) in 6.5-wide cells: Poisson counts around 27
    (dict(num_particles=1728, system_density=0.1, colloid_wall_option=1, colloid_radius=2.0, max_displacement=0.5),
     50, 56),
    # 4 cells per axis of 4.7, ~32 rods per cell (the lattice start's 4 x 4 x 4
    # sites in the fullest cells go to the FP64 hand-over for the first sweeps)
    (dict(num_particles=2000, system_density=0.30, colloid_wall_option=1, colloid_radius=3.0), 45, 48),
    # NPT: the same rule (over-full cells of a compressed box go to the FP64
    # hand-over); an explicit capacity wins
    (dict(num_particles=11000, system_density=0.30, mc_ensemble_type=2), 35, 48),
    (dict(num_particles=11000, system_density=0.30, mc_ensemble_type=2, cell_capacity=56), 56, 56),
])
def test_cell_capacity_rule(kw, lo, cls):
    import ctypes as C
    p = lcmc.default_params(**kw)
    cap, klass = C.c_int(), C.c_int()
    assert _lib.lib().lcmc_cell_capacity(C.byref(p), C.byref(cap), C.byref(klass)) == 0
    assert cap.value >= lo and klass.value == cls, (cap.value, klass.value)


def _gb_pair_terms(pos, u, L, rmax=3.6):
    """FP64 numpy restatement of pij_GB (MCnptColloid.c:2618-2681) for
    GB(3, 5, 2, 1), sigma0 = eps0 = 1, over all pairs closer than rmax
    (test infrastructure): (terms, distreal)."""
    import numpy as np
    from scipy.spatial import cKDTree

    pairs = cKDTree(pos, boxsize=L * (1 + 1e-12)).query_pairs(rmax, output_type="ndarray")
    i, j = pairs[:, 0], pairs[:, 1]
    d = pos[j] - pos[i]
    d -= L * np.round(d / L)
    r = np.linalg.norm(d, axis=1)
    rh = d / r[:, None]
    chi, kp = 0.8, np.sqrt(5.0)
    chip = (kp - 1) / (kp + 1)
    a, b, c = (rh * u[i]).sum(1), (rh * u[j]).sum(1), (u[i] * u[j]).sum(1)

    def g(w):
        return 1 - 0.5 * w * ((a + b) ** 2 / (1 + w * c) + (a - b) ** 2 / (1 - w * c))

    dr = r - 1 / np.sqrt(g(chi)) + 1
    R = 1 / np.maximum(dr, 1e-3)
    phi = np.where(dr < 0.001, 1e9, 4 / np.sqrt(1 - chi ** 2 * c ** 2) * g(chip) ** 2 * R ** 6 * (R ** 6 - 1))
    return phi, dr


def test_body_centred_lattice_start_has_no_overlaps():
    """init_lattice = 1 (host only): N sites of a body-centred tetragonal
    lattice with layers 1.05 sigma_ee apart along z.  With orientations drawn
    within 20 degrees of z some tilted neighbours still overlap (about 1 % of
    pairs above 100 eps0), but no pair is inside the reference's 1e9 clamp or
    beside it (distreal > 0.2, terms below 1e9), so every overlap relaxes;
    the simple-cubic start at this density holds clamped pairs."""
    import numpy as np
    from parellel_mc_mpi_for_liquidcrystalsystems_b200 import mc

    n = 32768
    p = mc.default_params(num_particles=n, system_density=0.32, init_orientation_cone_deg=20.0, init_lattice=1,
                          rng_seed=5)
    (px, py, pz, ox, oy, oz), box = mc.lattice(p)
    L = box[0]
    assert np.all((px >= 0) & (px < L) & (py >= 0) & (py < L) & (pz >= 0) & (pz < L))
    pos = np.stack([px, py, pz], 1)
    assert len(np.unique(np.round(pos * 1e6).astype(np.int64), axis=0)) == n
    assert np.all(oz >= np.cos(np.radians(20.0)) - 1e-12)
    phi, dr = _gb_pair_terms(pos, np.stack([ox, oy, oz], 1), L)
    assert dr.min() > 0.2 and phi.max() < 1e9
    assert np.mean(phi > 100.0) < 0.02
    p0 = mc.default_params(num_particles=n, system_density=0.32, init_orientation_cone_deg=20.0, rng_seed=5)
    (qx, qy, qz, ux, uy, uz), box0 = mc.lattice(p0)
    phi0, dr0 = _gb_pair_terms(np.stack([qx, qy, qz], 1), np.stack([ux, uy, uz], 1), box0[0])
    assert dr0.min() < 0.001 and phi0.max() >= 1e9
