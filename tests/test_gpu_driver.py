"""The cycle-loop driver (run_simulation) over the library on the GPU: it
writes the reference's files at the reference's intervals, and a run resumed
from its fortSphere.1 (with the exact sidecar) ends where one uninterrupted run
of the same length ends, bit for bit."""
import numpy as np
import pytest

import parellel_mc_mpi_for_liquidcrystalsystems_b200 as lcmc

pytestmark = pytest.mark.gpu

KEYS = ("mc_ensemble_type 1\nnum_particles 1000\nsystem_density 0.30\nsystem_temperature 1.0\n"
        "system_pressure 2.0\ngb_sigma_sidetoside 1.0\ngb_epsilon0 1.0\ngb_kappa 3.0\ngb_kappa_prime 5.0\n"
        "gb_mu_exponent 2.0\ngb_nu_exponent 1.0\nmax_displacement 0.1\nmax_rotation 0.1\n"
        "initial_configuration_type {init}\ncutoff_radius 4.0\nverlet_radius 4.8\ntotal_mc_cycles {cycles}\n"
        "configuration_save_interval 2000\nstatistics_print_interval 1000\ncolloid_wall_option 0\n"
        "colloid_interaction_epsilon 15\ncolloid_interaction_amplitude 1.5\ncolloid_radius 0.0\nrng_seed 31\n")


def write_params(d, init, cycles):
    f = d / "parametersFile.txt"
    f.write_text(KEYS.format(init=init, cycles=cycles))
    return f


def sidecar_state(path):
    raw = np.fromfile(str(path) + ".lcmc", dtype=np.uint8)
    return raw[8 + 8:]  # past the magic and the particle count: sweep, seed, energy, box, state


def test_run_simulation_writes_the_reference_files(tmp_path):
    lines = []
    res = lcmc.run_simulation(write_params(tmp_path, 2, 5000), tmp_path, log=lines.append)
    assert res["sweeps"] == 5 and res["stats"]["attempted"] == 5000
    assert len(lines) == 2  # sweeps 2 and 4 (every 2000 attempts)
    traj = (tmp_path / "Configuraciones.dat").read_text().splitlines()
    assert len(traj) == 2 * (2 + 1000) and traj[0].split() == ["1000"]
    assert (tmp_path / "qmga_mcnvtGB.cnf").read_text().splitlines()[0] == "1000"
    hist = np.loadtxt(tmp_path / "Histograma_Movimientos.dat", dtype=np.int64)
    assert hist.shape == (1000, 2) and hist[:, 1].sum() == res["stats"]["accepted"]
    head = (tmp_path / "fortSphere.1").read_text().splitlines()
    assert len(head) == 1 + 4 * 1000 and head[0].split()[0] == "1000"
    assert 0.0 < res["P2"] < 1.0 and abs(res["rho"] - 0.30) < 1e-9


def test_resumed_run_ends_where_one_run_ends(tmp_path):
    one, two = tmp_path / "one", tmp_path / "two"
    one.mkdir()
    two.mkdir()
    lcmc.run_simulation(write_params(one, 2, 8000), one, histogram=False)
    lcmc.run_simulation(write_params(two, 2, 4000), two, histogram=False)
    lcmc.run_simulation(write_params(two, 0, 4000), two, histogram=False)  # resume from two/fortSphere.1
    a, b = sidecar_state(one / "fortSphere.1"), sidecar_state(two / "fortSphere.1")
    assert a.size == b.size and np.array_equal(a, b)


def test_c_host_writes_what_run_simulation_writes(tmp_path):
    """tests/c_host/lcmc_run.c (the cycle loop in C over include/lcmc.h) and
    run_simulation, on one parameter file: the same status lines and the same
    bytes in every output file (Configuraciones.dat, fortSphere.1 and its
    sidecar, qmga_mcnvtGB.cnf, Histograma_Movimientos.dat)."""
    import subprocess

    from test_c_host_cpu import build_c_host

    exe = build_c_host(tmp_path / "lcmc_run")
    c_dir, py_dir = tmp_path / "c", tmp_path / "py"
    c_dir.mkdir()
    py_dir.mkdir()
    params = write_params(tmp_path, 2, 5000)
    r = subprocess.run([str(exe), str(params), str(c_dir)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = []
    lcmc.run_simulation(params, py_dir, log=lines.append)
    c_lines = r.stdout.splitlines()
    assert c_lines[:-1] == lines and c_lines[-1].startswith("done: 5 sweeps")
    for name in ("Configuraciones.dat", "fortSphere.1", "fortSphere.1.lcmc", "qmga_mcnvtGB.cnf",
                 "Histograma_Movimientos.dat"):
        assert (c_dir / name).read_bytes() == (py_dir / name).read_bytes(), name
