"""The reference's configuration files (no GPU): liblcmc.so's writers produce
the bytes that the reference's own esc_fort1, print_Trayectoria and
print_Qmga produced (tests/golden/io_golden.npz, made by
tests/golden/make_io_golden.py), and its reader returns what
read_initial_configuration returned, including the first-N rule for a file
holding more particles."""
import ctypes as C

import numpy as np

from parellel_mc_mpi_for_liquidcrystalsystems_b200 import _lib

DP = _lib.DP


def ptrs(arrs):
    return [np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(DP) for a in arrs]


def test_writers_match_the_reference_bytes(golden, tmp_path):
    g = golden("io_golden.npz")
    L = _lib.lib()
    arrs = [np.ascontiguousarray(a) for a in (*g["pos"], *g["ori"])]
    p = [a.ctypes.data_as(DP) for a in arrs]
    box = np.ascontiguousarray(g["box"])
    n = arrs[0].size
    f1 = str(tmp_path / "fortSphere.1").encode()
    assert L.lcmc_write_fort1(f1, n, *p, box.ctypes.data_as(DP), float(g["colloid_R"])) == 0
    assert open(f1, "rb").read() == g["fort1"].tobytes()
    tr = str(tmp_path / "Configuraciones.dat").encode()
    assert L.lcmc_write_trajectory(tr, 0, n, *p, box.ctypes.data_as(DP)) == 0
    assert L.lcmc_write_trajectory(tr, 1, n, *p, box.ctypes.data_as(DP)) == 0
    assert open(tr, "rb").read() == g["traj"].tobytes()
    qm = str(tmp_path / "qmga_mcnvtGB.cnf").encode()
    assert L.lcmc_write_qmga(qm, 0, n, *p, box.ctypes.data_as(DP)) == 0
    assert open(qm, "rb").read() == g["qmga"].tobytes()


def test_reader_matches_read_initial_configuration(golden, tmp_path):
    g = golden("io_golden.npz")
    path = tmp_path / "fortSphere.1"
    path.write_bytes(g["read_text"].tobytes())
    n = g["read_arrays"].shape[1]
    out = [np.zeros(n) for _ in range(6)]
    box = np.zeros(3)
    R = C.c_double()
    n_read = C.c_int()
    rc = _lib.lib().lcmc_read_fort1(str(path).encode(), n, *[a.ctypes.data_as(DP) for a in out],
                                    box.ctypes.data_as(DP), C.byref(R), C.byref(n_read))
    assert rc == 0 and n_read.value == n + 10
    assert np.array_equal(np.stack(out), g["read_arrays"])
    assert np.array_equal(box, g["read_box"]) and R.value == float(g["read_R"])


def test_round_trip_and_errors(tmp_path):
    rng = np.random.default_rng(3)
    n = 40
    arrs = [rng.uniform(0, 9, n) for _ in range(3)] + [rng.normal(size=n) for _ in range(3)]
    box = np.array([9.0, 9.5, 10.0])
    path = str(tmp_path / "f").encode()
    L = _lib.lib()
    assert L.lcmc_write_fort1(path, n, *ptrs(arrs), box.ctypes.data_as(DP), 0.0) == 0
    out = [np.zeros(n) for _ in range(6)]
    b2, R, nr = np.zeros(3), C.c_double(), C.c_int()
    assert L.lcmc_read_fort1(path, n, *[a.ctypes.data_as(DP) for a in out], b2.ctypes.data_as(DP), C.byref(R),
                             C.byref(nr)) == 0
    for a, b in zip(arrs, out):
        assert np.max(np.abs(a - b)) <= 5e-9  # 8 decimals
    assert L.lcmc_read_fort1(str(tmp_path / "missing").encode(), n, *[a.ctypes.data_as(DP) for a in out],
                             b2.ctypes.data_as(DP), C.byref(R), C.byref(nr)) == _lib.ENOFILE
    (tmp_path / "short").write_text("5 1 1 1 0\n1 2 3\n")
    assert L.lcmc_read_fort1(str(tmp_path / "short").encode(), 5, *[a.ctypes.data_as(DP) for a in out],
                             b2.ctypes.data_as(DP), C.byref(R), C.byref(nr)) == _lib.EPARAM
