#!/usr/bin/env python3
"""Configuration files written and read by the reference's OWN functions.

Runs where the reference source is available: loads
oracle/_ref/libmcref_serial.so (MCnptColloid.c built by oracle/build_ref.sh)
and, in a temporary directory (the reference writes to fixed file names),
calls esc_fort1 (MCnptColloid.c:3193), print_Trayectoria (3081, options 0 and
1) and print_Qmga (3110) on a seeded 50-particle configuration, then
read_initial_configuration (2786) on a fortSphere.1 holding 60 particles.
Stores the inputs, the files' bytes and what the reader returned in
io_golden.npz beside this script.
"""
import ctypes as C
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF_SO = os.path.join(REPO, "oracle", "_ref", "libmcref_serial.so")
N = 50

PARAM_TEXT = f"""mc_ensemble_type 1
num_particles {N}
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
initial_configuration_type 1
cutoff_radius 4.0
verlet_radius 4.8
total_mc_cycles 1000
configuration_save_interval 100
statistics_print_interval 100
colloid_wall_option 1
colloid_interaction_epsilon 15
colloid_interaction_amplitude 1.5
colloid_radius 1.25
"""

DP = C.POINTER(C.c_double)


def main():
    ref = C.CDLL(REF_SO)
    ref.load_initial_conditions.argtypes = [C.c_char_p]
    ref.refdrv_set_box.argtypes = [C.c_int, DP]
    for name in ("esc_fort1", "read_initial_configuration"):
        getattr(ref, name).argtypes = [DP] * 6
    for name in ("print_Trayectoria", "print_Qmga"):
        getattr(ref, name).argtypes = [DP] * 6 + [C.c_int]
    rng = np.random.default_rng(2024)
    box = np.array([11.5, 12.25, 13.125])
    pos = [np.ascontiguousarray(rng.uniform(0, L, N)) for L in box]
    u = rng.normal(size=(N, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    ori = [np.ascontiguousarray(u[:, k]) for k in range(3)]
    ptr = [a.ctypes.data_as(DP) for a in pos + ori]
    cwd = os.getcwd()
    out = {}
    with tempfile.TemporaryDirectory() as d:
        os.chdir(d)
        try:
            with open("p.txt", "w") as f:
                f.write(PARAM_TEXT)
            ref.load_initial_conditions(b"p.txt")
            ref.refdrv_set_box(N, box.ctypes.data_as(DP))
            ref.esc_fort1(*ptr)
            out["fort1"] = np.frombuffer(open("fortSphere.1", "rb").read(), dtype=np.uint8)
            ref.print_Trayectoria(*ptr, 0)
            ref.print_Trayectoria(*ptr, 1)
            out["traj"] = np.frombuffer(open("Configuraciones.dat", "rb").read(), dtype=np.uint8)
            ref.print_Qmga(*ptr, 0)
            out["qmga"] = np.frombuffer(open("qmga_mcnvtGB.cnf", "rb").read(), dtype=np.uint8)
            # a 60-particle file read with num_particles = 50: the reader takes the first 50
            big = N + 10
            with open("fortSphere.1", "w") as f:
                f.write(f"{big} 20.5 21.25 22.0 2.5\n")
                for i in range(big):
                    f.write(f"{1.0 + 0.1 * i:15.8f} {2.0 + 0.01 * i:15.8f} {3.0 - 0.02 * i:15.8f}\n")
                    f.write(f"{0.0:15.8f} {0.0:15.8f} {0.0:15.8f}\n")
                    f.write(f"{0.6:15.8f} {0.0:15.8f} {-0.8:15.8f}\n")
                    f.write(f"{0.0:15.8f} {0.0:15.8f} {0.0:15.8f}\n")
            out["read_text"] = np.frombuffer(open("fortSphere.1", "rb").read(), dtype=np.uint8)
            got = [np.zeros(N) for _ in range(6)]
            ref.read_initial_configuration(*[a.ctypes.data_as(DP) for a in got])
            out["read_arrays"] = np.stack(got)
            bs = (C.c_double * 3).in_dll(ref, "box_size")
            out["read_box"] = np.array(list(bs))
            out["read_R"] = np.array(C.c_double.in_dll(ref, "colloid_radius").value)
        finally:
            os.chdir(cwd)
    np.savez(os.path.join(HERE, "io_golden.npz"), box=box, pos=np.stack(pos), ori=np.stack(ori), colloid_R=1.25,
             **out)
    print("wrote io_golden.npz", {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
