"""Time the reference's own cuFFT build against this library on one grid.

TEST INFRASTRUCTURE ONLY.  Runs oracle/_ref/libqvti_ref.so (the reference's
unmodified cuviscoelas_3D.cu plus oracle/ref_harness.cu, built by
``make -C oracle ref``) through its C ABI, and the product (libqvti.so)
through its Python binding, on the same seeded homogeneous isotropic case.
Needs a GPU.  Usage::

    python oracle/time_reference.py N PML     # e.g. 256 30

The reference harness times the whole ``cuda_forward_acoustic_3D`` call
(setup, time loop, record copy-back; cuviscoelas_3D.cu:1137-1652), so its
per-step time is the difference of two runs, (t(45) - t(25)) / 20 steps,
which cancels the setup.  This library's per-step time is the wall time of
40 steps after 5 warm-up steps, on its own stream.  Both print one line:
``<which> n=N ms_per_step=T gcell=G`` with G in Gcell-steps/s.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
sys.path.insert(0, os.path.join(ROOT, "q-vti_b200"))

import qvti_cases as qc  # noqa: E402


def case(n, pml):
    return qc.homogeneous_case(n=(n, n, n), pml=pml, d=(10.0, 10.0, 10.0), dt=0.45e-3, nt=45, f0=20.0,
                               src=(n // 2, n // 2, n // 2), r_iz=pml + 5, name="timing")


def time_reference(c):
    import make_golden as mg
    lib = mg.load_ref()
    ms = {}
    for nt in (5, 25, 45):
        ms[nt] = mg.run_reference(lib, c, nt=nt, want_fields=False)[2]
    return (ms[45] - ms[25]) / 20.0


def time_library(c, vti):
    import qvti
    shape = c["velp"].shape
    with qvti.simulation_for_case(c, vti=vti) as sim:
        sim.set_model(c["velp"], c["vels"], c["rho"], c["gama_p"], c["gama_s"],
                      np.full(shape, 0.1, np.float32) if vti else None,
                      np.full(shape, 0.05, np.float32) if vti else None)
        sim.set_receivers(c["r_iz"], c["r_ix"], c["r_iy"])
        sim.set_source(c["s_ix"], c["s_iy"], int(c["s_iz"]) + 10, np.asarray(c["rik"], np.float32))
        sim.reset()
        sim.step(5)
        sim.sync()
        t0 = time.perf_counter()
        sim.step(40)
        sim.sync()
        return (time.perf_counter() - t0) * 1e3 / 40


def main():
    n, pml = int(sys.argv[1]), int(sys.argv[2])
    c = case(n, pml)
    cells = float(n) ** 3
    for which, fn in (("reference_cufft", lambda: time_reference(c)),
                      ("library_iso", lambda: time_library(c, False)),
                      ("library_vti", lambda: time_library(c, True))):
        t = fn()
        print("%s n=%d ms_per_step=%.3f gcell=%.3f" % (which, n, t, cells / t / 1e6), flush=True)


if __name__ == "__main__":
    main()
