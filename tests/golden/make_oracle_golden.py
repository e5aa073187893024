"""Generate golden fixtures from the FP64 CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE.  The oracle is pinned separately to the reference's own
cuFFT build (tests/test_oracle.py against the fixtures of make_golden.py);
these fixtures extend parity to cases the reference cannot run or that are
too large to compare field by field:

* ``vti_crop128`` -- a centred 128^3 crop of the 256^3 VTI benchmark model
  (``models.layered_vti``, seed 2024: 6 layers, eps/delta/Q per layer, 5 %
  Gaussian perturbations), at the benchmark's dt (the nominal 0.8 ms capped
  to 80 % of the stability bound of the full model: 0.45 ms), 20-cell C-PML,
  20 Hz Ricker force on vx at (64, 64, 25), 400 steps.  The reference is
  isotropic only, so VTI is pinned through the oracle.
* ``vti512_crop128`` -- the same crop of the 512 x 512 x 256 model of the
  precision configuration (the generator at that size, seed 2024; its dt
  from that model's stability bound), 400 steps.
* ``config1_force_planes`` -- the small configuration with the reference's
  own force source, the FP64 counterpart of the reference-build fixture
  tests/golden/config1.npz (planes 12 cells beside the source).
* ``config1_explosive`` -- the small isotropic configuration as specified
  (96^3, 20-cell C-PML, Vp 2500, Vs 1443, rho 2000, Qp 100, Qs 50, 25 Hz,
  dt 1 ms, 500 steps) with the explosive source at the grid centre, which the
  reference's build only has as commented-out code (cuviscoelas_3D.cu:775-776).

Each fixture stores the case scalars, wavelet and receivers, the seismograms
``rec_vx/vy/vz`` ([it][ir]) and, every 100 steps, two planes of vx, vy, vz
(``plane_y_<k>`` = the x-z plane through the source, ``plane_z_<k>`` = the x-y
plane at the source depth; full fields at these sizes are 25 MB each), plus
float64 sums of the model arrays so a test can tell that it rebuilt the same
model.  Usage::

    python tests/golden/make_oracle_golden.py [OUTDIR] [--only NAME]

(default OUTDIR tests/golden/oracle/, where the committed fixtures live).
"""
import importlib.util
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import qvti_cases as qc  # noqa: E402

MODEL_KEYS = ("velp", "vels", "rho", "gama_p", "gama_s", "eps", "delta")


def _models():
    spec = importlib.util.spec_from_file_location("qvti_models", os.path.join(ROOT, "q-vti_b200", "models.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def crop128_case(full_shape, name, nt=400, model=None):
    """The centred 128^3 crop of the VTI generator's model at `full_shape`
    (case dict in the conventions of tests/qvti_cases.py; the source depth is
    final, no +10 offset), at the dt of the full model.  `model`: that full
    model when the caller has built it already."""
    md = _models()
    full = model if model is not None else md.layered_vti(tuple(full_shape), 10.0, seed=2024)
    dt, _, _ = md.choose_dt(full, 10.0, 20.0, 0.8e-3, vti=True)
    sl = tuple(slice((g - 128) // 2, (g - 128) // 2 + 128) for g in full_shape)
    n, pml = 128, 20
    gx = np.arange(0, n, 8, dtype=np.int32)
    c = dict(name=name, ntx=n, nty=n, ntz=n, pml=pml, nt=nt, dx=10.0, dy=10.0, dz=10.0, dt=dt, f0=20.0,
             rik=md.ricker(nt, dt, 20.0), s_ix=64, s_iy=64, s_iz=pml + 5, r_iz=pml,
             r_ix=np.repeat(gx, gx.size), r_iy=np.tile(gx, gx.size), rnx_max=gx.size, rny_max=gx.size,
             vti=1, src_type=0, plane_y=64, plane_z=pml + 5)
    for k in MODEL_KEYS:
        c[k] = np.ascontiguousarray(full[k][sl])
    return c


def vti_crop128_case(nt=400):
    """Centred 128^3 crop of the 256^3 VTI benchmark model."""
    return crop128_case((256, 256, 256), "vti_crop128", nt)


def vti512_crop128_case(nt=400):
    """Centred 128^3 crop of the 512 x 512 x 256 precision-configuration
    model (same generator and seed; its own perturbation fields)."""
    return crop128_case((512, 512, 256), "vti512_crop128", nt)


def config1_explosive_case(nt=500):
    c = qc.config1_case(nt=nt)
    c["name"] = "config1_explosive"
    c["s_iz"] = 48  # explosive source at the centre, no offset
    c.update(vti=0, src_type=1, plane_y=48, plane_z=48)
    return c


def config1_force_planes_case(nt=500):
    """The small configuration with the reference's own source (force on vx at
    s_iz + 10, the centre), as in tests/golden/config1.npz from the
    reference's cuFFT build: the FP64 result on the x-z plane 12 cells
    beside the source (vy is antisymmetric about the source's own plane)."""
    c = qc.config1_case(nt=nt)
    c["name"] = "config1_force_planes"
    c.update(vti=0, src_type=0, ref_offset=1, plane_y=60, plane_z=-1)
    return c


def cases():
    return {"vti_crop128": vti_crop128_case, "config1_explosive": config1_explosive_case,
            "vti512_crop128": vti512_crop128_case, "config1_force_planes": config1_force_planes_case}


def model_sums(c):
    keys = MODEL_KEYS if c["vti"] else MODEL_KEYS[:5]
    return np.array([np.asarray(c[k], np.float64).sum() for k in keys])


def save_case(outdir, c):
    import oracle
    snaps = list(range(100, int(c["nt"]) + 1, 100))
    t0 = time.time()
    r = oracle.run_case(c, snaps=snaps, src_type=int(c["src_type"]), vti=bool(c["vti"]),
                        ref_offset=bool(c.get("ref_offset", 0)))
    write_case(outdir, c, r)
    print("oracle %.0f s" % (time.time() - t0), flush=True)


def write_case(outdir, c, r):
    """The fixture of case c from an oracle run r (run_case's result)."""
    snaps = list(range(100, int(c["nt"]) + 1, 100))
    out = {k: np.asarray(v) for k, v in c.items() if k not in MODEL_KEYS}
    out["model_sums"] = model_sums(c)
    out["rec_vx"], out["rec_vy"], out["rec_vz"] = r["rec"]
    for k in snaps:
        out["plane_y_%d" % k] = r["snaps"][k][:, :, int(c["plane_y"]), :].copy()
        if int(c["plane_z"]) >= 0:
            out["plane_z_%d" % k] = r["snaps"][k][:, :, :, int(c["plane_z"])].copy()
    path = os.path.join(outdir, c["name"] + ".npz")
    np.savez_compressed(path, **out)
    print("wrote %s" % path, flush=True)


def main():
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("outdir", nargs="?", default=os.path.join(HERE, "oracle"))
    ap.add_argument("--only", default=None)
    a = ap.parse_args()
    os.makedirs(a.outdir, exist_ok=True)
    for name, make in cases().items():
        if a.only and name != a.only:
            continue
        save_case(a.outdir, make())


if __name__ == "__main__":
    main()
