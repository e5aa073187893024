"""Generate golden fixtures by running the reference's own CUDA build.

TEST INFRASTRUCTURE.  Needs a GPU and oracle/_ref/libqvti_ref.so (built by
``make -C oracle ref`` from the reference's unmodified cuviscoelas_3D.cu plus
oracle/ref_harness.cu).  Usage on a GPU machine::

    python tests/golden/make_golden.py OUTDIR

writes one compressed ``.npz`` per case into OUTDIR; the committed fixtures in
tests/golden/ are exactly these files.  Each holds the case inputs (scalars,
model arrays when heterogeneous, wavelet, receivers) and the reference's
outputs: seismograms ``rec_vx/vy/vz`` ([it][ir], viscoelas_3D.cpp:416-435)
and wavefield snapshots ``snap_<k>`` (vx, vy, vz after k steps); for the
96^3 configuration, whose full fields are too large to commit, the x-z plane
12 cells beside the source ``plane_y_<k>`` (vx, vy, vz) every 100 steps and the
per-field norms of the final state.  ``--only NAME`` regenerates one case.
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import qvti_cases as qc  # noqa: E402

REF_SO = os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle", "_ref", "libqvti_ref.so")

_f = ctypes.POINTER(ctypes.c_float)
_i = ctypes.POINTER(ctypes.c_int)


def load_ref(path=REF_SO):
    lib = ctypes.CDLL(path)
    lib.qref_run.restype = ctypes.c_int
    lib.qref_run.argtypes = [ctypes.c_int] * 5 + [ctypes.c_float] * 5 + [_f] * 6 + \
        [ctypes.c_int] * 4 + [_i, _i, ctypes.c_int, ctypes.c_int] + [_f] * 4 + \
        [ctypes.POINTER(ctypes.c_double)]
    return lib


def _p(a, t=_f):
    return a.ctypes.data_as(t)


def run_reference(lib, c, nt=None, want_fields=True):
    """Run one shot through the reference; returns (rec[3,nt,rn], fields[9,...] or None, ms)."""
    nt = c["nt"] if nt is None else nt
    ntp = c["ntx"] * c["nty"] * c["ntz"]
    rn = c["rnx_max"] * c["rny_max"]
    rec = np.zeros((3, nt, rn), np.float32)
    fields = np.zeros((9, c["ntx"], c["nty"], c["ntz"]), np.float32) if want_fields else None
    arr = {k: np.ascontiguousarray(c[k], dtype=np.float32) for k in ("velp", "gama_p", "vels", "gama_s", "rho")}
    rik = np.ascontiguousarray(c["rik"][:nt], np.float32)
    rix = np.ascontiguousarray(c["r_ix"], np.int32)
    riy = np.ascontiguousarray(c["r_iy"], np.int32)
    ms = ctypes.c_double(0.0)
    rc = lib.qref_run(c["ntx"], c["nty"], c["ntz"], c["pml"], nt,
                      c["dx"], c["dy"], c["dz"], c["dt"], c["f0"],
                      _p(rik), _p(arr["velp"]), _p(arr["gama_p"]), _p(arr["vels"]), _p(arr["gama_s"]), _p(arr["rho"]),
                      c["s_ix"], c["s_iy"], c["s_iz"], c["r_iz"], _p(rix, _i), _p(riy, _i), c["rnx_max"], c["rny_max"],
                      _p(rec[0]), _p(rec[1]), _p(rec[2]),
                      _p(fields) if want_fields else None, ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError("reference run failed with %d" % rc)
    assert ntp == fields[0].size if want_fields else True
    return rec, fields, ms.value


def golden_cases():
    return [
        (qc.homogeneous_case(name="homog32"), [60, 120]),
        (qc.heterogeneous_case(name="hetero24x40x32"), [100]),
        (qc.config1_case(nt=500), [100, 200, 300, 400, 500]),
    ]


def _run_isolated(c, nt, tries=3):
    """Run the reference in a fresh process.  Its C-PML profile kernel reads
    mirror entries that other blocks write (cuviscoelas_3D.cu:248-250 vs
    293-306); in a process that already ran a shot the recycled device memory
    can feed that race a zero gamma and the whole run turns to NaN.  A fresh
    process per run, checked for finiteness, avoids it."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    for _ in range(tries):
        with ctx.Pool(1) as pool:
            rec, fields, ms = pool.apply(_worker, (c, nt))
        if np.isfinite(rec).all() and np.isfinite(fields).all():
            return rec, fields, ms
        print("reference run returned non-finite values, retrying", flush=True)
    raise RuntimeError("reference run non-finite after %d tries" % tries)


def _worker(c, nt):
    return run_reference(load_ref(), c, nt=nt, want_fields=True)


def save_case(outdir, c, snaps, lib=None):
    rec, fields, ms = _run_isolated(c, c["nt"])
    out = {k: (np.asarray(v) if not isinstance(v, str) else np.array(v)) for k, v in c.items()}
    homog = all(np.all(c[k] == c[k].flat[0]) for k in ("velp", "vels", "rho", "gama_p", "gama_s"))
    if homog:  # keep fixtures small: homogeneous models are stored as scalars
        for k in ("velp", "vels", "rho", "gama_p", "gama_s"):
            out[k] = np.array(c[k].flat[0], np.float32)
    out["rec_vx"], out["rec_vy"], out["rec_vz"] = rec[0], rec[1], rec[2]
    out["ref_ms"] = np.array(ms)
    if c["ntx"] * c["nty"] * c["ntz"] <= 64 ** 3:
        out["snap_%d" % c["nt"]] = fields[:3].copy()
        out["final9"] = fields
        for k in snaps:
            if k == c["nt"]:
                continue
            _, f, _ = _run_isolated(c, k)
            out["snap_%d" % k] = f[:3].copy()
    else:  # large case: per-field norms of the final state, x-z planes through the source
        out["final_norms"] = np.array([np.linalg.norm(f.astype(np.float64)) for f in fields])
        py = int(c["s_iy"]) + 12  # off the source's plane: vy is antisymmetric about it
        out["plane_y"] = np.array(py)
        for k in snaps:
            f = fields if k == c["nt"] else _run_isolated(c, k)[1]
            out["plane_y_%d" % k] = f[:3, :, py, :].copy()
    path = os.path.join(outdir, c["name"] + ".npz")
    np.savez_compressed(path, **out)
    print("wrote", path, "ref %.1f ms" % ms, flush=True)


def main():
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("outdir", nargs="?", default="golden_out")
    ap.add_argument("--only", default=None)
    a = ap.parse_args()
    os.makedirs(a.outdir, exist_ok=True)
    for c, snaps in golden_cases():
        if a.only and c["name"] != a.only:
            continue
        save_case(a.outdir, c, snaps)


if __name__ == "__main__":
    main()
