"""ctypes binding of the FP64 CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY -- imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker; never by the product.

``run_case(case)`` runs one shot described by a dict in the conventions of
tests/qvti_cases.py (the reference's: force source at s_iz + 10).  The oracle
restates cuviscoelas_3D.cu:22-1134 and the time loop cuviscoelas_3D.cu:1255-1630
in double precision; see qvti_oracle.h.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")


class QoParams(ctypes.Structure):
    _fields_ = [("ntx", ctypes.c_int), ("nty", ctypes.c_int), ("ntz", ctypes.c_int),
                ("pml", ctypes.c_int), ("nt", ctypes.c_int),
                ("dx", ctypes.c_float), ("dy", ctypes.c_float), ("dz", ctypes.c_float),
                ("dt", ctypes.c_float), ("f0", ctypes.c_float),
                ("vti", ctypes.c_int), ("src_type", ctypes.c_int),
                ("s_ix", ctypes.c_int), ("s_iy", ctypes.c_int), ("s_iz", ctypes.c_int),
                ("r_iz", ctypes.c_int), ("rn", ctypes.c_int), ("nthreads", ctypes.c_int)]


_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE], stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        f = ctypes.POINTER(ctypes.c_float)
        i = ctypes.POINTER(ctypes.c_int)
        d = ctypes.POINTER(ctypes.c_double)
        L.qo_run.restype = ctypes.c_int
        L.qo_run.argtypes = [ctypes.POINTER(QoParams), f, f, f, f, f, f, f, f, i, i, f, f, f,
                             ctypes.c_int, i, f, d]
        L.qo_fft3d.restype = None
        L.qo_fft3d.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, d, ctypes.c_int]
        L.qo_shift_tables.argtypes = [ctypes.c_int, ctypes.c_float, d, d]
        L.qo_wavenumbers.argtypes = [ctypes.c_int, ctypes.c_float, d]
        L.qo_q_coeffs.argtypes = [ctypes.c_int, f, f, f, ctypes.c_float, d]
        L.qo_pml_profile.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_float, d, d]
        _lib = L
    return _lib


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)) if a is not None else None


def _full(c, key, shape):
    a = np.asarray(c[key], np.float32)
    if a.ndim == 0:
        a = np.full(shape, a, np.float32)
    if a.shape != shape:  # the C restatement indexes the full grid
        raise ValueError("%s has shape %s, the grid is %s" % (key, a.shape, shape))
    return np.ascontiguousarray(a)


def run_case(c, nt=None, snaps=(), src_type=0, vti=False, nthreads=0, want_state=False, ref_offset=True):
    """Run a case dict.  Returns dict(rec=[3,nt,rn] float32, snaps={k: [3,...]},
    state=[9,...] float64 or None).  ``ref_offset`` adds the reference's +10
    to s_iz (cuviscoelas_3D.cu:772)."""
    L = lib()
    nt = int(c["nt"] if nt is None else nt)
    shape = (int(c["ntx"]), int(c["nty"]), int(c["ntz"]))
    ntp = shape[0] * shape[1] * shape[2]
    rn = int(c["rnx_max"]) * int(c["rny_max"])
    p = QoParams(shape[0], shape[1], shape[2], int(c["pml"]), nt,
                 float(c["dx"]), float(c["dy"]), float(c["dz"]), float(c["dt"]), float(c["f0"]),
                 1 if vti else 0, int(src_type), int(c["s_ix"]), int(c["s_iy"]),
                 int(c["s_iz"]) + (10 if ref_offset else 0), int(c["r_iz"]), rn, int(nthreads))
    arrs = [_full(c, k, shape) for k in ("velp", "vels", "rho", "gama_p", "gama_s")]
    eps = _full(c, "eps", shape) if vti else None
    dl = _full(c, "delta", shape) if vti else None
    rik = np.ascontiguousarray(np.asarray(c["rik"], np.float32)[:nt])
    rix = np.ascontiguousarray(c["r_ix"], np.int32)
    riy = np.ascontiguousarray(c["r_iy"], np.int32)
    rec = np.zeros((3, nt, rn), np.float32)
    snaps = sorted(int(s) for s in snaps)
    sn = np.zeros((max(len(snaps), 1), 3) + shape, np.float32)
    sarr = np.array(snaps if snaps else [0], np.int32)
    state = np.zeros((9,) + shape, np.float64) if want_state else None
    ip = ctypes.POINTER(ctypes.c_int)
    rc = L.qo_run(ctypes.byref(p), _fp(rik), _fp(arrs[0]), _fp(arrs[1]), _fp(arrs[2]), _fp(arrs[3]),
                  _fp(arrs[4]), _fp(eps), _fp(dl), rix.ctypes.data_as(ip), riy.ctypes.data_as(ip),
                  _fp(rec[0]), _fp(rec[1]), _fp(rec[2]), len(snaps), sarr.ctypes.data_as(ip), _fp(sn),
                  state.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if want_state else None)
    if rc != 0:
        raise RuntimeError("oracle failed with status %d" % rc)
    assert ntp == sn[0, 0].size
    return dict(rec=rec, snaps={k: sn[i] for i, k in enumerate(snaps)}, state=state)


def fft3d(a, sign):
    """Unnormalised 3D C2C FFT of a complex128 array (sign -1 forward)."""
    L = lib()
    a = np.ascontiguousarray(a, np.complex128).copy()
    L.qo_fft3d(a.shape[0], a.shape[1], a.shape[2], a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(sign))
    return a


def shift_tables(n, d):
    f = np.zeros(2 * n)
    b = np.zeros(2 * n)
    dp = ctypes.POINTER(ctypes.c_double)
    lib().qo_shift_tables(n, d, f.ctypes.data_as(dp), b.ctypes.data_as(dp))
    return f[0::2] + 1j * f[1::2], b[0::2] + 1j * b[1::2]


def wavenumbers(n, d):
    k = np.zeros(n)
    lib().qo_wavenumbers(n, d, k.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return k


def q_coeffs(vel, gam, rho, f0):
    vel, gam, rho = (np.ascontiguousarray(x, np.float32).ravel() for x in (vel, gam, rho))
    out = np.zeros(5 * vel.size)
    lib().qo_q_coeffs(vel.size, _fp(vel), _fp(gam), _fp(rho), f0, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return out.reshape(5, vel.size)


def pml_profile(n, pml, d, f0):
    a = np.zeros(n)
    b = np.zeros(n)
    dp = ctypes.POINTER(ctypes.c_double)
    lib().qo_pml_profile(n, pml, d, f0, a.ctypes.data_as(dp), b.ctypes.data_as(dp))
    return a, b
