"""Python binding of libqvti.so (ctypes over the C ABI in include/qvti.h).

The engine is the CUDA library; this module only marshals host arrays.  It
mirrors the reference's operator surface for the path: a shot is the call of
``cuda_forward_acoustic_3D`` (cuviscoelas_3D.cu:1137-1652) with the model,
wavelet, source and receivers of viscoelas_3D.cpp, returning the three
seismograms ``[it][ir]``.  There is no CPU fallback: loading fails loudly when
the library is missing.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqvti.so")

SRC_FORCE_X = 0
SRC_EXPLOSIVE = 1
FORM_PLAIN = 0  # every transform stage as FP32 butterflies
FORM_TC = 1     # 256-point y transforms as split-precision tensor-core contractions
MEDIA_VISCOELASTIC, MEDIA_DISPERSION_ONLY, MEDIA_LOSSLESS, MEDIA_Q_COMPENSATED = 1, 2, 3, 4
FIELDS = ("vx", "vy", "vz", "pxx", "pyy", "pzz", "pxy", "pxz", "pyz")


class QvtiError(RuntimeError):
    pass


class Config(ctypes.Structure):
    _fields_ = [("ntx", ctypes.c_int), ("nty", ctypes.c_int), ("ntz", ctypes.c_int), ("pml", ctypes.c_int),
                ("dx", ctypes.c_float), ("dy", ctypes.c_float), ("dz", ctypes.c_float),
                ("dt", ctypes.c_float), ("f0", ctypes.c_float), ("vti", ctypes.c_int),
                ("device", ctypes.c_int), ("w0", ctypes.c_float)]


class Shot(ctypes.Structure):
    """qvti_shot: one shot of a batch or a serving request."""
    _fields_ = [("ntx", ctypes.c_int), ("nty", ctypes.c_int), ("ntz", ctypes.c_int), ("pml", ctypes.c_int),
                ("dx", ctypes.c_float), ("dy", ctypes.c_float), ("dz", ctypes.c_float),
                ("dt", ctypes.c_float), ("f0", ctypes.c_float), ("vti", ctypes.c_int),
                ("velp", ctypes.POINTER(ctypes.c_float)), ("vels", ctypes.POINTER(ctypes.c_float)),
                ("rho", ctypes.POINTER(ctypes.c_float)), ("gama_p", ctypes.POINTER(ctypes.c_float)),
                ("gama_s", ctypes.POINTER(ctypes.c_float)), ("eps", ctypes.POINTER(ctypes.c_float)),
                ("delta", ctypes.POINTER(ctypes.c_float)),
                ("src_type", ctypes.c_int), ("s_ix", ctypes.c_int), ("s_iy", ctypes.c_int), ("s_iz", ctypes.c_int),
                ("wavelet", ctypes.POINTER(ctypes.c_float)), ("nt", ctypes.c_int),
                ("r_iz", ctypes.c_int), ("rn", ctypes.c_int),
                ("r_ix", ctypes.POINTER(ctypes.c_int)), ("r_iy", ctypes.POINTER(ctypes.c_int)),
                ("rec_vx", ctypes.POINTER(ctypes.c_float)), ("rec_vy", ctypes.POINTER(ctypes.c_float)),
                ("rec_vz", ctypes.POINTER(ctypes.c_float))]


class ShotResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("queue_s", ctypes.c_double), ("latency_s", ctypes.c_double),
                ("device_ms", ctypes.c_float)]


NUM_TILES = 6  # k_vy, k_vx, k_fz, k_cy, k_mx, k_sigma (QVTI_TILE_*)


class Tuning(ctypes.Structure):
    _fields_ = [("active", ctypes.c_int), ("kz_batch", ctypes.c_int), ("form", ctypes.c_int),
                ("gcell_steps", ctypes.c_double), ("tiles", ctypes.c_int * NUM_TILES)]


class RtmOpts(ctypes.Structure):
    _fields_ = [("media", ctypes.c_int), ("snap_every", ctypes.c_int), ("illum_eps", ctypes.c_float)]


SCHED_FIFO = 0            # first submitted, first admitted
SCHED_SMALLEST_FIRST = 1  # fewest cell-steps first (bounded passing)


class SchedOpts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("mem_budget", ctypes.c_size_t), ("max_active", ctypes.c_int),
                ("policy", ctypes.c_int)]


_lib = None
_F = ctypes.POINTER(ctypes.c_float)
_I = ctypes.POINTER(ctypes.c_int)
_D = ctypes.POINTER(ctypes.c_double)
_V = ctypes.c_void_p


def lib():
    """Load libqvti.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise QvtiError("libqvti.so not found at %s: build it with `make -C q-vti_b200`" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        sig = {
            "qvti_footprint_bytes": (ctypes.c_size_t, [ctypes.c_int] * 5),
            "qvti_create": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(_V)]),
            "qvti_destroy": (ctypes.c_int, [_V]),
            "qvti_get_config": (ctypes.c_int, [_V, ctypes.POINTER(Config)]),
            "qvti_sims_created": (ctypes.c_longlong, []),
            "qvti_set_model": (ctypes.c_int, [_V, _F, _F, _F, _F, _F, _F, _F, ctypes.c_int]),
            "qvti_set_source": (ctypes.c_int, [_V, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _F,
                                               ctypes.c_int]),
            "qvti_set_receivers": (ctypes.c_int, [_V, ctypes.c_int, _I, _I, ctypes.c_int]),
            "qvti_reset": (ctypes.c_int, [_V]),
            "qvti_step": (ctypes.c_int, [_V, ctypes.c_int]),
            "qvti_step_timed": (ctypes.c_int, [_V, ctypes.c_int, _F]),
            "qvti_sync": (ctypes.c_int, [_V]),
            "qvti_steps_done": (ctypes.c_int, [_V]),
            "qvti_get_records": (ctypes.c_int, [_V, _F, _F, _F]),
            "qvti_get_fields": (ctypes.c_int, [_V, ctypes.c_int, ctypes.c_int, _F]),
            "qvti_device_field": (ctypes.c_int, [_V, ctypes.c_int, ctypes.POINTER(_F)]),
            "qvti_field_norms": (ctypes.c_int, [_V, _D, _I]),
            "qvti_state_bytes": (ctypes.c_int, [_V, ctypes.POINTER(ctypes.c_size_t)]),
            "qvti_save_state": (ctypes.c_int, [_V, _V, ctypes.c_size_t]),
            "qvti_load_state": (ctypes.c_int, [_V, _V, ctypes.c_size_t]),
            "qvti_forward_shot": (ctypes.c_int, [_V, _F, _F, _F, _F, _F, _F, _F, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_int, ctypes.c_int, _F, ctypes.c_int, ctypes.c_int, _I,
                                                 _I, ctypes.c_int, _F, _F, _F]),
            "qvti_derivative_1d": (ctypes.c_int, [_V, ctypes.c_int, ctypes.c_int, _F, _F]),
            "qvti_q_derivative": (ctypes.c_int, [_V, ctypes.c_int, ctypes.c_int, ctypes.c_int, _F, _F]),
            "qvti_q_derivative_noalloc": (ctypes.c_int, [_V, _V, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                         ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                                         ctypes.c_int, ctypes.c_int, ctypes.c_int, _V]),
            "qvti_profile_step": (ctypes.c_int, [_V, ctypes.c_int, ctypes.c_int, _I, ctypes.c_char_p, _F, _D]),
            "qvti_get_stream": (ctypes.c_int, [_V, ctypes.POINTER(_V)]),
            "qvti_set_kz_batch": (ctypes.c_int, [_V, ctypes.c_int]),
            "qvti_set_form": (ctypes.c_int, [_V, ctypes.c_int]),
            "qvti_set_tiles": (ctypes.c_int, [_V, _I]),
            "qvti_get_tiles": (ctypes.c_int, [_V, _I, _I]),
            "qvti_autotune_tiles": (ctypes.c_int, [_V, ctypes.c_int, _I, _F]),
            "qvti_set_media": (ctypes.c_int, [_V, ctypes.c_int]),
            "qvti_probe_bounded_wait": (ctypes.c_int, [_V, ctypes.c_double]),
            "qvti_set_injection": (ctypes.c_int, [_V, _F, _F, _F, ctypes.c_int]),
            "qvti_rtm_shot": (ctypes.c_int, [ctypes.POINTER(Config), _F, _F, _F, _F, _F, _F, _F, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_int, ctypes.c_int, _F, ctypes.c_int, ctypes.c_int,
                                             _I, _I, ctypes.c_int, _F, _F, _F, ctypes.POINTER(RtmOpts), _F, _F]),
            "qvti_server_create": (ctypes.c_int, [ctypes.POINTER(SchedOpts), ctypes.POINTER(_V)]),
            "qvti_server_submit": (ctypes.c_int, [_V, ctypes.POINTER(Shot), ctypes.POINTER(ctypes.c_longlong)]),
            "qvti_server_wait": (ctypes.c_int, [_V, ctypes.c_longlong, ctypes.c_double,
                                                ctypes.POINTER(ShotResult)]),
            "qvti_server_load": (ctypes.c_int, [_V, _I, _I, ctypes.POINTER(ctypes.c_size_t)]),
            "qvti_server_destroy": (ctypes.c_int, [_V]),
            "qvti_run_batch": (ctypes.c_int, [ctypes.POINTER(Shot), ctypes.c_int, ctypes.POINTER(SchedOpts),
                                              ctypes.POINTER(ShotResult), _D]),
            "qvti_autotune": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.c_int, ctypes.c_int, _I, _I, _D]),
            "qvti_autotune_ex": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.c_int, ctypes.c_int,
                                                ctypes.POINTER(Tuning)]),
            "qvti_last_error": (ctypes.c_int, []),
            "qvti_error_string": (ctypes.c_char_p, [ctypes.c_int]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(rc, what):
    if rc != 0:
        raise QvtiError("%s failed: %s (%d)" % (what, lib().qvti_error_string(rc).decode(), rc))


def _fp(a):
    return None if a is None else a.ctypes.data_as(_F)


def _f32(a, shape=None):
    a = np.asarray(a, np.float32)
    if shape is not None and a.ndim == 0:
        a = np.full(shape, a, np.float32)
    return np.ascontiguousarray(a)


def footprint_bytes(ntx, nty, ntz, pml, vti=False):
    return int(lib().qvti_footprint_bytes(ntx, nty, ntz, int(pml), 1 if vti else 0))


class Simulation:
    """One shot on one GPU: grid, model, source, receivers, wavefield state."""

    def __init__(self, ntx, nty, ntz, pml, dx, dy, dz, dt, f0, vti=False, device=0, w0=0.0):
        self.shape = (int(ntx), int(nty), int(ntz))
        self.vti = bool(vti)
        cfg = Config(int(ntx), int(nty), int(ntz), int(pml), float(dx), float(dy), float(dz), float(dt), float(f0),
                     1 if vti else 0, int(device), float(w0))
        h = _V()
        _check(lib().qvti_create(ctypes.byref(cfg), ctypes.byref(h)), "qvti_create")
        self._h = h
        self.rn = 0
        self.nt = 0

    def close(self):
        if getattr(self, "_h", None):
            lib().qvti_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_model(self, velp, vels, rho, gama_p, gama_s, eps=None, delta=None):
        sh = self.shape
        arrs = [_f32(a, sh) for a in (velp, vels, rho, gama_p, gama_s)]
        e = _f32(eps, sh) if self.vti else None
        d = _f32(delta, sh) if self.vti else None
        for a in arrs:
            if a.shape != sh:
                raise QvtiError("model array shape %s != grid %s" % (a.shape, sh))
        _check(lib().qvti_set_model(self._h, *[_fp(a) for a in arrs], _fp(e), _fp(d), 0), "qvti_set_model")

    def set_model_device(self, ptrs):
        """ptrs: device addresses (ints) of velp, vels, rho, gama_p, gama_s[, eps, delta]."""
        p = [ctypes.cast(ctypes.c_void_p(int(x)), _F) for x in ptrs] + [None] * (7 - len(ptrs))
        _check(lib().qvti_set_model(self._h, *p, 1), "qvti_set_model")

    def set_source(self, s_ix, s_iy, s_iz, wavelet, kind=SRC_FORCE_X):
        w = _f32(wavelet)
        self.nt = w.size
        _check(lib().qvti_set_source(self._h, int(kind), int(s_ix), int(s_iy), int(s_iz), _fp(w), w.size),
               "qvti_set_source")

    def set_receivers(self, r_iz, r_ix, r_iy):
        rx = np.ascontiguousarray(r_ix, np.int32)
        ry = np.ascontiguousarray(r_iy, np.int32)
        self.rn = rx.size
        _check(lib().qvti_set_receivers(self._h, int(r_iz), rx.ctypes.data_as(_I), ry.ctypes.data_as(_I), rx.size),
               "qvti_set_receivers")

    def set_form(self, form):
        """FORM_PLAIN or FORM_TC (qvti_set_form)."""
        _check(lib().qvti_set_form(self._h, int(form)), "qvti_set_form")

    def set_tiles(self, tiles):
        """Per-kernel tiles, NUM_TILES ints, 0 = default (qvti_set_tiles)."""
        t = (ctypes.c_int * NUM_TILES)(*[int(v) for v in tiles])
        _check(lib().qvti_set_tiles(self._h, t), "qvti_set_tiles")

    def tiles(self):
        """(tiles the step launches take, runtime-kernel flags) (qvti_get_tiles)."""
        t, r = (ctypes.c_int * NUM_TILES)(), (ctypes.c_int * NUM_TILES)()
        _check(lib().qvti_get_tiles(self._h, t, r), "qvti_get_tiles")
        return list(t), list(r)

    def autotune_tiles(self, probe_steps=3):
        """qvti_autotune_tiles: (chosen settings, their ms per kernel)."""
        b, m = (ctypes.c_int * NUM_TILES)(), (ctypes.c_float * NUM_TILES)()
        _check(lib().qvti_autotune_tiles(self._h, int(probe_steps), b, m), "qvti_autotune_tiles")
        return list(b), list(m)

    def set_media(self, media):
        """MEDIA_* (qvti_set_media); call before set_model."""
        _check(lib().qvti_set_media(self._h, int(media)), "qvti_set_media")

    def set_injection(self, vx=None, vy=None, vz=None):
        """Time-reversed traces ([nt, rn] each, any may be None) added at the
        receivers from the next step on (qvti_set_injection)."""
        arrs = [None if a is None else _f32(a) for a in (vx, vy, vz)]
        nt = next(a.shape[0] for a in arrs if a is not None)
        _check(lib().qvti_set_injection(self._h, *[_fp(a) for a in arrs], int(nt)), "qvti_set_injection")

    def reset(self):
        _check(lib().qvti_reset(self._h), "qvti_reset")

    def step(self, n=1):
        _check(lib().qvti_step(self._h, int(n)), "qvti_step")

    def step_timed(self, n):
        ms = ctypes.c_float(0)
        _check(lib().qvti_step_timed(self._h, int(n), ctypes.byref(ms)), "qvti_step_timed")
        return ms.value

    def sync(self):
        _check(lib().qvti_sync(self._h), "qvti_sync")

    @property
    def steps_done(self):
        return lib().qvti_steps_done(self._h)

    def records(self):
        n = self.steps_done
        out = np.zeros((3, n, self.rn), np.float32)
        _check(lib().qvti_get_records(self._h, _fp(out[0]), _fp(out[1]), _fp(out[2])), "qvti_get_records")
        return out

    def fields(self, first=0, count=9):
        out = np.zeros((count,) + self.shape, np.float32)
        _check(lib().qvti_get_fields(self._h, int(first), int(count), _fp(out)), "qvti_get_fields")
        return out

    def device_field(self, which):
        p = _F()
        _check(lib().qvti_device_field(self._h, int(which), ctypes.byref(p)), "qvti_device_field")
        return ctypes.cast(p, ctypes.c_void_p).value

    def norms(self):
        out = np.zeros(9)
        bad = ctypes.c_int(0)
        rc = lib().qvti_field_norms(self._h, out.ctypes.data_as(_D), ctypes.byref(bad))
        return out, bool(bad.value), rc

    def save_state(self):
        """Snapshot of the time-stepping state (qvti_save_state) as a uint8 array."""
        n = ctypes.c_size_t(0)
        _check(lib().qvti_state_bytes(self._h, ctypes.byref(n)), "qvti_state_bytes")
        buf = np.empty(n.value, np.uint8)
        _check(lib().qvti_save_state(self._h, buf.ctypes.data_as(_V), buf.size), "qvti_save_state")
        return buf

    def load_state(self, buf):
        """Resume from a snapshot taken by save_state (after set_source/set_receivers)."""
        b = np.ascontiguousarray(buf, np.uint8)
        _check(lib().qvti_load_state(self._h, b.ctypes.data_as(_V), b.size), "qvti_load_state")

    def profile_step(self, nrep=3):
        """Per-kernel device time of one step: list of (name, ms, algorithmic bytes)."""
        maxk = 32
        names = ctypes.create_string_buffer(32 * maxk)
        ms = np.zeros(maxk, np.float32)
        by = np.zeros(maxk, np.float64)
        nk = ctypes.c_int(0)
        _check(lib().qvti_profile_step(self._h, int(nrep), maxk, ctypes.byref(nk), names, _fp(ms), by.ctypes.data_as(_D)),
               "qvti_profile_step")
        raw = names.raw
        return [(raw[32 * i:32 * i + 32].split(b"\0")[0].decode(), float(ms[i]), float(by[i])) for i in range(nk.value)]

    def q_derivative(self, field, axis, forward, power):
        """Re IFFT3(|k|^power T_axis FFT3(field)) / ntp (one constant-Q field)."""
        f = _f32(field)
        out = np.zeros_like(f)
        _check(lib().qvti_q_derivative(self._h, int(axis), 1 if forward else 0, int(power), _fp(f), _fp(out)),
               "qvti_q_derivative")
        return out

    def derivative_1d(self, field, axis, forward):
        f = _f32(field)
        out = np.zeros_like(f)
        _check(lib().qvti_derivative_1d(self._h, int(axis), 1 if forward else 0, _fp(f), _fp(out)),
               "qvti_derivative_1d")
        return out


def q_derivative_noalloc(d_in, d_out, shape, spacing, axis, forward, power, stream=0):
    """Allocation-free constant-Q derivative of a device array (addresses as
    ints) into a device array, asynchronous on `stream` (a cudaStream_t value;
    0 = default stream).  For callers that cannot allocate device memory; the
    library's fixed scratch limits the grid (see include/qvti.h)."""
    _check(lib().qvti_q_derivative_noalloc(_V(int(d_in)), _V(int(d_out)), int(shape[0]), int(shape[1]),
                                           int(shape[2]), float(spacing[0]), float(spacing[1]), float(spacing[2]),
                                           int(axis), 1 if forward else 0, int(power), _V(int(stream))),
           "qvti_q_derivative_noalloc")


def rtm_shot(c, obs, media=MEDIA_VISCOELASTIC, snap_every=5, illum_eps=1e-3, vti=False, src_type=SRC_FORCE_X,
             ref_offset=True, device=0):
    """Reverse-time migration of one shot (qvti_rtm_shot): case c gives the
    migration model, source and receivers; obs = [3, nt, rn] observed records
    (None entries are not injected).  Returns (cross-correlation image,
    source-normalised image), each [ntx, nty, ntz]."""
    shape = (int(c["ntx"]), int(c["nty"]), int(c["ntz"]))
    keep = [_f32(c[k], shape) for k in ("velp", "vels", "rho", "gama_p", "gama_s")]
    keep += [_f32(c["eps"], shape), _f32(c["delta"], shape)] if vti else [None, None]
    rik = _f32(c["rik"])
    nt = rik.size
    rx = np.ascontiguousarray(c["r_ix"], np.int32)
    ry = np.ascontiguousarray(c["r_iy"], np.int32)
    ob = [None if o is None else _f32(o) for o in obs]
    cfg = Config(*shape, int(c["pml"]), float(c["dx"]), float(c["dy"]), float(c["dz"]), float(c["dt"]),
                 float(c["f0"]), 1 if vti else 0, int(device), 0.0)
    opts = RtmOpts(int(media), int(snap_every), float(illum_eps))
    im = np.zeros(shape, np.float32)
    imn = np.zeros(shape, np.float32)
    _check(lib().qvti_rtm_shot(ctypes.byref(cfg), *[_fp(a) for a in keep], int(src_type), int(c["s_ix"]),
                               int(c["s_iy"]), int(c["s_iz"]) + (10 if ref_offset else 0), _fp(rik), nt,
                               int(c["r_iz"]), rx.ctypes.data_as(_I), ry.ctypes.data_as(_I), rx.size,
                               *[_fp(o) for o in ob], ctypes.byref(opts), _fp(im), _fp(imn)), "qvti_rtm_shot")
    return im, imn


def simulation_for_case(c, vti=False, device=0):
    return Simulation(c["ntx"], c["nty"], c["ntz"], c["pml"], c["dx"], c["dy"], c["dz"], c["dt"], c["f0"],
                      vti=vti, device=device)


def run_case(c, nt=None, snaps=(), src_type=SRC_FORCE_X, vti=False, ref_offset=True, device=0, want_state=False,
             form=FORM_PLAIN, media=MEDIA_VISCOELASTIC, tiles=None):
    """Run a shot described by a case dict (tests/qvti_cases.py conventions).

    Returns dict(rec=[3, nt, rn], snaps={k: [3, ...]}, state=[9, ...] or None).
    ``ref_offset`` adds the reference's +10 to s_iz (cuviscoelas_3D.cu:772);
    ``form`` selects the transforms' form (FORM_PLAIN, FORM_TC), ``media``
    the medium (MEDIA_*), ``tiles`` the per-kernel tiles (set_tiles)."""
    nt = int(c["nt"] if nt is None else nt)
    snaps = sorted(int(s) for s in snaps)
    with simulation_for_case(c, vti=vti, device=device) as sim:
        if form != FORM_PLAIN:
            sim.set_form(form)
        if media != MEDIA_VISCOELASTIC:
            sim.set_media(media)
        if tiles is not None:
            sim.set_tiles(tiles)
        sim.set_model(c["velp"], c["vels"], c["rho"], c["gama_p"], c["gama_s"],
                      c.get("eps") if vti else None, c.get("delta") if vti else None)
        sim.set_receivers(c["r_iz"], c["r_ix"], c["r_iy"])
        sim.set_source(c["s_ix"], c["s_iy"], int(c["s_iz"]) + (10 if ref_offset else 0),
                       np.asarray(c["rik"], np.float32)[:nt], kind=src_type)
        sim.reset()
        out = {}
        done = 0
        for k in snaps:
            sim.step(k - done)
            done = k
            out[k] = sim.fields(0, 3)
        sim.step(nt - done)
        rec = sim.records()
        state = sim.fields(0, 9) if want_state else None
    return dict(rec=rec, snaps=out, state=state)


# ------------------------------------------------------------ batches / serving
ERR_TIMEOUT = 7


class ShotRequest:
    """A shot for qvti_run_batch / the serving loop: owns the host arrays the
    C descriptor borrows (model, wavelet, receivers, record outputs).

    ``case`` follows tests/qvti_cases.py (velp, vels, rho, gama_p, gama_s,
    optional eps/delta, rik, s_ix/s_iy/s_iz, r_iz/r_ix/r_iy, grid and
    spacing); ``ref_offset`` adds the reference's +10 to s_iz like run_case."""

    def __init__(self, c, nt=None, vti=False, src_type=SRC_FORCE_X, ref_offset=True):
        self.nt = int(c["nt"] if nt is None else nt)
        shape = (int(c["ntx"]), int(c["nty"]), int(c["ntz"]))
        self.keep = [_f32(c[k]).reshape(-1) for k in ("velp", "vels", "rho", "gama_p", "gama_s")]
        eps = _f32(c["eps"]).reshape(-1) if vti else None
        delta = _f32(c["delta"]).reshape(-1) if vti else None
        self.keep += [eps, delta]
        self.wavelet = _f32(c["rik"])[: self.nt].copy()
        self.r_ix = np.ascontiguousarray(c["r_ix"], np.int32)
        self.r_iy = np.ascontiguousarray(c["r_iy"], np.int32)
        rn = len(self.r_ix)
        self.rec = np.zeros((3, self.nt, rn), np.float32)
        d = Shot()
        d.ntx, d.nty, d.ntz, d.pml = shape + (int(c["pml"]),)
        d.dx, d.dy, d.dz, d.dt, d.f0 = (float(c[k]) for k in ("dx", "dy", "dz", "dt", "f0"))
        d.vti = 1 if vti else 0
        d.velp, d.vels, d.rho, d.gama_p, d.gama_s, d.eps, d.delta = (_fp(a) for a in self.keep)
        d.src_type = src_type
        d.s_ix, d.s_iy = int(c["s_ix"]), int(c["s_iy"])
        d.s_iz = int(c["s_iz"]) + (10 if ref_offset else 0)
        d.wavelet, d.nt = _fp(self.wavelet), self.nt
        d.r_iz, d.rn = int(c["r_iz"]), rn
        d.r_ix = self.r_ix.ctypes.data_as(_I)
        d.r_iy = self.r_iy.ctypes.data_as(_I)
        d.rec_vx, d.rec_vy, d.rec_vz = (self.rec[i].ctypes.data_as(_F) for i in range(3))
        self.desc = d
        self.cells = shape[0] * shape[1] * shape[2]


def _opts(device, mem_budget, max_active, policy=SCHED_FIFO):
    o = SchedOpts()
    o.device, o.mem_budget, o.max_active, o.policy = int(device), int(mem_budget), int(max_active), int(policy)
    return o


def run_batch(requests, max_active=0, mem_budget=0, device=0, policy=SCHED_FIFO):
    """Run ShotRequests through qvti_run_batch; returns (results, wall_s).
    Records land in each request's ``rec`` ([3, nt, rn])."""
    n = len(requests)
    arr = (Shot * n)(*[r.desc for r in requests])
    res = (ShotResult * n)()
    wall = ctypes.c_double(0)
    rc = lib().qvti_run_batch(arr, n, ctypes.byref(_opts(device, mem_budget, max_active, policy)), res,
                              ctypes.byref(wall))
    _check(rc, "qvti_run_batch")
    return [dict(status=r.status, queue_s=r.queue_s, latency_s=r.latency_s, device_ms=r.device_ms) for r in res], \
        wall.value


def autotune(ntx, nty, ntz, pml, dx, dy, dz, dt, f0, vti=False, max_active=4, probe_steps=8, device=0):
    """qvti_autotune_ex: (shots in flight, kz batch, form, Gcell-steps/s,
    per-kernel tiles)."""
    cfg = Config(ntx, nty, ntz, pml, dx, dy, dz, dt, f0, 1 if vti else 0, device, 0.0)
    t = Tuning()
    _check(lib().qvti_autotune_ex(ctypes.byref(cfg), max_active, probe_steps, ctypes.byref(t)), "qvti_autotune_ex")
    return t.active, t.kz_batch, t.form, t.gcell_steps, list(t.tiles)


class Server:
    """The continuous serving loop (qvti_server_*): submit shots while others
    run; wait for them by ticket."""

    def __init__(self, max_active=0, mem_budget=0, device=0, policy=SCHED_FIFO):
        h = _V()
        _check(lib().qvti_server_create(ctypes.byref(_opts(device, mem_budget, max_active, policy)),
                                        ctypes.byref(h)), "qvti_server_create")
        self.h = h
        self.pending = {}

    def submit(self, req):
        t = ctypes.c_longlong(0)
        _check(lib().qvti_server_submit(self.h, ctypes.byref(req.desc), ctypes.byref(t)), "qvti_server_submit")
        self.pending[t.value] = req  # keep the borrowed arrays alive
        return t.value

    def wait(self, ticket, timeout=-1.0):
        r = ShotResult()
        rc = lib().qvti_server_wait(self.h, ticket, float(timeout), ctypes.byref(r))
        if rc == ERR_TIMEOUT:
            return None
        _check(rc, "qvti_server_wait")
        self.pending.pop(ticket, None)
        return dict(status=r.status, queue_s=r.queue_s, latency_s=r.latency_s, device_ms=r.device_ms)

    def load(self):
        q, a, b = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_size_t(0)
        _check(lib().qvti_server_load(self.h, ctypes.byref(q), ctypes.byref(a), ctypes.byref(b)), "qvti_server_load")
        return q.value, a.value, b.value

    def close(self):
        if self.h:
            lib().qvti_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
