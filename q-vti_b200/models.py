"""Seeded synthetic models and shot geometry for the benchmark configurations.

The reference reads its model from a raw float32 file that is not part of
the project (viscoelas_3D.cpp:541) and overrides vs/Q/rho with constants
(viscoelas_3D.cpp:658-677); the measured configurations are synthetic:

* ``layered_vti`` -- the 256^3 VTI workload: 6 equal-thickness horizontal
  layers in z with Vp 1800..4500 m/s increasing with depth, Vs = Vp/1.8,
  Gardner density rho = 310 Vp^0.25, per layer Thomsen eps ~ U[0.05, 0.25],
  delta ~ U[0, 0.12], Qp ~ U[30, 200], Qs = Qp/2, then every field multiplied
  by (1 + 0.05 g) with g an independent unit-variance Gaussian random field of
  80 m Gaussian correlation length (white noise convolved with a Gaussian of
  standard deviation L/2; exp(-r^2/L^2) correlation).
* ``stable_dt`` -- the staggered pseudospectral leapfrog bound
  (dt/2) |k|max v_eff <= 1 with |k|max = pi sqrt(1/dx^2+1/dy^2+1/dz^2) and
  v_eff the fastest phase velocity including the constant-Q dispersion
  factor at |k|max; the generator's dt is capped to 80 % of it when the
  nominal dt would be unstable (a stated deviation of the workload).
"""
import math

import numpy as np

PI_REF = 3.1415926


def gamma_of_q(q):
    """gamma = atan(1/Q)/pi (viscoelas_3D.cpp:287-288)."""
    return (np.arctan(1.0 / np.asarray(q, np.float64)) / PI_REF).astype(np.float32)


def ricker(nt, dt, f0):
    """Ricker wavelet with the reference's arithmetic (viscoelas_3D.cpp:494-502)."""
    t = (np.arange(nt).astype(np.float32) * np.float32(dt)).astype(np.float32)
    arg = (t - np.float32(1.0) / np.float32(f0)).astype(np.float32).astype(np.float64)
    tau = (PI_REF * float(np.float32(f0)) * arg) ** 2
    return ((1.0 - 2.0 * tau) * np.exp(-tau)).astype(np.float32)


def gaussian_field(shape, corr_cells, rng):
    """Unit-variance Gaussian random field with Gaussian correlation length
    ``corr_cells`` (in cells), float32."""
    import scipy.fft as sf
    w = rng.standard_normal(shape, dtype=np.float32)
    s = corr_cells / 2.0
    k = [np.fft.fftfreq(n).astype(np.float32) for n in shape[:-1]] + [np.fft.rfftfreq(shape[-1]).astype(np.float32)]
    g = [np.exp(-2.0 * (np.pi * s) ** 2 * kk ** 2).astype(np.float32) for kk in k]
    W = sf.rfftn(w, workers=-1)
    W *= g[0][:, None, None]
    W *= g[1][None, :, None]
    W *= g[2][None, None, :]
    f = sf.irfftn(W, s=shape, workers=-1).astype(np.float32)
    f -= f.mean()
    sd = f.std()
    return f / sd if sd > 0 else f


def layered_vti(n=(256, 256, 256), d=10.0, seed=2024, nlayers=6, vp_top=1800.0, vp_bot=4500.0,
                pert=0.05, corr_m=80.0, perturb=True):
    """Return dict of float32 [ix][iy][iz] fields: velp, vels, rho, gama_p,
    gama_s, eps, delta (and qp, qs)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = n
    vp_l = np.linspace(vp_top, vp_bot, nlayers)
    eps_l = rng.uniform(0.05, 0.25, nlayers)
    del_l = rng.uniform(0.0, 0.12, nlayers)
    qp_l = rng.uniform(30.0, 200.0, nlayers)
    layer = np.minimum((np.arange(nz) * nlayers) // nz, nlayers - 1)
    prof = {
        "velp": vp_l[layer],
        "vels": vp_l[layer] / 1.8,
        "rho": 310.0 * vp_l[layer] ** 0.25,
        "eps": eps_l[layer],
        "delta": del_l[layer],
        "qp": qp_l[layer],
        "qs": 0.5 * qp_l[layer],
    }
    out = {}
    corr_cells = corr_m / d
    for i, (name, p) in enumerate(prof.items()):
        f = np.broadcast_to(p.astype(np.float32)[None, None, :], n).astype(np.float32)
        if perturb:
            g = gaussian_field(n, corr_cells, np.random.default_rng([seed, i + 1]))
            f = f * (1.0 + pert * g)
        out[name] = np.ascontiguousarray(f, np.float32)
    out["gama_p"] = gamma_of_q(out["qp"])
    out["gama_s"] = gamma_of_q(out["qs"])
    return out


def layered_profiles(nz, seed, nlayers=6, vp_top=1800.0, vp_bot=4500.0):
    """1D (depth) profiles of the layered model, with the same per-layer draws
    as layered_vti: velp, vels, rho, eps, delta, qp, qs, gama_p, gama_s."""
    rng = np.random.default_rng(seed)
    vp_l = np.linspace(vp_top, vp_bot, nlayers)
    eps_l = rng.uniform(0.05, 0.25, nlayers)
    del_l = rng.uniform(0.0, 0.12, nlayers)
    qp_l = rng.uniform(30.0, 200.0, nlayers)
    layer = np.minimum((np.arange(nz) * nlayers) // nz, nlayers - 1)
    p = dict(velp=vp_l[layer], vels=vp_l[layer] / 1.8, rho=310.0 * vp_l[layer] ** 0.25, eps=eps_l[layer],
             delta=del_l[layer], qp=qp_l[layer], qs=0.5 * qp_l[layer])
    p = {k: v.astype(np.float32) for k, v in p.items()}
    p["gama_p"] = gamma_of_q(p["qp"])
    p["gama_s"] = gamma_of_q(p["qs"])
    return p


MODEL_FIELDS = ("velp", "vels", "rho", "gama_p", "gama_s", "eps", "delta")


def layered_fast(n, seed, vti=True, nlayers=6):
    """Unperturbed layered model built by broadcasting its depth profiles
    (the serving workload's "seeded layered models"): float32 [ix][iy][iz]."""
    p = layered_profiles(n[2], seed, nlayers)
    out = {}
    for k in MODEL_FIELDS[:5] + (MODEL_FIELDS[5:] if vti else ()):
        a = np.empty(n, np.float32)
        a[...] = p[k][None, None, :]
        out[k] = a
    return out


def perturbation_bases(n, seed, corr_m=80.0, d=10.0):
    """One unit Gaussian random field per model property for grid n, to be
    shared (shifted) by many shots of that grid (perturbed_layered)."""
    return {k: gaussian_field(n, corr_m / d, np.random.default_rng([seed, i + 1]))
            for i, k in enumerate(("velp", "vels", "rho", "eps", "delta", "qp", "qs"))}


def perturbed_layered(n, seed, bases, shift, pert=0.05, vti=True):
    """Layered model with this shot's own layer draws, perturbed by 5 % std
    with the grid's shared Gaussian fields rolled by `shift` cells."""
    p = layered_profiles(n[2], seed)
    out = {}
    for k in ("velp", "vels", "rho", "eps", "delta", "qp", "qs"):
        if k in ("eps", "delta") and not vti:
            continue
        g = np.roll(bases[k], tuple(int(x) for x in shift), axis=(0, 1, 2))
        out[k] = np.ascontiguousarray(p[k][None, None, :] * (1.0 + pert * g), np.float32)
    out["gama_p"] = gamma_of_q(out.pop("qp"))
    out["gama_s"] = gamma_of_q(out.pop("qs"))
    return out


def smooth_even(x, lo=16):
    """Nearest even 5-smooth integer (2^a 3^b 5^c) to x, at least lo."""
    best = None
    for m in range(max(lo, int(x * 0.8)), int(x * 1.25) + 2):
        if m % 2:
            continue
        r = m
        for f in (2, 3, 5):
            while r % f == 0:
                r //= f
        if r == 1 and (best is None or abs(m - x) < abs(best - x)):
            best = m
    return best


def stable_dt(model, d, f0, vti=True):
    """Largest stable dt of the staggered PS leapfrog for this model."""
    dx, dy, dz = (d, d, d) if np.isscalar(d) else d
    kmax = PI_REF * math.sqrt(1 / dx ** 2 + 1 / dy ** 2 + 1 / dz ** 2)
    w0 = 2 * PI_REF * f0
    vp = model["velp"].astype(np.float64)
    g = model["gama_p"].astype(np.float64)
    if vti:
        ani = np.maximum(np.maximum(model["eps"], model["delta"]), 0).astype(np.float64)
        v = vp * np.sqrt(1.0 + 2.0 * ani)
    else:
        v = vp
    c = v * np.cos(g * PI_REF / 2)
    x = c * kmax / w0
    disp = np.maximum(1.0 + g * (x - 1.0 / x), 1.0)
    veff = float((c * np.sqrt(disp)).max())
    return 2.0 / (kmax * veff), veff


def choose_dt(model, d, f0, dt_nominal, vti=True, safety=0.8):
    """dt_nominal if stable, else the largest multiple of 0.05 ms below
    safety x the stability bound."""
    lim, veff = stable_dt(model, d, f0, vti)
    if dt_nominal <= safety * lim:
        return dt_nominal, lim, veff
    dt = math.floor(safety * lim / 5e-5) * 5e-5
    return dt, lim, veff


def surface_receivers(nx, ny):
    """All nx*ny horizontal points, receiver ir = ix*ny + iy (cuviscoelas_3D.cu:787)."""
    ix, iy = np.meshgrid(np.arange(nx, dtype=np.int32), np.arange(ny, dtype=np.int32), indexing="ij")
    return ix.ravel().copy(), iy.ravel().copy()
