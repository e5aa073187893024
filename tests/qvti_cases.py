"""Seeded test cases shared by the golden-fixture generator and the tests.

A case is a plain dict of numpy arrays and scalars describing one shot in the
reference's conventions (viscoelas_3D.cpp / cuviscoelas_3D.cu):

* grid ``ntx, nty, ntz`` is the total padded grid, PML inside, ``pml`` cells
  on every face; fields are float32 ``[ix][iy][iz]`` with z fastest
  (ip = ix*nty*ntz + iy*ntz + iz, cuviscoelas_3D.cu:176);
* model: ``velp, vels, rho`` and the constant-Q exponents ``gama_p, gama_s``
  with gamma = atan(1/Q)/pi (viscoelas_3D.cpp:285-289);
* source: Ricker wavelet ``rik`` (viscoelas_3D.cpp:494-502) injected into vx
  at (s_ix, s_iy, s_iz + 10) -- the reference's own offset
  (cuviscoelas_3D.cu:772);
* receivers: ``r_ix, r_iy`` (padded indices, rnx_max*rny_max of them, receiver
  ir = ix*rny_max + iy) at depth index ``r_iz`` (cuviscoelas_3D.cu:782-791).
"""
import numpy as np

PI_REF = 3.1415926  # the reference's truncated pi (viscoelas_3D.cpp:14, cuviscoelas_3D.cu:15)


def ricker(nt, dt, f0):
    """Ricker wavelet with the reference's arithmetic (viscoelas_3D.cpp:494-502).

    ``it*dt`` and ``1/f0`` are float32 in the reference; the square and the
    exponential are evaluated in double and the result rounded to float32.
    """
    it = np.arange(nt, dtype=np.int64)
    t = (it.astype(np.float32) * np.float32(dt)).astype(np.float32)
    inv = np.float32(1.0) / np.float32(f0)
    arg = (t - inv).astype(np.float32).astype(np.float64)
    tmp = (PI_REF * float(np.float32(f0)) * arg) ** 2
    return ((1.0 - 2.0 * tmp) * np.exp(-tmp)).astype(np.float32)


def gamma_of_q(q):
    """gamma = atan(1/Q)/pi with the reference's pi (viscoelas_3D.cpp:287-288)."""
    q = np.asarray(q, dtype=np.float64)
    return (np.arctan(1.0 / q) / PI_REF).astype(np.float32)


def _smooth_field(rng, shape, corr_cells):
    """Zero-mean, unit-std Gaussian random field smoothed by a Gaussian kernel."""
    w = rng.standard_normal(shape)
    k = [np.fft.fftfreq(n) for n in shape]
    kx, ky, kz = np.meshgrid(*k, indexing="ij")
    s = corr_cells / 2.0
    filt = np.exp(-2.0 * (np.pi * s) ** 2 * (kx ** 2 + ky ** 2 + kz ** 2))
    f = np.real(np.fft.ifftn(np.fft.fftn(w) * filt))
    f -= f.mean()
    sd = f.std()
    return f / sd if sd > 0 else f


def homogeneous_case(n=(32, 32, 32), pml=8, d=(10.0, 10.0, 10.0), dt=1e-3, nt=120, f0=25.0,
                     vp=2500.0, vs=1443.0, rho=2000.0, qp=100.0, qs=50.0,
                     src=None, r_iz=None, name="homog"):
    ntx, nty, ntz = n
    shape = (ntx, nty, ntz)
    src = src if src is not None else (ntx // 2, nty // 2, ntz // 2)
    r_iz = r_iz if r_iz is not None else pml + 2
    r_ix = np.arange(ntx, dtype=np.int32)
    r_iy = np.full(ntx, nty // 2, dtype=np.int32)
    return dict(
        name=name, ntx=ntx, nty=nty, ntz=ntz, pml=pml, nt=nt,
        dx=d[0], dy=d[1], dz=d[2], dt=dt, f0=f0,
        velp=np.full(shape, vp, np.float32), vels=np.full(shape, vs, np.float32),
        rho=np.full(shape, rho, np.float32),
        gama_p=np.full(shape, gamma_of_q(qp), np.float32),
        gama_s=np.full(shape, gamma_of_q(qs), np.float32),
        rik=ricker(nt, dt, f0),
        s_ix=src[0], s_iy=src[1], s_iz=src[2] - 10, r_iz=r_iz,
        r_ix=r_ix, r_iy=r_iy, rnx_max=ntx, rny_max=1,
    )


def heterogeneous_case(n=(24, 40, 32), pml=6, d=(12.0, 10.0, 8.0), dt=0.8e-3, nt=100, f0=30.0,
                       seed=7, src=(12, 20, 16), r_iz=8, name="hetero"):
    """Smooth random isotropic model (vp 2000-3000 m/s, Q 30-200)."""
    ntx, nty, ntz = n
    shape = (ntx, nty, ntz)
    rng = np.random.default_rng(seed)
    vp = 2500.0 + 250.0 * np.clip(_smooth_field(rng, shape, 4.0), -2, 2)
    vs = vp / (1.6 + 0.1 * np.clip(_smooth_field(rng, shape, 4.0), -2, 2))
    rho = 2100.0 + 150.0 * np.clip(_smooth_field(rng, shape, 4.0), -2, 2)
    qp = 115.0 + 42.0 * np.clip(_smooth_field(rng, shape, 4.0), -2, 2)
    qs = 0.5 * qp
    rnx, rny = 4, 5
    gx = np.linspace(pml, ntx - pml - 1, rnx).astype(np.int32)
    gy = np.linspace(pml, nty - pml - 1, rny).astype(np.int32)
    r_ix = np.repeat(gx, rny).astype(np.int32)
    r_iy = np.tile(gy, rnx).astype(np.int32)
    return dict(
        name=name, ntx=ntx, nty=nty, ntz=ntz, pml=pml, nt=nt,
        dx=d[0], dy=d[1], dz=d[2], dt=dt, f0=f0,
        velp=vp.astype(np.float32), vels=vs.astype(np.float32), rho=rho.astype(np.float32),
        gama_p=gamma_of_q(qp), gama_s=gamma_of_q(qs),
        rik=ricker(nt, dt, f0),
        s_ix=src[0], s_iy=src[1], s_iz=src[2] - 10, r_iz=r_iz,
        r_ix=r_ix, r_iy=r_iy, rnx_max=rnx, rny_max=rny,
    )


def config1_case(nt=500):
    """Small isotropic homogeneous cube 96^3, 20-cell C-PML, 500 steps (the
    reference-runnable case): Vp 2500, Vs 1443, rho 2000, Qp 100, Qs 50,
    25 Hz Ricker at the centre, 96 receivers on a line at depth index 25."""
    c = homogeneous_case(n=(96, 96, 96), pml=20, d=(10.0, 10.0, 10.0), dt=1e-3, nt=nt, f0=25.0,
                         src=(48, 48, 48), r_iz=25, name="config1")
    return c


def relL2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a - b))


def snapshot_error(ours, ref, peak):
    """Error of one field of a snapshot plane against its reference: relative
    L2, except where the reference field is below 1 % of `peak` -- the
    largest norm of the whole wavefield (vx, vy, vz together) on that plane
    over the run -- where the L2 error is taken relative to that peak
    instead.  Two cases reach it: a component that vanishes by symmetry on
    the plane (vy through an x-directed or an explosive source), and a
    field that has decayed after the wave left through the C-PML.  There
    relative L2 measures FP32 rounding, not the scheme: the reference's own
    cuFFT build differs from the FP64 oracle by 1.1e-3 relative L2 on the
    96^3 configuration's plane at step 500, where the field is 5e-4 of its
    peak, against 2.5e-6..1.7e-5 at steps 100-400."""
    a = np.asarray(ours, np.float64)
    b = np.asarray(ref, np.float64)
    nb = np.linalg.norm(b)
    d = np.linalg.norm(a - b)
    return d / max(nb, 1e-2 * peak) if peak > 0 else d


def plane_peak(planes):
    """Largest norm of a wavefield plane ([3, ...] per snapshot) over a run."""
    return max(float(np.linalg.norm(np.asarray(p, np.float64))) for p in planes)
