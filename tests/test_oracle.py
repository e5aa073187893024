"""CPU tests of the FP64 oracle: its FFT, tables and coefficient builders
against independent formulas, and -- the pin -- its full shots against the
reference's own cuFFT build (golden fixtures produced by
tests/golden/make_golden.py on a GPU).
"""
import math

import numpy as np
import pytest

import qvti_cases as qc
from conftest import golden_names, load_golden, snap_keys

PI = qc.PI_REF


@pytest.mark.parametrize("shape", [(8, 6, 10), (12, 20, 7), (16, 16, 16), (24, 40, 30), (5, 9, 11)])
def test_fft_matches_numpy(oracle, shape):
    rng = np.random.default_rng(0)
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    f = oracle.fft3d(a, -1)
    assert np.abs(f - np.fft.fftn(a)).max() <= 1e-12 * np.abs(f).max()
    i = oracle.fft3d(a, +1)
    assert np.abs(i - np.fft.ifftn(a) * a.size).max() <= 1e-12 * np.abs(i).max()


def test_fft_impulse_and_tone(oracle):
    n = (12, 10, 16)
    a = np.zeros(n, complex)
    a[0, 0, 0] = 1
    assert np.allclose(oracle.fft3d(a, -1), 1.0)
    x = np.arange(16)
    a = np.broadcast_to(np.exp(2j * np.pi * 3 * x / 16), n).copy()
    f = oracle.fft3d(a, -1)
    expect = np.zeros(n, complex)
    expect[0, 0, 3] = a.size
    assert np.abs(f - expect).max() < 1e-9


@pytest.mark.parametrize("n", [16, 17, 30, 96])
def test_shift_tables(oracle, n):
    d = 12.5
    fw, bw = oracle.shift_tables(n, d)
    i = np.arange(n)
    ks = np.where(i <= n // 2, i, i - n) * 2 * PI / (n * d)  # signed, Nyquist positive
    assert np.allclose(fw, 1j * ks * np.exp(1j * ks * d / 2), atol=1e-12)
    assert np.allclose(bw, 1j * ks * np.exp(-1j * ks * d / 2), atol=1e-12)
    k = oracle.wavenumbers(n, d)
    assert np.allclose(k, np.abs(ks))


def test_spectral_derivative_of_sine(oracle):
    """d/dx sin(k x) sampled at x_i, with the forward shift, equals
    k cos(k (x_i + d/2)) (known answer for a band-limited tone; the tables use
    the reference's pi = 3.1415926, which leaves a ~1e-7 relative residue)."""
    n, d, m = 64, 10.0, 5
    x = np.arange(n) * d
    k = 2 * PI * m / (n * d)
    fw, bw = oracle.shift_tables(n, d)
    f = np.sin(k * x)
    dfw = np.real(np.fft.ifft(np.fft.fft(f) * fw))
    dbw = np.real(np.fft.ifft(np.fft.fft(f) * bw))
    assert np.abs(dfw - k * np.cos(k * (x + d / 2))).max() < 2e-6 * k
    assert np.abs(dbw - k * np.cos(k * (x - d / 2))).max() < 2e-6 * k


def test_q_coefficients(oracle):
    vel = np.array([2500.0, 1443.0], np.float32)
    q = np.array([100.0, 50.0])
    gam = qc.gamma_of_q(q)
    rho = np.array([2000.0, 2000.0], np.float32)
    f0 = 25.0
    out = oracle.q_coeffs(vel, gam, rho, f0)
    w0 = float(np.float32(2 * PI * f0))
    for i in range(2):
        g, r = float(gam[i]), float(rho[i])
        c = float(vel[i]) * math.cos(g * PI / 2)
        expect = [-r * c * g * w0, r * c * c, r * c ** 3 * g / w0, r * c * g * PI, r * c * c * g * g * PI / w0]
        assert np.allclose(out[:, i], expect, rtol=1e-12)
    # gamma = atan(1/Q)/pi
    assert abs(float(gam[0]) - math.atan(1 / 100.0) / PI) < 1e-8


def test_pml_profile(oracle):
    n, pml, d, f0 = 60, 10, 10.0, 20.0
    a, b = oracle.pml_profile(n, pml, d, f0)
    om_max = 4 * 5000.0 * math.log(100.0) / (2 * pml * d)
    assert b[0] == pytest.approx(om_max * ((pml - 1) / pml) ** 3, rel=1e-6)
    assert b[pml - 1] == 0 and b[pml] == 0 and b[n - pml] == 0
    assert a[pml] == pytest.approx(PI * f0)
    assert a[0] == pytest.approx(om_max * ((pml - 1) / pml) ** 3)  # alpha(0) = 0
    assert np.allclose(a, a[::-1]) and np.allclose(b, b[::-1])
    assert np.all(b[:pml - 1] > 0) and np.all(np.diff(b[:pml]) < 0)


def test_ricker():
    nt, dt, f0 = 200, 1e-3, 25.0
    r = qc.ricker(nt, dt, f0)
    t = np.arange(nt) * dt - 1 / f0
    tau = (PI * f0 * t) ** 2
    assert np.allclose(r, (1 - 2 * tau) * np.exp(-tau), atol=1e-6)
    assert np.argmax(r) == 40


ORACLE_VS_REF_TOL = 2e-5  # FP64 oracle vs the reference's FP32 cuFFT build


@pytest.mark.parametrize("name", [n for n in golden_names() if n != "config1"])
def test_oracle_matches_reference_golden(oracle, name):
    """The pin: the oracle reproduces the reference's own outputs."""
    c = load_golden(name)
    snaps = snap_keys(c)
    r = oracle.run_case(c, snaps=snaps, want_state=True)
    for i, comp in enumerate(("vx", "vy", "vz")):
        e = qc.relL2(r["rec"][i], c["rec_" + comp])
        assert e <= ORACLE_VS_REF_TOL, (comp, e)
    for k in snaps:
        for i in range(3):
            e = qc.relL2(r["snaps"][k][i], c["snap_%d" % k][i])
            assert e <= ORACLE_VS_REF_TOL, (k, i, e)
    for f in range(9):
        e = qc.relL2(r["state"][f], c["final9"][f])
        assert e <= ORACLE_VS_REF_TOL, (f, e)


def test_oracle_vti_zero_anisotropy_is_isotropic(oracle):
    c = qc.heterogeneous_case(n=(16, 16, 20), pml=4, nt=30, seed=2, src=(8, 8, 10), r_iz=5)
    c["eps"] = np.zeros_like(c["velp"])
    c["delta"] = np.zeros_like(c["velp"])
    a = oracle.run_case(c, vti=True)
    b = oracle.run_case(c, vti=False)
    for i in range(3):
        assert qc.relL2(a["rec"][i], b["rec"][i]) < 1e-12


def test_oracle_lossless_p_moveout(oracle):
    """Q -> infinity (gamma ~ 0): the direct P wave from an explosive source
    takes (200 m - 100 m) / vp to travel between receivers 10 and 20 cells
    away (known answer; difference of the peak times, within 3 steps)."""
    vp = 2000.0
    c = qc.homogeneous_case(n=(48, 24, 24), pml=4, d=(10.0, 10.0, 10.0), dt=1e-3, nt=170, f0=30.0,
                            vp=vp, vs=1000.0, rho=2000.0, qp=1e9, qs=1e9, src=(12, 12, 12), r_iz=12)
    c["r_ix"] = np.array([22, 32], np.int32)
    c["r_iy"] = np.array([12, 12], np.int32)
    c["rnx_max"], c["rny_max"] = 2, 1
    r = oracle.run_case(c, src_type=1, ref_offset=False)
    a, b = r["rec"][0][:, 0].astype(np.float64), r["rec"][0][:, 1].astype(np.float64)
    lag = int(np.argmax(np.abs(b))) - int(np.argmax(np.abs(a)))
    expect = 100.0 / vp / c["dt"]
    assert abs(lag - expect) <= 3, (lag, expect)


def test_oracle_attenuation_decreases_energy(oracle):
    base = dict(n=(32, 32, 32), pml=6, nt=70, f0=30.0, vp=2500.0, vs=1400.0, rho=2000.0, src=(16, 16, 16), r_iz=8)
    lo = qc.homogeneous_case(qp=20.0, qs=10.0, **base)
    hi = qc.homogeneous_case(qp=1000.0, qs=500.0, **base)
    e_lo = np.sum(oracle.run_case(lo, src_type=1, ref_offset=False, want_state=True)["state"][:3] ** 2)
    e_hi = np.sum(oracle.run_case(hi, src_type=1, ref_offset=False, want_state=True)["state"][:3] ** 2)
    assert e_lo < 0.95 * e_hi
