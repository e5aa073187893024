"""The 1D staggered spectral derivative (the building block of the velocity
update and of every transform) against numpy's FFT with the oracle's FP64
shift tables.  Tolerance: max error <= 2e-5 of the field's derivative scale."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _numpy_derivative(f, axis, d, forward, oracle):
    n = f.shape[axis]
    fw, bw = oracle.shift_tables(n, d)
    T = (fw if forward else bw).copy()
    if n % 2 == 0:
        T[n // 2] = T[n // 2].real  # the Hermitian part seen by the real output
    sh = [1, 1, 1]
    sh[axis] = n
    F = np.fft.fft(f.astype(np.float64), axis=axis)
    return np.real(np.fft.ifft(F * T.reshape(sh), axis=axis))


@pytest.mark.parametrize("shape", [(32, 48, 64), (96, 40, 24), (16, 20, 30)])
@pytest.mark.parametrize("axis", [0, 1, 2])
@pytest.mark.parametrize("forward", [True, False])
def test_derivative_1d(qvti, oracle, shape, axis, forward):
    rng = np.random.default_rng(1 + axis + 7 * forward)
    f = rng.standard_normal(shape).astype(np.float32)
    d = (10.0, 12.5, 8.0)
    with qvti.Simulation(*shape, 4, *d, 1e-3, 20.0) as sim:
        out = sim.derivative_1d(f, axis, forward)
    ref = _numpy_derivative(f, axis, d[axis], forward, oracle)
    err = np.abs(out - ref).max() / np.abs(ref).max()
    assert err < 2e-5, err


def _numpy_q_derivative(f, d, axis, forward, power, oracle):
    """Re IFFT3(|k|^power T(k_axis) FFT3(f)) in FP64 (cuviscoelas_3D.cu:188-190, 475-744)."""
    n = f.shape
    ks = [oracle.wavenumbers(n[a], d[a]) for a in range(3)]
    k2 = ks[0][:, None, None] ** 2 + ks[1][None, :, None] ** 2 + ks[2][None, None, :] ** 2
    k2[0, 0, 0] = 1e-10
    ap = k2 ** (0.5 * power)
    fw, bw = oracle.shift_tables(n[axis], d[axis])
    T = (fw if forward else bw).copy()
    if n[axis] % 2 == 0:
        T[n[axis] // 2] = T[n[axis] // 2].real
    sh = [1, 1, 1]
    sh[axis] = n[axis]
    F = np.fft.fftn(f.astype(np.float64))
    return np.real(np.fft.ifftn(F * ap * T.reshape(sh)))


@pytest.mark.parametrize("power", [-1, 0, 1])
@pytest.mark.parametrize("axis,forward", [(0, True), (1, False), (2, True), (2, False)])
def test_q_derivative(qvti, oracle, power, axis, forward):
    shape = (32, 48, 64)
    d = (10.0, 12.5, 8.0)
    rng = np.random.default_rng(3 + power + 5 * axis)
    f = rng.standard_normal(shape).astype(np.float32)
    with qvti.Simulation(*shape, 6, *d, 1e-3, 20.0) as sim:
        out = sim.q_derivative(f, axis, forward, power)
    ref = _numpy_q_derivative(f, d, axis, forward, power, oracle)
    err = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    assert err < 1e-5, err


@pytest.mark.parametrize("shape", [(48, 64, 96), (64, 64, 64)])
def test_q_derivative_repeated_calls(qvti, oracle, shape):
    """Several calls on one simulation: each call's upload must land before
    its transforms read it (the uploads are ordered on the simulation's
    stream)."""
    d = (10.0, 12.5, 8.0)
    rng = np.random.default_rng(17)
    with qvti.Simulation(*shape, 6, *d, 1e-3, 20.0) as sim:
        for axis, forward, power in [(0, True, -1), (2, False, 1), (1, True, 0), (0, True, -1)]:
            f = rng.standard_normal(shape).astype(np.float32)
            out = sim.q_derivative(f, axis, forward, power)
            ref = _numpy_q_derivative(f, d, axis, forward, power, oracle)
            err = np.linalg.norm(out - ref) / np.linalg.norm(ref)
            assert err < 1e-5, (axis, forward, power, err)
