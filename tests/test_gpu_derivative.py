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
