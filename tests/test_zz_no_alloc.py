"""The allocation-free entry point, qvti_q_derivative_noalloc, for callers
that cannot allocate device memory (a fixed serving footprint, a host
framework's own memory pool, a loop that cannot take cudaMalloc's device
synchronisation): its scratch lives in fixed library arrays, so the caller
only passes device input and output buffers.

Checked through the C ABI against the allocating entry point
qvti_q_derivative on the same inputs, two calls in a row (the second reuses
the scratch the first left behind), within the constant-Q derivative
tolerance of tests/test_gpu_derivative.py (relative L2 1e-5).  This file is
named to be collected last; it needs nothing from the other tests.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _rel(a, b):
    return float(np.linalg.norm(a.astype(np.float64) - b) / np.linalg.norm(b))


def test_noalloc_matches_allocating_entry_point(qvti):
    import torch

    shape = (48, 64, 96)            # half spectrum 49*48*64 values: inside the 4 MiB scratch
    spacing = (10.0, 12.5, 8.0)
    rng = np.random.default_rng(11)
    calls = [(0, True, -1), (2, False, 1)]
    fields = [rng.standard_normal(shape).astype(np.float32) for _ in calls]

    with qvti.Simulation(*shape, 6, *spacing, 1e-3, 20.0) as sim:
        expected = [sim.q_derivative(f, a, fw, pw) for f, (a, fw, pw) in zip(fields, calls)]

    d_in = torch.empty(shape, dtype=torch.float32, device="cuda")
    d_out = torch.empty(shape, dtype=torch.float32, device="cuda")
    for f, (a, fw, pw), exp in zip(fields, calls, expected):
        d_in.copy_(torch.from_numpy(f))
        d_out.fill_(float("nan"))
        torch.cuda.synchronize()
        qvti.q_derivative_noalloc(d_in.data_ptr(), d_out.data_ptr(), shape, spacing, a, fw, pw, stream=0)
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()
        assert np.isfinite(got).all()
        assert _rel(got, exp.astype(np.float64)) <= TOL


def test_noalloc_rejects_grids_beyond_its_scratch(qvti):
    import torch

    d = torch.empty(16, dtype=torch.float32, device="cuda")   # never touched: rejected first
    with pytest.raises(qvti.QvtiError, match="unsupported"):
        qvti.q_derivative_noalloc(d.data_ptr(), d.data_ptr(), (128, 128, 128), (10.0, 10.0, 10.0), 0, True, 0)
    assert qvti.lib().qvti_last_error() == 3  # QVTI_ERR_UNSUPPORTED, reported like every other entry point
    with pytest.raises(qvti.QvtiError, match="invalid argument"):
        qvti.q_derivative_noalloc(d.data_ptr(), d.data_ptr(), (32, 32, 32), (10.0, 10.0, 10.0), 3, True, 0)
    assert qvti.lib().qvti_last_error() == 1  # QVTI_ERR_ARG


def test_noalloc_matches_fp64_numpy(qvti, oracle):
    """The allocation-free derivative against an FP64 numpy restatement of
    the operator itself (tests/test_gpu_derivative.py: Re IFFT3(|k|^p T(k_a)
    FFT3(f)) with the oracle's k-space tables), not only against the
    allocating entry point."""
    import torch
    from test_gpu_derivative import _numpy_q_derivative

    shape, spacing = (32, 48, 40), (10.0, 8.0, 12.0)
    rng = np.random.default_rng(5)
    f = rng.standard_normal(shape).astype(np.float32)
    d_in = torch.from_numpy(f).cuda()
    d_out = torch.empty_like(d_in)
    for axis, fw, pw in ((1, True, 1), (0, False, -1), (2, True, 0)):
        d_out.fill_(float("nan"))
        torch.cuda.synchronize()
        qvti.q_derivative_noalloc(d_in.data_ptr(), d_out.data_ptr(), shape, spacing, axis, fw, pw, stream=0)
        torch.cuda.synchronize()
        want = _numpy_q_derivative(f, spacing, axis, fw, pw, oracle)
        assert _rel(d_out.cpu().numpy(), want) <= TOL
