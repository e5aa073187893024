"""The split-precision tensor-core form (qvti_set_form(QVTI_FORM_TC)): the
256-point y transforms run as 16-point DFT matrix products on tcgen05 with
TF32 hi/lo operands (three products, FP32 accumulation in TMEM).

Same tolerance as the plain form against the FP64 oracle (relative L2
<= 1e-4 on every seismogram component and snapshot field), and close to the
plain form's own result; grids without a 256-point y axis are rejected.
"""
import numpy as np
import pytest

import qvti_cases as qc
from test_gpu_parity import TOL, _compare, _ct_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [(16, 256, 24), (24, 256, 20)])
def test_tc_form_against_oracle(qvti, oracle, n):
    """Both y passes (forward with the y derivatives, inverse over the 21
    fields) on the tensor cores; VTI, heterogeneous, 120 steps.  ny = 256
    with 16 x 24 or 24 x 20 other axes: 31 or 45 lines per kz batch edge,
    so the 8-line tiles are ragged too."""
    nt = 120
    c = _ct_case(n, nt, pml=4)
    ours = qvti.run_case(c, snaps=[60, nt], vti=True, form=qvti.FORM_TC)
    ref = oracle.run_case(c, snaps=[60, nt], vti=True)
    _compare(ours, ref, "tc%dx%dx%d" % n)


def test_tc_form_close_to_plain(qvti):
    """64 x 256 x 48, 150 steps: the two forms differ by the rounding of the
    3xTF32 products only."""
    nt = 150
    c = _ct_case((64, 256, 48), nt)
    a = qvti.run_case(c, snaps=[nt], vti=True, form=qvti.FORM_TC)
    b = qvti.run_case(c, snaps=[nt], vti=True)
    for i in range(3):
        assert qc.relL2(a["rec"][i], b["rec"][i]) <= 1e-5
        assert qc.relL2(a["snaps"][nt][i], b["snaps"][nt][i]) <= 1e-5
    assert not np.array_equal(a["rec"], b["rec"])  # the tensor-core path really ran


def test_tc_form_needs_a_256_point_y_axis(qvti):
    with qvti.Simulation(32, 48, 32, 6, 10.0, 10.0, 10.0, 1e-3, 20.0) as sim:
        with pytest.raises(qvti.QvtiError, match="unsupported"):
            sim.set_form(qvti.FORM_TC)
        sim.set_form(qvti.FORM_PLAIN)
    with qvti.Simulation(32, 256, 32, 6, 10.0, 10.0, 10.0, 1e-3, 20.0) as sim:
        sim.set_form(qvti.FORM_TC)
        with pytest.raises(qvti.QvtiError, match="invalid argument"):
            sim.set_form(7)


def test_bounded_wait_reports_a_timeout_and_the_simulation_recovers(qvti):
    """The tensor-core rounds wait on an mbarrier with a time limit; when it
    runs out the kernel records QVTI_ERR_TIMEOUT in the engine's device flag
    and returns.  Exercised without a fault: a 50 ms wait on a barrier that
    nothing completes.  qvti_sync reports the timeout; after qvti_reset the
    simulation steps and records as before."""
    c = _ct_case((16, 256, 24), 40, pml=4)
    ref = qvti.run_case(c, vti=True, form=qvti.FORM_TC)["rec"]
    with qvti.simulation_for_case(c, vti=True) as sim:
        sim.set_form(qvti.FORM_TC)
        sim.set_model(c["velp"], c["vels"], c["rho"], c["gama_p"], c["gama_s"], c["eps"], c["delta"])
        sim.set_receivers(c["r_iz"], c["r_ix"], c["r_iy"])
        sim.set_source(c["s_ix"], c["s_iy"], int(c["s_iz"]) + 10, np.asarray(c["rik"], np.float32))
        sim.reset()
        qvti._check(qvti.lib().qvti_probe_bounded_wait(sim._h, 0.05), "qvti_probe_bounded_wait")
        with pytest.raises(qvti.QvtiError, match="timed out"):
            sim.sync()
        sim.reset()
        sim.step(40)
        sim.sync()
        assert np.array_equal(sim.records(), ref)
