"""Parity on the benchmark model and on the small configuration as specified,
against FP64 oracle fixtures (tests/golden/oracle/, made by
tests/golden/make_oracle_golden.py; the oracle itself is pinned to the
reference's cuFFT build in tests/test_oracle.py).

* vti_crop128: the centred 128^3 crop of the 256^3 VTI benchmark model at the
  benchmark's dt, 400 steps (the 128-point compiled kernels, a 20-cell
  C-PML, strong heterogeneity and anisotropy over a long run).
* config1_explosive: 96^3 isotropic, explosive source at the centre, 500
  steps.
* config1_force_planes: the same grid with the reference's force source,
  the FP64 counterpart of the reference-build fixture tests/golden/config1.npz.

Tolerance: relative L2 <= 1e-4 on every seismogram component and on the vx,
vy, vz planes of every snapshot (every 100 steps), each field relative to
its own norm unless that is below 1 % of the wavefield's peak on the plane
over the run (a component that vanishes there by symmetry, or a field
after the wave has left), then relative to that peak
(qvti_cases.snapshot_error).
"""
import os
import sys

import numpy as np
import pytest

import qvti_cases as qc

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "oracle")
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_oracle_golden as mog  # noqa: E402

TOL = 1e-4


def _fixture(name):
    path = os.path.join(FIX, name + ".npz")
    if not os.path.exists(path):
        pytest.fail("missing fixture %s (tests/golden/make_oracle_golden.py)" % path)
    return dict(np.load(path))


def _case(name):
    c = mog.cases()[name]()
    g = _fixture(name)
    sums = mog.model_sums(c)
    assert np.allclose(sums, g["model_sums"], rtol=1e-6, atol=0), "rebuilt model differs from the fixture's"
    return c, g


@pytest.mark.parametrize("name", sorted(mog.cases()))
def test_fixture_cases_rebuild_their_models(name):
    """CPU: the seeded generators rebuild the fixture's model and geometry."""
    c, g = _case(name)
    assert int(g["nt"]) == int(c["nt"]) and float(g["dt"]) == pytest.approx(float(c["dt"]))
    assert np.array_equal(g["r_ix"], c["r_ix"]) and np.array_equal(g["r_iy"], c["r_iy"])
    assert g["rec_vx"].shape == (int(c["nt"]), len(c["r_ix"]))
    assert np.isfinite(g["rec_vx"]).all() and np.abs(g["rec_vx"]).max() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(mog.cases()))
def test_against_oracle_fixture(qvti, name):
    c, g = _case(name)
    nt = int(c["nt"])
    snaps = list(range(100, nt + 1, 100))
    ours = qvti.run_case(c, snaps=snaps, src_type=int(c["src_type"]), vti=bool(c["vti"]),
                         ref_offset=bool(c.get("ref_offset", 0)))
    worst = 0.0
    for i, comp in enumerate(("vx", "vy", "vz")):
        e = qc.relL2(ours["rec"][i], g["rec_" + comp])
        worst = max(worst, e)
        assert e <= TOL, "%s seismogram %s relL2 %.3g" % (name, comp, e)
    py, pz = int(c["plane_y"]), int(c["plane_z"])
    for lab in ("y", "z") if pz >= 0 else ("y",):
        peak = qc.plane_peak([g["plane_%s_%d" % (lab, k)] for k in snaps])
        for i in range(3):
            ref = [g["plane_%s_%d" % (lab, k)][i] for k in snaps]
            for k, r in zip(snaps, ref):
                f = ours["snaps"][k][i]
                mine = f[:, py, :] if lab == "y" else f[:, :, pz]
                e = qc.snapshot_error(mine, r, peak)
                worst = max(worst, e)
                assert e <= TOL, "%s step %d field %d plane %s error %.3g" % (name, k, i, lab, e)
    print("%s worst error %.2e" % (name, worst))
