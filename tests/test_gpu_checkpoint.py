"""Checkpoint / resume (qvti_state_bytes, qvti_save_state, qvti_load_state).

Every step kernel is deterministic, so a run stopped after k steps, saved,
and resumed from the snapshot (in a new simulation, or in the same one after
it has moved on) must give exactly the seismograms and wavefields of an
uninterrupted run: the tests compare with exact equality.  A snapshot of
another grid, spacing, medium type or receiver count is rejected.
"""
import numpy as np
import pytest

import qvti_cases as qc

pytestmark = pytest.mark.gpu

NT, SPLIT = 70, 27


def _case(n=(48, 32, 40), vti=True, seed=5):
    c = qc.heterogeneous_case(n=n, pml=6, d=(10.0, 10.0, 10.0), dt=0.8e-3, nt=NT, f0=30.0, seed=seed,
                              src=(n[0] // 2, n[1] // 2, n[2] // 2), r_iz=n[2] // 2 - 6, name="ckpt")
    if vti:
        rng = np.random.default_rng(seed + 50)
        c["eps"] = (0.05 + 0.2 * rng.random(n)).astype(np.float32)
        c["delta"] = (0.12 * rng.random(n)).astype(np.float32)
    return c


def _prepared(qvti, c, vti):
    sim = qvti.simulation_for_case(c, vti=vti)
    sim.set_model(c["velp"], c["vels"], c["rho"], c["gama_p"], c["gama_s"],
                  c.get("eps") if vti else None, c.get("delta") if vti else None)
    sim.set_receivers(c["r_iz"], c["r_ix"], c["r_iy"])
    sim.set_source(c["s_ix"], c["s_iy"], int(c["s_iz"]) + 10, np.asarray(c["rik"], np.float32))
    sim.reset()
    return sim


@pytest.mark.parametrize("vti", [False, True])
def test_resume_is_bitwise(qvti, vti):
    c = _case(vti=vti)
    with _prepared(qvti, c, vti) as sim:
        sim.step(NT)
        rec_ref, state_ref = sim.records(), sim.fields(0, 9)

    with _prepared(qvti, c, vti) as sim:
        sim.step(SPLIT)
        snap = sim.save_state()
        rec_at_split = sim.records()
        sim.step(9)                      # move on, then roll back in place
        sim.load_state(snap)
        assert sim.steps_done == SPLIT
        assert np.array_equal(sim.records(), rec_at_split)
        sim.step(NT - SPLIT)
        assert np.array_equal(sim.records(), rec_ref)
        assert np.array_equal(sim.fields(0, 9), state_ref)

    with _prepared(qvti, c, vti) as sim:   # a fresh simulation of the same shot
        sim.load_state(snap)
        sim.step(NT - SPLIT)
        assert np.array_equal(sim.records(), rec_ref)
        assert np.array_equal(sim.fields(0, 9), state_ref)


def test_snapshot_size_and_header(qvti):
    c = _case(vti=True)
    with _prepared(qvti, c, True) as sim:
        sim.step(5)
        snap = sim.save_state()
    nx, ny, nz, pml = 48, 32, 40, int(c["pml"])
    ntp = nx * ny * nz
    rn = int(c["rnx_max"] * c["rny_max"])
    # 18 full-grid arrays (v, s, R, Q) and the 37 C-PML arrays of their slabs:
    # 13 of the x slab, 13 of the y slab, 11 of the z slab
    slab = 13 * 2 * pml * ny * nz + 13 * nx * 2 * pml * nz + 11 * nx * ny * 2 * pml
    assert snap.size == 72 + 18 * 4 * ntp + 4 * slab + 3 * 5 * rn * 4
    assert bytes(snap[:8]) == b"QVTIST02"


def test_mismatched_snapshots_are_rejected(qvti):
    c = _case(vti=True)
    with _prepared(qvti, c, True) as sim:
        sim.step(4)
        snap = sim.save_state()
        bad = snap.copy()
        bad[0] ^= 0xFF                       # not a snapshot
        with pytest.raises(qvti.QvtiError):
            sim.load_state(bad)
        with pytest.raises(qvti.QvtiError):  # truncated
            sim.load_state(snap[:-4])
        sim.load_state(snap)                 # the intact one still loads
        assert sim.steps_done == 4
    with _prepared(qvti, c, False) as iso:   # another medium type
        with pytest.raises(qvti.QvtiError):
            iso.load_state(snap)
    other = _case(n=(48, 32, 48), vti=True)
    with _prepared(qvti, other, True) as sim:  # another grid
        with pytest.raises(qvti.QvtiError):
            sim.load_state(snap)
    with _prepared(qvti, c, True) as sim:      # another receiver count
        sim.set_receivers(c["r_iz"], c["r_ix"][:3], c["r_iy"][:3])
        with pytest.raises(qvti.QvtiError):
            sim.load_state(snap)
