"""Parity of the CUDA path against the FP64 oracle and the reference's own
cuFFT build (golden fixtures), through the C ABI.

Tolerance: relative L2 <= 1e-4 on every seismogram component and every
snapshot field at the end of the run (FP32 against FP64 and against the
reference's FP32 cuFFT result).
"""
import numpy as np
import pytest

import qvti_cases as qc
from conftest import golden_names, load_golden, snap_keys

TOL = 1e-4
pytestmark = pytest.mark.gpu


def _compare(ours, ref, label):
    worst = 0.0
    for i, comp in enumerate(("vx", "vy", "vz")):
        e = qc.relL2(ours["rec"][i], ref["rec"][i])
        worst = max(worst, e)
        assert e <= TOL, "%s seismogram %s relL2 %.3g" % (label, comp, e)
    for k in ref.get("snaps", {}):
        for i in range(3):
            e = qc.relL2(ours["snaps"][k][i], ref["snaps"][k][i])
            worst = max(worst, e)
            assert e <= TOL, "%s snapshot %d field %d relL2 %.3g" % (label, k, i, e)
    return worst


@pytest.mark.parametrize("name", [n for n in golden_names() if n != "config1"])
def test_against_reference_golden(qvti, name):
    c = load_golden(name)
    snaps = snap_keys(c)
    ours = qvti.run_case(c, snaps=snaps, want_state=True)
    ref = dict(rec=np.stack([c["rec_vx"], c["rec_vy"], c["rec_vz"]]),
               snaps={k: c["snap_%d" % k] for k in snaps})
    _compare(ours, ref, name)
    for f in range(9):
        e = qc.relL2(ours["state"][f], c["final9"][f])
        assert e <= TOL, "%s final field %d relL2 %.3g" % (name, f, e)


def test_config1_against_reference_golden(qvti):
    """96^3, 20-cell C-PML, 500 steps: seismograms, vx, vy, vz on the x-z
    plane 12 cells beside the source every 100 steps (qvti_cases.
    snapshot_error: relative L2, or relative to the wavefield's peak on the
    plane where a field is below 1 % of it -- at step 500, after the wave
    has left), and the final-state norms."""
    c = load_golden("config1")
    planes = sorted(int(k.split("_")[2]) for k in c if k.startswith("plane_y_"))
    assert planes == [100, 200, 300, 400, 500], planes
    ours = qvti.run_case(c, snaps=planes, want_state=True)
    ref = dict(rec=np.stack([c["rec_vx"], c["rec_vy"], c["rec_vz"]]))
    _compare(ours, ref, "config1")
    py = int(c["plane_y"])
    peak = qc.plane_peak([c["plane_y_%d" % k] for k in planes])
    for i in range(3):
        for k in planes:
            e = qc.snapshot_error(ours["snaps"][k][i][:, py, :], c["plane_y_%d" % k][i], peak)
            assert e <= TOL, "config1 step %d field %d plane error %.3g" % (k, i, e)
    norms = np.array([np.linalg.norm(f.astype(np.float64)) for f in ours["state"]])
    rel = np.abs(norms - c["final_norms"]) / c["final_norms"]
    assert rel.max() <= TOL, rel


@pytest.mark.parametrize("name", [n for n in golden_names() if n != "config1"])
def test_against_oracle(qvti, oracle, name):
    c = load_golden(name)
    snaps = snap_keys(c)
    ours = qvti.run_case(c, snaps=snaps)
    ref = oracle.run_case(c, snaps=snaps)
    _compare(ours, ref, name)


def _vti_case(seed=3):
    c = qc.heterogeneous_case(n=(32, 32, 48), pml=8, d=(10.0, 10.0, 10.0), dt=0.8e-3, nt=90, f0=30.0,
                              seed=seed, src=(16, 16, 20), r_iz=10, name="vti")
    rng = np.random.default_rng(seed + 100)
    shape = c["velp"].shape
    c["eps"] = (0.05 + 0.2 * rng.random(shape)).astype(np.float32)
    c["delta"] = (0.12 * rng.random(shape)).astype(np.float32)
    return c


def test_vti_against_oracle(qvti, oracle):
    c = _vti_case()
    ours = qvti.run_case(c, snaps=[45], vti=True)
    ref = oracle.run_case(c, snaps=[45], vti=True)
    _compare(ours, ref, "vti")


def test_vti_zero_anisotropy_matches_isotropic(qvti):
    c = _vti_case(seed=5)
    c["eps"][:] = 0
    c["delta"][:] = 0
    a = qvti.run_case(c, vti=True)
    b = qvti.run_case(c, vti=False)
    for i in range(3):
        assert qc.relL2(a["rec"][i], b["rec"][i]) <= 1e-6


def test_explosive_source_against_oracle(qvti, oracle):
    c = qc.heterogeneous_case(n=(32, 48, 32), pml=6, seed=11, src=(16, 24, 16), r_iz=8, nt=80, name="expl")
    ours = qvti.run_case(c, snaps=[40], src_type=qvti.SRC_EXPLOSIVE, ref_offset=False)
    ref = oracle.run_case(c, snaps=[40], src_type=1, ref_offset=False)
    _compare(ours, ref, "explosive")


@pytest.mark.parametrize("n", [(64, 64, 64), (64, 128, 96), (160, 32, 48), (48, 144, 32), (32, 48, 192),
                               (120, 32, 48), (32, 108, 48), (40, 48, 100),
                               (64, 64, 100), (100, 108, 64), (64, 150, 64)])
def test_compile_time_path_against_oracle(qvti, oracle, n):
    """A kernel takes the compile-time FFT path when its transform length is
    compiled; the mixed grids put some kernels on it (x: k_vx, k_mx at 160
    and 120; y: k_vy, k_cy at 144 and 108; z: k_fz, k_sigma at the
    three-stage 192 and at 100) and the rest on the runtime path.  The last
    three have partial last tiles: z tiles of k_vy and k_vx (nz = 100), y
    tiles of k_fz and k_mx and the line tiles of k_cy (ny = 108, 33 x 100
    lines), and the y tiles of k_sigma (ny = 150, the masked instantiation).
    VTI, heterogeneous, receivers 6 cells above and within 3 cells of the
    source."""
    nt = 100 if n[0] * n[1] * n[2] <= 64 ** 3 else 80
    c = _ct_case(n, nt)
    ours = qvti.run_case(c, snaps=[nt], vti=True)
    ref = oracle.run_case(c, snaps=[nt], vti=True)
    _compare(ours, ref, "ct%dx%dx%d" % n)


@pytest.mark.parametrize("n", [(256, 16, 24), (16, 256, 24), (24, 16, 256)])
def test_256_point_kernels_against_oracle(qvti, oracle, n):
    """The benchmark grid is 256 points on every axis; each case puts one axis
    at 256 so the instantiations the benchmark times run against the FP64
    oracle: x = 256 -> k_vx<256> and k_mx<256> (k-space x pass); y = 256 ->
    k_vy<256> and both k_cy<256> passes; z = 256 -> k_fz<256> and
    k_sigma<256> (its in-place two-stage C2R).  VTI, heterogeneous, 120
    steps, seismograms and snapshots at steps 60 and 120."""
    nt = 120
    c = _ct_case(n, nt, pml=4)
    ours = qvti.run_case(c, snaps=[60, nt], vti=True)
    ref = oracle.run_case(c, snaps=[60, nt], vti=True)
    _compare(ours, ref, "256axis%dx%dx%d" % n)


@pytest.mark.parametrize("batch", [7, 17])
def test_kz_batches_match_one_pass(qvti, batch):
    """The k-space passes in batches of kz planes (ragged line tiles at every
    batch edge: 7 x 100 and 17 x 100 lines are not multiples of 8) give the
    same step bit for bit as one pass over all planes."""
    n, nt = (100, 108, 64), 30
    c = _ct_case(n, nt)
    full = qvti.run_case(c, vti=True, want_state=True)
    with qvti.simulation_for_case(c, vti=True) as sim:
        qvti._check(qvti.lib().qvti_set_kz_batch(sim._h, batch), "qvti_set_kz_batch")
        sim.set_model(c["velp"], c["vels"], c["rho"], c["gama_p"], c["gama_s"], c["eps"], c["delta"])
        sim.set_receivers(c["r_iz"], c["r_ix"], c["r_iy"])
        sim.set_source(c["s_ix"], c["s_iy"], int(c["s_iz"]) + 10, np.asarray(c["rik"], np.float32)[:nt])
        sim.reset()
        sim.step(nt)
        assert np.array_equal(sim.records(), full["rec"])
        assert np.array_equal(sim.fields(0, 9), full["state"])


def _ct_case(n, nt, pml=8):
    c = qc.heterogeneous_case(n=n, pml=pml, d=(10.0, 10.0, 10.0), dt=0.8e-3, nt=nt, f0=30.0, seed=21,
                              src=(n[0] // 2, n[1] // 2, n[2] // 2), r_iz=n[2] // 2 - 6, name="ct")
    # a 3 x 3 receiver patch beside the source: the direct wave reaches every
    # receiver within the run, so the seismograms carry signal, not noise
    sx, sy = n[0] // 2, n[1] // 2
    gx, gy = np.meshgrid(np.arange(sx - 3, sx + 4, 3), np.arange(sy - 3, sy + 4, 3), indexing="ij")
    c["r_ix"] = gx.ravel().astype(np.int32)
    c["r_iy"] = gy.ravel().astype(np.int32)
    c["rnx_max"], c["rny_max"] = 3, 3
    rng = np.random.default_rng(4)
    c["eps"] = (0.05 + 0.2 * rng.random(c["velp"].shape)).astype(np.float32)
    c["delta"] = (0.12 * rng.random(c["velp"].shape)).astype(np.float32)
    return c
