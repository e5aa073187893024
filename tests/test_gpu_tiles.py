"""Per-kernel tiles (qvti_set_tiles, qvti_get_tiles, qvti_autotune_tiles) and
the multi-step step graphs.

* Every step kernel on its runtime-length path, at every tile the grid
  admits, against the FP64 oracle at the parity bar (relative L2 <= 1e-4)
  and against the default tiling to FP32 rounding.  The grid mixes a length
  without a compiled kernel (x = 32: k_vx and k_mx run their runtime
  kernels by default) with compiled ones (y = 64, z = 96).
* The tile search returns settings the grid admits and leaves them set.
* Invalid tilings are rejected and leave the tiling unchanged.
* A call of qvti_step over many steps replays 16-step graphs; the result is
  bit-identical to the same steps taken one call at a time.
"""
import numpy as np
import pytest

import qvti_cases as qc
from test_gpu_parity import _compare, _ct_case

pytestmark = pytest.mark.gpu

GRID = (32, 64, 96)
NT = 80
KERNELS = ("k_vy", "k_vx", "k_fz", "k_cy", "k_mx", "k_sigma")
ROUNDING = 2e-5  # runtime against compiled kernels: the same radix plan, other rounding order


@pytest.fixture(scope="module")
def case():
    return _ct_case(GRID, NT, pml=6)


@pytest.fixture(scope="module")
def default_run(qvti, case):
    return qvti.run_case(case, snaps=[NT // 2, NT], vti=True)


@pytest.fixture(scope="module")
def oracle_run(oracle, case):
    return oracle.run_case(case, snaps=[NT // 2, NT], vti=True)


def _ready(qvti, sim, case):
    sim.set_model(case["velp"], case["vels"], case["rho"], case["gama_p"], case["gama_s"], case["eps"], case["delta"])
    sim.set_receivers(case["r_iz"], case["r_ix"], case["r_iy"])
    sim.set_source(case["s_ix"], case["s_iy"], int(case["s_iz"]) + 10, np.asarray(case["rik"], np.float32)[:NT])


def test_default_tiling_against_oracle(qvti, case, default_run, oracle_run):
    with qvti.simulation_for_case(case, vti=True) as sim:
        tiles, runtime = sim.tiles()
    # x = 32 has no compiled kernel: k_vx and k_mx (x transforms) run their
    # runtime kernels, the others their compiled ones
    assert runtime == [0, 1, 0, 0, 1, 0], runtime
    assert tiles == [16, 16, 16, 8, 16, 4], tiles
    _compare(default_run, oracle_run, "default tiling")


@pytest.mark.parametrize("kernel", range(6), ids=KERNELS)
def test_runtime_tiles_against_oracle(qvti, case, default_run, oracle_run, kernel):
    accepted = []
    for t in (2, 4, 8, 16, 32):
        tiles = [0] * qvti.NUM_TILES
        tiles[kernel] = t
        try:
            ours = qvti.run_case(case, snaps=[NT // 2, NT], vti=True, tiles=tiles)
        except qvti.QvtiError as e:
            # only the largest tiles may exceed the shared memory of a block
            assert t >= 16 and "unsupported" in str(e), (t, str(e))
            continue
        accepted.append(t)
        _compare(ours, oracle_run, "%s tile %d" % (KERNELS[kernel], t))
        for i in range(3):
            e = qc.relL2(ours["rec"][i], default_run["rec"][i])
            assert e <= ROUNDING, "%s tile %d seismogram %d vs default %.3g" % (KERNELS[kernel], t, i, e)
            e = qc.relL2(ours["snaps"][NT][i], default_run["snaps"][NT][i])
            assert e <= ROUNDING, "%s tile %d field %d vs default %.3g" % (KERNELS[kernel], t, i, e)
    assert {2, 4, 8} <= set(accepted), accepted


def test_tiles_reported_as_set(qvti, case):
    with qvti.simulation_for_case(case, vti=True) as sim:
        sim.set_tiles([8, 4, 2, 16, 8, 2])
        tiles, runtime = sim.tiles()
        assert tiles == [8, 4, 2, 16, 8, 2] and runtime == [1] * 6
        sim.set_tiles([0] * 6)
        assert sim.tiles()[1] == [0, 1, 0, 0, 1, 0]


@pytest.mark.parametrize("bad", [
    [3, 0, 0, 0, 0, 0],    # odd
    [0, 0, 0, 0, 64, 0],   # above 32
    [0, 0, 0, 0, 0, 1],    # below 2
    [0, 0, 0, 0, 0, -2],   # negative
    [0, 0, 12, 0, 0, 0],   # does not divide ny = 64
])
def test_invalid_tiles_rejected(qvti, case, bad):
    with qvti.simulation_for_case(case, vti=True) as sim:
        sim.set_tiles([4, 0, 0, 0, 0, 0])
        with pytest.raises(qvti.QvtiError, match="unsupported"):
            sim.set_tiles(bad)
        tiles, runtime = sim.tiles()
        assert tiles[0] == 4 and runtime[0] == 1  # unchanged


def test_autotune_tiles_leaves_a_valid_setting(qvti, case, default_run):
    with qvti.simulation_for_case(case, vti=True) as sim:
        _ready(qvti, sim, case)
        best, ms = sim.autotune_tiles(probe_steps=2)
        assert all(b == 0 or b in (2, 4, 8, 16, 32) for b in best), best
        assert all(m > 0 for m in ms), ms
        tiles, runtime = sim.tiles()
        for i, b in enumerate(best):
            if b:
                assert tiles[i] == b and runtime[i] == 1
        # the search left the simulation reset: a full run matches the default
        # tiling to rounding
        sim.step(NT)
        rec = sim.records()
    for i in range(3):
        assert qc.relL2(rec[i], default_run["rec"][i]) <= ROUNDING


def test_multi_step_graphs_match_single_steps(qvti, case):
    """40 steps in one call (two 16-step graphs and eight one-step ones)
    against 40 calls of one step: the same kernels in the same order."""
    def run(chunks):
        with qvti.simulation_for_case(case, vti=True) as sim:
            _ready(qvti, sim, case)
            sim.reset()
            for n in chunks:
                sim.step(n)
            return sim.records(), sim.fields(0, 9)
    rec_a, f_a = run([40])
    rec_b, f_b = run([1] * 40)
    rec_c, f_c = run([17, 16, 7])
    assert np.array_equal(rec_a, rec_b) and np.array_equal(f_a, f_b)
    assert np.array_equal(rec_a, rec_c) and np.array_equal(f_a, f_c)
