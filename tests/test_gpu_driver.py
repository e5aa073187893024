"""The C++ host driver (q-vti_b200/host/qvti_driver.cpp), which keeps the
reference's host surface (viscoelas_3D.cpp: run parameters, observation
system, source_xy.txt / source_trnum.txt, raw float32 seismograms [it][ir]
per shot and component) on top of the drop-in C ABI.

A two-shot run on a 32^3 padded grid: the files the reference writes exist
with their sizes and formats, and each shot's seismograms equal the same
shot run through the Python binding of the extended ABI (bit for bit: same
kernels, same inputs).  The JSON-lines run log has one line per shot; a
stepped run adds the energy norms, which equal the binding's.
"""
import ctypes
import json
import os
import subprocess

import numpy as np
import pytest

import qvti_cases as qc
from conftest import ROOT

pytestmark = pytest.mark.gpu

RUN = dict(nx=20, ny=20, nz=20, pml=6, nt=60, nsx=2, nsy=1, dsx=6, dsy=6, nsx0=7, nsy0=10, depth=4, dr=4,
           dx=10.0, dy=10.0, dz=10.0, dt=0.8e-3, f0=30.0, velp_const=2500.0, vs_ratio=1.5, qp=200.0, qs=150.0,
           rho=1800.0)


def _driver():
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "q-vti_b200"), "driver"])
    return os.path.join(ROOT, "q-vti_b200", "qvti_driver")


def _run(tmp_path, **extra):
    exe = _driver()
    desc = dict(RUN, outdir=str(tmp_path / "output"), recdir=str(tmp_path / "record"), **extra)
    f = tmp_path / "run.txt"
    f.write_text("".join("%s = %s\n" % kv for kv in desc.items()))
    out = subprocess.run([exe, str(f)], cwd=str(tmp_path), capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    return desc


def _shot_case(desc, isx):
    r = desc
    pml, nx, ny, nz = r["pml"], r["nx"], r["ny"], r["nz"]
    n = (nx + 2 * pml, ny + 2 * pml, nz + 2 * pml)
    rnx, rny = nx // r["dr"], ny // r["dr"]
    ip = np.arange(rnx * rny)
    vp = np.full(n, r["velp_const"], np.float32)
    return dict(ntx=n[0], nty=n[1], ntz=n[2], pml=pml, nt=r["nt"], dx=r["dx"], dy=r["dy"], dz=r["dz"],
                dt=r["dt"], f0=r["f0"], velp=vp, vels=vp / np.float32(r["vs_ratio"]),
                rho=np.full(n, r["rho"], np.float32), gama_p=np.full(n, qc.gamma_of_q(r["qp"]), np.float32),
                gama_s=np.full(n, qc.gamma_of_q(r["qs"]), np.float32), rik=qc.ricker(r["nt"], r["dt"], r["f0"]),
                s_ix=isx * r["dsx"] + pml + r["nsx0"], s_iy=pml + r["nsy0"], s_iz=pml + r["depth"],
                r_iz=pml + r["depth"], r_ix=(pml + ip // rny * r["dr"]).astype(np.int32),
                r_iy=(pml + ip % rny * r["dr"]).astype(np.int32))


def test_driver_writes_the_reference_outputs(qvti, tmp_path):
    desc = _run(tmp_path)
    out, rec = tmp_path / "output", tmp_path / "record"
    xy = (out / "source_xy.txt").read_bytes().decode().split("\r\n")
    assert xy[0] == "%10d %10d" % (desc["nsx0"], desc["nsy0"])
    assert xy[1] == "%10d %10d" % (desc["dsx"] + desc["nsx0"], desc["nsy0"])
    rn = (desc["nx"] // desc["dr"]) * (desc["ny"] // desc["dr"])
    assert (out / "source_trnum.txt").read_bytes().decode() == "%d\r\n%d\r\n" % (rn, rn)
    for shot in range(2):
        c = _shot_case(desc, shot)
        ref = qvti.run_case(c)["rec"]
        for i, comp in enumerate(("vx", "vy", "vz")):
            a = np.fromfile(rec / ("Q1dep_%s_small_shot%d.bin" % (comp, shot)), np.float32)
            assert a.size == desc["nt"] * rn
            assert np.array_equal(a.reshape(desc["nt"], rn), ref[i])
        assert np.abs(ref[0]).max() > 0
    log = [json.loads(line) for line in (out / "run.jsonl").read_text().splitlines()]
    assert [e["shot"] for e in log] == [0, 1]
    assert all(e["status"] == "ok" and e["seconds"] > 0 and e["gcell_steps_per_s"] > 0 for e in log)
    assert all("energy" not in e for e in log)  # whole-shot ABI calls: no wavefield access


def test_driver_snapshots_match_fields(qvti, tmp_path):
    desc = _run(tmp_path, snap_every=30, nsx=1)
    out, pml = tmp_path / "output", desc["pml"]
    c = _shot_case(desc, 0)
    res = qvti.run_case(c, snaps=[30, 60])
    for k in (30, 60):
        for i, comp in enumerate("xyz"):
            a = np.fromfile(out / ("shot0snap%d_v%s.bin" % (k, comp)), np.float32)
            want = res["snaps"][k][i][pml:-pml, pml:-pml, pml:-pml]
            assert a.size == want.size
            assert np.array_equal(a.reshape(want.shape), want)
    (entry,) = [json.loads(line) for line in (out / "run.jsonl").read_text().splitlines()]
    assert entry["shot"] == 0 and entry["status"] == "ok" and entry["nonfinite"] is False
    state = qvti.run_case(c, want_state=True)["state"].astype(np.float64)
    want = (state.reshape(9, -1) ** 2).sum(axis=1)
    assert np.allclose(entry["energy"], want, rtol=1e-9, atol=0)


class _Source(ctypes.Structure):
    _fields_ = [("s_iz", ctypes.c_int), ("s_ix", ctypes.c_int), ("s_iy", ctypes.c_int), ("r_iz", ctypes.c_int),
                ("r_ix", ctypes.POINTER(ctypes.c_int)), ("r_iy", ctypes.POINTER(ctypes.c_int)), ("r_n", ctypes.c_int)]


class _MultiGPU(ctypes.Structure):
    _fields_ = [("record", ctypes.POINTER(ctypes.c_float)), ("record2", ctypes.POINTER(ctypes.c_float)),
                ("record3", ctypes.POINTER(ctypes.c_float)), ("sim", ctypes.c_void_p),
                ("ntx", ctypes.c_int), ("nty", ctypes.c_int), ("ntz", ctypes.c_int), ("nt", ctypes.c_int),
                ("rnmax", ctypes.c_int)]


def test_void_abi_keeps_its_engine_across_shots(qvti):
    """The reference allocates once (cuda_Device_malloc) and runs every shot
    on the same buffers (viscoelas_3D.cpp:355-405).  Three shots through
    cuda_forward_acoustic_3D: the second (same grid and constants, another
    source position) reuses the first shot's engine -- no qvti_create -- and
    both equal qvti_forward_shot bit for bit; the third changes dt and gets a
    new engine."""
    L = qvti.lib()
    F = ctypes.POINTER(ctypes.c_float)
    L.qvti_sims_created.restype = ctypes.c_longlong
    L.cuda_forward_acoustic_3D.restype = None
    L.cuda_forward_acoustic_3D.argtypes = [ctypes.c_int] * 11 + [ctypes.c_float] * 7 + [F] * 6 + \
        [ctypes.POINTER(_Source), ctypes.POINTER(_MultiGPU)] + [ctypes.c_int] * 5
    c = qc.heterogeneous_case(n=(32, 32, 32), pml=6, nt=60, seed=9, src=(16, 16, 16), r_iz=8)
    ntx, nty, ntz, nt = c["ntx"], c["nty"], c["ntz"], c["nt"]
    ntp = ntx * nty * ntz
    rnx, rny = int(c["rnx_max"]), int(c["rny_max"])
    rn = rnx * rny
    rix, riy = np.ascontiguousarray(c["r_ix"], np.int32), np.ascontiguousarray(c["r_iy"], np.int32)
    IP = ctypes.POINTER(ctypes.c_int)
    srcs = (_Source * 3)(*[_Source(int(c["s_iz"]), sx, 16, int(c["r_iz"]), rix.ctypes.data_as(IP),
                                   riy.ctypes.data_as(IP), rn) for sx in (16, 13, 19)])
    plan = (_MultiGPU * 1)()
    L.cuda_Device_malloc(ntx, nty, ntz, ntp, ntx - 12, nty - 12, ntz - 12, nt, rn, plan, 1)
    L.cuda_Host_initialization(ntp, nt, rn, plan, 1)
    model = [np.ascontiguousarray(c[k], np.float32) for k in ("velp", "gama_p", "vels", "gama_s", "rho")]
    rik = np.ascontiguousarray(c["rik"], np.float32)
    w0 = float(np.float32(2 * qc.PI_REF * c["f0"]))
    try:
        created = []
        for shot, dt in ((0, c["dt"]), (1, c["dt"]), (2, 0.5 * c["dt"])):
            L.cuda_forward_acoustic_3D(0, shot, nt, ntx, nty, ntz, ntp, ntx - 12, nty - 12, ntz - 12, c["pml"],
                                       c["dx"], c["dy"], c["dz"], dt, c["f0"], w0, 5000.0, rik.ctypes.data_as(F),
                                       *[m.ctypes.data_as(F) for m in model], srcs, plan, 1, rn, rnx, rny, 4)
            created.append(L.qvti_sims_created())
            got = np.stack([np.ctypeslib.as_array(getattr(plan[0], r), shape=(nt, rn)).copy()
                            for r in ("record", "record2", "record3")])
            want = qvti.run_case(dict(c, s_ix=srcs[shot].s_ix, dt=dt))["rec"]
            assert np.array_equal(got, want), "shot %d differs from qvti_forward_shot" % shot
            assert np.abs(got).max() > 0
        # run_case creates one simulation per call; the void ABI one on shot 0 and one on shot 2
        assert created[1] - created[0] == 1, created   # only run_case's own simulation
        assert created[2] - created[1] == 2, created   # a new engine for the new dt, plus run_case's
    finally:
        L.cuda_Device_free(plan, 1)


def test_forward_shot_matches_the_step_by_step_calls(qvti):
    """qvti_forward_shot queues the model upload and the state clear without
    waiting and stages the model in spectrum scratch; two shots in a row on
    one simulation (VTI, the second from another source position, the host
    model in page-locked memory for one and pageable for the other) equal
    the same shots through set_model / set_receivers / set_source / reset /
    step bit for bit."""
    torch = pytest.importorskip("torch")
    c = qc.heterogeneous_case(n=(32, 48, 64), pml=6, nt=70, seed=12, src=(16, 24, 30), r_iz=10)
    rng = np.random.default_rng(3)
    c["eps"] = (0.05 + 0.2 * rng.random(c["velp"].shape)).astype(np.float32)
    c["delta"] = (0.1 * rng.random(c["velp"].shape)).astype(np.float32)
    names = ("velp", "vels", "rho", "gama_p", "gama_s", "eps", "delta")
    nt, rn = int(c["nt"]), len(c["r_ix"])
    F = ctypes.POINTER(ctypes.c_float)
    IP = ctypes.POINTER(ctypes.c_int)
    rix = np.ascontiguousarray(c["r_ix"], np.int32)
    riy = np.ascontiguousarray(c["r_iy"], np.int32)
    rik = np.ascontiguousarray(c["rik"], np.float32)[:nt]
    pinned = {k: torch.from_numpy(np.ascontiguousarray(c[k], np.float32)).pin_memory() for k in names}
    pageable = {k: np.ascontiguousarray(c[k], np.float32) for k in names}

    def ptr(a):
        return ctypes.cast(ctypes.c_void_p(a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data), F)

    with qvti.simulation_for_case(c, vti=True) as sim:
        for sx, model in ((16, pinned), (11, pageable)):
            rec = np.zeros((3, nt, rn), np.float32)
            rc = qvti.lib().qvti_forward_shot(sim._h, *[ptr(model[k]) for k in names], qvti.SRC_FORCE_X, sx,
                                              int(c["s_iy"]), int(c["s_iz"]) + 10, rik.ctypes.data_as(F), nt,
                                              int(c["r_iz"]), rix.ctypes.data_as(IP), riy.ctypes.data_as(IP), rn,
                                              *[rec[i].ctypes.data_as(F) for i in range(3)])
            assert rc == 0, qvti.lib().qvti_error_string(rc)
            want = qvti.run_case(dict(c, s_ix=sx), vti=True)["rec"]
            assert np.abs(want).max() > 0
            assert np.array_equal(rec, want), "source x %d" % sx
