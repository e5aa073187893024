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
