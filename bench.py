"""Benchmark: Gcell-steps/s of the 3D viscoelastic pseudospectral time step on
the 256^3 VTI workload, one shot per GPU.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one time step of the whole padded 256^3 grid (PML inside); value =
cells x steps x ranks / max-over-ranks device time of the K timed steps
(CUDA events on the engine's stream).  Shots are independent, so N GPUs run
N replicas of the shot with no data-path collective ("scaling": "weak");
torch.distributed only provides the barrier and the max over ranks.

``--workload batch`` (the batching form: 48 seeded VTI shots over the grids
128^3, 160x160x128, 192^3, 256x256x192, nt scaled by --nt-scale) and
``--workload serve`` (the serving form: Poisson arrivals, log-uniform grids
between 96^3 and 384x384x256, iso/VTI 50/50, 150 GB admission budget) print
one JSON line each for those forms; the default is the 256^3 step.

``--impl reference`` times the reference's CPU counterpart: the reference has
no CPU implementation of the path (it is CUDA + cuFFT), so the arm runs the
FP64 CPU restatement (oracle/) on all host cores, each step a bounded sample
(one time step of the centred 128^3 crop of the same model, at most 20 timed
steps so the run ends in a few minutes), on rank 0 only.  Our arm's
``cpu_baseline`` times the same crop the same way with 4 steps, and its
``reference_gpu`` entry times the reference's own cuFFT build on this GPU
(256^3 isotropic, outside the timed region).
"""
import argparse
import contextlib
import ctypes
import importlib.util
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "q-vti_b200")

GRID = (256, 256, 256)
PML = 30  # C-PML cells per face (the 256^3 workload)
DX = 10.0
F0 = 20.0
DT_NOMINAL = 0.8e-3
SEED = 2024
METRIC = "Gcell-steps/s 256^3 VTI"
UNIT = "Gcell-steps/s"


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class Dist:
    """Barrier and max-reduce over ranks: torch.distributed over NCCL on GPUs
    (gloo when no GPU is visible, e.g. the CPU tests of this logic).  Shots
    are independent, so this is the only cross-rank traffic."""

    def __init__(self, world, local, backend=None):
        self.world = world
        self.pg = None
        if world > 1:
            import datetime

            import torch
            import torch.distributed as td
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            self.device = None
            if backend == "nccl":
                torch.cuda.set_device(local)
                self.device = torch.device("cuda", local)
            td.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.td, self.torch, self.local = td, torch, local
            self.pg = True

    def barrier(self):
        if self.pg:
            if self.device is not None:
                self.td.barrier(device_ids=[self.local])
            else:
                self.td.barrier()

    def max(self, x):
        if not self.pg:
            return x
        t = self.torch.tensor([float(x)], dtype=self.torch.float64, device=self.device)
        self.td.all_reduce(t, op=self.td.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.td.destroy_process_group()


def aggregate_value(cells, steps, world, ms_max):
    """Whole-job Gcell-steps/s: every rank advances its own shot `steps` steps."""
    return cells * steps * world / (ms_max / 1e3) / 1e9


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                p = [x.strip() for x in line.split(",")]
                if len(p) >= 9 and p[1].replace(".", "").isdigit():
                    rows.append(p)
        except OSError:
            pass
        finally:
            with contextlib.suppress(OSError):
                os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic(kernel):
    """dram read+write bytes per launch of `kernel` from the committed ncu
    summaries (a line `traffic_bytes_per_launch <kernel> <bytes>`), or None."""
    pdir = os.path.join(ROOT, "profiles")
    if not os.path.isdir(pdir):
        return None
    for fn in sorted(os.listdir(pdir)):
        if not fn.endswith((".md", ".txt")):
            continue
        for line in open(os.path.join(pdir, fn)):
            p = line.strip().strip("`").split()
            if len(p) == 3 and p[0] == "traffic_bytes_per_launch" and p[1] == kernel:
                return float(p[2])
    return None


def make_model(models):
    m = models.layered_vti(tuple(GRID), DX, seed=SEED)
    dt, lim, veff = models.choose_dt(m, DX, F0, DT_NOMINAL, vti=True)
    return m, dt, lim, veff


def workload_desc(dt):
    return ("256^3 VTI: 6 layers Vp 1800-4500 m/s, Vs=Vp/1.8, Gardner rho, eps U[0.05,0.25], delta U[0,0.12], "
            "Qp U[30,200], Qs=Qp/2, 5%% Gaussian perturbations (80 m), pml 30, dx 10 m, dt %.2f ms "
            "(0.8 ms capped to 80%% of the CFL bound), 20 Hz Ricker force at (128,128,35), "
            "256x256 receivers at iz=30, seed %d" % (dt * 1e3, SEED))


# ----------------------------------------------------------------- CPU leg --
CPU_CROP = 128  # edge of the centred crop both CPU legs time (clamped to the grid)


def oracle_case(model, crop, nt, dt):
    """Case dict of a centred crop^3 of the model (crop clamped to the grid)."""
    crop = min(crop, min(GRID))
    c0 = [(g - crop) // 2 for g in GRID]
    sl = tuple(slice(a, a + crop) for a in c0)
    pml = max(4, min(PML, crop // 6))
    case = dict(ntx=crop, nty=crop, ntz=crop, pml=pml, nt=nt, dx=DX, dy=DX, dz=DX, dt=dt, f0=F0,
                s_ix=crop // 2, s_iy=crop // 2, s_iz=pml + 5, r_iz=pml, r_ix=np.arange(crop, dtype=np.int32),
                r_iy=np.full(crop, crop // 2, np.int32), rnx_max=crop, rny_max=1)
    for k in ("velp", "vels", "rho", "gama_p", "gama_s", "eps", "delta"):
        case[k] = np.ascontiguousarray(model[k][sl])
    models = _load("qvti_models", os.path.join(PKG, "models.py"))
    case["rik"] = models.ricker(nt, dt, F0)
    return case, crop


def oracle_rate(model, crop, steps, dt, nthreads):
    """Gcell-steps/s of the FP64 oracle on a centred crop^3 of the model.

    Two runs of the same case, of 1 and 1 + `steps` steps: their difference
    is the time of `steps` steps with the setup (tables, coefficients) and
    the first step cancelled; the 1-step run is the warm-up.  At the default
    128^3 crop a step takes seconds, far above timing noise.  Returns (rate,
    seconds of the timed steps, crop)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    case, crop = oracle_case(model, crop, 1 + steps, dt)
    t0 = time.perf_counter()
    orc.run_case(case, nt=1, vti=True, ref_offset=False, nthreads=nthreads)
    t1 = time.perf_counter()
    orc.run_case(case, nt=1 + steps, vti=True, ref_offset=False, nthreads=nthreads)
    t2 = time.perf_counter()
    sec = (t2 - t1) - (t1 - t0)
    if sec <= 0:
        raise RuntimeError("oracle timing: %d steps took no measurable time (%.3f s, %.3f s)"
                           % (steps, t1 - t0, t2 - t1))
    return crop ** 3 * steps / sec / 1e9, sec, crop


def cpu_sample(crop, steps, sec, cores):
    return ("FP64 CPU restatement (oracle/) on a centred %d^3 crop of the same model: %d timed steps (%.1f s), "
            "setup and first step cancelled by differencing a 1-step and a %d-step run, %d threads; the rate "
            "per cell-step is taken as the %dx%dx%d rate (not scaled for the FFTs' log n growth, %.2fx at "
            "that size)" % (crop, steps, sec, 1 + steps, cores, GRID[0], GRID[1], GRID[2],
                             math.log(GRID[0] * GRID[1] * GRID[2]) / math.log(crop ** 3)))


def reference_arm(args, world, rank):
    if rank != 0:
        return 0
    models = _load("qvti_models", os.path.join(PKG, "models.py"))
    model, dt, _, _ = make_model(models)
    cores = os.cpu_count() or 1
    # each timed step is one step of the crop (a bounded sample of the
    # workload's step); at most 20 of them so the arm ends in a few minutes
    steps = max(1, min(args.steps, 20))
    rate, sec, crop = oracle_rate(model, CPU_CROP, steps, dt, cores)
    line = {
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec / steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": workload_desc(dt), "sample": "%d^3 crop" % crop,
                                        "timed_steps": steps},
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": cpu_sample(crop, steps, sec, cores)},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def reference_gpu_timing(n, pml):
    """The reference's own cuFFT build (oracle/_ref, compiled from its
    unmodified sources) timed on the same B200 by oracle/time_reference.py in
    a separate process, outside this bench's timed region: 256^3 isotropic
    (the reference has no VTI), per-step time from the difference of a 45-
    and a 25-step call, beside this library's isotropic and VTI steps on the
    same case.  None when the build is absent."""
    so = os.path.join(ROOT, "oracle", "_ref", "libqvti_ref.so")
    if not os.path.exists(so):
        return None
    try:
        out = subprocess.run([sys.executable, os.path.join(ROOT, "oracle", "time_reference.py"), str(n), str(pml)],
                             capture_output=True, text=True, timeout=600)
    except subprocess.TimeoutExpired:
        return {"error": "timed out"}
    res = {}
    for line in out.stdout.splitlines():
        p = line.split()
        if len(p) == 4 and p[1] == "n=%d" % n:
            res[p[0]] = {"ms_per_step": float(p[2].split("=")[1]), "gcell_steps_per_s": float(p[3].split("=")[1])}
    if "reference_cufft" not in res:
        return {"error": (out.stderr or out.stdout)[-300:]}
    r = res["reference_cufft"]["ms_per_step"]
    return {"grid": [n, n, n], "pml": pml, "medium": "isotropic homogeneous", "timing": res,
            "speedup_iso": r / res["library_iso"]["ms_per_step"] if "library_iso" in res else None,
            "source": "oracle/_ref (reference cuviscoelas_3D.cu + cuFFT, unmodified, sm_100a), wall time of "
                      "cuda_forward_acoustic_3D: (t(45) - t(25)) / 20"}


# ----------------------------------------------------------------- our arm --
def tc_form(qv, sim, K, W, nprof, ntp, world, dist, ms_plain):
    """The split-precision tensor-core form on the same simulation: W warm-up
    and K timed steps (CUDA events on the engine's stream, max over ranks),
    its per-kernel times, and its agreement with the plain form: both forms
    run the same 60 steps from rest and their seismograms and final
    velocities are compared (relative L2)."""
    try:
        sim.set_form(qv.FORM_TC)
    except qv.QvtiError as e:
        return {"unavailable": str(e)}
    sim.step(W)
    sim.sync()
    dist.barrier()
    ms = dist.max(sim.step_timed(K))
    kernels = sim.profile_step(nprof)
    value = aggregate_value(ntp, K, world, ms)
    agree = {}
    runs = {}
    for form in (qv.FORM_PLAIN, qv.FORM_TC):
        sim.set_form(form)
        sim.reset()
        sim.step(60)
        runs[form] = (sim.records(), sim.fields(0, 3))
    sim.set_form(qv.FORM_TC)
    rel = lambda a, b: float(np.linalg.norm((a - b).astype(np.float64)) / max(np.linalg.norm(b.astype(np.float64)), 1e-30))
    for i, comp in enumerate(("vx", "vy", "vz")):
        agree["rec_" + comp] = rel(runs[qv.FORM_TC][0][i], runs[qv.FORM_PLAIN][0][i])
        agree["field_" + comp] = rel(runs[qv.FORM_TC][1][i], runs[qv.FORM_PLAIN][1][i])
    return {"form": "256-point y transforms as 16-point DFT products on tcgen05 (kind::tf32, 3 hi/lo terms, FP32 "
                    "accumulate in TMEM); other transforms FP32",
            "value": value, "ms_per_step": ms / K, "tc_vs_plain": (ms_plain / K) / (ms / K),
            "kernels": [{"name": n, "ms": round(m, 4), "gbs": round(b / (m / 1e3) / 1e9, 1)} for n, m, b in kernels],
            "relL2_vs_plain_60_steps": agree}


def our_arm(args, world, rank, local):
    qv = _load("qvti_b200", os.path.join(PKG, "qvti.py"))
    models = _load("qvti_models", os.path.join(PKG, "models.py"))
    dist = Dist(world, local)
    model, dt, lim, veff = make_model(models)
    nx, ny, nz = GRID
    ntp = nx * ny * nz
    K, W = args.steps, args.warmup
    nprof = 3
    nt = 2 * (W + K + nprof) + 60  # the plain form, the tensor-core form, their 60-step comparison
    rik = models.ricker(nt, dt, F0)
    r_ix, r_iy = models.surface_receivers(nx, ny)
    src = (nx // 2, ny // 2, PML + 5)

    sim = qv.Simulation(nx, ny, nz, PML, DX, DX, DX, dt, F0, vti=True, device=local)
    if args.form == "tc":
        sim.set_form(qv.FORM_TC)
    sim.set_model(model["velp"], model["vels"], model["rho"], model["gama_p"], model["gama_s"],
                  model["eps"], model["delta"])
    sim.set_receivers(PML, r_ix, r_iy)
    sim.set_source(*src, rik, kind=qv.SRC_FORCE_X)
    sim.reset()
    sim.step(W)
    sim.sync()

    dist.barrier()
    with ClockSampler(local) as clk:
        ms = sim.step_timed(K)  # CUDA events on the engine's stream, synchronised
    dist.barrier()
    ms_max = dist.max(ms)
    value = aggregate_value(ntp, K, world, ms_max)
    clocks = clk.summary()

    kernels = sim.profile_step(nprof)
    norms, nonfinite, _ = sim.norms()
    tc = None if args.no_tc else tc_form(qv, sim, K, W, nprof, ntp, world, dist, ms_max)
    sim.close()

    if args.no_e2e:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "grid": list(GRID),
                              "kernels": kernels, "finite": not nonfinite}), flush=True)
        dist.close()
        return 0
    # end to end through the public C ABI: host model (pinned), host wavelet,
    # receivers, K steps, seismograms back to host -- one call
    import torch
    pinned = {k: torch.from_numpy(model[k]).pin_memory() for k in
              ("velp", "vels", "rho", "gama_p", "gama_s", "eps", "delta")}
    recs = torch.empty((3, K, nx * ny), dtype=torch.float32).pin_memory()
    e2e_sim = qv.Simulation(nx, ny, nz, PML, DX, DX, DX, dt, F0, vti=True, device=local)
    F = ctypes.POINTER(ctypes.c_float)
    I = ctypes.POINTER(ctypes.c_int)

    def fp(t):
        return ctypes.cast(ctypes.c_void_p(t.data_ptr()), F)

    rik_k = np.ascontiguousarray(rik[:K])
    dist.barrier()
    t0 = time.perf_counter()
    rc = qv.lib().qvti_forward_shot(e2e_sim._h, *[fp(pinned[k]) for k in ("velp", "vels", "rho", "gama_p",
                                                                            "gama_s", "eps", "delta")],
                                    qv.SRC_FORCE_X, src[0], src[1], src[2], rik_k.ctypes.data_as(F), K, PML,
                                    r_ix.ctypes.data_as(I), r_iy.ctypes.data_as(I), nx * ny,
                                    fp(recs[0]), fp(recs[1]), fp(recs[2]))
    t_e2e = time.perf_counter() - t0
    e2e_sim.close()
    if rc != 0:
        raise SystemExit("qvti_forward_shot failed: %d" % rc)
    t_e2e = dist.max(t_e2e)
    e2e_value = ntp * K * world / t_e2e / 1e9
    h2d = 7 * ntp * 4 + K * 4 + 2 * nx * ny * 4
    d2h = 3 * K * nx * ny * 4

    top = max(kernels, key=lambda k: k[1])
    peak, peak_kind = measured_peaks()
    achieved = top[2] / (top[1] / 1e3) / 1e9
    traffic = ncu_traffic(top[0])
    step_ms = sum(k[1] for k in kernels)
    alg_bytes = sum(k[2] for k in kernels)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        # the reference arm's crop and method, fewer timed steps (about 20 s
        # of CPU work)
        cores = os.cpu_count() or 1
        rate, sec, crop = oracle_rate(model, CPU_CROP, 4, dt, cores)
        cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port", "sample": cpu_sample(crop, 4, sec, cores)}
    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_ref_gpu:
        ref_gpu = reference_gpu_timing(GRID[0], PML)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_desc(dt), "grid": list(GRID), "pml": PML, "dt_s": dt,
                       "cfl_dt_limit_s": lim, "form": "plain FP32",
                       "l2": "inputs larger than L2 (~14 GB of fields and spectra per step)",
                       "parallelism": "shot replicas, one per GPU" if world > 1 else "single GPU"},
            "roofline": {"bound": "hbm", "kernel": top[0], "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "alg_bytes_per_launch": top[2], "ms_per_launch": top[1]},
            "step_roofline": {"alg_bytes_per_cell_step": alg_bytes / ntp, "achieved_gbs": alg_bytes / (step_ms / 1e3) / 1e9,
                              "canonical_B_alg_T63": 1177},
            "kernels": [{"name": n, "ms": round(m, 4), "gbs": round(b / (m / 1e3) / 1e9, 1)} for n, m, b in kernels],
            "cpu_baseline": cpu,
            "reference_gpu": ref_gpu,
            "tc": tc,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K,
                    "seconds": t_e2e},
            "gpu_launches": len(kernels) * K,
            "clocks": clocks,
            "finite": not nonfinite,
        }
        print(json.dumps(line), flush=True)
    dist.close()
    return 0


# ------------------------------------------------------- batching form --
def _shot_case(md, model, n, pml, dt, nt, src, r_step):
    rik = md.ricker(nt, dt, F0)
    gx = np.arange(0, n[0], r_step, dtype=np.int32)
    gy = np.arange(0, n[1], r_step, dtype=np.int32)
    c = dict(ntx=n[0], nty=n[1], ntz=n[2], pml=pml, nt=nt, dx=DX, dy=DX, dz=DX, dt=dt, f0=F0, rik=rik,
             s_ix=int(src[0]), s_iy=int(src[1]), s_iz=int(src[2]), r_iz=pml,
             r_ix=np.repeat(gx, len(gy)), r_iy=np.tile(gy, len(gx)))
    c.update(model)
    return c


def batch_arm(args):
    """48 shots, grids drawn uniformly from {128^3, 160x160x128, 192^3,
    256x256x192}, each with its own seeded layered VTI model (5 % Gaussian
    perturbations, 80 m correlation: one field set per grid, rolled by a
    seeded shift per shot), source uniform in x, y and in the top 20 % below
    the C-PML, nt ~ U[1000, 2500] x --nt-scale, receivers every 4th surface
    point.  Runs the batch sequentially (one shot in flight) and with the
    autotuned scheduler; value = cell-steps of the batch / wall time."""
    qv = _load("qvti_b200", os.path.join(PKG, "qvti.py"))
    md = _load("qvti_models", os.path.join(PKG, "models.py"))
    rng = np.random.default_rng(SEED + 4)
    shapes = [(128, 128, 128), (160, 160, 128), (192, 192, 192), (256, 256, 192)]
    pml = 20
    bases = {n: md.perturbation_bases(n, SEED + 10 + i) for i, n in enumerate(shapes)}
    reqs, cells = [], 0
    for i in range(args.shots):
        n = shapes[int(rng.integers(len(shapes)))]
        nt = max(1, int(round(int(rng.integers(1000, 2501)) * args.nt_scale)))
        model = md.perturbed_layered(n, SEED + 100 + i, bases[n], rng.integers(0, n, size=3))
        dt, _, _ = md.choose_dt(model, DX, F0, DT_NOMINAL, vti=True)
        top = pml + max(1, int(0.2 * (n[2] - 2 * pml)))
        src = (rng.integers(pml, n[0] - pml), rng.integers(pml, n[1] - pml), rng.integers(pml, top))
        reqs.append(qv.ShotRequest(_shot_case(md, model, n, pml, dt, nt, src, 4), vti=True, ref_offset=False))
        cells += n[0] * n[1] * n[2] * nt
    del bases
    seq_res, seq_wall = qv.run_batch(reqs, max_active=1)
    seq_recs = [r.rec.copy() for r in reqs]
    res, wall = qv.run_batch(reqs, max_active=0)
    same = all(np.array_equal(a, r.rec) for a, r in zip(seq_recs, reqs))
    lat = sorted(r["latency_s"] for r in res)
    out = {"metric": "Gcell-steps/s, batch of %d uneven VTI shots" % args.shots, "value": cells / wall / 1e9,
           "unit": UNIT, "higher_is_better": True, "n_gpus": 1, "dtype": "f32", "data": "synthetic",
           "config": {"workload": "batching form: grids {128^3, 160x160x128, 192^3, 256x256x192}, layered VTI "
                                  "with 5%% perturbations, pml %d, nt U[1000,2500] x %g, receivers every 4th "
                                  "surface point" % (pml, args.nt_scale), "shots": args.shots,
                      "cell_steps": cells},
           "wall_s": wall, "sequential": {"value": cells / seq_wall / 1e9, "wall_s": seq_wall},
           "speedup_vs_sequential": seq_wall / wall, "identical_to_sequential": bool(same),
           "latency_s": {"p50": lat[len(lat) // 2], "p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))]},
           "status_ok": all(r["status"] == 0 for r in res + seq_res)}
    print(json.dumps(out), flush=True)
    return 0


# -------------------------------------------------------- serving form --
def serve_arm(args):
    """Poisson arrivals (rate --rate per s, for --duration s) of shots with
    grid axes log-uniform between 96 and 384 (x, y) and 96 and 256 (z),
    rounded to the nearest even 5-smooth size; nt ~ U[800, 3000] x
    --nt-scale; isotropic or VTI 50/50; seeded unperturbed layered models;
    admission by HBM footprint under a 150 GB budget.  A producer thread
    builds each request's model ahead of its arrival, a collector thread
    waits for results in submission order; latency is submit to seismograms
    on the host.  value = aggregate Gcell-steps/s."""
    import queue
    import threading
    qv = _load("qvti_b200", os.path.join(PKG, "qvti.py"))
    md = _load("qvti_models", os.path.join(PKG, "models.py"))
    rng = np.random.default_rng(SEED + 5)
    arrivals, t = [], 0.0
    while True:
        t += float(rng.exponential(1.0 / args.rate))
        if t > args.duration:
            break
        arrivals.append(t)
    specs = []
    for i in range(len(arrivals)):
        lx, ly, lz = (math.exp(rng.uniform(math.log(96), math.log(hi))) for hi in (384, 384, 256))
        n = (md.smooth_even(lx), md.smooth_even(ly), md.smooth_even(lz))
        nt = max(1, int(round(int(rng.integers(800, 3001)) * args.nt_scale)))
        vti = bool(rng.integers(2))
        pml = 20
        src = (int(rng.integers(pml, n[0] - pml)), int(rng.integers(pml, n[1] - pml)), pml + 5)
        specs.append((n, nt, vti, pml, src, SEED + 1000 + i))
    ready = queue.Queue(maxsize=6)

    def produce():
        for n, nt, vti, pml, src, seed in specs:
            prof = md.layered_profiles(n[2], seed)
            dt, _, _ = md.choose_dt(prof, DX, F0, DT_NOMINAL, vti=vti)
            model = md.layered_fast(n, seed, vti=vti)
            c = _shot_case(md, model, n, pml, dt, nt, src, 8)
            ready.put((qv.ShotRequest(c, vti=vti, ref_offset=False), n[0] * n[1] * n[2] * nt))

    th = threading.Thread(target=produce, daemon=True)
    th.start()
    late = 0.0
    done = queue.Queue()
    res = []
    policy = qv.SCHED_SMALLEST_FIRST if args.policy == "smallest_first" else qv.SCHED_FIFO
    with qv.Server(max_active=0, mem_budget=int(150e9), policy=policy) as srv:
        def collect():  # waits in submission order, releasing each request's host arrays
            while True:
                item = done.get()
                if item is None:
                    return
                tk, cs = item
                res.append((srv.wait(tk, timeout=-1.0), cs))

        col = threading.Thread(target=collect, daemon=True)
        col.start()
        t0 = time.perf_counter()
        for a in arrivals:
            req, cs = ready.get()
            now = time.perf_counter() - t0
            if now < a:
                time.sleep(a - now)
            else:
                late = max(late, now - a)
            done.put((srv.submit(req), cs))
            del req
        done.put(None)
        col.join()
        t_end = time.perf_counter() - t0
    ok = all(r["status"] == 0 for r, _ in res)
    lat = sorted(r["latency_s"] for r, _ in res)
    cells = sum(cs for _, cs in res)
    q = lambda p: lat[min(len(lat) - 1, int(p * len(lat)))]
    out = {"metric": "shot latency p50/p99 and aggregate Gcell-steps/s, serving", "value": cells / t_end / 1e9,
           "unit": UNIT, "higher_is_better": True, "n_gpus": 1, "dtype": "f32", "data": "synthetic",
           "latency_s": {"p50": q(0.5), "p99": q(0.99), "max": lat[-1]},
           "requests": len(res), "offered_rate_per_s": args.rate, "arrival_window_s": args.duration,
           "admission": args.policy,
           "max_submit_lag_s": late, "run_s": t_end, "status_ok": ok,
           "config": {"workload": "serving form: Poisson %.1f/s, axes log-uniform 96..384 (x,y), 96..256 (z) "
                                  "rounded to even 5-smooth, nt U[800,3000] x %g, iso/VTI 50/50, layered, pml 20, "
                                  "150 GB budget" % (args.rate, args.nt_scale)}}
    print(json.dumps(out), flush=True)
    return 0


# ------------------------------------------------------ precision form --
def precision_arm(args):
    """Precision form: the VTI generator at 512 x 512 x 256 (seed 2024, its
    own perturbation fields, dt from its stability bound), pml 30, 20 Hz
    force at (256, 256, 35), receivers every 4th surface point; --nt steps
    (3000) from rest in the plain FP32 form and, where the grid has one, the
    tensor-core form, each timed whole with CUDA events.  Accuracy: the
    centred 128^3 crop of the same model (400 steps) run in each form and
    compared with the FP64 oracle's run of that crop
    (tests/golden/oracle/vti512_crop128.npz): relative L2 of each seismogram
    component and of vx, vy, vz on two planes every 100 steps (worst over
    the snapshots), and the peak seismogram error max|d| / max|ref|."""
    qv = _load("qvti_b200", os.path.join(PKG, "qvti.py"))
    md = _load("qvti_models", os.path.join(PKG, "models.py"))
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import make_oracle_golden as mog
    shape, pml, nt = (512, 512, 256), 30, args.nt
    model = md.layered_vti(shape, DX, seed=SEED)
    dt, lim, _ = md.choose_dt(model, DX, F0, DT_NOMINAL, vti=True)
    gx = np.arange(0, shape[0], 4, dtype=np.int32)
    gy = np.arange(0, shape[1], 4, dtype=np.int32)
    r_ix, r_iy = np.repeat(gx, gy.size), np.tile(gy, gx.size)
    rik = md.ricker(nt, dt, F0)
    forms = {}
    with qv.Simulation(*shape, pml, DX, DX, DX, dt, F0, vti=True) as sim:
        sim.set_model(*[model[k] for k in ("velp", "vels", "rho", "gama_p", "gama_s", "eps", "delta")])
        sim.set_receivers(pml, r_ix, r_iy)
        sim.set_source(shape[0] // 2, shape[1] // 2, pml + 5, rik)
        for name, form in (("plain", qv.FORM_PLAIN), ("tc", qv.FORM_TC)):
            try:
                sim.set_form(form)
            except qv.QvtiError as e:
                forms[name] = {"unavailable": str(e)}
                continue
            sim.reset()
            sim.step(5)  # graph build and first launches, untimed
            sim.reset()
            with ClockSampler(0) as clk:
                ms = sim.step_timed(nt)
            norms, bad, _ = sim.norms()
            forms[name] = {"value": shape[0] * shape[1] * shape[2] * nt / (ms / 1e3) / 1e9, "seconds": ms / 1e3,
                           "ms_per_step": ms / nt, "finite": not bad, "clocks": clk.summary()}
    crop = mog.crop128_case(shape, "vti512_crop128", 400, model=model)
    del model
    path = os.path.join(ROOT, "tests", "golden", "oracle", "vti512_crop128.npz")
    acc = {}
    if os.path.exists(path):
        g = dict(np.load(path))
        snaps = list(range(100, 401, 100))
        for name, form in (("plain", qv.FORM_PLAIN), ("tc", qv.FORM_TC)):
            try:
                ours = qv.run_case(crop, snaps=snaps, vti=True, ref_offset=False, form=form)
            except qv.QvtiError as e:
                acc[name] = {"unavailable": str(e)}
                continue
            rel = lambda a, b: float(np.linalg.norm((a - b).astype(np.float64)) / np.linalg.norm(b.astype(np.float64)))
            e = {}
            for i, comp in enumerate(("vx", "vy", "vz")):
                e["rec_" + comp] = rel(ours["rec"][i], g["rec_" + comp])
                e["field_" + comp] = max(max(rel(ours["snaps"][k][i][:, int(crop["plane_y"]), :], g["plane_y_%d" % k][i]),
                                             rel(ours["snaps"][k][i][:, :, int(crop["plane_z"])], g["plane_z_%d" % k][i]))
                                         for k in snaps)
            ref = np.stack([g["rec_vx"], g["rec_vy"], g["rec_vz"]])
            e["peak_seismogram_err"] = float(np.abs(ours["rec"] - ref).max() / np.abs(ref).max())
            e["worst_relL2"] = max(v for k, v in e.items() if k != "peak_seismogram_err")
            acc[name] = e
    else:
        acc = {"unavailable": "oracle fixture tests/golden/oracle/vti512_crop128.npz missing"}
    out = {"metric": "Gcell-steps/s 512x512x256 VTI, %d steps; per-field relL2 vs FP64 oracle (128^3 crop)" % nt,
           "value": forms["plain"]["value"], "unit": UNIT, "higher_is_better": True, "n_gpus": 1, "dtype": "f32",
           "data": "synthetic", "forms": forms, "accuracy_crop128_400_steps": acc,
           "config": {"workload": "precision form: VTI generator at 512x512x256 (6 layers, eps/delta/Q per layer, 5%% "
                                  "Gaussian perturbations, seed %d), pml %d, dt %.2f ms (0.8 ms capped to 80%% of the "
                                  "stability bound %.2f ms), 20 Hz force at (256,256,%d), receivers every 4th surface "
                                  "point; accuracy on the centred 128^3 crop (pml 20, 400 steps) against the FP64 "
                                  "oracle" % (SEED, pml, dt * 1e3, lim * 1e3, pml + 5),
                      "grid": list(shape), "steps": nt}}
    print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--no-ref-gpu", action="store_true", help="skip timing the reference's cuFFT build")
    ap.add_argument("--no-tc", action="store_true", help="skip the tensor-core form")
    ap.add_argument("--grid", type=int, default=256, help="cube edge (profiling of smaller cases)")
    ap.add_argument("--ny", type=int, default=0, help="y length other than --grid (profiling of smaller cases)")
    ap.add_argument("--form", default="plain", choices=["plain", "tc"],
                    help="form of the timed steps (profiling; the default line times the plain form and "
                         "reports the tensor-core form beside it)")
    ap.add_argument("--workload", default="step", choices=["step", "batch", "serve", "precision"])
    ap.add_argument("--nt", type=int, default=3000, help="precision: steps of the 512x512x256 run")
    ap.add_argument("--shots", type=int, default=48, help="batch: number of shots")
    ap.add_argument("--nt-scale", type=float, default=0.1, help="batch/serve: fraction of the nominal nt")
    ap.add_argument("--rate", type=float, default=4.0, help="serve: arrivals per second")
    ap.add_argument("--policy", default="fifo", choices=["fifo", "smallest_first"],
                    help="serve: admission order of waiting shots")
    ap.add_argument("--duration", type=float, default=60.0, help="serve: arrival window (s)")
    args = ap.parse_args()
    if args.workload == "batch":
        return batch_arm(args)
    if args.workload == "serve":
        return serve_arm(args)
    if args.workload == "precision":
        return precision_arm(args)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    world, rank, local = dist_setup()
    if args.grid != 256 or args.ny:
        global GRID, PML
        GRID = (args.grid, args.ny or args.grid, args.grid)
        PML = min(30, max(4, min(GRID) // 8))
    if args.impl == "reference":
        return reference_arm(args, world, rank)
    return our_arm(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
