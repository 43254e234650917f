"""Throughput of the FMT2D forward hot path on B200: eikonal time fields per second.

Workload (one step): every OBS source x every stage of the Pg and PmP phases of
the joint velocity + Moho model, 2001 x 401 nodes at 0.1 km (30 OBS every
6.5 km; Pg = 1 field, PmP = 2 stages down to the Moho and back up), i.e. 90
eikonal time fields, solved through the library's public entry point.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

* value  : fields/s with the model resident on the device (device-timed with
           CUDA events on the library's stream, max over ranks).
* e2e    : the same metric through the public API from host buffers: model
           upload (host arrays -> device), the forward solve, and the read-back
           of every terminal-stage traveltime field to host memory.
* roofline: the field solve (k_solve) against the measured HBM bandwidth,
           with the algorithmic traffic of one field: 16 B per region node
           (4 B slowness read, 4 B time and 8 B gradient written, the FP32
           figure of the traveltime contract; the FP64 fields this build keeps
           move 36 B per node, reported beside it), over the forward's device
           time (the solves of independent stage chains overlap).
* max_err_ms: the largest traveltime difference, over every reached node of
           every field of one source, against the FP64 heap fast marching
           restatement (oracle/, the checker); reached sets must agree.
* rays, lsqr: ray backtrace + Frechet rows of every Pg and PmP pick of the
           model (picks/s, device-timed), and the LSQR solve on those rows
           (s per LSQR iteration).
* adjoint: the misfit gradient w.r.t. the grid slowness by the discrete
           adjoint of the same fields (fmt2d_misfit_gradient, s per gradient).
* cpu_baseline: the FP64 CPU restatement of the reference algorithm (oracle/)
           on the host cores, over a bounded sample of the same workload
           (pool warmed first, median of 3 timed repetitions).
* --impl reference: the CPU restatement timed on all host cores (the reference
           Fortran cannot be built here: no Fortran compiler in the image).

Multi-GPU: one process per GPU (torchrun).  Sources are independent, so the
ranks share out a larger source set: rank r solves the model's 30 OBS
positions shifted by r/N of the OBS spacing (30 N distinct sources in all),
with no collective on the data path (weak scaling); the step time is the max
over ranks.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

PHASES = (1, 3)          # Pg, PmP
WORKLOAD = "fmt2d forward, 2001x401 joint velocity+Moho model, 30 OBS, Pg+PmP (90 fields)"
METRIC = "eikonal fields/s @2001x401 (<=0.5 ms err)"


def _env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


# ---------------------------------------------------------------- CPU arms
_CPU_STATE = {}


def _cpu_init():
    if "o" not in _CPU_STATE:
        sys.path.insert(0, os.path.join(HERE, "oracle"))
        import pyoracle
        from fmt2d_b200 import synth
        m = synth.config(1)
        _CPU_STATE.update(m=m, o=pyoracle.Oracle(m))


def _cpu_worker(args):
    """One process of the CPU restatement: solve the given sources, return seconds.
    The model is generated and built once per process, outside the timing."""
    src_idx, phases = args
    _cpu_init()
    from fmt2d_b200.api import phase_mask
    m, o = _CPU_STATE["m"], _CPU_STATE["o"]
    mask = phase_mask(phases)
    t0 = time.perf_counter()
    for s in src_idx:
        o.forward(0, float(m.obs_x[s]), mask)
    return time.perf_counter() - t0


def _cpu_fields_of_source(args):
    """The checker: the CPU restatement's traveltimes of every field of one
    source (FP64 heap fast marching)."""
    sx, phases = args
    _cpu_init()
    from fmt2d_b200.api import fields_of, phase_mask
    o = _CPU_STATE["o"]
    mask = phase_mask(phases)
    o.forward(0, float(sx), mask)
    return {tf: o.field(0, tf)[0] for tf in fields_of(mask)}


def cpu_fields_per_s(nsrc: int, procs: int, reps: int = 3, check_x=None):
    """Fields/s of the CPU restatement over `nsrc` sources on `procs` processes
    (the pool is warmed by one untimed pass; median of `reps` timed passes),
    the processes' mean single-core rate, the wall times and, for check_x,
    the checker's fields of a source at that x."""
    from fmt2d_b200.api import fields_of, phase_mask
    nf_src = len(fields_of(phase_mask(PHASES)))
    ctx = mp.get_context("spawn")
    chunks = [list(range(i, nsrc, procs)) for i in range(procs)]
    chunks = [c for c in chunks if c]
    checked = None
    with ctx.Pool(len(chunks), initializer=_cpu_init) as pool:
        pool.map(_cpu_worker, [(c[:1], PHASES) for c in chunks])
        if check_x is not None:
            checked = pool.map(_cpu_fields_of_source, [(check_x, PHASES)])[0]
        walls, rates = [], []
        for _ in range(reps):
            t0 = time.perf_counter()
            secs = pool.map(_cpu_worker, [(c, PHASES) for c in chunks])
            walls.append(time.perf_counter() - t0)
            rates += [len(c) * nf_src / t for c, t in zip(chunks, secs) if t > 0]
    one = float(np.mean(rates)) if rates else 0.0
    return nsrc * nf_src / float(np.median(walls)), len(chunks), walls, one, checked


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu, self.rows, self.proc = gpu, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in self.rows if len(r) >= 8 and num(r[1]) is not None]
        mx = [num(r[2]) for r in self.rows if len(r) >= 8 and num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) >= 8
                          for i in range(4) if r[4 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


# ---------------------------------------------------------------- helpers
def measured_peak_hbm():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        for k in ("hbm_gbs", "hbm_GBps", "hbm"):
            if k in d:
                return float(d[k]), "measured"
    except (OSError, ValueError):
        pass
    return 6650.0, "fallback"


# DRAM bytes (read + write) per region node of the field solve (k_solve), from
# an ncu capture of one launch on 4 Pg fields of this model (2,581,316 region
# nodes, 163.5 MB read + 127.6 MB written): profiles/k_solve_2001x401_pg_4src.md
K_SOLVE_DRAM_BYTES_PER_NODE = 112.8


def traffic_per_step(nodes_step: float):
    """DRAM traffic of the step's field solves, scaled from the captured
    launch by region nodes (the solve's traffic grows with the nodes)."""
    if K_SOLVE_DRAM_BYTES_PER_NODE is None:
        return None
    return round(K_SOLVE_DRAM_BYTES_PER_NODE * nodes_step)


def dist_setup(n_gpus):
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE); NCCL
    when a CUDA device is present, gloo otherwise (host-only runs and tests).
    Only the timing is reduced across ranks: the sources are independent."""
    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local = _env_int("LOCAL_RANK", 0)
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(x: float, world: int, device) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------- arms
def run_reference(args, world, rank):
    """CPU restatement of the reference path on all host cores (rank 0 only)."""
    if rank != 0:
        return
    from fmt2d_b200 import synth
    from fmt2d_b200.api import fields_of, phase_mask
    cores = os.cpu_count() or 1
    m = synth.config(1)
    nsrc_all = len(m.obs_x)
    # each step: a bounded sample of the workload (sources spread over the cores)
    nsrc = min(nsrc_all, max(cores, 4))
    nf_src = len(fields_of(phase_mask(PHASES)))
    ctx = mp.get_context("spawn")
    procs = min(cores, nsrc)
    chunks = [list(range(i, nsrc, procs)) for i in range(procs)]
    walls, rates = [], []
    with ctx.Pool(procs, initializer=_cpu_init) as pool:
        for step in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            secs = pool.map(_cpu_worker, [(c, PHASES) for c in chunks])
            if step >= args.warmup:
                walls.append(time.perf_counter() - t0)
                rates += [len(c) * nf_src / t for c, t in zip(chunks, secs) if t > 0]
    sec = float(np.sum(walls))
    value = nsrc * nf_src * len(walls) / sec
    out = {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "fields/s",
           "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(1e3 * sec / len(walls), 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": WORKLOAD, "sample_sources": nsrc, "fields_per_step":
                      nsrc * nf_src},
           "cpu_baseline": {"value": round(value, 3), "unit": "fields/s", "cores": procs,
                            "kind": "port",
                            "sample": f"{nsrc} of {nsrc_all} sources x Pg+PmP stages per step, "
                                      f"FP64 heap fast marching, {procs} processes",
                            "single_core": {"value": round(float(np.mean(rates)), 3)
                                            if rates else None, "unit": "fields/s",
                                            "sample": "mean rate of one process (one core)"}},
           "e2e": {"value": round(value, 3), "unit": "fields/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0},
           "gpu_launches": 0}
    print(json.dumps(out), flush=True)


def source_set(m, rank: int, world: int) -> np.ndarray:
    """Sources of one rank: the model's OBS positions shifted by rank/world of
    the OBS spacing (on grid nodes), so the ranks solve distinct sources."""
    x = np.asarray(m.obs_x, dtype=np.float64)
    if world > 1 and x.size > 1:
        x = x + rank * (x[1] - x[0]) / world
        x = np.round(x / m.dx) * m.dx
        x = np.clip(x, m.xpos[1], m.xpos[-2])
    return x


def max_error_ms(g, checked, mask):
    """Largest |T_device - T_checker| (ms) over the nodes both reach, and the
    number of nodes reached by one side only, over every field of source 0."""
    from fmt2d_b200.api import fields_of
    worst, reach_diff = 0.0, 0
    for tf in fields_of(mask):
        To = checked[tf]
        Tg = g.field(0, tf)[0]
        ro, rg = To < 1e19, Tg < 1e19
        reach_diff += int((ro != rg).sum())
        both = ro & rg
        if both.any():
            worst = max(worst, float(np.abs(To[both] - Tg[both]).max()))
    return worst * 1e3, reach_diff


def timed_on(stream, fn):
    """Run fn and return (its result, device ms between events on stream)."""
    import torch
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    out = fn()
    b.record(stream)
    b.synchronize()
    return out, a.elapsed_time(b)


def rays_and_lsqr(g, m, stream, nsrc=None, phases=None):
    """Ray backtrace + Frechet rows of every pick of the model on the fields
    of the last forward (picks/s), then the damped, smoothed LSQR solve on the
    selected rows (s per LSQR iteration).  Observed times are the computed
    ones plus seeded 40 ms Gaussian noise (config-1 pick noise).  nsrc /
    phases: only the picks of the first nsrc sources and of those phases
    (the fields a reduced run solved)."""
    from fmt2d_b200.api import select_data
    P = m.picks
    if nsrc is not None:
        P = P[P[:, 0] < nsrc]
    if phases is not None:
        P = P[np.isin(P[:, 1], phases)]
    src = P[:, 0].astype(np.int32)
    ph = P[:, 1].astype(np.int32)
    rx, rz = P[:, 2].copy(), P[:, 3].copy()
    g.trace(src, ph, rx, rz)                       # warm (tables, buffers)
    (t, valid, nnz), tr_ms = timed_on(stream, lambda: g.trace(src, ph, rx, rz))
    rp, gi, gv = g.frechet_rows()
    rng = np.random.default_rng(1)
    obs = np.where(valid, t + rng.normal(0.0, 0.040, t.size), -1.0)
    _, nvp, npar = g.inv_index()
    mv = np.ones(npar)
    srp, sgi, sgv, res, wt, _ = select_data(ph, obs, t, valid, rp, gi, gv, mv, crit_chi=1.0)
    nd = srp.size - 1
    g.set_frechet(nd, npar, srp, sgi, sgv)
    gtg = g.gtg_diag()
    eps_min = max(1e-6, 1e-4 * float(gtg.max()))
    iters = 100
    g.lsqr(res, np.zeros(npar), gtg, wdv=1.0, wdv_iface=1.0, w_smooth=10.0,
           w_smooth_iface=10.0, eps_min=0.0, max_iter=8)  # warm (graph, buffers)
    _, it, _, _, _ = g.lsqr(res, np.zeros(npar), gtg, wdv=1.0, wdv_iface=1.0, w_smooth=10.0,
                            w_smooth_iface=10.0, eps_min=eps_min, max_iter=iters)
    ls = g.lsqr_stats()
    rays = {"value": round(P.shape[0] / (tr_ms / 1e3), 1), "unit": "picks/s",
            "picks": int(P.shape[0]), "valid": int(valid.sum()), "frechet_nnz": int(nnz),
            "ms": round(tr_ms, 3), "note": "fmt2d_trace, device-timed, fields resident"}
    lsqr = {"value": round(ls["ms"] / 1e3 / max(it, 1), 6), "unit": "s per LSQR iteration",
            "iterations": int(it), "ndata": int(nd), "nparm": int(npar), "nnz": int(sgi.size),
            "ms": round(ls["ms"], 3), "smooth_type": 1,
            "note": "fmt2d_lsqr, damping 1, Laplacian 10, device-timed"}
    # misfit gradient w.r.t. the grid slowness by the discrete adjoint of the
    # same fields (the call traces the picks again), wall time of the call
    g.misfit_gradient(src, ph, rx, rz, obs, 0.040)       # warm
    t0 = time.perf_counter()
    out = g.misfit_gradient(src, ph, rx, rz, obs, 0.040)
    adj_s = time.perf_counter() - t0
    info = out["info"]
    if np.any(info[:3] != 0):
        raise RuntimeError(f"adjoint could not follow the forward: {info[:3].tolist()}")
    adjoint = {"value": round(adj_s, 4), "unit": "s per misfit gradient",
               "fields": int(info[4]), "nodes": int(info[5]), "sweep_rounds": int(info[3]),
               "picks": int(P.shape[0]),
               "note": "fmt2d_misfit_gradient: trace + discrete adjoint of every field + map "
                       "onto the 2001x401 slowness grid, wall time, fields resident"}
    return rays, lsqr, adjoint


def inversion_iterations(local, n_iter: int = 2, cfg: int = 1):
    """Seconds per outer inversion iteration (the lsqr_inversion2d loop body,
    fmt2d_b200.inversion) through the public API.  Observed times are the
    checkerboard model's (device forward + rays, seeded Gaussian noise), the
    inversion starts from the smooth model with a flat Moho, alternating
    velocity / interface updates.  cfg 1: the 2001x401 model, 30 OBS, Pg+PmP,
    40 ms noise, fixed damping 1, Laplacian smoothing 10.  cfg 4: the 4001x601
    model, 100 OBS, all five phases, 30-60 ms noise by phase, auto damping
    and hybrid smoothing.  Each iteration: forward + rays + Frechet rows,
    selection, damped LSQR solves, line-search forwards with model steps."""
    from fmt2d_b200 import synth
    from fmt2d_b200.api import Fmt2d
    from fmt2d_b200.inversion import Inversion, InversionParams
    true, start = synth.config(cfg), synth.start_model(cfg)
    P = true.picks
    if cfg == 4:
        phases = (1, 2, 3, 4, 5)
        sigma = np.array([0.0, 0.030, 0.040, 0.050, 0.060, 0.060])[P[:, 1].astype(int)]
        params = InversionParams(phases=phases, lam_damp=0.0, lam_smooth=10.0,
                                 lam_smooth_iface=10.0, smooth_type=3, corr_x_iface=2.0,
                                 lsqr_max_iter=500, crit_chi=1.0, alt_inv_mode=-1)
    else:
        phases = PHASES
        sigma = np.full(P.shape[0], 0.040)
        params = InversionParams(phases=phases, lam_damp=1.0, lam_smooth=10.0,
                                 lam_smooth_iface=10.0, crit_chi=1.0, alt_inv_mode=-1)
    t0 = time.perf_counter()
    g = Fmt2d(local).upload(true)
    g.forward(true.obs_x, phases)
    t, valid, _ = g.trace(P[:, 0].astype(np.int32), P[:, 1].astype(np.int32), P[:, 2], P[:, 3])
    g.close()
    rng = np.random.default_rng(cfg)
    obs = np.where(valid, t + rng.normal(0.0, 1.0, t.size) * sigma, -1.0)
    t_obs = time.perf_counter() - t0
    g = Fmt2d(local).upload(start)
    tune = g.autotune(start.obs_x, phases)
    inv = Inversion(g, start.obs_x, P, obs, params)
    rows = []
    for _ in range(n_iter):
        r = inv.iteration()
        rows.append({"s": round(r.seconds, 3), "rms_orig_ms": round(1e3 * r.rms_orig, 3),
                     "rms_new_ms": round(1e3 * r.rms_new, 3), "step": r.step, "ndata": r.ndata,
                     "mode": r.mode, "forwards": r.forwards, "lsqr_solves": r.lsqr_solves,
                     "phases_s": {k: round(v, 3) for k, v in r.phases_s.items()}})
    g.close()
    grid = f"{true.nx}x{synth.config(cfg).pgrid_nz()}"
    return {"value": round(float(np.mean([x["s"] for x in rows])), 3),
            "unit": "s per inversion iteration", "iterations": rows,
            "workload": f"config {cfg}: {grid}, {true.obs_x.size} OBS, phases {phases}, "
                        f"{P.shape[0]} picks, start: smooth model, flat Moho",
            "observed_times_s": round(t_obs, 3), "autotune": tune,
            "note": "wall clock through the public API, 1 GPU"}


def uneven_batch(local, n_models: int, stream_dev):
    """The uneven multi-model batch: n_models seeded models of grid sizes from
    401x121 to 2001x401, up to 20 OBS each, all five phases, solved in one
    fmt2d_forward_batch call; the same models one fmt2d_forward after another
    beside it.  Fields/s, wall clock on the device's work (the calls return
    when their fields are solved)."""
    from fmt2d_b200 import synth
    from fmt2d_b200.api import Fmt2d, fields_of, forward_batch, phase_mask
    phases = (1, 2, 3, 4, 5)
    models = [synth.uneven_model(k, max_obs=20) for k in range(n_models)]
    ctxs = [Fmt2d(local).upload(m) for m in models]
    srcs = [np.asarray(m.obs_x, dtype=np.float64) for m in models]
    nf = sum(x.size for x in srcs) * len(fields_of(phase_mask(phases)))
    forward_batch(ctxs, srcs, phases)                       # warm (field stores)
    t0 = time.perf_counter()
    forward_batch(ctxs, srcs, phases)
    tb = time.perf_counter() - t0
    t0 = time.perf_counter()
    for g, x in zip(ctxs, srcs):
        g.forward(x, phases)
    ts = time.perf_counter() - t0
    sizes = [f"{m.nx}x{g.nz}" for m, g in zip(models, ctxs)]
    for g in ctxs:
        g.close()
    return {"value": round(nf / tb, 3), "unit": "fields/s", "models": n_models, "fields": nf,
            "s": round(tb, 3), "one_model_at_a_time": {"value": round(nf / ts, 3),
                                                       "s": round(ts, 3)},
            "grids": sizes, "phases": "all five",
            "note": "fmt2d_forward_batch over the models' contexts vs fmt2d_forward per model"}


def run_ours(args, world, rank, local):
    from fmt2d_b200 import synth
    from fmt2d_b200.api import fields_of, phase_mask
    global PHASES
    if args.phases:
        PHASES = tuple(int(p) for p in args.phases.split(","))
    m = synth.config(1)
    src = source_set(m, rank, world)
    if args.sources > 0:
        src = src[:args.sources]
    mask = phase_mask(PHASES)
    cpu, checked = None, None
    if rank == 0 and world == 1 and not args.no_cpu:
        # before the first CUDA call: the CPU restatement on the host cores,
        # and the checker's fields of source 0
        cores = os.cpu_count() or 1
        nsrc = min(30, max(4, cores))
        procs = min(cores, nsrc)
        v, used, walls, one, checked = cpu_fields_per_s(nsrc, procs, reps=3,
                                                        check_x=float(src[0]))
        cpu = {"value": round(v, 3), "unit": "fields/s", "cores": used, "kind": "port",
               "sample": f"{nsrc} sources x Pg+PmP stages of the same model, FP64 heap fast "
                         f"marching, {used} processes, pool warmed, median of "
                         f"{len(walls)} passes ({', '.join(f'{w:.1f}' for w in walls)} s wall)",
               "single_core": {"value": round(one, 3), "unit": "fields/s",
                               "sample": "mean rate of one process (one core) in that run"}}
    import torch
    from fmt2d_b200.api import Fmt2d, TF_REGION
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    g = Fmt2d(local).upload(m)
    stream = torch.cuda.ExternalStream(g.stream(), device=dev)
    nf = len(fields_of(mask)) * src.size
    # the last stage of each phase (ray tracing starts there)
    terminal = sorted({{1: 1, 2: 3, 3: 5, 4: 8, 5: 12}[p] for p in PHASES})

    # the solve block size for this workload (bit-identical results for every
    # size), picked by the library's autotuner before the warm-up
    tune = g.autotune(src, PHASES)
    for _ in range(args.warmup):
        g.forward(src, PHASES)
    torch.cuda.synchronize()

    # ---- device-resident timing (fmt2d_forward raises Fmt2dNotConverged if a
    # field does not reach its fixed point; the counters are checked too)
    launches, nodes, capped, unsettled = 0, 0, 0, 0
    with ClockSampler(local) as clk:
        barrier(world)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            g.forward(src, PHASES)
            st = g.stats()
            launches += st["launches"]
            nodes += st["nodes"]
            capped += st["capped"]
            unsettled += st["unsettled"]
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        barrier(world)
        ms = e0.elapsed_time(e1)
    if capped or unsettled:
        raise RuntimeError(f"forward not converged: capped={capped} unsettled={unsettled}")
    ms = max_over_ranks(ms, world, dev)
    step_ms = ms / args.steps
    value = world * nf / (step_ms / 1e3)
    solver = {k: st[k] for k in ("steps", "steps_all", "evals", "writes", "passes")}

    err_ms, reach_diff = (None, None)
    if checked is not None:
        err_ms, reach_diff = max_error_ms(g, checked, mask)
        if err_ms > 0.5 or reach_diff > 2 * len(checked):
            raise RuntimeError(f"traveltime error {err_ms:.4f} ms, reach differs at "
                               f"{reach_diff} nodes")

    # ---- end to end through the public API from host buffers
    bufs = {}
    for tf in terminal:
        n = g.region_nnode(TF_REGION[tf])
        bufs[tf] = np.zeros(n)
    h2d = sum(np.asarray(a).nbytes for a in (m.xpos, m.topo, m.zrel, m.vel, m.sed_z, m.moho_z))
    h2d += src.nbytes
    d2h = sum(src.size * bufs[tf].nbytes for tf in terminal)

    def e2e_step():
        g.upload(m)
        g.forward(src, PHASES)
        for s in range(src.size):
            for tf in terminal:
                g._check(g.L.fmt2d_get_field(g.h, s, tf, bufs[tf].ctypes.data, None, None),
                         "fmt2d_get_field")

    e2e_step()
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    e2e_steps = max(1, min(args.steps, 3))
    for _ in range(e2e_steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / e2e_steps, world, dev)
    e2e_value = world * nf / e2e_s

    # ---- rays + Frechet rows and LSQR on the same fields (every rank, the
    # same steps, outside the timed region)
    try:
        g.forward(src, PHASES)
        rays, lsqr, adjoint = rays_and_lsqr(g, m, stream, src.size, PHASES)
    except Exception as ex:  # the eikonal line is the result; report why these are absent
        rays = lsqr = adjoint = {"unavailable": str(ex)[:200]}

    # ---- s per inversion iteration (rank 0 of a 1-GPU run; outside the
    # timed region)
    inversion = None
    if world == 1 and not args.no_inversion:
        try:
            inversion = inversion_iterations(local, args.inversion_iters, args.inversion_config)
        except Exception as ex:
            inversion = {"unavailable": str(ex)[:200]}

    # ---- the uneven multi-model batch (outside the timed region)
    batch = None
    if world == 1 and args.models > 0:
        try:
            batch = uneven_batch(local, args.models, dev)
        except Exception as ex:
            batch = {"unavailable": str(ex)[:200]}

    # ---- the plain form, one source (its stage solves) per fmt2d_forward call,
    # on a few sources: the denominator of "batched vs plain"
    try:
        k = int(min(3, src.size))
        torch.cuda.synchronize()
        _, plain_ms = timed_on(stream, lambda: [g.forward(src[i:i + 1], PHASES)
                                                for i in range(k)])
        plain = {"value": round(k * len(fields_of(mask)) / (plain_ms / 1e3), 3),
                 "unit": "fields/s", "sources_timed": k,
                 "note": "one source per fmt2d_forward call, device-timed"}
    except Exception as ex:
        plain = {"unavailable": str(ex)[:200]}

    if rank != 0:
        g.close()
        return
    peak, peak_kind = measured_peak_hbm()
    nodes_step = nodes / args.steps
    alg_bytes = 16.0 * nodes_step                  # per step, all fields
    achieved = alg_bytes / (step_ms / 1e3) / 1e9
    out = {"metric": METRIC, "value": round(value, 3), "unit": "fields/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(step_ms, 3),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic",
           "config": {"workload": WORKLOAD, "grid": "2001x401", "sources_per_gpu": int(src.size),
                      "fields_per_gpu": nf, "l2": "field data per step (> 1 GB) exceeds L2",
                      "parallelism": f"sources x {world} gpus, independent"},
           "max_err_ms": round(err_ms, 5) if err_ms is not None else None,
           "reach_diff_nodes": reach_diff,
           "converged": {"capped": int(capped), "unsettled": int(unsettled)},
           "e2e": {"value": round(e2e_value, 3), "unit": "fields/s", "h2d_bytes_per_step": int(h2d),
                   "d2h_bytes_per_step": int(d2h), "includes": "model upload, forward, "
                   "terminal-stage traveltime read-back"},
           "roofline": {"bound": "hbm", "kernel": "k_solve",
                        "achieved": round(achieved, 4), "peak": peak, "unit": "GB/s",
                        "frac": round(achieved / peak, 7), "peak_kind": peak_kind,
                        "traffic": traffic_per_step(nodes_step),
                        "algorithmic_bytes_per_step": alg_bytes,
                        "bytes_per_node": 16, "fp64_bytes_per_node": 36,
                        "fp64_frac": round(36.0 * nodes_step / (step_ms / 1e3) / 1e9 / peak, 7)},
           "solver": solver, "autotune": tune,
           "rays": rays, "lsqr": lsqr, "adjoint": adjoint, "inversion": inversion, "uneven_batch": batch,
           "plain": plain,
           "gpu_launches": int(launches), "clocks": clk.summary(),
           "cpu_baseline": cpu}
    print(json.dumps(out), flush=True)
    g.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-inversion", action="store_true",
                    help="skip the s-per-inversion-iteration leg")
    ap.add_argument("--inversion-config", type=int, default=1, choices=[1, 4],
                    help="model of the inversion leg: 1 (2001x401) or 4 (4001x601, minutes)")
    ap.add_argument("--inversion-iters", type=int, default=2)
    ap.add_argument("--models", type=int, default=8,
                    help="models of the uneven multi-model batch leg (0: skip)")
    ap.add_argument("--sources", type=int, default=0,
                    help="solve only the first N sources (profiling captures; 0: all 30)")
    ap.add_argument("--phases", default="",
                    help="comma-separated phase ids to solve (profiling captures; default 1,3)")
    args = ap.parse_args()
    if args.impl == "reference":
        # host-core arm: rank 0 alone runs it, the other ranks exit without work
        run_reference(args, _env_int("WORLD_SIZE", 1), _env_int("RANK", 0))
        return
    world, rank, local = dist_setup(args.gpus)
    try:
        run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
