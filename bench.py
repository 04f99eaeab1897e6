"""Throughput of the coupled phase-field step on B200.

Workload (one step = one time step of the whole grid): Ti-10at%Nb
directional solidification, 2048 x 2048 cells (Nx_all x Ny_all, 2046^2
interior), exact CALPHAD chemistry, frozen temperature G = 5e6 K/m,
V = 0.5 m/s, moving frame on (pull-back every step_pull_back = 1008 steps),
seeded Philox interface noise of amplitude 0.01.  Synthetic input: seeded
planar front.  The headline line computes in FP64, the reference's
arithmetic (its CPU arm, `--impl reference`, runs the same configuration);
the FP32 bulk path, the surrogate, the ensemble, the 3D variant, the
reference's own 256^2 workload and grids far beyond L2 are side legs.

Metric: Gcell-steps/s = interior cells x steps / s (whole job over N GPUs).

Device timing: CUDA events on the launching stream around each step.  The
step's input fields fit in the 126 MB L2, so L2 is flushed between timed
steps (outside the events): a 256 MiB buffer is written, then another
256 MiB buffer is read, so that the step reads its fields from HBM and does
not pay the write-back of the flush's dirty lines.
e2e: one output interval of the reference loop (step_fields = 200 steps,
fun.cu:437-446) through the C-ABI from pinned host buffers: H2D of the
fields (a restart), every step's FP64 solute-mass reduction read back to the
host, D2H of the fields (the snapshot), all in one event-timed region.

python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference]
Under torchrun each rank runs an independent replica (the path has no
exchange step); time is the max over ranks.
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "2d-rapid-solidification_b200"))

METRIC = "Gcell-steps/s, %HBM peak; surrogate vs exact CALPHAD at ≤0.5% tip-speed error"
UNIT = "Gcell-steps/s"
BYTES_PER_CELL = {"f32": 16, "f64": 32}  # psi, c read once + written once
WORKLOAD = ("Ti-10Nb directional solidification 2048x2048, exact CALPHAD, frozen T G=5e6 K/m V=0.5 m/s, "
            "moving frame, interface noise 0.01")
# kernels a step launches: the FP32 tile path (column table + tile, plus the
# mass reduction as a programmatic dependent launch when the mass is read),
# the FP64 tile path (the same), and the register-prefetch kernel that
# pull-back steps take (plus one reduction launch for the mass)
# (kernel of the roofline, launches of a step without pull-back, whether the
# mass reduction is fused into that kernel)
STEP_PATH = {"f32": ("rs::tile_kernel<false>", 2, False),
             "f64": ("rs::tile_kernel_f64", 2, False)}
# the tile steps' kernel (RS_OPT_PIPELINE): 0 one tile per CTA, 1 the
# persistent warp-role pipeline (the other one is timed beside it)
PIPELINE = 0


def rank_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(x, dist, device):
    """Largest value of x over all ranks (time of the slowest replica)."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, cells, steps, max_ms):
    """Whole-job Gcell-steps/s: every rank advances its own replica."""
    return world * cells * steps / (max_ms * 1e-3) / 1e9


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(kernel_tag):
    """DRAM bytes per launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(kernel_tag)
    except Exception:
        return None


def workload_config(p, d):
    """The workload both arms run (identical keys and values)."""
    return {"workload": WORKLOAD, "grid": [p.nx_all, p.ny_all], "interior_cells": (p.nx_all - 2) * (p.ny_all - 2),
            "dx_W": p.dx, "dt_tau0": d.dt, "step_pull_back": d.step_pull_back}


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


class Flush:
    """L2 flush between timed steps: write a 256 MiB buffer (larger than the
    126 MB L2), then read another 256 MiB buffer, so L2 holds clean lines of
    unrelated data when the next step starts."""

    def __init__(self):
        import torch
        n = 256 * 1024 * 1024 // 4
        self.w = torch.empty(n, dtype=torch.float32, device="cuda")
        self.r = torch.ones(n, dtype=torch.float32, device="cuda")
        self.acc = None

    def __call__(self, k):
        self.w.fill_(float(k))
        self.acc = self.r.sum()


class Loop:
    """The reference main() loop body on one field set pair through the
    library (main.cu:156-240): pull-back every step_pull_back steps (coarse
    tip reduced on the device, 4-byte read), then the fused step; counts the
    library's kernel launches."""

    def __init__(self, p, dtype, ic_seed=None, options=None):
        import torch
        from rapidsolid import configs, lib
        self.torch = torch
        self.p, self.dtype = p, dtype
        self.prec = "f64" if dtype == torch.float64 else "f32"
        self.ctx = lib.Context(p)
        for k, v in (options or {}).items():
            self.ctx.set_option(k, v)
        self.d = self.ctx.d
        self.a, self.b = lib.FieldSet(p, dtype), lib.FieldSet(p, dtype)
        self.ctx.initial_planar(self.a, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ,
                                configs.IC_SEED if ic_seed is None else ic_seed)
        self.itip = torch.zeros(1, dtype=torch.int32, device="cuda")
        self.n, self.hist, self.l = 0, 0, 0.0
        self.launches = 0

    def step(self, mass_out=None):
        p, d, n = self.p, self.d, self.n
        pb = None
        if n % d.step_pull_back == 0:
            self.ctx.itip(self.a, self.itip)
            self.launches += 2  # block partials + final reduction
            pb = int(self.itip.item()) - p.i_tip_target
            self.hist += pb
        self.ctx.step(self.a, self.b, n, i_offset_history=self.hist, l_offset_Vp=self.l, pull_back=pb,
                      mass_out=mass_out)
        # every step, pull-back steps included (the tile kernel gathers the
        # shifted tile), launches the column table and the tile kernel, which
        # reduces the mass itself
        red = 1 if mass_out is not None else 0
        _, nl, fused = STEP_PATH[self.prec]
        self.launches += nl + (0 if fused else red)
        self.l += p.Vp * d.dt * d.tau0 / (p.S * p.W0)
        self.a, self.b = self.b, self.a
        self.n = n + 1

    def close(self):
        self.ctx.close()


def timed_steps(loop, steps, flush, st, nvtx=None):
    """CUDA-event time (ms) of each of `steps` steps, L2 flushed before each.
    `nvtx` names an NVTX range around them (a profiler can capture just the
    timed launches with it; without a profiler the range costs nothing)."""
    torch = loop.torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    loop.launches = 0
    if nvtx:
        torch.cuda.nvtx.range_push(nvtx)
    for k in range(steps):
        flush(k)
        ev[k][0].record(st)
        loop.step()
        ev[k][1].record(st)
    if nvtx:
        torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    return [s.elapsed_time(e) for s, e in ev], loop.launches


def e2e_interval(loop, nsteps, dist, world, st):
    """One output interval of the reference loop through the C-ABI, from
    pinned host fields: H2D of psi and c (a restart), nsteps steps each with
    its FP64 solute mass written by the device into mapped host memory, D2H
    of psi and c (the field snapshot of set_fields_output, fun.cu:621-666)."""
    torch = loop.torch
    p = loop.p
    h_psi = torch.empty((p.ny_all, p.nx_all), dtype=loop.dtype, pin_memory=True)
    h_c = torch.empty_like(h_psi).pin_memory()
    h_psi.copy_(loop.a.psi)
    h_c.copy_(loop.a.c)
    # every step's mass goes straight into mapped page-locked host memory
    # (rs_host_alloc): the step's reduction writes it there, no copy call
    from rapidsolid import lib
    h_mass = lib.HostBuffer(nsteps)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    loop.a.psi.copy_(h_psi, non_blocking=True)
    loop.a.c.copy_(h_c, non_blocking=True)
    for k in range(nsteps):
        loop.step(mass_out=h_mass.device + 8 * k)
    h_psi.copy_(loop.a.psi, non_blocking=True)
    h_c.copy_(loop.a.c, non_blocking=True)
    e1.record(st)
    torch.cuda.synchronize()
    import numpy as np
    masses = h_mass.host.copy()
    h_mass.close()
    if not (np.isfinite(masses).all() and masses.min() > 0):
        raise RuntimeError("e2e: a step's mass did not arrive in host memory")
    ms = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
    cells = (p.nx_all - 2) * (p.ny_all - 2)
    field_bytes = 2 * h_psi.numel() * h_psi.element_size()
    return {"value": round(job_throughput(world, cells, nsteps, ms), 4), "unit": UNIT,
            "h2d_bytes_per_step": round(field_bytes / nsteps, 1),
            "d2h_bytes_per_step": round(8 + field_bytes / nsteps, 1), "ms_per_step": round(ms / nsteps, 5),
            "interval_steps": nsteps,
            "note": "C-ABI rs_step over one output interval of the reference loop (step_fields steps): H2D of "
                    "psi and c from pinned memory, every step's FP64 mass written by the device into mapped "
                    "page-locked host memory (rs_host_alloc), D2H of psi and c; no L2 flush"}


def kernel_name(prec, options):
    from rapidsolid import _abi
    if (options or {}).get(_abi.RS_OPT_PIPELINE, 0):
        return f"rs::pipe_kernel_{prec}"
    return STEP_PATH[prec][0]


def roofline(prec, cells, kern_ms, peak, peak_kind, kernel):
    alg = BYTES_PER_CELL[prec] * cells
    achieved = alg / (kern_ms * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_source": peak_kind, "algorithmic_bytes_per_launch": alg,
            "kernel": kernel, "kernel_ms_median": round(kern_ms, 5),
            "traffic": profiled_traffic(f"step_{prec}_2048")}


def run_arm(p, dtype, args, flush, st, dist, world, clocks=None, options=None, e2e=True):
    """Warm-up, timed steps (L2 flushed), roofline and e2e of one precision."""
    loop = Loop(p, dtype, options=options)
    for _ in range(args.warmup):
        loop.step()
    loop.torch.cuda.synchronize()
    if dist:
        dist.barrier()
    loop.torch.cuda.synchronize()
    if clocks is not None:
        # clocks are sampled from before to after the timed region (200 ms
        # period): untimed steps keep the GPU under load while it starts
        clocks.start()
        t_pre = time.time()
        while time.time() - t_pre < args.clock_preroll:
            for _ in range(20):
                loop.step()
            loop.torch.cuda.synchronize()
    # the timed window starts on the step after a pull-back step, so that its
    # K consecutive steps hold the loop's cadence (one pull-back step in
    # step_pull_back) whatever the pre-roll took; the pull-back step itself is
    # timed on its own afterwards
    spb = loop.d.step_pull_back
    while loop.n % spb != 1:
        loop.step()
    loop.torch.cuda.synchronize()
    if dist:
        dist.barrier()
    n0 = loop.n
    t_wall = time.time()
    ms_steps, launches = timed_steps(loop, args.steps, flush, st, nvtx=f"timed_{loop.prec}")
    t_wall = time.time() - t_wall
    if dist:
        dist.barrier()
    while loop.n % spb != 0:
        loop.step()
    pb_ms, _ = timed_steps(loop, 1, flush, st)
    clk = None
    if clocks is not None:
        t_post = time.time()
        while time.time() - t_post < 0.3:
            for _ in range(20):
                loop.step()
            loop.torch.cuda.synchronize()
        clk = clocks.stop()
    total_ms = max_over_ranks(sum(ms_steps), dist, "cuda")
    cells = (p.nx_all - 2) * (p.ny_all - 2)
    srt = sorted(ms_steps)
    kern_ms = srt[len(srt) // 2]
    peak, peak_kind = measured_peak()
    out = {"value": round(job_throughput(world, cells, args.steps, total_ms), 4),
           "ms_per_step": round(total_ms / args.steps, 5),
           "roofline": roofline(loop.prec, cells, kern_ms, peak, peak_kind, kernel_name(loop.prec, options)),
           "gpu_launches": launches, "wall_s_timed": round(t_wall, 3), "clocks": clk,
           "first_timed_step": n0, "pull_back_step_ms": round(pb_ms[0], 5), "step_pull_back": spb}
    if e2e:
        # an output interval that starts after a pull-back step, like the window above
        while loop.n % spb != 1:
            loop.step()
        out["e2e"] = e2e_interval(loop, loop.d.step_fields, dist, world, st)
    loop.close()
    return out


def run_ours(args):
    import torch
    from rapidsolid import configs

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    p = configs.scale()
    from rapidsolid import lib
    d = lib.derive(p)
    st = torch.cuda.current_stream()
    flush = Flush()
    from rapidsolid import _abi
    head = run_arm(p, torch.float64, args, flush, st, dist, world, clocks=ClockSampler(local),
                   options={_abi.RS_OPT_PIPELINE: PIPELINE})

    line = {
        "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp64",
        "data": "synthetic (seeded planar Ti-10Nb front, Philox noise)",
        "config": workload_config(p, d), "parallelism": f"replicas x{world}",
        "l2": "flushed between timed steps (256 MiB written, then 256 MiB read)",
        "roofline": head["roofline"], "e2e": head["e2e"], "gpu_launches": head["gpu_launches"],
        "clocks": head["clocks"], "wall_s_timed": head["wall_s_timed"],
        "first_timed_step": head["first_timed_step"], "pull_back_step_ms": head["pull_back_step_ms"],
        "step_pull_back": head["step_pull_back"],
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(p, seconds=args.cpu_seconds)
    if rank == 0 and world == 1 and not args.no_side_legs:
        alt = run_arm(p, torch.float64, args, flush, st, None, 1, options={_abi.RS_OPT_PIPELINE: 1 - PIPELINE},
                      e2e=False)
        alt.pop("clocks")
        line["fp64_other_kernel"] = {"pipeline": 1 - PIPELINE, "value": alt["value"],
                                     "ms_per_step": alt["ms_per_step"], "roofline": alt["roofline"]}
        fp32 = run_arm(p, torch.float32, args, flush, st, None, 1, options={_abi.RS_OPT_PIPELINE: PIPELINE})
        alt32 = run_arm(p, torch.float32, args, flush, st, None, 1, options={_abi.RS_OPT_PIPELINE: 1 - PIPELINE},
                        e2e=False)
        fp32["other_kernel"] = {"pipeline": 1 - PIPELINE, "value": alt32["value"],
                                "ms_per_step": alt32["ms_per_step"], "roofline": alt32["roofline"]}
        fp32.pop("clocks")
        line["fp32_exact"] = fp32
        line["fp32_exact_vs_fp64_exact"] = round(fp32["value"] / head["value"], 3)
        line["c1_plain_small"] = c1_leg()
        line["surrogate"] = surrogate_leg(p, flush, fp32["value"], head["value"])
        line["ensemble"] = ensemble_leg(flush)
        del flush
        torch.cuda.empty_cache()
        line["beyond_l2"] = beyond_l2_leg()
        torch.cuda.empty_cache()
        line["peritectic_3d"] = peritectic_3d_leg(measured_peak()[0])
        torch.cuda.empty_cache()
        line["tinb_3d"] = tinb_3d_leg(measured_peak()[0])
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


def c1_leg(nsteps=500):
    """The reference's own workload: 256^2 FP64, frozen T
    G = 1e6 K/m, V = 0.05 m/s, 500 steps with the pull-back of step 0
    (main.cu's cadence), timed as one run launch by launch, and with steps
    1..499 replayed from a CUDA graph captured once (the step arguments of a
    frozen-temperature run are known in advance; step_pull_back = 10082)."""
    import torch
    from rapidsolid import configs
    p = configs.plain_small()
    cells = (p.nx_all - 2) * (p.ny_all - 2)
    warm = Loop(p, torch.float64)
    for _ in range(3):  # first launches of each kernel, not timed
        warm.step()
    torch.cuda.synchronize()
    warm.close()
    out = {}
    # launch by launch: the whole run
    loop = Loop(p, torch.float64)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(nsteps):
        loop.step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    out["eager"] = {"value": round(cells * nsteps / (ms * 1e-3) / 1e9, 3), "ms_run": round(ms, 4),
                    "us_per_step": round(ms * 1e3 / nsteps, 3)}
    loop.close()
    # step 0 (pull-back, coarse tip read back) eagerly, then steps 1..499 as
    # one graph; the capture does not execute, so the replay starts from the
    # state after step 0
    loop = Loop(p, torch.float64)
    loop.step()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    cs = torch.cuda.Stream()
    cs.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(cs):
        with torch.cuda.graph(g, stream=cs):
            for _ in range(nsteps - 1):
                loop.step()
    torch.cuda.synchronize()
    e0.record()
    g.replay()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    out["graph"] = {"value": round(cells * (nsteps - 1) / (ms * 1e-3) / 1e9, 3), "ms_steps_1_499": round(ms, 4),
                    "us_per_step": round(ms * 1e3 / (nsteps - 1), 3)}
    del g
    loop.close()
    out["note"] = ("256x256 FP64, 500 steps; the reference arm (bench.py --impl reference) times the reference's "
                   "own kernels on this run (reference_kernels_b200.fp64_2d_256_c1)")
    return out


def beyond_l2_leg(n=8192, steps=10):
    """The C2 step on an 8192 x 8192 grid (FP32: 512 MiB per field set,
    FP64: 1 GiB), far beyond the 126 MB L2: no flush is needed and the
    sustained HBM fraction is read directly from back-to-back steps."""
    import torch
    from rapidsolid import _abi, configs
    p = configs.scale()
    p.nx_all = p.ny_all = n
    cells = (n - 2) * (n - 2)
    peak, peak_kind = measured_peak()
    out = {}
    for prec, dtype in (("f32", torch.float32), ("f64", torch.float64)):
        loop = Loop(p, dtype, options={_abi.RS_OPT_PIPELINE: PIPELINE})
        for _ in range(3):
            loop.step()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for k in range(steps):
            ev[k][0].record()
            loop.step()
            ev[k][1].record()
        torch.cuda.synchronize()
        ts = sorted(s.elapsed_time(e) for s, e in ev)
        ms = ts[len(ts) // 2]
        rl = roofline(prec, cells, ms, peak, peak_kind, kernel_name(prec, {_abi.RS_OPT_PIPELINE: PIPELINE}))
        rl.pop("traffic")
        out[prec] = {"value": round(cells / (ms * 1e-3) / 1e9, 3), "ms_per_step": round(ms, 5), "roofline": rl}
        loop.close()
        torch.cuda.empty_cache()
    out["grid"] = [n, n]
    return out


def _timed_steps(ctx, p, d, a, b, flush, n0, nsteps):
    """Median CUDA-event time (ms) of nsteps steps, L2 flushed between them."""
    import torch
    ts = []
    for k in range(nsteps):
        flush(k)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ctx.step(a, b, n0 + k)
        e1.record()
        a, b = b, a
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    ts.sort()
    return ts[len(ts) // 2]


def surrogate_leg(p, flush, fp32_value, fp64_value, nsteps=30, seeds=(1, 2, 3)):
    """The FP32 step with the learned CALPHAD surrogate (trained here on the
    GPU by the library's kernels, deterministically for a seed): speed with
    the network of the workload definition's wide box, and tip speed and
    position against the exact FP32 step over the full 20000-step run, for
    three training seeds of the wide box and for the box fitted to the run."""
    import torch
    from rapidsolid import configs, lib, run, surrogate
    trained = {}
    for name, bx, seed in [("wide", surrogate.default_box, sd) for sd in seeds] + \
                          [("fitted", surrogate.fitted_box, seeds[0])]:
        t0 = time.time()
        w, box, hist = surrogate.train(p, box=bx(), epochs=40, seed=seed)
        torch.cuda.synchronize()
        trained[(name, seed)] = (w, box, hist, time.time() - t0)
    w, box = trained[("wide", seeds[0])][:2]
    ctx = lib.Context(p)
    ctx.set_surrogate(w, box)
    a, b = lib.FieldSet(p, torch.float32), lib.FieldSet(p, torch.float32)
    ctx.initial_planar(a, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, configs.IC_SEED)
    for k in range(1, 6):
        ctx.step(a, b, k)
        a, b = b, a
    ms = _timed_steps(ctx, p, ctx.d, a, b, flush, 6, nsteps)
    ctx.close()
    cells = (p.nx_all - 2) * (p.ny_all - 2)
    value = cells / (ms * 1e-3) / 1e9
    x0, v0, _, _, _ = run.tip_run(p, torch.float32, configs.STEPS["scale_fp32"])
    accuracy = {}
    for (name, seed), (w, box, hist, t_train) in trained.items():
        x1, v1, audit, m0, m1 = run.tip_run(p, torch.float32, configs.STEPS["scale_fp32"], surrogate=(w, box))
        accuracy[f"{name}_seed{seed}"] = {
            "tip_speed_error": round(abs(v1 - v0) / v0, 6), "tip_speed_m_s": [round(v0, 6), round(v1, 6)],
            "tip_position_max_dx": round(max(abs(u - q) for u, q in zip(x0, x1)) / p.dx, 4),
            "solute_drift_rel": (m1 - m0) / m0,
            "box": {"T": [round(box.T_lo, 3), round(box.T_hi, 3)], "c": [box.c_lo, box.c_hi]},
            "train_s": round(t_train, 2), "train_scaled_mse": hist[-1],
            "audit": {"max_err_mu_J_mol": audit[0], "max_err_dG_J_mol": audit[1], "fallback_cells": audit[2],
                      "audited_cells": audit[3]}}
    wide = [v["tip_speed_error"] for k, v in accuracy.items() if k.startswith("wide")]
    return {"value": round(value, 3), "ms_per_step": round(ms, 5), "vs_fp32_exact": round(value / fp32_value, 3),
            "vs_fp64_exact": round(value / fp64_value, 3), "box_of_speed": "wide", "accuracy": accuracy,
            "wide_tip_speed_error_spread": [min(wide), max(wide)],
            "note": "3->32->32->2 SiLU, FP16 mma.sync hidden layers; the network evaluates every cell that is "
                    "not bulk melt (the melt keeps its exact series form); exact fallback out of box and "
                    "1/1024 audit; 20000 steps, tip every 1000"}


def _time3(ctx, a, b, k0, ntimed):
    """median CUDA-event time (ms) of ntimed 3D steps from step k0; returns (ms, a, b)"""
    import torch
    ts = []
    for k in range(k0, k0 + ntimed):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ctx.step(a, b, k)
        e1.record()
        a, b = b, a
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return sorted(ts)[len(ts) // 2], a, b


def tinb_3d_leg(peak, nsteps_run=5000, ntimed=10):
    """The 3D three-phase structure with the Ti-Nb CALPHAD energy (energy 1):
    512 x 512 x 1024 FP32, two BCC grains under a seeded planar front at
    z = 24 +- 0.5 dx, melt x_Nb = 0.10, G = 2e6 K/m, V = 0.2 m/s, on the exact
    CALPHAD path and with the learned surrogate (trained here on the box of
    the run's states, inputs T, c and the interpolation weight).  Step times
    by CUDA events (1 GiB per field: far beyond L2, no flush), roofline
    against 24 algorithmic bytes per cell-step, and the whole 5000-step run
    on both paths: front advance (mean solid thickness per column, the sum
    over z of 1 - phi1), front speed over the second half, solute drift, and
    the surrogate's front-speed and front-position differences from the exact
    run.  The FP64 kernel at 512 x 512 x 256."""
    import torch
    from rapidsolid import configs, lib, surrogate
    out = {}
    p = configs.tinb_3d()
    cl, cs = configs.tinb_compositions()
    ic = configs.IC3_TINB
    cells = (p.nx - 2) * (p.ny - 2) * (p.nz - 2)
    p2 = configs.scale()
    d2 = lib.derive(p2)
    m_per_cell = 0.8 * p2.S * p2.W0 * 1e-9
    s_per_step = p.dt * d2.tau0 * 1e-9
    p2.cinf = p.c_ref
    t0 = time.time()
    w, box, hist = surrogate.train(p2, box=surrogate.fitted_box(), epochs=40, seed=1, g_input=True)
    torch.cuda.synchronize()
    t_train = time.time() - t0

    def front(fs):  # mean solid thickness per (x, y) column, in cells: sum over z of 1 - phi1
        return float((1.0 - fs.phi1[1:-1, 1:-1, 1:-1].double()).sum(0).mean())

    for name, use in (("fp32_exact", False), ("fp32_surrogate", True)):
        ctx = lib.Context3(p)
        if use:
            ctx.set_surrogate(w, box)
        a, b = lib.FieldSet3(p, torch.float32), lib.FieldSet3(p, torch.float32)
        ctx.initial_grains(a, ic["z_front"], ic["amp"], cl, cs, ic["seed"])
        for k in range(3):
            ctx.step(a, b, k)
            a, b = b, a
        ms, a, b = _time3(ctx, a, b, 3, ntimed)
        # the whole run from the initial state
        m = torch.zeros(2, dtype=torch.float64, device="cuda")
        ctx.initial_grains(a, ic["z_front"], ic["amp"], cl, cs, ic["seed"])
        ctx.mass(a, m[0:1])
        if use:
            ctx.surrogate_audit()
        fr = [front(a)]
        r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        r0.record()
        for k in range(nsteps_run):
            ctx.step(a, b, k)
            a, b = b, a
            if k + 1 == nsteps_run // 2:
                fr.append(front(a))
        r1.record()
        ctx.mass(a, m[1:2])
        torch.cuda.synchronize()
        ctx.device_status()
        fr.append(front(a))
        run_ms = r0.elapsed_time(r1)
        m0, m1 = m.tolist()
        alg = 24 * cells
        achieved = alg / (ms * 1e-3) / 1e9
        speed = (fr[2] - fr[1]) * m_per_cell / ((nsteps_run - nsteps_run // 2) * s_per_step)
        out[name] = {"value": round(cells / (ms * 1e-3) / 1e9, 3), "unit": "Gcell-steps/s",
                     "ms_per_step": round(ms, 4), "grid": [p.nx, p.ny, p.nz], "interior_cells": cells,
                     "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                                  "frac": round(achieved / peak, 4), "algorithmic_bytes_per_launch": alg,
                                  "kernel": "rs::tinb_kernel<float> (surrogate)" if use
                                  else "rs::tinb_x2_kernel (packed FP32 pairs)"},
                     "run": {"steps": nsteps_run, "ms": round(run_ms, 1), "front_cells": [round(x, 4) for x in fr],
                             "front_speed_m_s": round(speed, 6), "solute_drift_rel": (m1 - m0) / m0}}
        if use:
            em, eg, nfb, naud = ctx.surrogate_audit()
            out[name]["audit"] = {"max_err_mu_J_mol": em, "max_err_dG_J_mol": eg, "fallback_cells": nfb,
                                  "audited_cells": naud}
            out[name]["box"] = {"T": [round(box.T_lo, 3), round(box.T_hi, 3)], "c": [box.c_lo, box.c_hi]}
            out[name]["train_s"] = round(t_train, 2)
        ctx.close()
        del a, b
        torch.cuda.empty_cache()
    ve, vs = out["fp32_exact"]["run"]["front_speed_m_s"], out["fp32_surrogate"]["run"]["front_speed_m_s"]
    out["fp32_surrogate"]["vs_exact"] = round(out["fp32_surrogate"]["value"] / out["fp32_exact"]["value"], 3)
    out["fp32_surrogate"]["front_speed_error"] = round(abs(vs - ve) / abs(ve), 6) if ve else None
    out["fp32_surrogate"]["front_position_diff_cells"] = round(
        out["fp32_surrogate"]["run"]["front_cells"][-1] - out["fp32_exact"]["run"]["front_cells"][-1], 6)
    # FP64 at 512 x 512 x 256
    q = configs.tinb_3d(nz=256)
    cells = (q.nx - 2) * (q.ny - 2) * (q.nz - 2)
    ctx = lib.Context3(q)
    a, b = lib.FieldSet3(q, torch.float64), lib.FieldSet3(q, torch.float64)
    ctx.initial_grains(a, ic["z_front"], ic["amp"], cl, cs, ic["seed"])
    for k in range(3):
        ctx.step(a, b, k)
        a, b = b, a
    ms, a, b = _time3(ctx, a, b, 3, ntimed)
    ctx.device_status()
    achieved = 48 * cells / (ms * 1e-3) / 1e9
    out["fp64"] = {"value": round(cells / (ms * 1e-3) / 1e9, 3), "unit": "Gcell-steps/s", "ms_per_step": round(ms, 4),
                   "grid": [q.nx, q.ny, q.nz],
                   "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                                "frac": round(achieved / peak, 4), "algorithmic_bytes_per_launch": 48 * cells,
                                "kernel": "rs::tinb_kernel<double>"}}
    ctx.close()
    del a, b
    torch.cuda.empty_cache()
    out["note"] = ("TiAg.cu's three-phase structure with the Ti-Nb CALPHAD energy of the 2D model (mu = g1 Glc + "
                   "(1 - g1) Gsc, driving force Gl - Gs), two BCC grains; one table launch (per-plane CALPHAD "
                   "groups) and one fused z-march launch per step")
    return out


def peritectic_3d_leg(peak, nsteps_run=5000, ntimed=10):
    """The 3D three-phase variant (the reference's TiAg.cu model) on one GPU:
    512 x 512 x 1024 FP32 with a frozen gradient (G = 2e6 K/m, V = 0.2 m/s),
    beta front at z = 24 +- 0.5 dx with four alpha caps.  Step time by CUDA
    events (three fields of 1 GiB each per set: far beyond L2, no flush),
    roofline against 24 algorithmic bytes per cell-step, the whole run's time
    and solute drift; the FP64 kernel at the reference's own 512 x 512 x 128."""
    import torch
    from rapidsolid import configs, lib
    out = {}
    p = configs.peritectic_3d()
    cells = (p.nx - 2) * (p.ny - 2) * (p.nz - 2)
    ctx = lib.Context3(p)
    a, b = lib.FieldSet3(p, torch.float32), lib.FieldSet3(p, torch.float32)
    ctx.initial(a, **configs.IC3)
    m = torch.zeros(2, dtype=torch.float64, device="cuda")
    ctx.mass(a, m[0:1])
    for k in range(3):
        ctx.step(a, b, k)
        a, b = b, a
    ts = []
    for k in range(3, 3 + ntimed):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ctx.step(a, b, k)
        e1.record()
        a, b = b, a
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    ms = sorted(ts)[len(ts) // 2]
    # the whole run: nsteps_run steps from the initial state
    ctx.initial(a, **configs.IC3)
    r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    r0.record()
    for k in range(nsteps_run):
        ctx.step(a, b, k)
        a, b = b, a
    r1.record()
    ctx.mass(a, m[1:2])
    torch.cuda.synchronize()
    ctx.device_status()
    run_ms = r0.elapsed_time(r1)
    m0, m1 = m.tolist()
    alg = 24 * cells
    achieved = alg / (ms * 1e-3) / 1e9
    out["fp32"] = {"value": round(cells / (ms * 1e-3) / 1e9, 3), "unit": "Gcell-steps/s", "ms_per_step": round(ms, 4),
                   "grid": [p.nx, p.ny, p.nz], "interior_cells": cells,
                   "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                                "frac": round(achieved / peak, 4), "algorithmic_bytes_per_launch": alg,
                                "kernel": "rs::peri3d_x2_kernel"},
                   "run": {"steps": nsteps_run, "ms": round(run_ms, 1),
                           "gcell_steps_s": round(cells * nsteps_run / (run_ms * 1e-3) / 1e9, 3),
                           "solute_drift_rel": (m1 - m0) / m0},
                   "G_T_per_cell": p.G_T, "V_T_cells_per_step": p.V_T}
    ctx.close()
    del a, b
    torch.cuda.empty_cache()
    q = configs.peritectic_3d(nz=128)
    q.G_T = q.V_T = 0.0
    cells = (q.nx - 2) * (q.ny - 2) * (q.nz - 2)
    ctx = lib.Context3(q)
    a, b = lib.FieldSet3(q, torch.float64), lib.FieldSet3(q, torch.float64)
    ctx.initial(a, 100.0, 0.5, 4, 30.0, 5)
    for k in range(3):
        ctx.step(a, b, k)
        a, b = b, a
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for k in range(3, 3 + ntimed):
        ctx.step(a, b, k)
        a, b = b, a
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / ntimed
    achieved = 48 * cells / (ms * 1e-3) / 1e9
    out["fp64_reference_size"] = {"value": round(cells / (ms * 1e-3) / 1e9, 3), "unit": "Gcell-steps/s",
                                  "ms_per_step": round(ms, 4), "grid": [q.nx, q.ny, q.nz],
                                  "roofline_frac": round(achieved / peak, 4), "kernel": "rs::peri3d_kernel<double>",
                                  "note": "isothermal, the reference's Nx x Ny x devNz; the reference arm "
                                          "(bench.py --impl reference) times its own kernels at this size"}
    ctx.close()
    out["note"] = ("one fused launch per step (computeMu + boundaryMu + diffuse + boundary of TiAg.cu); "
                   "no CALPHAD in this model, so no surrogate path")
    return out


def _ensemble(runs, sur=None):
    import torch
    from rapidsolid import lib
    ens = lib.Ensemble([p for p, _, _ in runs])
    for r, (p, cl, cs) in enumerate(runs):
        a, b = lib.FieldSet(p, torch.float32), lib.FieldSet(p, torch.float32)
        ens.ctx[r].initial_planar(a, cl, cs, 7 + r)
        if sur is not None:
            ens.ctx[r].set_surrogate(*sur)
        ens.bind(r, a, b)
    return ens


def _ensemble_tips(ens, runs):
    """x of every run's precise tip, (i_offset_history + tip.x) dx in W."""
    import ctypes as C
    import torch
    from rapidsolid import _abi, lib
    buf = torch.zeros(C.sizeof(_abi.Tip), dtype=torch.uint8, device="cuda")
    xs = []
    for r, (p, _, _) in enumerate(runs):
        _, hist, _, cur = ens.state(r)
        ens.ctx[r].precise_tip(cur, buf)
        t = lib.tip_from_bytes(buf.cpu().numpy().tobytes())
        xs.append((hist + t.x) * p.dx)
    return xs


# the ensemble's stepping paths (rs_ensemble_autotune): per tile shape (rows x
# 128 columns), per-step launches replayed from a CUDA graph or the persistent
# walk, each with three tile orders
ENS_PATHS = [f"{rows}x128 tiles, {form}, {order}" for rows in (16, 8, 32) for form in ("graph", "walk")
             for order in ("run by run", "largest first", "interleaved")]


def _timed_ensemble(ens, flush, nsteps):
    import torch
    ens.steps(3)  # step 0 pulls every run back (eager), then graph replays
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    flush(1)
    e0.record()
    ens.steps(nsteps)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def ensemble_leg(flush, nruns=64, nsteps=100, vel_steps=4000):
    """The batched ensemble of uneven runs (64 Ti-Nb runs, sizes 256^2 ..
    1024x2048, V 0.01-2 m/s, G 1e5-1e7 K/m, x_Nb 0.05-0.20, seeded): aggregate
    Gcell-steps/s of the batched step (per-step launches replayed from a
    CUDA graph, or the persistent walk, as the autotuner picks; both timed
    with its tile order), exact FP32 and
    through the learned surrogate (one network trained on a box that spans
    every run's compositions and temperatures), against the same runs stepped
    one rs_step at a time; per-run tip velocity of the surrogate ensemble
    against each run stepped alone on the exact path."""
    import torch
    from rapidsolid import configs, run, surrogate
    runs = configs.ensemble(nruns)
    ps = [p for p, _, _ in runs]
    cells = sum((p.nx_all - 2) * (p.ny_all - 2) for p in ps)
    out = {"runs": nruns, "cells": cells, "steps": nsteps}
    # exact path
    ens = _ensemble(runs)
    choice, tune_ms = ens.autotune(reps=5)
    ms = _timed_ensemble(ens, flush, nsteps)
    out["exact"] = {"value": round(cells * nsteps / (ms * 1e-3) / 1e9, 3), "ms_per_step": round(ms / nsteps, 5),
                    "autotune": {"choice": ENS_PATHS[choice], "ms_per_step_of_path": [round(x, 5) for x in tune_ms]}}
    # the two stepping paths with the autotuned tile shape and order
    for name, path in (("graph", 6 * (choice // 6) + choice % 3), ("walk", 6 * (choice // 6) + 3 + choice % 3)):
        ens.set_path(path)
        msp = _timed_ensemble(ens, flush, nsteps)
        out["exact"]["path_" + name] = {"value": round(cells * nsteps / (msp * 1e-3) / 1e9, 3),
                                        "ms_per_step": round(msp / nsteps, 5)}
    ens.set_path(choice)
    # the same runs one by one (two launches per run and step)
    ctxs = [ens.ctx[r] for r in range(nruns)]
    cur = [ens.state(r)[3] for r in range(nruns)]
    nxt = [ens.sets[r][0] if cur[r] is ens.sets[r][1] else ens.sets[r][1] for r in range(nruns)]
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record()
    for k in range(10):
        for r in range(nruns):
            ctxs[r].step(cur[r], nxt[r], 1)
    s1.record()
    torch.cuda.synchronize()
    ms_single = s0.elapsed_time(s1) / 10
    out["one_by_one"] = {"value": round(cells / (ms_single * 1e-3) / 1e9, 3), "ms_per_step": round(ms_single, 5)}
    ens.close()
    # surrogate path: one network on a box over all runs
    box = surrogate.ensemble_box(ps)
    w, box, hist = surrogate.train(ps[0], box=box, epochs=40, seed=1)
    ens = _ensemble(runs, (w, box))
    choice, tune_ms = ens.autotune(reps=5)
    ms = _timed_ensemble(ens, flush, nsteps)
    out["surrogate"] = {"value": round(cells * nsteps / (ms * 1e-3) / 1e9, 3), "ms_per_step": round(ms / nsteps, 5),
                        "autotune": {"choice": ENS_PATHS[choice],
                                     "ms_per_step_of_path": [round(x, 5) for x in tune_ms]},
                        "box": {"T": [round(box.T_lo, 2), round(box.T_hi, 2)], "c": [box.c_lo, box.c_hi]}}
    ens.close()
    # per-run tip velocity over the second half of vel_steps: the surrogate
    # ensemble against each run stepped alone on the exact path
    ens = _ensemble(runs, (w, box))
    x0 = _ensemble_tips(ens, runs)
    ens.steps(vel_steps // 2)
    xh = _ensemble_tips(ens, runs)
    ens.steps(vel_steps - vel_steps // 2)
    x1 = _ensemble_tips(ens, runs)
    audit = [ens.ctx[r].surrogate_audit() for r in range(nruns)]
    ens.close()
    errs = []
    for r, (p, cl, cs) in enumerate(runs):
        xs, v_exact, _, _, _ = run.tip_run(p, torch.float32, vel_steps, every=vel_steps // 2, ic_seed=7 + r,
                                           initial=(cl, cs))
        d = lib_derive(p)
        v_ens = (x1[r] - xh[r]) * p.S * p.W0 / ((vel_steps - vel_steps // 2) * d.tau0 * d.dt)
        errs.append({"run": r, "grid": [p.nx_all, p.ny_all], "V_pull": round(p.Vp, 4),
                     "tip_speed_m_s": [round(v_exact, 5), round(v_ens, 5)],
                     "rel_error": round(abs(v_ens - v_exact) / max(abs(v_exact), 1e-12), 5)})
    rel = sorted(e["rel_error"] for e in errs)
    out["surrogate"]["tip_velocity_vs_single_exact_runs"] = {
        "steps": vel_steps, "median_rel_error": rel[len(rel) // 2], "max_rel_error": rel[-1],
        "fallback_cells": int(sum(a[2] for a in audit)), "per_run": errs}
    out["value"] = out["exact"]["value"]
    out["note"] = ("CUDA graph replays between pull-backs; every run equals its single run bit for bit on both "
                   "paths (tests)")
    return out


def lib_derive(p):
    from rapidsolid import lib
    return lib.derive(p)


def cpu_baseline(p, seconds=12.0, steps=None):
    """The CPU FP64 restatement (oracle, OpenMP on all host threads) timed on a
    bounded sample of the same workload: the full grid for a few steps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from rapidsolid import configs
    d = pyoracle.derive(p)
    s = pyoracle.initial_planar(p, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, configs.IC_SEED)
    t0 = time.time()
    pyoracle.run(p, d, s, 1)
    t1 = time.time() - t0
    n = steps or max(1, min(50, int(seconds / max(t1, 1e-3))))
    t0 = time.time()
    pyoracle.run(p, d, s, n)
    dt = time.time() - t0
    cells = (p.nx_all - 2) * (p.ny_all - 2)
    return {"value": round(cells * n / dt / 1e9, 5), "unit": UNIT, "cores": pyoracle.lib().ro_num_threads(),
            "kind": "port", "sample": f"{n} FP64 steps of the {p.nx_all}x{p.ny_all} grid ({dt:.1f} s)",
            "cpu": _cpu_model()}


def _cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return None


def run_reference(args):
    """The reference path has no CPU implementation of its own (its step is
    CUDA); its CPU form is the FP64 restatement in oracle/ (OpenMP, all host
    threads), timed on the same workload as the headline arm with the same
    warm-up and step count (each step one full-grid step, capped so that the
    run stays within minutes)."""
    rank, world, _ = rank_info()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from rapidsolid import configs
    p = configs.scale()
    d = pyoracle.derive(p)
    s = pyoracle.initial_planar(p, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, configs.IC_SEED)
    steps = max(1, min(args.steps, REF_MAX_STEPS))
    warm = max(0, min(args.warmup, REF_MAX_STEPS))
    if warm:
        s = pyoracle.run(p, d, s, warm)
    t0 = time.time()
    pyoracle.run(p, d, s, steps, step0=warm)
    dt = time.time() - t0
    cells = (p.nx_all - 2) * (p.ny_all - 2)
    value = cells * steps / dt / 1e9
    cores = pyoracle.lib().ro_num_threads()
    sample = f"{steps} FP64 steps of the {p.nx_all}x{p.ny_all} grid after {warm} warm-up steps"
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 5), "unit": UNIT, "n_gpus": world,
            "steps": steps, "warmup": warm, "ms_per_step": round(dt * 1e3 / steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp64", "data": "synthetic",
            "config": workload_config(p, d),
            "cpu_baseline": {"value": round(value, 5), "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": sample, "cpu": _cpu_model()},
            "e2e": {"value": round(value, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    gpu = _reference_kernels_gpu(pyoracle)
    if gpu:
        line["reference_kernels_b200"] = gpu
    print(json.dumps(line))


REF_MAX_STEPS = 400  # about 30 s of the 2048^2 FP64 step on 16 host threads


def _reference_kernels_gpu(pyoracle):
    """The reference's own CUDA kernels, built from its sources into
    oracle/_ref/ (FP64): the 2D step (compute_phi, compute_psi,
    compute_c_CALPHAD at 2048 x 2048) and the 3D step (TiAg.cu computeMu,
    boundaryMu, diffuse, boundary at its own 512 x 512 x 128).  Reported
    beside the CPU arm; skipped without a GPU or without the binaries."""
    import subprocess
    try:
        import torch
        if not torch.cuda.is_available():
            return None
    except ImportError:
        return None
    out = {}
    for key, args in (("fp64_2d_2048", ["ref_harness_2048", "bench", "100", "0.144"]),
                      ("fp64_2d_256_c1", ["ref_harness_256", "bench", "500", "0.144"]),
                      ("fp64_3d_512x512x128", ["ref3_harness_512", "bench", "10"])):
        binary = pyoracle.ref_binary(args[0])
        if not os.path.exists(binary):
            continue
        try:
            r = subprocess.run([binary] + args[1:], capture_output=True, text=True, timeout=300, check=True)
            out[key] = json.loads(r.stdout.strip().splitlines()[-1])
        except (subprocess.SubprocessError, ValueError, IndexError) as e:
            out[key] = {"error": str(e)[:200]}
    return out or None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--clock-preroll", type=float, default=1.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-side-legs", action="store_true", help="skip the FP64 and surrogate legs")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
