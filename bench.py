"""Throughput of the coupled phase-field step on B200.

Workload (one step = one time step of the whole grid):
  Ti-10at%Nb directional solidification, 2048 x 2048 cells (Nx_all x Ny_all,
  2046^2 interior), FP32 fields (psi, c - cinf) double-buffered, exact CALPHAD
  chemistry, frozen temperature G = 5e6 K/m, V = 0.5 m/s, moving frame on
  (pull-back every step_pull_back = 1008 steps), seeded Philox interface
  noise of amplitude 0.01.  Synthetic input: seeded planar front.

Metric: Gcell-steps/s = interior cells x steps / s (whole job over N GPUs).

Device timing: CUDA events on the launching stream around each step; the
64 MiB working set fits in L2, so a 256 MiB buffer is written between timed
steps (outside the events) and every step reads its fields from HBM.
e2e: the same steps through the C-ABI from pinned host buffers: H2D of the
initial fields, every step's fused FP64 solute-mass reduction read back to
the host, D2H of the final fields, all inside one event-timed region.

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


def run_ours(args):
    import torch
    from rapidsolid import configs, lib

    rank, world, local = rank_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    p = configs.scale_fp32()
    ctx = lib.Context(p)
    d = ctx.d
    dtype = torch.float32
    a, b = lib.FieldSet(p, dtype), lib.FieldSet(p, dtype)
    ctx.initial_planar(a, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, configs.IC_SEED)
    st = torch.cuda.current_stream()
    cells = (p.nx_all - 2) * (p.ny_all - 2)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    itip = torch.zeros(1, dtype=torch.int32, device="cuda")

    state = {"step": 0, "hist": 0, "l": 0.0, "a": a, "b": b}
    launches = [0]

    def vp_dl(n):
        return p.Vp * d.dt * d.tau0 / (p.S * p.W0)

    def one_step(mass_out=None):
        """main.cu loop body: pull-back every step_pull_back steps (coarse tip
        reduced on the device, 4-byte read), fused step."""
        n = state["step"]
        pb = None
        if n % d.step_pull_back == 0:
            ctx.itip(state["a"], itip)
            launches[0] += 2
            pb = int(itip.item()) - p.i_tip_target
            state["hist"] += pb
        ctx.step(state["a"], state["b"], n, i_offset_history=state["hist"], l_offset_Vp=state["l"],
                 pull_back=pb, mass_out=mass_out)
        # a pull-back step is one register-kernel launch (+1 for its mass
        # reduction); the others launch the column-table kernel and the tile
        # kernel, which reduces the mass itself
        launches[0] += (1 if pb is not None else 2) + (1 if mass_out is not None and pb is not None else 0)
        state["l"] += vp_dl(n)
        state["a"], state["b"] = state["b"], state["a"]
        state["step"] = n + 1

    for _ in range(args.warmup):
        one_step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    # clocks are sampled from before to after the timed region (200 ms period):
    # untimed steps keep the GPU under load while the sampler starts
    clocks = ClockSampler(local)
    clocks.start()
    t_pre = time.time()
    while time.time() - t_pre < args.clock_preroll:
        for _ in range(20):
            one_step()
        torch.cuda.synchronize()
    launches[0] = 0
    t_wall = time.time()
    for k in range(args.steps):
        flush.fill_(float(k))
        ev[k][0].record(st)
        one_step()
        ev[k][1].record(st)
    torch.cuda.synchronize()
    t_wall = time.time() - t_wall
    gpu_launches = launches[0]
    t_post = time.time()
    while time.time() - t_post < 0.3:
        for _ in range(20):
            one_step()
        torch.cuda.synchronize()
    clk = clocks.stop()
    ms_steps = [s.elapsed_time(e) for s, e in ev]
    total_ms = max_over_ranks(sum(ms_steps), dist, "cuda")
    ms_per_step = total_ms / args.steps
    value = job_throughput(world, cells, args.steps, total_ms)

    # roofline of the step kernel: median launch duration
    srt = sorted(ms_steps)
    kern_ms = srt[len(srt) // 2]
    alg_bytes = BYTES_PER_CELL["f32"] * cells
    achieved = alg_bytes / (kern_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak()
    # the same bytes moved by a plain device copy (half read, half written)
    # under the same flush: the floor of one step of this size
    src = torch.ones(alg_bytes // 8, dtype=torch.float32, device="cuda")
    dst = torch.empty_like(src)
    cts = []
    for k in range(max(args.steps, 10)):
        flush.fill_(float(k))
        c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        c0.record(st)
        dst.copy_(src)
        c1.record(st)
        torch.cuda.synchronize()
        cts.append(c0.elapsed_time(c1))
    copy_ms = sorted(cts)[len(cts) // 2]
    del src, dst

    # ---- e2e through the C-ABI with host buffers
    e2e_steps = args.steps
    h_psi = torch.empty((p.ny_all, p.nx_all), dtype=dtype, pin_memory=True)
    h_c = torch.empty_like(h_psi).pin_memory()
    h_psi.copy_(state["a"].psi)
    h_c.copy_(state["a"].c)
    h_mass = torch.zeros(e2e_steps, dtype=torch.float64, pin_memory=True)
    d_mass = torch.zeros(e2e_steps, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # each step's solute mass is read back on a copy stream, so the read
    # overlaps the next step instead of holding the compute stream
    cs = torch.cuda.Stream()
    done = [torch.cuda.Event() for _ in range(e2e_steps)]
    e0.record(st)
    state["a"].psi.copy_(h_psi, non_blocking=True)
    state["a"].c.copy_(h_c, non_blocking=True)
    for k in range(e2e_steps):
        one_step(mass_out=d_mass[k:k + 1])
        done[k].record(st)
        cs.wait_event(done[k])
        with torch.cuda.stream(cs):
            h_mass[k:k + 1].copy_(d_mass[k:k + 1], non_blocking=True)
    h_psi.copy_(state["a"].psi, non_blocking=True)
    h_c.copy_(state["a"].c, non_blocking=True)
    st.wait_stream(cs)
    e1.record(st)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
    field_bytes = 2 * h_psi.numel() * h_psi.element_size()
    e2e = {"value": job_throughput(world, cells, e2e_steps, e2e_ms), "unit": UNIT,
           "h2d_bytes_per_step": field_bytes / e2e_steps, "d2h_bytes_per_step": 8 + field_bytes / e2e_steps,
           "ms_per_step": e2e_ms / e2e_steps,
           "note": "C-ABI rs_step from pinned host fields; per-step FP64 mass read back on a copy stream; "
                   "no L2 flush"}

    line = {
        "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32 (FP64 column CALPHAD groups, FP64 mass sum)",
        "data": "synthetic (seeded planar Ti-10Nb front, Philox noise)",
        "config": {"workload": "Ti-10Nb directional solidification 2048x2048 FP32 exact CALPHAD, frozen T "
                               "G=5e6 K/m V=0.5 m/s, moving frame, interface noise 0.01",
                   "grid": [p.nx_all, p.ny_all], "interior_cells": cells, "dx_W": p.dx, "dt_tau0": d.dt,
                   "step_pull_back": d.step_pull_back, "l2": "flushed between timed steps (256 MiB write)",
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": alg_bytes, "kernel": "rs::tile_kernel",
                     "kernel_ms_median": round(kern_ms, 5), "traffic": profiled_traffic("step_f32_2048"),
                     "copy_floor": {"ms": round(copy_ms, 5),
                                    "frac": round(alg_bytes / (copy_ms * 1e-3) / 1e9 / peak, 4),
                                    "note": "device copy of the same bytes under the same L2 flush"}},
        "e2e": e2e, "gpu_launches": gpu_launches, "clocks": clk, "wall_s_timed": round(t_wall, 3),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(p, seconds=args.cpu_seconds)
    if rank == 0 and world == 1 and not args.no_side_legs:
        fp64 = fp64_leg(p, flush)
        line["fp64_exact"] = fp64
        line["fp32_exact_vs_fp64_exact"] = round(value / fp64["value"], 3)
        line["surrogate"] = surrogate_leg(p, flush, value, fp64["value"])
        line["ensemble"] = ensemble_leg(flush)
        del flush
        torch.cuda.empty_cache()
        line["peritectic_3d"] = peritectic_3d_leg(peak)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


def _timed_steps(ctx, p, d, a, b, flush, n0, nsteps):
    """Median CUDA-event time (ms) of nsteps steps, L2 flushed between them."""
    import torch
    ts = []
    for k in range(nsteps):
        flush.fill_(float(k))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ctx.step(a, b, n0 + k)
        e1.record()
        a, b = b, a
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    ts.sort()
    return ts[len(ts) // 2]


def fp64_leg(p, flush, nsteps=30):
    """The exact FP64 step (the drop-in's precision) on the same workload."""
    import torch
    from rapidsolid import configs, lib
    ctx = lib.Context(p)
    a, b = lib.FieldSet(p, torch.float64), lib.FieldSet(p, torch.float64)
    ctx.initial_planar(a, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, configs.IC_SEED)
    for k in range(1, 6):
        ctx.step(a, b, k)
        a, b = b, a
    ms = _timed_steps(ctx, p, ctx.d, a, b, flush, 6, nsteps)
    cells = (p.nx_all - 2) * (p.ny_all - 2)
    ctx.close()
    return {"value": round(cells / (ms * 1e-3) / 1e9, 3), "ms_per_step": round(ms, 5), "steps": nsteps,
            "kernel": "rs::step_kernel<double, H, 3, false> (register prefetch)",
            "note": "median of CUDA-event step times, L2 flushed"}


def _tip_run(p, use_w, box, nsteps=20000, every=1000):
    """The C2 loop (moving frame, tip every `every` steps): tip positions."""
    import ctypes as C
    import torch
    from rapidsolid import _abi, configs, lib
    ctx = lib.Context(p)
    d = ctx.d
    if use_w is not None:
        ctx.set_surrogate(use_w, box)
    a, b = lib.FieldSet(p, torch.float32), lib.FieldSet(p, torch.float32)
    ctx.initial_planar(a, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, configs.IC_SEED)
    itip = torch.zeros(1, dtype=torch.int32, device="cuda")
    tipbuf = torch.zeros(C.sizeof(_abi.Tip), dtype=torch.uint8, device="cuda")
    hist, l, xs = 0, 0.0, []
    for n in range(nsteps + 1):
        if n % every == 0:
            ctx.precise_tip(a, tipbuf)
            t = lib.tip_from_bytes(tipbuf.cpu().numpy().tobytes())
            xs.append((hist + t.x) * p.dx)
            if n == nsteps:
                break
        pb = None
        if n % d.step_pull_back == 0:
            ctx.itip(a, itip)
            pb = int(itip.item()) - p.i_tip_target
            hist += pb
        ctx.step(a, b, n, i_offset_history=hist, l_offset_Vp=l, pull_back=pb)
        l += p.Vp * d.dt * d.tau0 / (p.S * p.W0)
        a, b = b, a
    torch.cuda.synchronize()
    audit = ctx.surrogate_audit() if use_w is not None else None
    ctx.close()
    half = len(xs) // 2
    v = (xs[-1] - xs[half]) * p.S * p.W0 / ((nsteps - half * every) * d.tau0 * d.dt)
    return xs, v, audit


def surrogate_leg(p, flush, fp32_value, fp64_value, nsteps=30):
    """The FP32 step with the learned CALPHAD surrogate (trained here on the
    GPU by the library's kernels): speed, and tip speed against the exact FP32
    step over the full 20000-step run, for the box fitted to the run and for
    the wide training box of the workload definition."""
    import torch
    from rapidsolid import configs, lib, surrogate
    boxes = {"fitted": surrogate.fitted_box(), "wide": surrogate.default_box()}
    trained = {}
    for name, bx in boxes.items():
        t0 = time.time()
        w, box, hist = surrogate.train(p, box=bx, epochs=40)
        torch.cuda.synchronize()
        trained[name] = (w, box, hist, time.time() - t0)
    w, box = trained["fitted"][:2]
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
    x0, v0, _ = _tip_run(p, None, None)
    accuracy = {}
    for name, (w, box, hist, t_train) in trained.items():
        x1, v1, audit = _tip_run(p, w, box)
        accuracy[name] = {
            "tip_speed_error": round(abs(v1 - v0) / v0, 5), "tip_speed_m_s": [round(v0, 6), round(v1, 6)],
            "tip_position_max_dx": round(max(abs(u - q) for u, q in zip(x0, x1)) / p.dx, 4),
            "box": {"T": [round(box.T_lo, 3), round(box.T_hi, 3)], "c": [box.c_lo, box.c_hi]},
            "train_s": round(t_train, 2), "train_scaled_mse": hist[-1],
            "audit": {"max_err_mu_J_mol": audit[0], "max_err_dG_J_mol": audit[1], "fallback_cells": audit[2],
                      "audited_cells": audit[3]}}
    return {"value": round(value, 3), "ms_per_step": round(ms, 5), "vs_fp32_exact": round(value / fp32_value, 3),
            "vs_fp64_exact": round(value / fp64_value, 3), "box_of_speed": "fitted", "accuracy": accuracy,
            "note": "3->32->32->2 SiLU, FP16 mma.sync hidden layers; the network evaluates every cell that is "
                    "not bulk melt (the melt keeps its exact series form); exact fallback out of box and "
                    "1/1024 audit"}


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


def ensemble_leg(flush, nruns=64, nsteps=100):
    """The batched ensemble of uneven runs (64 Ti-Nb runs, sizes 256^2 ..
    1024x2048, V 0.01-2 m/s, G 1e5-1e7 K/m, x_Nb 0.05-0.20, seeded): aggregate
    Gcell-steps/s of the one-launch, graph-replayed step, against the same runs
    stepped one rs_step at a time."""
    import torch
    from rapidsolid import configs, lib
    runs = configs.ensemble(nruns)
    ps = [p for p, _, _ in runs]
    cells = sum((p.nx_all - 2) * (p.ny_all - 2) for p in ps)
    ens = lib.Ensemble(ps)
    for r, (p, cl, cs) in enumerate(runs):
        a, b = lib.FieldSet(p, torch.float32), lib.FieldSet(p, torch.float32)
        ens.ctx[r].initial_planar(a, cl, cs, 7 + r)
        ens.bind(r, a, b)
    choice, tune_ms = ens.autotune(reps=5)
    ens.steps(3)  # step 0 pulls every run back (eager), then graph replays
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    flush.fill_(1.0)
    e0.record()
    ens.steps(nsteps)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
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
    ens.close()
    return {"value": round(cells * nsteps / (ms * 1e-3) / 1e9, 3), "runs": nruns, "cells": cells,
            "ms_per_step": round(ms / nsteps, 5), "steps": nsteps,
            "one_by_one": {"value": round(cells / (ms_single * 1e-3) / 1e9, 3), "ms_per_step": round(ms_single, 5)},
            "autotune": {"choice": ["run by run", "largest first", "interleaved"][choice],
                         "ms_per_launch": [round(x, 5) for x in tune_ms]},
            "note": "FP32 exact path (the surrogate is slower, see its leg); CUDA graph "
                    "replays between pull-backs; every run equals its single run bit for bit (tests)"}


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
    threads), timed on a bounded sample: each step is one full-grid step."""
    rank, world, _ = rank_info()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    from rapidsolid import configs
    p = configs.scale_fp32()
    d = pyoracle.derive(p)
    s = pyoracle.initial_planar(p, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, configs.IC_SEED)
    steps = max(1, min(args.steps, 20))
    warm = max(0, min(args.warmup, 1))
    if warm:
        s = pyoracle.run(p, d, s, warm)
    t0 = time.time()
    pyoracle.run(p, d, s, steps, step0=warm)
    dt = time.time() - t0
    cells = (p.nx_all - 2) * (p.ny_all - 2)
    value = cells * steps / dt / 1e9
    cores = pyoracle.lib().ro_num_threads()
    sample = f"{steps} FP64 steps of the {p.nx_all}x{p.ny_all} grid after {warm} warm-up"
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 5), "unit": UNIT, "n_gpus": world,
            "steps": steps, "warmup": warm, "ms_per_step": round(dt * 1e3 / steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp64", "data": "synthetic",
            "config": {"workload": "Ti-10Nb directional solidification 2048x2048, exact CALPHAD, frozen T",
                       "grid": [p.nx_all, p.ny_all]},
            "cpu_baseline": {"value": round(value, 5), "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": sample, "cpu": _cpu_model()},
            "e2e": {"value": round(value, 5), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    gpu = _reference_kernels_gpu(pyoracle)
    if gpu:
        line["reference_kernels_b200"] = gpu
    print(json.dumps(line))


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
