"""Run a named workload through the C-ABI for a number of steps.

    python -m rapidsolid.run --config scale_fp32 --precision f32 --steps 8
    python -m rapidsolid.run --config peritectic_3d --nz 256 --steps 3
    (from 2d-rapid-solidification_b200/, or with it on PYTHONPATH)

Used for profiling: every step is one rs_step launch on the whole grid,
starting from the seeded planar Ti-10Nb front of the configuration.  The
moving frame (pull-back every step_pull_back steps) and the per-step frozen
temperature follow the reference loop (main.cu:156-240).
"""
import argparse
import sys

from . import _abi, configs, lib


def main(argv=None):
    import torch
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--config", default="scale_fp32", choices=["plain_small", "scale_fp32", "peritectic_3d"])
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"])
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--grid", type=int, default=0, help="override Nx_all = Ny_all")
    ap.add_argument("--no-tma", action="store_true", help="use the register-prefetch kernel")
    ap.add_argument("--pipeline", action="store_true", help="FP64: the persistent warp-role tile kernel")
    ap.add_argument("--surrogate", action="store_true",
                    help="FP32: train the CALPHAD surrogate on the wide box (10 epochs) and step through it")
    ap.add_argument("--nz", type=int, default=0, help="3D: override the number of z planes")
    ap.add_argument("--tfc", action="store_true",
                    help="2D: the coarse-grid temperature, initialised and then held fixed (the step alone)")
    a = ap.parse_args(argv)
    if a.config == "peritectic_3d":
        return run3(a)
    p = getattr(configs, a.config)()
    if a.grid:
        p.nx_all = p.ny_all = a.grid
    if a.tfc:  # coarse T: a 4 um sample, the front 30 cells above Tcold
        p.tfc = 1
        p.length_sample_um = 4.0
        p.Tcold = p.T_ref - p.GG * p.dx * p.S * p.W0 * (p.i_tip_target + 30)
    ctx = lib.Context(p)
    if a.no_tma:
        ctx.set_option(_abi.RS_OPT_TMA, 0)
    if a.pipeline:
        ctx.set_option(_abi.RS_OPT_PIPELINE, 1)
    if a.surrogate:
        from . import surrogate
        w, box, _ = surrogate.train(p, box=surrogate.default_box(), epochs=10, seed=1)
        ctx.set_surrogate(w, box)
    d = ctx.d
    dt = torch.float64 if a.precision == "f64" else torch.float32
    cur, nxt = lib.FieldSet(p, dt), lib.FieldSet(p, dt)
    ctx.initial_planar(cur, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, configs.IC_SEED)
    T, ile = None, 0
    if a.tfc:
        T = torch.zeros(d.NxT_all * d.NyT_all, dtype=torch.float64, device="cuda")
        ctx.temperature_init(T)
        ile = d.i_left_end_initial
    itip = torch.zeros(1, dtype=torch.int32, device="cuda")
    mass = torch.zeros(1, dtype=torch.float64, device="cuda")
    hist, l = 0, 0.0
    for n in range(a.steps):
        pb = None
        if n % d.step_pull_back == 0:
            ctx.itip(cur, itip)
            pb = int(itip.item()) - p.i_tip_target
            hist += pb
        ctx.step(cur, nxt, n, i_offset_history=hist, l_offset_Vp=l, pull_back=pb, T_coarse=T, i_left_end=ile,
                 i_left_end_T=ile)
        l += p.Vp * d.dt * d.tau0 / (p.S * p.W0)
        cur, nxt = nxt, cur
    ctx.mass(cur, mass)
    torch.cuda.synchronize()
    ctx.device_status()
    print(f"{a.config} {a.precision} grid {p.nx_all}x{p.ny_all}: {a.steps} steps, "
          f"solute mass {mass.item():.12g}")
    return 0


def tip_run(p, dtype, nsteps, every=1000, surrogate=None, ic_seed=None, initial=None):
    """The reference loop (main.cu:156-240) on the workload p from its seeded
    planar front: pull-back every step_pull_back steps, the precise tip every
    `every` steps as set_tip_output does (fun.cu:3024-3050).  surrogate:
    (weights, box) of a trained network, or None for the exact evaluation.
    initial: (c_liquid, c_solid) of the planar front (default Ti-10Nb).
    Returns (tip positions x = (i_offset_history + tip.x) dx in units of W,
    tip velocity in m/s over the second half of the run, the surrogate's
    audit (or None), solute mass at the start and at the end)."""
    import ctypes as C

    import torch
    ctx = lib.Context(p)
    d = ctx.d
    if surrogate is not None:
        ctx.set_surrogate(*surrogate)
    a, b = lib.FieldSet(p, dtype), lib.FieldSet(p, dtype)
    cl, cs = initial if initial is not None else (configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ)
    ctx.initial_planar(a, cl, cs, configs.IC_SEED if ic_seed is None else ic_seed)
    itip = torch.zeros(1, dtype=torch.int32, device="cuda")
    tipbuf = torch.zeros(C.sizeof(_abi.Tip), dtype=torch.uint8, device="cuda")
    mass = torch.zeros(2, dtype=torch.float64, device="cuda")
    ctx.mass(a, mass[0:1])
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
    ctx.mass(a, mass[1:2])
    torch.cuda.synchronize()
    ctx.device_status()
    audit = ctx.surrogate_audit() if surrogate is not None else None
    ctx.close()
    half = len(xs) // 2
    v = (xs[-1] - xs[half]) * p.S * p.W0 / ((nsteps - half * every) * d.tau0 * d.dt)
    m0, m1 = mass.tolist()
    return xs, v, audit, m0, m1


def run3(a):
    """The 3D three-phase workload: rs3_initial, then a.steps rs3_step launches."""
    import torch
    p = configs.peritectic_3d(nz=a.nz) if a.nz else configs.peritectic_3d()
    ctx = lib.Context3(p)
    dt = torch.float64 if a.precision == "f64" else torch.float32
    cur, nxt = lib.FieldSet3(p, dt), lib.FieldSet3(p, dt)
    ctx.initial(cur, **configs.IC3)
    for n in range(a.steps):
        ctx.step(cur, nxt, n)
        cur, nxt = nxt, cur
    mass = torch.zeros(1, dtype=torch.float64, device="cuda")
    ctx.mass(cur, mass)
    torch.cuda.synchronize()
    ctx.device_status()
    print(f"peritectic_3d {a.precision} grid {p.nx}x{p.ny}x{p.nz}: {a.steps} steps, solute mass {mass.item():.12g}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
