"""The learned CALPHAD surrogate: training data, forward and backward kernels
against the CPU restatement (oracle/pymlp.py) and the exact evaluator."""
import numpy as np
import pytest

import pymlp
from rapidsolid import _abi, configs, lib, run, surrogate

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def exact_targets(p, box, x):
    """mu'' = mu(T, c, phi) - Glc(T, cinf) and dG = Gl - Gs from the host build
    of the reference evaluator (fun.cu:1671-1720)."""
    x = x.astype(np.float64)
    T = box.T_lo + (box.T_hi - box.T_lo) * (x[:, 0] + 1.0) / 2.0
    c = box.c_lo + (box.c_hi - box.c_lo) * (x[:, 1] + 1.0) / 2.0
    phi = x[:, 2]
    g = phi * (1.875 + phi * phi * (-1.25 + 0.375 * phi * phi))
    Glc, Gsc = lib.calphad_eval(2, T, c), lib.calphad_eval(3, T, c)
    mu = 0.5 * (1 + g) * Gsc + 0.5 * (1 - g) * Glc
    ref = lib.calphad_eval(2, T, np.full_like(T, p.cinf))
    return np.stack([mu - ref, lib.calphad_eval(0, T, c) - lib.calphad_eval(1, T, c)], axis=1)


def test_samples_are_exact_targets():
    p = configs.scale_fp32()
    box = surrogate.default_box()
    x, y = surrogate.sample(p, box, 4096, seed=5)
    xh, yh = x.cpu().numpy(), y.cpu().numpy().astype(np.float64)
    assert np.abs(xh).max() <= 1.0
    ye = exact_targets(p, box, xh)
    # the GPU evaluates in FP64 from the unrounded draw and stores FP32
    assert np.abs(yh - ye).max() <= 2e-6 * np.abs(ye).max() + 1e-2


def test_forward_and_gradient_match_numpy():
    p = configs.scale_fp32()
    box = surrogate.default_box()
    x, y = surrogate.sample(p, box, 512, seed=9)
    box.y_mean[0], box.y_mean[1], box.y_scale[0], box.y_scale[1] = 100.0, -50.0, 3000.0, 800.0
    w = surrogate.init_weights(3)
    w += np.random.default_rng(4).normal(0, 0.05, w.shape).astype(np.float32)  # non-zero biases
    wt = torch.from_numpy(w).cuda()
    out = surrogate.forward(box, wt, x).cpu().numpy()
    o_ref, _ = pymlp.forward(w, x.cpu().numpy())
    out_ref = o_ref * np.array(box.y_scale[:]) + np.array(box.y_mean[:])
    assert np.abs(out - out_ref).max() <= 1e-5 * np.abs(out_ref).max()
    g, loss = surrogate.grad(box, wt, x, y)
    l_ref, g_ref = pymlp.loss_and_grad(w, x.cpu().numpy(), y.cpu().numpy(), box.y_mean[:], box.y_scale[:])
    assert abs(loss.item() - l_ref) <= 1e-5 * l_ref
    g = g.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(g - g_ref) <= 1e-5 * np.linalg.norm(g_ref)
    # every parameter block is exercised
    for a, b in ((0, 96), (96, 128), (128, 1152), (1152, 1184), (1184, 1248), (1248, 1250)):
        assert np.abs(g_ref[a:b]).max() > 0


def test_training_reduces_the_error():
    p = configs.scale_fp32()
    w, box, hist = surrogate.train(p, n_samples=1 << 16, epochs=6, batch=2048, lr=3e-3, seed=2)
    assert hist[-1] < 0.2 * hist[0]
    x, y = surrogate.sample(p, box, 8192, seed=77)
    emax, erms = surrogate.errors(box, w, x, y)
    # six short epochs: well below the spread of the targets, not converged
    assert erms[0] < 0.5 * box.y_scale[0] and erms[1] < 0.5 * box.y_scale[1]


def test_training_is_reproducible():
    """Every random source of the training is seeded (Philox samples, Glorot
    initial weights, the shuffle) and the gradient of a batch is summed in a
    fixed order (one cluster, partial sums added in rank order), so two
    trainings with one seed give the same weights bit for bit."""
    p = configs.scale()
    runs = [surrogate.train(p, n_samples=1 << 15, epochs=3, batch=2048, seed=11) for _ in range(2)]
    assert torch.equal(runs[0][0], runs[1][0])
    assert runs[0][2] == runs[1][2]
    other = surrogate.train(p, n_samples=1 << 15, epochs=3, batch=2048, seed=12)
    assert not torch.equal(runs[0][0], other[0])


def test_surrogate_tip_speed_on_the_run_box():
    """The learned surrogate on the scale workload (2048^2 FP32, G = 5e6 K/m,
    V = 0.5 m/s, noise 0.01, the full 20000 steps, moving frame), trained on
    the box the run's states occupy (T in [T_solidus - 30, T_liquidus + 10] K,
    x_Ti in [0.84, 0.96]; 2^20 samples, 40 epochs, seed 1): against the exact
    FP32 run, tip velocity over the second half within 0.5 % and tip position
    within 0.25 dx at every sample (every 1000 steps; measured 0.004 % and
    0.13 dx); no cell falls outside the box.  On the wide box of the workload
    definition (T in [T_solidus - 200, T_liquidus + 50] K, x_Nb <= 0.40) the
    same network misses the target (1.8-7.3 % over three seeds, the bench's
    surrogate leg): over a box that wide its FP16 layers resolve Gl - Gs to
    about 1 J/mol, too coarse for the front's kinetics."""
    p = configs.scale()
    w, box, _ = surrogate.train(p, box=surrogate.fitted_box(), epochs=40, seed=1)
    n = configs.STEPS["scale_fp32"]
    x0, v0, _, _, _ = run.tip_run(p, torch.float32, n)
    x1, v1, audit, m0, m1 = run.tip_run(p, torch.float32, n, surrogate=(w, box))
    assert abs(v1 - v0) <= 0.005 * abs(v0), (v0, v1)
    assert max(abs(a - b) for a, b in zip(x0, x1)) <= 0.25 * p.dx, (x0, x1)
    assert audit[2] == 0 and audit[3] > 0


def test_surrogate_step_runs_with_audit():
    """The FP32 step with the surrogate in place of the exact per-cell
    evaluation of every cell that is not bulk melt: finite fields, the audit
    visits about one such cell in 1024 per step and finds no out-of-box cell
    on this workload, and a learned form that still moves the front (its
    accuracy is measured, not asserted to a tolerance: see the surrogate
    notes of the design document)."""
    p = configs.scale_fp32()
    p.nx_all = p.ny_all = 512
    w, box, _ = surrogate.train(p, n_samples=1 << 18, epochs=8, batch=4096, lr=3e-3, seed=4)
    out = {}
    for use in (False, True):
        ctx = lib.Context(p)
        if use:
            ctx.set_surrogate(w, box)
        a, b = lib.FieldSet(p, torch.float32), lib.FieldSet(p, torch.float32)
        ctx.initial_planar(a, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, configs.IC_SEED)
        for n in range(1, 301):
            ctx.step(a, b, n)
            a, b = b, a
        torch.cuda.synchronize()
        ctx.device_status()
        out[use] = (a.psi.cpu().numpy(), a.c.cpu().numpy(), ctx.surrogate_audit() if use else None)
    psi, c, (emu, edg, nfb, naud) = out[True]
    assert np.isfinite(psi).all() and np.isfinite(c).all()
    # cells the network evaluates: psi not exactly -1 (the melt keeps its
    # exact series form), plus tile halo columns next to them
    non_melt = int((out[False][0] != -1.0).sum())
    assert nfb == 0
    assert 0.3 * 300 * non_melt / 1024 < naud < 3.0 * 300 * non_melt / 1024
    assert 0.0 < emu and 0.0 < edg
    # the front stays where the exact run has it to within a few cells
    ifront = lambda ps: (ps.reshape(p.ny_all, p.nx_all)[1:-1, 1:-1] > 0).sum(1).mean()
    assert abs(ifront(psi) - ifront(out[False][0])) < 3.0


def test_surrogate_skips_deep_solid_rows():
    """A wide solid (psi exactly +1) with a liquid pocket: tile rows whose 3x3
    neighbourhoods are all solid take no network pass (their mu'' enters no
    flux).  One step with the surrogate against the exact FP32 step: the deep
    solid is left exactly unchanged, and the c increments near the pocket
    agree to within the network's error (a row wrongly taken as deep would
    lose its whole flux there).  The network is trained on the box fitted to
    the workload (the pocket's T and c lie inside it), whose mu'' error is a
    few per cent of the mu'' differences that drive the pocket's fluxes."""
    from test_gpu_step import download, solid_with_pocket, upload
    p = configs.small(640, 70, i_tip_target=400, G=5e6, V=0.5)
    s = solid_with_pocket(p, 5)
    w, box, _ = surrogate.train(p, box=surrogate.fitted_box(), epochs=40, seed=4)
    out = {}
    for use in (False, True):
        ctx = lib.Context(p)
        if use:
            ctx.set_surrogate(w, box)
        cur, nxt = upload(p, s, torch.float32), lib.FieldSet(p, torch.float32)
        s32 = download(p, cur)
        ctx.step(cur, nxt, 0)
        torch.cuda.synchronize()
        ctx.device_status()
        out[use] = download(p, nxt)
    g, e = out[True], out[False]
    assert np.isfinite(g.psi).all() and np.isfinite(g.c).all()
    solid = s32.psi == 1.0
    deep = solid.copy()
    for dj in (-1, 0, 1):
        for di in (-1, 0, 1):
            deep &= np.roll(np.roll(solid, dj, 0), di, 1)
    deep[[0, -1], :] = deep[:, [0, -1]] = False
    assert np.array_equal(g.c[deep], s32.c[deep]) and np.array_equal(g.psi[deep], s32.psi[deep])
    near = np.zeros_like(deep)
    near[20:47, 175:206] = True  # the pocket and its interface
    de = e.c - s32.c
    assert np.abs(de[near]).max() > 1e-6
    err, ref = np.abs((g.c - s32.c) - de)[near].max(), np.abs(de[near]).max()
    assert err <= 0.5 * ref, (err, ref, ctx.surrogate_audit())
