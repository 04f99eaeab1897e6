"""The 3D step with the Ti-Nb CALPHAD energy (rs3_params.energy = 1) on the
GPU against the FP64 oracle (oracle/rs3_oracle.c, whose energy 1 is pinned to
the reference's 2D CALPHAD step in test_oracle_tinb3.py).

Tolerances: FP64 within 1e-13 of the oracle after one step and 1e-10 after
100 steps (the oracle does not contract multiply-adds, the kernel does; the
kernel's per-plane CALPHAD groups come from the device evaluator); FP32
within 2e-4 in phi1, phi2 and 2e-6 in c of the FP64 oracle after 200 steps,
solute mass within 1e-7 (relative) of its start."""
import numpy as np
import pytest
import torch

import pyoracle
from rapidsolid import configs, lib, surrogate
from test_gpu_peri3d import maxdiff, run_gpu, to_gpu, to_host

pytestmark = pytest.mark.gpu

X_NB = 0.10


def params(nx=40, ny=22, nz=45, **kw):
    p = configs.tinb_3d(nx=nx, ny=ny, nz=nz, z_front=12.0)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def initial(p, seed=5):
    cl, cs = configs.tinb_compositions(X_NB)
    return pyoracle.initial_grains3(p, 12.0, 0.5, cl, cs, seed)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_initial_grains_match_oracle(dtype):
    p = params()
    cl, cs = configs.tinb_compositions(X_NB)
    ctx = lib.Context3(p)
    s = lib.FieldSet3(p, dtype)
    ctx.initial_grains(s, 12.0, 0.5, cl, cs, 5)
    torch.cuda.synchronize()
    got = to_host(s, p)
    ref = initial(p)
    tol = 0.0 if dtype == torch.float64 else 1e-7
    assert maxdiff(got, ref) <= tol
    ctx.close()


def test_mu_matches_oracle():
    p = params()
    f = pyoracle.run3(p, initial(p), 3)  # smooth interfaces
    ctx = lib.Context3(p)
    s = to_gpu(p, f, torch.float64)
    mu = torch.empty_like(s.c)
    ctx.mu(s, mu)
    ref = pyoracle.mu3(p, *f)
    np.testing.assert_allclose(mu.cpu().numpy(), ref, rtol=1e-13, atol=1e-9)
    ctx.close()


@pytest.mark.parametrize("nsteps,tol", [(1, 1e-13), (100, 1e-10)])
def test_fp64_matches_oracle(nsteps, tol):
    p = params()
    f = initial(p)
    out = run_gpu(p, f, nsteps)
    ref = pyoracle.run3(p, f, nsteps)
    assert maxdiff(out, ref) <= tol


def test_fp64_with_solid_diffusion_and_moving_isotherms():
    p = params(Da=0.1, Db=0.05, V_T=0.05)
    f = pyoracle.run3(p, initial(p), 2)
    out = run_gpu(p, f, 3, step0=2)
    ref = pyoracle.run3(p, f, 3, step0=2)
    assert maxdiff(out, ref) <= 1e-13


def test_fp32_close_to_fp64():
    p = params()
    f = initial(p)
    out = run_gpu(p, f, 200, dtype=torch.float32)
    ref = pyoracle.run3(p, f, 200)
    assert float(np.abs(out[0] - ref[0]).max()) <= 2e-4
    assert float(np.abs(out[1] - ref[1]).max()) <= 2e-4
    assert float(np.abs(out[2] - ref[2]).max()) <= 2e-6
    m0, m1 = pyoracle.mass3(p, f[2]), pyoracle.mass3(p, np.ascontiguousarray(out[2]))
    assert abs(m1 - m0) <= 1e-7 * m0


def front(p1):
    """mean number of solid cells (phi1 < 1/2) per (x, y) column"""
    return float((p1[1:-1, 1:-1, 1:-1] < 0.5).sum(0).mean())


def test_surrogate_follows_the_exact_step():
    """FP32 with the learned CALPHAD surrogate (inputs T, c and the
    interpolation weight g, trained on the box of the run's states) against
    the exact FP32 step over 400 steps: the front within 0.25 cell on
    average, no cell outside the box, audited cells and bounded errors."""
    p = params(nx=64, ny=32, nz=64)
    p2 = configs.scale()
    p2.cinf = p.c_ref
    w, box, _ = surrogate.train(p2, box=surrogate.fitted_box(), n_samples=1 << 18, epochs=20, batch=4096, seed=3,
                                g_input=True)
    f = initial(p)
    out = {}
    for use in (False, True):
        ctx = lib.Context3(p)
        if use:
            ctx.set_surrogate(w, box)
        a, b = to_gpu(p, f, torch.float32), lib.FieldSet3(p, torch.float32)
        for k in range(400):
            ctx.step(a, b, k)
            a, b = b, a
        torch.cuda.synchronize()
        ctx.device_status()
        out[use] = (to_host(a, p), ctx.surrogate_audit() if use else None)
        ctx.close()
    (ex, _), (su, (emu, edg, nfb, naud)) = out[False], out[True]
    assert np.isfinite(su[0]).all() and np.isfinite(su[2]).all()
    assert nfb == 0 and naud > 0
    assert emu < 500.0 and edg < 20.0
    assert abs(front(su[0]) - front(ex[0])) <= 0.25
