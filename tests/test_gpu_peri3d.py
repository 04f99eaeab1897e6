"""The 3D three-phase step on the GPU (rs3_step, one TMA z-march kernel)
against the FP64 oracle and the reference's own kernels (TiAg.cu).

Tolerances: FP64 within 1e-13 of the oracle after one step and 1e-10 after
200 steps (the oracle does not contract multiply-adds, the kernel does);
FP32 within 5e-5 of the FP64 oracle in phi1, phi2 and c after 200 steps, and
solute mass within 1e-8 (relative) of its start over 200 full-size steps."""
import os
import subprocess
import tempfile

import numpy as np
import pytest
import torch

import pyoracle
from helpers import golden
from rapidsolid import configs, lib

pytestmark = pytest.mark.gpu


def params(nx=32, ny=32, nz=20, **kw):
    p = lib.default_params3()
    p.nx, p.ny, p.nz = nx, ny, nz
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def to_gpu(p, f, dtype):
    """FP32 sets hold c - c_offset3 (rs3_c_offset)."""
    s = lib.FieldSet3(p, dtype)
    off = lib.c_offset3(p) if dtype == torch.float32 else 0.0
    for dst, src in zip((s.phi1, s.phi2, s.c), (f[0], f[1], f[2] - off)):
        dst.copy_(torch.from_numpy(src))
    s.off = off
    return s


def to_host(s, p=None):
    off = getattr(s, "off", None)
    if off is None:
        off = lib.c_offset3(p) if s.dtype == torch.float32 else 0.0
    return [s.phi1.double().cpu().numpy(), s.phi2.double().cpu().numpy(), s.c.double().cpu().numpy() + off]


def run_gpu(p, f, nsteps, dtype=torch.float64, step0=0):
    ctx = lib.Context3(p)
    a, b = to_gpu(p, f, dtype), lib.FieldSet3(p, dtype)
    for k in range(nsteps):
        ctx.step(a, b, step0 + k)
        a, b = b, a
    torch.cuda.synchronize()
    ctx.device_status()
    out = to_host(a, p)
    ctx.close()
    return out


def maxdiff(a, b):
    return max(float(np.abs(x - y).max()) for x, y in zip(a, b))


@pytest.mark.parametrize("nsteps,tol", [(1, 1e-13), (200, 1e-10)])
def test_fp64_matches_reference_kernels(nsteps, tol):
    z = golden("peri3d_32.npz")
    p = params()
    out = run_gpu(p, [z["phi1"], z["phi2"], z["c"]], nsteps)
    ref = [z[f"{n}_{nsteps}"] for n in ("phi1", "phi2", "c")]
    assert maxdiff(out, ref) <= tol


def test_mu_matches_reference_kernels():
    z = golden("peri3d_32.npz")
    p = params()
    ctx = lib.Context3(p)
    s = to_gpu(p, [z["phi1"], z["phi2"], z["c"]], torch.float64)
    mu = torch.empty_like(s.c)
    ctx.mu(s, mu)
    np.testing.assert_allclose(mu.cpu().numpy(), z["mu0"], rtol=0, atol=1e-15)
    ctx.close()


@pytest.mark.parametrize("shape", [(36, 27, 13), (64, 48, 9), (128, 16, 70)])
def test_fp64_ragged_sizes_match_oracle(shape):
    """Partial tiles in x and y, planes not a multiple of the z chunk."""
    p = params(*shape)
    f = pyoracle.initial3(p, 5.0, 0.5, 2, 4.0, 9)
    out = run_gpu(p, f, 30)
    ref = pyoracle.run3(p, f, 30)
    assert maxdiff(out, ref) <= 1e-11


@pytest.mark.parametrize("z_chunk", [1, 2, 3, 5, 64])
def test_z_chunks_give_identical_results(z_chunk):
    p = params(64, 32, 24)
    f = pyoracle.initial3(p, 8.0, 0.5, 2, 5.0, 1)
    base = run_gpu(p, f, 10)
    p.z_chunk = z_chunk
    assert maxdiff(run_gpu(p, f, 10), base) == 0.0


def test_gradient_extension_matches_oracle():
    p = params(64, 32, 40, G_T=-2e-4, V_T=0.05, z_T=12.0)
    f = pyoracle.initial3(p, 12.0, 0.5, 3, 6.0, 4)
    out = run_gpu(p, f, 50, step0=100)
    ref = pyoracle.run3(p, f, 50, step0=100)
    assert maxdiff(out, ref) <= 1e-11


def test_initial_state_matches_oracle():
    p = params(64, 48, 30)
    ctx = lib.Context3(p)
    s = lib.FieldSet3(p, torch.float64)
    ctx.initial(s, 10.0, 0.5, 3, 6.0, 21)
    ref = pyoracle.initial3(p, 10.0, 0.5, 3, 6.0, 21)
    assert maxdiff(to_host(s), ref) == 0.0
    ctx.close()


def test_fp32_within_tolerance_of_fp64_oracle():
    z = golden("peri3d_32.npz")
    p = params()
    f = [z["phi1"], z["phi2"], z["c"]]
    out = run_gpu(p, f, 200, dtype=torch.float32)
    ref = [z[f"{n}_200"] for n in ("phi1", "phi2", "c")]
    assert maxdiff(out, ref) <= 5e-5


@pytest.mark.parametrize("shape", [(36, 27, 13), (64, 48, 9), (132, 40, 70)])
def test_fp32_ragged_sizes_within_tolerance(shape):
    """The packed-pair FP32 kernel on partial tiles (x pairs beside the ghost
    columns, rows past the last full tile) against the FP64 oracle."""
    p = params(*shape)
    f = pyoracle.initial3(p, 5.0, 0.5, 2, 4.0, 9)
    out = run_gpu(p, f, 30, dtype=torch.float32)
    ref = pyoracle.run3(p, f, 30)
    assert maxdiff(out, ref) <= 2e-5


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-11), (torch.float32, 5e-5)])
def test_nonzero_a1_and_solid_diffusion(dtype, tol):
    """a1 and the solid diffusivities Da, Db (zero in the reference's set)
    switch on the kernels' optional terms."""
    p = params(64, 32, 24, a1=1.5, Da=0.3, Db=0.2)
    f = pyoracle.initial3(p, 8.0, 0.5, 2, 5.0, 6)
    out = run_gpu(p, f, 40, dtype=dtype)
    ref = pyoracle.run3(p, f, 40)
    assert maxdiff(out, ref) <= tol


def test_mass_reduction():
    p = params(64, 48, 30)
    f = pyoracle.initial3(p, 10.0, 0.5, 3, 6.0, 2)
    ctx = lib.Context3(p)
    s = to_gpu(p, f, torch.float64)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    ctx.mass(s, out)
    # summation orders differ: within the accumulated rounding of 92 160 terms
    assert out.item() == pytest.approx(pyoracle.mass3(p, f[2]), rel=1e-11)
    ctx.close()


def test_fp32_initial_state_and_mu_carry_the_offset():
    p = params(64, 48, 30)
    ctx = lib.Context3(p)
    s = lib.FieldSet3(p, torch.float32)
    ctx.initial(s, 10.0, 0.5, 3, 6.0, 21)
    ref = pyoracle.initial3(p, 10.0, 0.5, 3, 6.0, 21)
    assert maxdiff(to_host(s, p), ref) <= 1e-7
    mu = torch.empty_like(s.c)
    ctx.mu(s, mu)
    assert np.abs(mu.double().cpu().numpy() - pyoracle.mu3(p, *ref)).max() <= 1e-6
    m = torch.zeros(1, dtype=torch.float64, device="cuda")
    ctx.mass(s, m)
    assert m.item() == pytest.approx(pyoracle.mass3(p, ref[2]), rel=1e-7)
    ctx.close()


def test_full_size_fp32_run_conserves_solute():
    """The workload's 512 x 512 x 1024 FP32 grid: 200 steps, finite fields,
    solute mass within 1e-8 (relative) of its start (FP32 sets hold c minus
    the melt's composition; what drifts is solid-side updates below the
    rounding of c there)."""
    p = configs.peritectic_3d()
    ctx = lib.Context3(p)
    a, b = lib.FieldSet3(p, torch.float32), lib.FieldSet3(p, torch.float32)
    ctx.initial(a, **configs.IC3)
    m = torch.zeros(2, dtype=torch.float64, device="cuda")
    ctx.mass(a, m[0:1])
    for k in range(200):
        ctx.step(a, b, k)
        a, b = b, a
    ctx.mass(a, m[1:2])
    torch.cuda.synchronize()
    ctx.device_status()
    m0, m1 = m.tolist()
    assert abs(m1 - m0) <= 1e-8 * abs(m0)
    assert torch.isfinite(a.phi1).all() and torch.isfinite(a.c).all()
    ctx.close()


def test_live_reference_at_its_own_size():
    """512 x 512 x 128 (TiAg.cu's own Nx, Ny, devNz), FP64: 20 steps of the
    reference's kernels (oracle/_ref/ref3_harness_512) against rs3_step."""
    binary = pyoracle.ref_binary("ref3_harness_512")
    if not os.path.exists(binary):
        pytest.skip("reference harness not built (oracle/ref_build.sh)")
    p = params(512, 512, 128)
    ctx = lib.Context3(p)
    s = lib.FieldSet3(p, torch.float64)
    ctx.initial(s, 40.0, 0.5, 4, 30.0, 17)
    f = to_host(s)
    ctx.close()
    with tempfile.TemporaryDirectory() as td:
        din, dout = os.path.join(td, "in"), os.path.join(td, "out")
        os.makedirs(din)
        os.makedirs(dout)
        for name, a in zip(("phi1", "phi2", "c"), f):
            a.tofile(os.path.join(din, name + ".bin"))
        subprocess.run([binary, "step", din, dout, "20"], check=True)
        ref = [np.fromfile(os.path.join(dout, n + ".bin"), dtype=np.float64).reshape(f[0].shape)
               for n in ("phi1", "phi2", "c")]
    out = run_gpu(p, f, 20)
    assert maxdiff(out, ref) <= 1e-12
