"""Parity of the CUDA step (through the C-ABI) with the CPU FP64 oracle."""
import ctypes as C

import numpy as np
import pytest

import pyoracle
from helpers import fix_ghosts, golden, maxabs, perturbed_state
from rapidsolid import _abi, configs, lib

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def upload(p, s, dtype=torch.float64, with_phi=False):
    fs = lib.FieldSet(p, dtype, with_phi=with_phi)
    fs.psi.copy_(torch.from_numpy(s.psi))
    if dtype == torch.float64:
        fs.c.copy_(torch.from_numpy(s.c))
    else:
        fs.c.copy_(torch.from_numpy(s.c - p.cinf))
    if with_phi:
        fs.phi.copy_(torch.from_numpy(s.phi))
    return fs


def download(p, fs):
    s = pyoracle.State(p)
    s.psi[:] = fs.psi.double().cpu().numpy()
    c = fs.c.double().cpu().numpy()
    s.c[:] = c if fs.dtype == torch.float64 else c + p.cinf
    s.phi[:] = np.clip(s.psi, -1, 1) if fs.phi is None else fs.phi.double().cpu().numpy()
    return s


VARIANTS = {
    "default": {},
    "noise": dict(noise_amplitude=0.05, seed=12345),
    "two_eps": dict(one_eps=0, eps2=0.01, eps1=0.03, epk1=0.1),
    "noflux": dict(periodic_j=0),
    "steep": dict(G=5e6, V=0.5),
}


def make(name, nx=64, ny=48):
    kw = dict(VARIANTS[name])
    p = configs.small(nx, ny, i_tip_target=22, G=kw.pop("G", 1e6), V=kw.pop("V", 0.05), **kw)
    return p


@pytest.mark.parametrize("tma", [1, 0])
@pytest.mark.parametrize("name", sorted(VARIANTS))
def test_single_step_f64(name, tma):
    p = make(name)
    d = pyoracle.derive(p)
    s = perturbed_state(p, 17, amp=0.25)
    ctx = lib.Context(p)
    ctx.set_option(_abi.RS_OPT_TMA, tma)
    cur = upload(p, s, with_phi=True)
    nxt = lib.FieldSet(p, torch.float64, with_phi=True)
    ctx.step(cur, nxt, 3, i_offset_history=2, l_offset_Vp=0.37)
    torch.cuda.synchronize()
    o = pyoracle.step(p, d, s, 3, 2, 0.37)
    g = download(p, nxt)
    for k in ("psi", "phi", "c"):
        assert maxabs(getattr(g, k), getattr(o, k)) <= 1e-13, k
    ctx.device_status()


def test_f64_series_rows_match_oracle_log_form():
    """The FP64 kernel takes log(c/(1-c)) - log(cinf/(1-cinf)) as the atanh
    series of s = delta/(2 cinf (1-c) + delta) on rows whose cells all have
    |s| < 1/9, the oracle (like the reference) takes the logarithm.  A melt
    with seeded solute noise (|s| about 0.024 on average, 82 % of the warp rows
    in the series range, the others on the logarithm) gives one step within
    the single-step tolerance."""
    p = make("default", 160, 64)
    d = pyoracle.derive(p)
    s = perturbed_state(p, 29, amp=0.2)
    rng = np.random.default_rng(29)
    liquid = s.psi < -0.999
    s.c[:] = np.where(liquid, p.cinf + 0.0055 * rng.standard_normal(s.c.shape), s.c)
    fix_ghosts(p, s)
    delta = s.c - p.cinf
    sv = delta / (2 * p.cinf * (1 - s.c) + delta)
    assert np.abs(sv[liquid]).max() > 1 / 9 and np.abs(sv[liquid]).mean() > 0.02
    ctx = lib.Context(p)
    cur, nxt = upload(p, s), lib.FieldSet(p, torch.float64)
    ctx.step(cur, nxt, 0)
    o = pyoracle.step(p, d, s, 0)
    g = download(p, nxt)
    assert maxabs(g.psi, o.psi) <= 1e-13 and maxabs(g.c, o.c) <= 1e-13


def test_f64_far_melt_rows_match_oracle_log_form():
    """Far-melt rows (psi = -1 and |c - cinf| <= 1e-3 min(cinf, 1 - cinf) on
    every cell of the warp's row) take the solute log term as its Taylor
    polynomial in c - cinf.  A melt whose solute noise grows along the
    growth axis from 1e-12 to 1e-3 (so warp rows fall on the polynomial, on
    the atanh series and on the logarithm), with exact zeros in part of it,
    gives one step and twenty steps within the tolerances of the oracle's
    logarithm."""
    p = make("default", 256, 64)
    d = pyoracle.derive(p)
    s = perturbed_state(p, 31, amp=0.2)
    rng = np.random.default_rng(31)
    liquid = s.psi < -0.999
    i = np.arange(p.nx_all)[None, :]
    amp = 10.0 ** (-12.0 + 9.0 * i / p.nx_all)
    noise = amp * rng.standard_normal(s.c.shape)
    noise[:, 200:230] = 0.0
    s.c[:] = np.where(liquid, p.cinf + noise, s.c)
    fix_ghosts(p, s)
    tiny = 1e-3 * min(p.cinf, 1 - p.cinf)
    far = liquid & (np.abs(s.c - p.cinf) <= tiny)
    assert far.mean() > 0.3 and (liquid & ~far).any()
    ctx = lib.Context(p)
    cur, nxt = upload(p, s), lib.FieldSet(p, torch.float64)
    ctx.step(cur, nxt, 0)
    o = pyoracle.step(p, d, s, 0)
    g = download(p, nxt)
    assert maxabs(g.psi, o.psi) <= 1e-13 and maxabs(g.c, o.c) <= 1e-13
    for n in range(1, 20):
        ctx.step(nxt, cur, n)
        cur, nxt = nxt, cur
        o = pyoracle.step(p, d, o, n)
    g = download(p, nxt)
    assert maxabs(g.psi, o.psi) <= 1e-12 and maxabs(g.c, o.c) <= 1e-12


def test_rotated_orientation_f64():
    p = make("default")
    a, b, gm = np.radians([20.0, 10.0, 35.0])
    R = [np.cos(b) * np.cos(gm), np.sin(a) * np.sin(b) * np.cos(gm) - np.cos(a) * np.sin(gm),
         np.cos(a) * np.sin(b) * np.cos(gm) + np.sin(a) * np.sin(gm), np.cos(b) * np.sin(gm),
         np.sin(a) * np.sin(b) * np.sin(gm) + np.cos(a) * np.cos(gm),
         np.cos(a) * np.sin(b) * np.sin(gm) - np.sin(a) * np.cos(gm), -np.sin(b), np.sin(a) * np.cos(b),
         np.cos(a) * np.cos(b)]
    for k in range(9):
        p.orientation[k] = R[k]
    d = pyoracle.derive(p)
    s = perturbed_state(p, 4, amp=0.3)
    ctx = lib.Context(p)
    cur, nxt = upload(p, s), lib.FieldSet(p, torch.float64)
    ctx.step(cur, nxt, 0)
    o = pyoracle.step(p, d, s, 0)
    g = download(p, nxt)
    assert maxabs(g.psi, o.psi) <= 1e-13 and maxabs(g.c, o.c) <= 1e-13


@pytest.mark.parametrize("tma", [1, 0])
@pytest.mark.parametrize("off", [-2, 0, 3, 40])
def test_fused_pull_back_step_f64(off, tma):
    """A pull-back step fused into rs_step (the tile kernel gathers its
    shifted tile; the register kernel remaps its loads) against the oracle's
    pull_back then step; off = 40 fills most columns from the right edge."""
    p = make("default")
    d = pyoracle.derive(p)
    s = perturbed_state(p, 23, amp=0.2)
    ctx = lib.Context(p)
    ctx.set_option(_abi.RS_OPT_TMA, tma)
    cur, nxt = upload(p, s), lib.FieldSet(p, torch.float64)
    ctx.step(cur, nxt, 0, i_offset_history=off, pull_back=off)
    o = pyoracle.step(p, d, pyoracle.pull_back(p, s, off), 0, off, 0.0)
    g = download(p, nxt)
    assert maxabs(g.psi, o.psi) <= 1e-13 and maxabs(g.c, o.c) <= 1e-13


@pytest.mark.parametrize("tma", [1, 0])
@pytest.mark.parametrize("off", [-2, 3, 40])
def test_fused_pull_back_step_f32(off, tma):
    p = make("steep", 64, 48)
    d = pyoracle.derive(p)
    s = perturbed_state(p, 8, amp=0.25)
    ctx = lib.Context(p)
    ctx.set_option(_abi.RS_OPT_TMA, tma)
    cur, nxt = upload(p, s, torch.float32), lib.FieldSet(p, torch.float32)
    ctx.step(cur, nxt, 0, i_offset_history=off, pull_back=off)
    sp = pyoracle.pull_back(p, s, off)
    o = pyoracle.step(p, d, sp, 0, off, 0.0)
    g = download(p, nxt)
    # increments over the shifted state, as for the unshifted FP32 step
    assert maxabs(g.psi - sp.psi, o.psi - sp.psi) <= 5e-6
    assert maxabs(g.c - sp.c, o.c - sp.c) <= 5e-8


def run_gpu(ctx, p, d, s, nsteps, dtype=torch.float64):
    a, b = upload(p, s, dtype), lib.FieldSet(p, dtype)
    l = 0.0
    for n in range(nsteps):
        ctx.step(a, b, n, l_offset_Vp=l)
        l += pyoracle.l_offset_increment(p, d, n)
        a, b = b, a
    torch.cuda.synchronize()
    return download(p, a)


@pytest.mark.parametrize("tma", [1, 0])
def test_many_steps_f64(tma):
    p = make("steep", 256, 200)
    d = pyoracle.derive(p)
    s = perturbed_state(p, 31, amp=0.3)
    ctx = lib.Context(p)
    ctx.set_option(_abi.RS_OPT_TMA, tma)
    g = run_gpu(ctx, p, d, s, 200)
    ctx.device_status()
    o = s
    l = 0.0
    for n in range(200):
        o = pyoracle.step(p, d, o, n, 0, l)
        l += pyoracle.l_offset_increment(p, d, n)
    assert maxabs(g.psi, o.psi) <= 1e-11 and maxabs(g.c, o.c) <= 1e-11


def test_plain_small_500_steps_parity():
    """256x256 Ti-10Nb, frozen T: pull_back at step 0 then 500 steps;
    max |dphi|, |dc| <= 1e-10 against the oracle (and the reference kernels)."""
    p = configs.plain_small()
    d = pyoracle.derive(p)
    s = pyoracle.initial_planar(p, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, configs.IC_SEED)
    ctx = lib.Context(p)
    a, b = lib.FieldSet(p, torch.float64), lib.FieldSet(p, torch.float64)
    ctx.initial_planar(a, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, configs.IC_SEED)
    itip = torch.zeros(1, dtype=torch.int32, device="cuda")
    ctx.itip(a, itip)
    off = int(itip.item()) - p.i_tip_target
    assert off == pyoracle.itip(p, s.psi) - p.i_tip_target
    l = 0.0
    for n in range(500):
        ctx.step(a, b, n, i_offset_history=off if n == 0 else off, l_offset_Vp=l,
                 pull_back=off if n == 0 else None)
        l += pyoracle.l_offset_increment(p, d, n)
        a, b = b, a
    g = download(p, a)
    o = pyoracle.run(p, d, pyoracle.pull_back(p, s, off), 500, i_offset_history=off)
    assert maxabs(g.psi, o.psi) <= 1e-10
    assert maxabs(g.c, o.c) <= 1e-10
    try:
        z = golden("c1_500.npz")
    except FileNotFoundError:
        return
    assert off == 0  # the fixture replays the reference loop with i_offset_history = 0
    for tag in ("fma", "nofma"):
        assert maxabs(g.psi[1:-1, 1:-1], z[f"{tag}_psi"][1:-1, 1:-1]) <= 1e-10
        assert maxabs(g.c[1:-1, 1:-1], z[f"{tag}_c"][1:-1, 1:-1]) <= 1e-10


@pytest.mark.parametrize("tma", [1, 0])
def test_single_step_f32_close_to_oracle(tma):
    p = make("steep", 64, 48)
    d = pyoracle.derive(p)
    s = perturbed_state(p, 8, amp=0.25)
    ctx = lib.Context(p)
    ctx.set_option(_abi.RS_OPT_TMA, tma)
    cur, nxt = upload(p, s, torch.float32), lib.FieldSet(p, torch.float32)
    ctx.step(cur, nxt, 0)
    o = pyoracle.step(p, d, s, 0)
    g = download(p, nxt)
    # inputs are rounded to FP32 first; compare increments
    assert maxabs(g.psi - s.psi, o.psi - s.psi) <= 5e-6
    assert maxabs(g.c - s.c, o.c - s.c) <= 5e-8


def solid_with_pocket(p, seed):
    """Planar front at i_tip_target with a wide solid behind it (psi exactly
    +1 in FP32 from about 16 cells behind the front) holding a liquid pocket
    of radius 5 at (i, j) = (190, 33), and seeded c noise in the solid: tile
    rows of the solid are deep solid except those next to the pocket."""
    s = pyoracle.initial_planar(p, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, seed)
    ny, nx = s.psi.shape
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    pocket = np.tanh((np.hypot(i - 190.0, j - 33.0) - 5.0) * p.dx / np.sqrt(2.0))
    psi = np.minimum(s.psi, pocket)
    c = s.c + 0.5 * (1.0 - pocket) * (configs.C_LIQUID_TI10NB - configs.C_SOLID_AT_TLIQ)
    c = c + 2e-3 * np.random.default_rng(seed).standard_normal(c.shape) * (psi > 0.9)
    s.psi[:] = psi
    s.phi[:] = psi
    s.c[:] = c
    fix_ghosts(p, s)
    return s


@pytest.mark.parametrize("tma", [1, 0])
def test_f32_step_with_deep_solid_close_to_oracle(tma):
    """Rows whose 3x3 neighbourhoods are all psi = +1 skip the per-cell mu''
    (every face weight there is 0); rows beside the pocket's interface must
    not.  One step against the FP64 oracle, increments compared as in the
    single-step test, and the deep solid left exactly unchanged."""
    p = configs.small(640, 70, i_tip_target=400, G=5e6, V=0.5)
    d = pyoracle.derive(p)
    s = solid_with_pocket(p, 5)
    ctx = lib.Context(p)
    ctx.set_option(_abi.RS_OPT_TMA, tma)
    cur, nxt = upload(p, s, torch.float32), lib.FieldSet(p, torch.float32)
    s32 = download(p, cur)  # the FP32-rounded input
    ctx.step(cur, nxt, 0)
    o = pyoracle.step(p, d, s32, 0)
    g = download(p, nxt)
    assert maxabs(g.psi - s32.psi, o.psi - s32.psi) <= 5e-6
    assert maxabs(g.c - s32.c, o.c - s32.c) <= 5e-8
    deep = np.ones_like(s32.psi, dtype=bool)
    for dj in (-1, 0, 1):
        for di in (-1, 0, 1):
            deep &= np.roll(np.roll(s32.psi == 1.0, dj, 0), di, 1)
    deep[[0, -1], :] = deep[:, [0, -1]] = False
    assert deep[1:-1, 130:380].mean() > 0.5
    assert np.array_equal(g.c[deep], s32.c[deep]) and np.array_equal(g.psi[deep], s32.psi[deep])


@pytest.mark.parametrize("tma", [1, 0])
def test_f64_step_with_deep_solid_matches_oracle(tma):
    """The FP64 tile kernel's deep-solid rows (S = mu'' = 0, every face
    weight there 0) and the interface rows around a liquid pocket: one step
    against the oracle within 1e-13, the deep solid left exactly unchanged."""
    p = configs.small(640, 70, i_tip_target=400, G=5e6, V=0.5)
    d = pyoracle.derive(p)
    s = solid_with_pocket(p, 5)
    ctx = lib.Context(p)
    ctx.set_option(_abi.RS_OPT_TMA, tma)
    cur, nxt = upload(p, s), lib.FieldSet(p, torch.float64)
    ctx.step(cur, nxt, 0)
    o = pyoracle.step(p, d, s, 0)
    g = download(p, nxt)
    assert maxabs(g.psi, o.psi) <= 1e-13 and maxabs(g.c, o.c) <= 1e-13
    deep = np.ones_like(s.psi, dtype=bool)
    for dj in (-1, 0, 1):
        for di in (-1, 0, 1):
            deep &= np.roll(np.roll(s.psi == 1.0, dj, 0), di, 1)
    deep[[0, -1], :] = deep[:, [0, -1]] = False
    assert np.array_equal(g.c[deep], s.c[deep]) and np.array_equal(g.psi[deep], s.psi[deep])


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("shape", [(64, 48), (300, 130), (1032, 1038)])
def test_pipeline_kernel_equals_tile_kernel(shape, dtype):
    """The persistent warp-role kernels (RS_OPT_PIPELINE) run the same
    per-cell arithmetic as the one-tile-per-CTA kernels: fields and the fused
    solute mass and coarse tip bit for bit, over 30 steps with noise, on grids
    whose tiles do not divide them (1032 x 1038: several tiles per CTA)."""
    dt = torch.float64 if dtype == "f64" else torch.float32
    p = configs.small(*shape, i_tip_target=22, G=5e6, V=0.5, noise_amplitude=0.05, seed=7)
    d = pyoracle.derive(p)
    s = perturbed_state(p, 3, amp=0.3)
    out = []
    for pipe in (0, 1):
        ctx = lib.Context(p)
        ctx.set_option(_abi.RS_OPT_PIPELINE, pipe)
        a, b = upload(p, s, dt, with_phi=True), lib.FieldSet(p, dt, with_phi=True)
        m = torch.zeros(30, dtype=torch.float64, device="cuda")
        it = torch.zeros(30, dtype=torch.int32, device="cuda")
        l = 0.0
        for n in range(30):
            ctx.step(a, b, n, l_offset_Vp=l, mass_out=m[n:n + 1], itip_out=it[n:n + 1])
            l += pyoracle.l_offset_increment(p, d, n)
            a, b = b, a
        torch.cuda.synchronize()
        ctx.device_status()
        g = download(p, a)
        out.append((g.psi, g.c, a.phi.cpu().numpy(), m.cpu().numpy(), it.cpu().numpy()))
        ctx.close()
    for x, y in zip(out[0], out[1]):
        assert np.array_equal(x, y)


def test_tma_and_register_paths_agree():
    """Both kernels run the same per-cell arithmetic; they differ only where
    the compiler contracts a multiply-add differently."""
    for dtype, tol_psi, tol_c in ((torch.float64, 1e-13, 1e-13), (torch.float32, 1e-5, 1e-7)):
        p = make("noise", 300, 130)
        d = pyoracle.derive(p)
        s = perturbed_state(p, 77, amp=0.3)
        out = []
        for tma in (1, 0):
            ctx = lib.Context(p)
            ctx.set_option(_abi.RS_OPT_TMA, tma)
            out.append(run_gpu(ctx, p, d, s, 30, dtype))
            ctx.device_status()
        assert maxabs(out[0].psi, out[1].psi) <= tol_psi and maxabs(out[0].c, out[1].c) <= tol_c


def test_f32_tracks_f64_over_steps():
    p = make("steep", 128, 64)
    d = pyoracle.derive(p)
    s = perturbed_state(p, 2, amp=0.2)
    ctx = lib.Context(p)
    g64 = run_gpu(ctx, p, d, s, 400)
    g32 = run_gpu(ctx, p, d, s, 400, torch.float32)
    assert maxabs(g32.psi, g64.psi) <= 2e-4
    assert maxabs(g32.c, g64.c) <= 2e-6
    m64, m32 = pyoracle.mass(p, g64.c), pyoracle.mass(p, g32.c)
    assert abs(m32 - m64) / m64 <= 1e-9


def test_mass_into_mapped_host_memory():
    """rs_host_alloc: a step given the device address of mapped page-locked
    host memory as mass_out / itip_out writes its reductions there; after the
    stream synchronises the host reads the same values the step writes into
    device memory, on both tile paths and on a pull-back step."""
    p = make("default")
    s = perturbed_state(p, 8, amp=0.3)
    ctx = lib.Context(p)
    hb = lib.HostBuffer(4)
    hi = lib.HostBuffer(4, np.int32)
    for dtype in (torch.float64, torch.float32):
        for pb in (None, 2):
            cur, nxt = upload(p, s, dtype), lib.FieldSet(p, dtype)
            ctx.step(cur, nxt, 0, pull_back=pb, mass_out=hb.device, itip_out=hi.device)
            m = torch.zeros(1, dtype=torch.float64, device="cuda")
            it = torch.zeros(1, dtype=torch.int32, device="cuda")
            ctx.step(cur, nxt, 0, pull_back=pb, mass_out=m, itip_out=it)
            torch.cuda.synchronize()
            assert hb.host[0] == m.item() and hi.host[0] == it.item(), (dtype, pb)
            assert hb.host[1] == 0.0
    hb.close()
    hi.close()


def test_fused_reductions_match_standalone():
    p = make("default")
    s = perturbed_state(p, 6, amp=0.3)
    ctx = lib.Context(p)
    for dtype in (torch.float64, torch.float32):
        cur, nxt = upload(p, s, dtype), lib.FieldSet(p, dtype)
        m = torch.zeros(2, dtype=torch.float64, device="cuda")
        it = torch.zeros(2, dtype=torch.int32, device="cuda")
        ctx.step(cur, nxt, 0, mass_out=m[0:1], itip_out=it[0:1])
        ctx.mass(nxt, m[1:2])
        ctx.itip(nxt, it[1:2])
        g = download(p, nxt)
        mm = m.cpu().numpy()
        assert abs(mm[0] - mm[1]) <= 1e-12 * abs(mm[1])
        assert abs(mm[1] - pyoracle.mass(p, g.c)) <= 1e-12 * abs(mm[1])
        assert it[0].item() == it[1].item() == pyoracle.itip(p, g.psi)
