"""Row bands on the GPU (rs_step in band mode): two and three bands of one
domain, held on one device and swapping edge rows by rapidsolid.bands.
exchange_local, equal the single-domain rs_step bit for bit, FP32 and FP64,
with interface noise and a pull-back from the global coarse tip; and one band
exchanging with itself is the periodic domain."""
import pytest
import torch

from rapidsolid import bands, configs, lib

pytestmark = pytest.mark.gpu


def _params(nx=256, ny=200):
    p = configs.small(nx, ny, i_tip_target=20)
    p.noise_amplitude = 0.02
    p.seed = 123
    return p


def _single(p, dtype, nsteps):
    ctx = lib.Context(p)
    a, b = lib.FieldSet(p, dtype), lib.FieldSet(p, dtype)
    ctx.initial_planar(a, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, 3)
    itip = torch.zeros(1, dtype=torch.int32, device="cuda")
    ctx.itip(a, itip)
    off = int(itip.item()) - p.i_tip_target
    for n in range(nsteps):
        ctx.step(a, b, n, i_offset_history=off, pull_back=off if n == 0 else None)
        a, b = b, a
    torch.cuda.synchronize()
    ctx.device_status()
    return a.psi[1:-1].clone(), a.c[1:-1].clone(), off


def _banded(p, dtype, nsteps, world):
    ctxs, cur, nxt = [], [], []
    for r in range(world):
        q = bands.band_params(p, r, world)
        ctxs.append(lib.Context(q))
        cur.append(lib.FieldSet(q, dtype))
        nxt.append(lib.FieldSet(q, dtype))
        ctxs[r].initial_planar(cur[r], configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, 3)
    bands.exchange_local([[f.psi, f.c] for f in cur])
    itip = torch.zeros(world, dtype=torch.int32, device="cuda")
    for r in range(world):
        ctxs[r].itip(cur[r], itip[r:r + 1])
    off = int(itip.max().item()) - p.i_tip_target  # the max over the bands
    for n in range(nsteps):
        for r in range(world):
            ctxs[r].step(cur[r], nxt[r], n, i_offset_history=off, pull_back=off if n == 0 else None)
        cur, nxt = nxt, cur
        bands.exchange_local([[f.psi, f.c] for f in cur])
    torch.cuda.synchronize()
    for c in ctxs:
        c.device_status()
    psi = torch.cat([f.psi[1:-1] for f in cur])
    c = torch.cat([f.c[1:-1] for f in cur])
    return psi, c, off


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("world", [1, 2, 3])
def test_bands_equal_the_single_domain(dtype, world):
    p = _params()
    psi0, c0, off0 = _single(p, dtype, 40)
    psi1, c1, off1 = _banded(p, dtype, 40, world)
    assert off0 == off1
    assert torch.equal(psi0, psi1) and torch.equal(c0, c1)


def test_band_mode_rejects_what_needs_the_whole_domain():
    p = _params()
    q = bands.band_params(p, 0, 2)
    ctx = lib.Context(q)
    f = lib.FieldSet(q, torch.float64)
    tip = torch.zeros(64, dtype=torch.uint8, device="cuda")
    with pytest.raises(lib.RsError):
        ctx.precise_tip(f, tip)
    q.tfc = 1
    with pytest.raises(lib.RsError):
        lib.Context(q)
