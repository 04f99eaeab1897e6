"""A tile kernel whose bounded wait for its TMA load gives up skips its tile
(no phase runs on a partly filled tile, nothing is stored), reports the
failure through rs_device_status, and leaves the context usable.  The give-up
path is reached by the RS_OPT_WAIT_LIMIT test option (one try), not by a
fault."""
import numpy as np
import pytest

import pyoracle
from helpers import maxabs, perturbed_state
from rapidsolid import _abi, configs, lib
from test_gpu_step import download, upload

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SENTINEL = 7.0


@pytest.mark.parametrize("dtype", ["f32", "f64", "f32_pipeline", "f64_pipeline"])
def test_wait_that_gives_up_skips_the_tile(dtype):
    dt = torch.float32 if dtype.startswith("f32") else torch.float64
    p = configs.small(256, 130, i_tip_target=40, G=5e6, V=0.5)
    d = pyoracle.derive(p)
    s = perturbed_state(p, 5, amp=0.2)
    ctx = lib.Context(p)
    ctx.set_option(_abi.RS_OPT_PIPELINE, 1 if dtype.endswith("pipeline") else 0)
    cur = upload(p, s, dt)
    nxt = lib.FieldSet(p, dt)
    nxt.psi.fill_(SENTINEL)
    nxt.c.fill_(SENTINEL)
    mass = torch.zeros(1, dtype=torch.float64, device="cuda")
    ctx.set_option(_abi.RS_OPT_WAIT_LIMIT, 1)
    ctx.step(cur, nxt, 0, mass_out=mass)
    with pytest.raises(lib.RsError) as e:
        ctx.device_status()
    assert e.value.code == _abi.RS_E_STATE
    # a skipped tile stores nothing: its cells keep the sentinel
    assert bool((nxt.psi[1:-1, 1:-1] == SENTINEL).any())
    # the context stays usable: with the default limit the step equals the oracle's
    ctx.set_option(_abi.RS_OPT_WAIT_LIMIT, 0)
    ctx.step(cur, nxt, 0, mass_out=mass)
    torch.cuda.synchronize()
    ctx.device_status()
    ref = pyoracle.step(p, d, s, 0)
    g = download(p, nxt)
    tol_psi, tol_c = (5e-6, 5e-8) if dt == torch.float32 else (1e-13, 1e-13)
    assert maxabs(g.psi, ref.psi) <= tol_psi and maxabs(g.c, ref.c) <= tol_c
    m_ref = pyoracle.mass(p, ref.c)
    assert abs(mass.item() - m_ref) <= (1e-8 if dt == torch.float32 else 1e-13) * m_ref
    ctx.close()
