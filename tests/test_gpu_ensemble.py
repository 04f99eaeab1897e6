"""Batched ensemble (rs_ensemble_*): runs of uneven size stepped by one
launch, pull-back-free stretches replayed from a CUDA graph or taken by one
persistent launch (device-side grid barriers between tables and tiles and
between steps), must equal the same runs stepped one by one through rs_step,
bit for bit."""
import numpy as np
import pytest

from rapidsolid import configs, lib, surrogate

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

# (nx_all, ny_all, V m/s, G K/m): different pull-back cadences and sizes
RUNS = [(256, 200, 2.0, 5e6), (384, 136, 1.5, 2e6), (200, 300, 0.9, 8e6), (132, 132, 0.5, 1e6), (516, 72, 0.3, 3e6)]
STEPS = 600


def params():
    out = []
    for k, (nx, ny, V, G) in enumerate(RUNS):
        p = configs._ti10nb(configs.default_params(), nx, ny, G, V, T0=configs.T_SOLIDUS_TI10NB)
        p.noise_amplitude, p.seed = 0.01, 100 + k
        out.append(p)
    return out


def single(p, sur=None):
    ctx = lib.Context(p)
    if sur is not None:
        ctx.set_surrogate(*sur)
    d = ctx.d
    a, b = lib.FieldSet(p, torch.float32), lib.FieldSet(p, torch.float32)
    ctx.initial_planar(a, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, 7)
    itip = torch.zeros(1, dtype=torch.int32, device="cuda")
    hist, l = 0, 0.0
    for n in range(STEPS):
        pb = None
        if n % d.step_pull_back == 0:
            ctx.itip(a, itip)
            pb = int(itip.item()) - p.i_tip_target
            hist += pb
        ctx.step(a, b, n, i_offset_history=hist, l_offset_Vp=l, pull_back=pb)
        l += p.Vp * d.dt * d.tau0 / (p.S * p.W0)
        a, b = b, a
    torch.cuda.synchronize()
    return a.psi.cpu().numpy(), a.c.cpu().numpy(), hist, l


# paths: tile shape path // 6 (16, 8 or 32 rows by 128 columns), per-step
# launches (path % 6 < 3) or the persistent walk, tile order path % 3
@pytest.mark.parametrize("path", ["autotuned", 0, 4, 6, 11, 13, 15])
def test_ensemble_equals_single_runs(path):
    ps = params()
    ens = lib.Ensemble(ps)
    for r, p in enumerate(ps):
        a, b = lib.FieldSet(p, torch.float32), lib.FieldSet(p, torch.float32)
        ens.ctx[r].initial_planar(a, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, 7)
        ens.bind(r, a, b)
    choice, ms = ens.autotune(reps=3)
    assert choice in range(lib.ENS_PATHS) and len(ms) == lib.ENS_PATHS and all(m > 0 for m in ms)
    if path != "autotuned":
        ens.set_path(path)
    ens.steps(250)
    ens.steps(STEPS - 250)
    torch.cuda.synchronize()
    assert any(ps[r].Vp >= 1.0 for r in range(len(ps)))  # some run pulls back inside the stretch
    for r, p in enumerate(ps):
        step, hist, l, cur = ens.state(r)
        assert step == STEPS
        psi, c, hist1, l1 = single(p)
        assert hist == hist1 and l == l1
        assert np.array_equal(cur.psi.cpu().numpy(), psi), r
        assert np.array_equal(cur.c.cpu().numpy(), c), r
    ens.ctx[0].device_status()
    ens.close()


@pytest.mark.parametrize("path", [1, 5, 8, 16])
def test_ensemble_surrogate_path_equals_single_runs(path):
    """With a network set on every run's context, the batched launch takes
    the surrogate path of the tile kernel: each run equals the same run
    stepped alone through rs_step with the same network, bit for bit."""
    ps = params()
    w, box, _ = surrogate.train(ps[0], n_samples=1 << 15, epochs=3, batch=2048, seed=3)
    ens = lib.Ensemble(ps)
    for r, p in enumerate(ps):
        a, b = lib.FieldSet(p, torch.float32), lib.FieldSet(p, torch.float32)
        ens.ctx[r].initial_planar(a, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, 7)
        ens.ctx[r].set_surrogate(w, box)
        ens.bind(r, a, b)
    ens.set_path(path)
    ens.steps(STEPS)
    torch.cuda.synchronize()
    for r, p in enumerate(ps):
        step, hist, l, cur = ens.state(r)
        psi, c, hist1, l1 = single(p, (w, box))
        assert hist == hist1 and l == l1
        assert np.array_equal(cur.psi.cpu().numpy(), psi), r
        assert np.array_equal(cur.c.cpu().numpy(), c), r
        assert ens.ctx[r].surrogate_audit()[3] > 0  # the run's cells went through its network
    ens.close()


def test_walk_barrier_that_gives_up_reports_and_ends():
    """The persistent walk's grid barriers are bounded: with run 0's wait
    limit at one poll, early arrivals give up at once (the others have not
    arrived yet), the CTAs that gave up stop working but keep arriving, the
    launch ends, rs_device_status reports RS_E_STATE, and the context stays
    usable (a walk with the default limit then runs clean).  No fault and no
    hang: every wait is a bounded poll."""
    from rapidsolid import _abi
    ps = params()[:3]
    ens = lib.Ensemble(ps)
    for r, p in enumerate(ps):
        a, b = lib.FieldSet(p, torch.float32), lib.FieldSet(p, torch.float32)
        ens.ctx[r].initial_planar(a, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, 7)
        ens.bind(r, a, b)
    ens.set_path(3)
    ens.steps(2)  # step 0 pulls every run back (eager), step 1 is a walk
    torch.cuda.synchronize()
    ens.ctx[0].device_status()
    ens.ctx[0].set_option(_abi.RS_OPT_WAIT_LIMIT, 1)
    ens.steps(5)
    torch.cuda.synchronize()
    with pytest.raises(lib.RsError) as e:
        ens.ctx[0].device_status()
    assert e.value.code == _abi.RS_E_STATE
    ens.ctx[0].set_option(_abi.RS_OPT_WAIT_LIMIT, 0)
    ens.steps(5)
    torch.cuda.synchronize()
    ens.ctx[0].device_status()
    ens.close()
