"""Moving frame, reductions, tip tracker, initial conditions and the coarse
temperature on the GPU against the oracle."""
import ctypes as C

import numpy as np
import pytest

import pyoracle
from helpers import TFC_CASES, golden, maxabs, perturbed_state, tfc_input, tfc_T_mask
from helpers import tfc_params as ref_tfc_params
from rapidsolid import _abi, configs, lib
from test_gpu_step import download, upload

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("off", [-5, 0, 2, 40])
def test_pull_back_standalone(dtype, off):
    dt = torch.float64 if dtype == "f64" else torch.float32
    p = configs.small(64, 40, i_tip_target=20)
    s = perturbed_state(p, 11, amp=0.2)
    if dt == torch.float32:  # compare on FP32-representable inputs
        s.psi[:] = s.psi.astype(np.float32)
        s.c[:] = (s.c - p.cinf).astype(np.float32).astype(np.float64) + p.cinf
    ctx = lib.Context(p)
    cur, nxt = upload(p, s, dt), lib.FieldSet(p, dt)
    ctx.pull_back(cur, nxt, off)
    g = download(p, nxt)
    o = pyoracle.pull_back(p, s, off)
    assert maxabs(g.psi, o.psi) == 0.0
    assert maxabs(g.c, o.c) <= (0.0 if dt == torch.float64 else 1e-15)


def test_itip_and_mass():
    p = configs.small(96, 72, i_tip_target=30)
    s = perturbed_state(p, 13, amp=0.4)
    ctx = lib.Context(p)
    fs = upload(p, s)
    out_i = torch.zeros(1, dtype=torch.int32, device="cuda")
    out_m = torch.zeros(1, dtype=torch.float64, device="cuda")
    ctx.itip(fs, out_i)
    ctx.mass(fs, out_m)
    assert out_i.item() == pyoracle.itip(p, s.psi)
    assert abs(out_m.item() - pyoracle.mass(p, s.c)) <= 1e-13 * pyoracle.mass(p, s.c)
    # all-liquid field: get_itip_all_grain returns 1
    fs.psi.fill_(-1.0)
    ctx.itip(fs, out_i)
    assert out_i.item() == 1


@pytest.mark.parametrize("idx", range(5))
def test_precise_tip_matches_reference_fixture(idx):
    z = golden("tip_ref.npz")
    name = str(z["names"][idx])
    ref = z["tips"][idx]
    p = configs.small(64, 64, i_tip_target=24)
    psi = z["psi_" + name]
    ctx = lib.Context(p)
    fs = lib.FieldSet(p, torch.float64)
    fs.psi.copy_(torch.from_numpy(psi))
    out = torch.zeros(C.sizeof(_abi.Tip), dtype=torch.uint8, device="cuda")
    ctx.precise_tip(fs, out)
    t = lib.tip_from_bytes(out.cpu().numpy().tobytes())
    assert (t.i, t.j) == (int(ref[1]), int(ref[2]))
    assert t.status == 0
    assert abs(t.x - ref[3]) <= 1e-12 * max(1, abs(ref[3]))
    assert abs(t.y - ref[4]) <= 1e-12 * max(1, abs(ref[4]))
    assert abs(t.R - ref[5]) <= 1e-9 * max(1, abs(ref[5]))


def test_precise_tip_on_evolved_fields_f32():
    p = configs.small(128, 96, i_tip_target=40, G=5e6, V=0.5)
    d = pyoracle.derive(p)
    s = perturbed_state(p, 21, amp=0.6)
    s = pyoracle.run(p, d, s, 50)
    psi32 = s.psi.astype(np.float32)
    ctx = lib.Context(p)
    fs = lib.FieldSet(p, torch.float32)
    fs.psi.copy_(torch.from_numpy(psi32))
    out = torch.zeros(C.sizeof(_abi.Tip), dtype=torch.uint8, device="cuda")
    ctx.precise_tip(fs, out)
    t = lib.tip_from_bytes(out.cpu().numpy().tobytes())
    o = pyoracle.precise_tip(p, d, psi32.astype(np.float64))
    assert (t.i, t.j, t.status) == (o.i, o.j, o.status)
    assert abs(t.x - o.x) <= 1e-11 and abs(t.y - o.y) <= 1e-11


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_initial_conditions(dtype):
    dt = torch.float64 if dtype == "f64" else torch.float32
    tol = 1e-14 if dt == torch.float64 else 1e-7
    p = configs.small(64, 48, i_tip_target=20)
    ctx = lib.Context(p)
    fs = lib.FieldSet(p, dt)
    ctx.initial(fs)
    g = download(p, fs)
    o = pyoracle.initial_reference(p)
    assert maxabs(g.psi, o.psi) <= tol and maxabs(g.c, o.c) <= tol
    ctx.initial_planar(fs, 0.9, 0.88, 99)
    g = download(p, fs)
    o = pyoracle.initial_planar(p, 0.9, 0.88, 99)
    assert maxabs(g.psi, o.psi) <= tol and maxabs(g.c, o.c) <= tol


def tfc_params(G=1e7):
    p = configs.small(64, 42, i_tip_target=20, tfc=1, G=G, V=0.5)
    p.length_sample_um = 1.0
    # coarse domain starts 30 cells left of the window (i_left_end ~ 30)
    p.Tcold = p.T_ref - p.GG * p.dx * p.S * p.W0 * (p.i_tip_target + 30)
    return p


def test_temperature_kernels():
    p = tfc_params()
    d = pyoracle.derive(p)
    ctx = lib.Context(p)
    nT = d.NxT_all * d.NyT_all
    T = torch.zeros(nT, dtype=torch.float64, device="cuda")
    ctx.temperature_init(T)
    To = np.zeros(nT)
    pyoracle.lib().ro_initial_temperature(C.byref(p), C.byref(d), pyoracle._p(To))
    assert maxabs(T.cpu().numpy(), To) == 0.0
    # source from a psi change, then one temperature step
    s = perturbed_state(p, 3, amp=0.3)
    s2 = pyoracle.step(p, d, s, 0, T_fine=np.full(s.c.shape, configs.T_LIQUIDUS_TI10NB))
    cur, nxt = upload(p, s), upload(p, s2)
    ile = 3
    dphidt = torch.zeros(nT, dtype=torch.float64, device="cuda")
    ctx.integrate_phi(cur, nxt, dphidt, ile)
    Do = np.zeros(nT)
    pyoracle.lib().ro_integrate_phi(C.byref(p), C.byref(d), pyoracle._p(Do), pyoracle._p(s.psi),
                                    pyoracle._p(s2.psi), ile)
    assert maxabs(dphidt.cpu().numpy(), Do) == 0.0
    Tn = torch.empty_like(T)
    ctx.temperature_step(T, Tn, dphidt, 7)
    a, b = To.copy(), To.copy()
    for _ in range(d.ratio_dt_dtT):
        pyoracle.lib().ro_compute_temperature(C.byref(p), C.byref(d), pyoracle._p(a), pyoracle._p(b),
                                              pyoracle._p(Do), 7)
        a, b = b, a
    g = T.cpu().numpy().reshape(d.NyT_all, d.NxT_all)
    o = a.reshape(d.NyT_all, d.NxT_all)
    assert maxabs(g[:d.NyT, :d.NxT], o[:d.NyT, :d.NxT]) <= 1e-12
    Tf = torch.zeros((p.ny_all, p.nx_all), dtype=torch.float64, device="cuda")
    ctx.interpolate_temperature(T, Tf, ile)
    Tfo = np.zeros((p.ny_all, p.nx_all))
    pyoracle.lib().ro_interpolate_temperature(C.byref(p), C.byref(d), pyoracle._p(np.ascontiguousarray(o.ravel())),
                                              pyoracle._p(Tfo), ile)
    assert maxabs(Tf.cpu().numpy(), Tfo) <= 1e-11


@pytest.mark.parametrize("G", [1e7, 5e8])
def test_tfc_step_f64(G):
    """The fused step evaluates the fine T by bilinear interpolation of the
    coarse T on the fly; same result as interpolate_temperature + step.  At
    G = 1e7 K/m every cell is within 4 K of its tile's reference temperature
    (K + C0 by its Taylor polynomial); at 5e8 K/m (0.5 K per cell) most cells
    are not, and take the cell form."""
    p = tfc_params(G)
    d = pyoracle.derive(p)
    ctx = lib.Context(p)
    nT = d.NxT_all * d.NyT_all
    T = torch.zeros(nT, dtype=torch.float64, device="cuda")
    ctx.temperature_init(T)
    ile = d.i_left_end_initial
    Tf = np.zeros((p.ny_all, p.nx_all))
    pyoracle.lib().ro_interpolate_temperature(C.byref(p), C.byref(d), pyoracle._p(T.cpu().numpy()),
                                              pyoracle._p(Tf), ile)
    s = perturbed_state(p, 19, amp=0.3)
    cur, nxt = upload(p, s), lib.FieldSet(p, torch.float64)
    ctx.step(cur, nxt, 0, T_coarse=T, i_left_end=ile, i_left_end_T=ile)
    o = pyoracle.step(p, d, s, 0, T_fine=Tf)
    g = download(p, nxt)
    assert maxabs(g.psi, o.psi) <= 1e-13 and maxabs(g.c, o.c) <= 1e-13


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_tfc_back_to_back_tile_steps(dtype):
    """Coarse-grid-temperature steps on the TMA tile kernels, launched back to
    back with no other kernel between them (no reduction, fixed T), against
    the same steps on the register-window kernel (RS_OPT_TMA = 0): each step
    must read the previous step's finished fields.  The two kernels group the
    arithmetic differently, so they agree to rounding, not bit for bit (FP32:
    to its rounding over 40 steps)."""
    dt = getattr(torch, dtype)
    tol_psi, tol_c = (1e-11, 1e-11) if dt == torch.float64 else (2e-4, 2e-5)
    p = configs.small(256, 250, i_tip_target=40, tfc=1, G=1e7, V=0.5)
    p.length_sample_um = 2.0
    p.Tcold = p.T_ref - p.GG * p.dx * p.S * p.W0 * (p.i_tip_target + 30)
    d = pyoracle.derive(p)
    s = perturbed_state(p, 31, amp=0.3)
    out = []
    for tma in (1, 0):
        ctx = lib.Context(p)
        ctx.set_option(_abi.RS_OPT_TMA, tma)
        T = torch.zeros(d.NxT_all * d.NyT_all, dtype=torch.float64, device="cuda")
        ctx.temperature_init(T)
        ile = d.i_left_end_initial
        a, b = upload(p, s, dt), lib.FieldSet(p, dt)
        for n in range(40):
            ctx.step(a, b, n, T_coarse=T, i_left_end=ile, i_left_end_T=ile)
            a, b = b, a
        torch.cuda.synchronize()
        ctx.device_status()
        out.append(download(p, a))
        ctx.close()
    assert maxabs(out[0].psi, out[1].psi) <= tol_psi and maxabs(out[0].c, out[1].c) <= tol_c


def test_tfc_loop_with_pull_back_f64():
    """The coarse-temperature loop of fun.cu:431-514 over 120 steps, pull-back
    every 30 steps with non-zero shifts, on the GPU (pull-back fused into
    rs_step, rs_integrate_phi reading cur through the same shift) against the
    oracle doing the reference's order: pull_back, step, integrate_phi on the
    shifted field, ratio_dt_dtT temperature sub-steps, interpolate_temperature."""
    p = tfc_params()
    p.step_pull_back = 30
    d = pyoracle.derive(p)
    nsteps, nT = 120, d.NxT_all * d.NyT_all
    # the front starts 5 cells ahead of i_tip_target, so the frame shifts
    p0 = tfc_params()
    p0.i_tip_target += 5
    s0 = perturbed_state(p0, 23, amp=0.2)
    L = pyoracle.lib()
    pr = lambda a: pyoracle._p(np.ascontiguousarray(a))
    # oracle
    s = s0.copy()
    T = np.zeros(nT)
    L.ro_initial_temperature(C.byref(p), C.byref(d), pr(T))
    ile = d.i_left_end_initial
    Tf = np.zeros((p.ny_all, p.nx_all))
    L.ro_interpolate_temperature(C.byref(p), C.byref(d), pr(T), pr(Tf), ile)
    hist, l, shifts = 0, 0.0, []
    for n in range(nsteps):
        if n % d.step_pull_back == 0:
            off = pyoracle.itip(p, s.psi) - p.i_tip_target
            shifts.append(off)
            hist += off
            ile = d.i_left_end_initial + hist - int(l / p.dx)
            s = pyoracle.pull_back(p, s, off)
        s2 = pyoracle.step(p, d, s, n, i_offset_history=hist, l_offset_Vp=l, T_fine=Tf)
        D = np.zeros(nT)
        L.ro_integrate_phi(C.byref(p), C.byref(d), pr(D), pr(s.psi), pr(s2.psi), ile)
        a, b = T.copy(), T.copy()
        for _ in range(d.ratio_dt_dtT):
            L.ro_compute_temperature(C.byref(p), C.byref(d), pr(a), pr(b), pr(D), n)
            a, b = b, a
        T = a
        L.ro_interpolate_temperature(C.byref(p), C.byref(d), pr(T), pr(Tf), ile)
        s = s2
        l += pyoracle.l_offset_increment(p, d, n)
    assert any(shifts), shifts
    # GPU
    ctx = lib.Context(p)
    ga, gb = upload(p, s0), lib.FieldSet(p, torch.float64)
    Tg = torch.zeros(nT, dtype=torch.float64, device="cuda")
    Tn, dphidt = torch.zeros_like(Tg), torch.zeros_like(Tg)
    ctx.temperature_init(Tg)
    itip = torch.zeros(1, dtype=torch.int32, device="cuda")
    hist, l = 0, 0.0
    ile = ile_T = d.i_left_end_initial
    for n in range(nsteps):
        pb = None
        if n % d.step_pull_back == 0:
            ctx.itip(ga, itip)
            pb = int(itip.item()) - p.i_tip_target
            hist += pb
            ile = d.i_left_end_initial + hist - int(l / p.dx)
        ctx.step(ga, gb, n, i_offset_history=hist, l_offset_Vp=l, pull_back=pb, T_coarse=Tg, i_left_end=ile,
                 i_left_end_T=ile_T)
        ctx.integrate_phi(ga, gb, dphidt, ile)
        ctx.temperature_step(Tg, Tn, dphidt, n)
        ile_T = ile
        l += pyoracle.l_offset_increment(p, d, n)
        ga, gb = gb, ga
    g = download(p, ga)
    assert maxabs(g.psi, s.psi) <= 1e-10 and maxabs(g.c, s.c) <= 1e-10
    Tgh = Tg.cpu().numpy().reshape(d.NyT_all, d.NxT_all)
    To = T.reshape(d.NyT_all, d.NxT_all)
    assert maxabs(Tgh[:d.NyT, :d.NxT], To[:d.NyT, :d.NxT]) <= 1e-9


def _gpu_tfc_loop(p, d, s0, dtype, nsteps):
    """The coarse-temperature loop through the C-ABI (as in the test above)."""
    nT = d.NxT_all * d.NyT_all
    ctx = lib.Context(p)
    ga, gb = upload(p, s0, dtype), lib.FieldSet(p, dtype)
    Tg = torch.zeros(nT, dtype=torch.float64, device="cuda")
    Tn, dphidt = torch.zeros_like(Tg), torch.zeros_like(Tg)
    ctx.temperature_init(Tg)
    itip = torch.zeros(1, dtype=torch.int32, device="cuda")
    mass = torch.zeros(1, dtype=torch.float64, device="cuda")
    hist, l = 0, 0.0
    ile = ile_T = d.i_left_end_initial
    for n in range(nsteps):
        pb = None
        if n % d.step_pull_back == 0:
            ctx.itip(ga, itip)
            pb = int(itip.item()) - p.i_tip_target
            hist += pb
            ile = d.i_left_end_initial + hist - int(l / p.dx)
        ctx.step(ga, gb, n, i_offset_history=hist, l_offset_Vp=l, pull_back=pb, T_coarse=Tg, i_left_end=ile,
                 i_left_end_T=ile_T)
        ctx.integrate_phi(ga, gb, dphidt, ile)
        ctx.temperature_step(Tg, Tn, dphidt, n)
        ile_T = ile
        l += pyoracle.l_offset_increment(p, d, n)
        ga, gb = gb, ga
    ctx.mass(ga, mass)
    torch.cuda.synchronize()
    ctx.device_status()
    return download(p, ga), Tg.cpu().numpy(), mass.item()


def test_tfc_loop_fp32_against_fp64():
    """The coarse-temperature loop in FP32 (register-window kernel, CALPHAD
    groups of each cell's bilinear T in FP64, their differences in FP64)
    against the same loop in FP64: 300 steps with pull-backs; psi within 2e-4,
    c within 2e-6, solute mass within 1e-8 (measured 2.2e-9), and the coarse
    T (about 2100 K, driven by the latent heat of the FP32 dphi/dt) within
    1e-4 K (measured 1.2e-5 K)."""
    p = tfc_params()
    p.step_pull_back = 60
    d = pyoracle.derive(p)
    p0 = tfc_params()
    p0.i_tip_target += 5
    s0 = perturbed_state(p0, 23, amp=0.2)
    s64, T64, m64 = _gpu_tfc_loop(p, d, s0, torch.float64, 300)
    s32, T32, m32 = _gpu_tfc_loop(p, d, s0, torch.float32, 300)
    assert maxabs(s32.psi, s64.psi) <= 2e-4 and maxabs(s32.c, s64.c) <= 2e-6
    assert abs(m32 - m64) <= 1e-8 * abs(m64), (m32, m64)
    assert maxabs(T32, T64) <= 1e-4


@pytest.mark.parametrize("name", sorted(TFC_CASES))
def test_tfc_loop_matches_reference_kernels(name):
    """The FP64 coarse-temperature loop through the C-ABI against the
    reference's own TFC kernels (fixture of its main() loop body with
    ifTFC 1, pull-backs inside the run), with the tolerances of the oracle's
    pin (test_oracle_tfc.py: the reference's own FMA and no-FMA builds differ
    by 1.0e-9 in psi and 2.9e-9 K in T after the run): interior psi within
    5e-9, c within 1e-10, the coarse T within 1e-8 K."""
    z = golden(name + ".npz")
    nx, ny, nsteps, spb = TFC_CASES[name]
    p = ref_tfc_params(nx, ny, spb)
    d = pyoracle.derive(p)
    g, T, _ = _gpu_tfc_loop(p, d, tfc_input(p), torch.float64, nsteps)
    T = T.reshape(d.NyT_all, d.NxT_all)
    for tag in ("fma", "nofma"):
        assert maxabs(g.psi[1:-1, 1:-1], z[f"{tag}_psi"][1:-1, 1:-1]) <= 5e-9
        assert maxabs(g.c[1:-1, 1:-1], z[f"{tag}_c"][1:-1, 1:-1]) <= 1e-10
        cols = list(z[f"{tag}_T_cols"])
        m = tfc_T_mask(d, cols)
        assert maxabs(T[:d.NyT, cols][m], z[f"{tag}_T"][:d.NyT][m]) <= 1e-8
