"""The C++ host driver (lib/rs_run): the reference's main() loop on the C-ABI.

The driver's run (FP64, and FP32 with --precision f32) must equal, bit for
bit, the same loop written in
Python over the same entry points (pull-back cadence, frozen temperature with
the Vp ramp, fun.cu:431-514), and a restart that loads its own check point and
runs no step must write the same files back (save/load_check_point,
save/load_parameters)."""
import math
import os
import subprocess

import numpy as np
import pytest

from rapidsolid import _abi, lib

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DRIVER = os.path.join(os.path.dirname(lib.LIB_PATH), "rs_run")
NX, NY, ITIP, STEPS = 256, 128, 64, 300


def run_driver(out, *extra):
    if not os.path.exists(DRIVER):
        pytest.fail(f"{DRIVER} is missing: build it with make")
    r = subprocess.run([DRIVER, "--nx", str(NX), "--ny", str(NY), "--i-tip", str(ITIP), "--out", str(out),
                        "--no-fields", *extra], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def python_loop(steps, tfc, dtype=torch.float64):
    """The loop body of fun.cu:431-514 over the Python binding (no files)."""
    p = lib.default_params()
    p.nx_all, p.ny_all, p.i_tip_target, p.tfc = NX, NY, ITIP, tfc
    ctx = lib.Context(p)
    d = ctx.d
    a, b = lib.FieldSet(p, dtype), lib.FieldSet(p, dtype)
    ctx.initial(a)
    itip = torch.zeros(1, dtype=torch.int32, device="cuda")
    T = Tn = dphidt = None
    if tfc:
        T = torch.zeros(d.NxT_all * d.NyT_all, dtype=torch.float64, device="cuda")
        Tn, dphidt = torch.zeros_like(T), torch.zeros_like(T)
        ctx.temperature_init(T)
    hist, l = p.i_offset_history_initial, p.l_offset_Vp_initial
    ile = ile_T = d.i_left_end_initial
    for n in range(steps):
        pb = None
        if n % d.step_pull_back == 0:  # set_pull_back, fun.cu:693-742
            ctx.itip(a, itip)
            pb = int(itip.item()) - p.i_tip_target
            hist += pb
            if tfc:
                ile = d.i_left_end_initial + hist - int(l / p.dx)
        ctx.step(a, b, n, i_offset_history=hist, l_offset_Vp=l, pull_back=pb, T_coarse=T, i_left_end=ile,
                 i_left_end_T=ile_T)
        if tfc:  # fun.cu:486-497
            ctx.integrate_phi(a, b, dphidt, ile)
            ctx.temperature_step(T, Tn, dphidt, n)
            ile_T = ile
        t_ns = n * d.tau0 * d.dt
        vp = p.Vp + 0.0107587 * (t_ns * 0.001) if p.vp_ramp else p.Vp  # Vp_ramp, fun.cu:1974-1981
        l += vp * d.dt * d.tau0 / (p.S * p.W0)
        a, b = b, a
    torch.cuda.synchronize()
    c = a.c.double().cpu().numpy().reshape(NY, NX)
    if dtype == torch.float32:  # FP32 sets hold c - cinf
        c = p.cinf + c
    phi = np.clip(a.psi.double().cpu().numpy().reshape(NY, NX), -1.0, 1.0)
    Th = None if T is None else T.cpu().numpy()
    return c, phi, hist, l, Th, d


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("tfc", [1, 0])
def test_driver_equals_python_loop(tmp_path, tfc, precision):
    out = run_driver(tmp_path, "--steps", str(STEPS), "--tfc", str(tfc), "--tip-every", "100",
                     "--check-every", "1000000", "--precision", precision)
    c = np.fromfile(tmp_path / "data" / "check_point_c.bin", dtype=np.float64).reshape(NY, NX)
    phi = np.fromfile(tmp_path / "data" / "check_point_phi.bin", dtype=np.float64).reshape(NY, NX)
    c_ref, phi_ref, hist, l, T, d = python_loop(STEPS, tfc, torch.float32 if precision == "f32" else torch.float64)
    assert np.array_equal(c, c_ref)
    assert np.array_equal(phi, phi_ref)
    s = lib.read_parameters(tmp_path / "parameters.txt", tfc=tfc)
    assert s.step == STEPS and s.i_offset_history == hist
    assert math.isclose(s.l_offset_Vp, l, rel_tol=1e-5)  # the file holds %g
    if tfc:  # coarse temperature check point: the NyT x NxT block
        Tf = np.fromfile(tmp_path / "data" / "check_point_temperature.bin", dtype=np.float64)
        assert np.array_equal(Tf, T.reshape(d.NyT_all, d.NxT_all)[:d.NyT, :d.NxT].ravel())
    # tip rows at steps 0, 100, 200 on stdout and in tip.txt
    rows = [r for r in out.splitlines() if r and r.split()[0].isdigit()]
    assert [int(r.split()[0]) for r in rows] == [0, 100, 200]
    assert (tmp_path / "tip.txt").read_text().count("\n") == 2 + 3


def test_restart_round_trip(tmp_path):
    run_driver(tmp_path, "--steps", "120", "--tip-every", "50", "--check-every", "1000000")
    names = ["data/check_point_c.bin", "data/check_point_phi.bin", "parameters.txt",
             "data/check_point_temperature.bin"]
    before = {n: (tmp_path / n).read_bytes() for n in names}
    run_driver(tmp_path, "--load", "--steps", "0", "--check-every", "1000000")
    for n in names:
        assert (tmp_path / n).read_bytes() == before[n], n
