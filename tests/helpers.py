"""Shared helpers of the test suite (paths, seeded inputs, comparisons)."""
import os

import numpy as np

import pyoracle  # oracle/pyoracle.py: CPU FP64 checker
from rapidsolid import configs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def perturbed_state(p, seed, amp=0.02):
    """Planar Ti-10Nb front plus smooth seeded perturbations of psi and c, with
    ghost cells made consistent (zero-gradient i, periodic/mirrored j)."""
    rng = np.random.default_rng(seed)
    s = pyoracle.initial_planar(p, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, seed)
    ny, nx = s.psi.shape
    j = np.arange(ny)[:, None]
    i = np.arange(nx)[None, :]
    bump = amp * np.sin(2 * np.pi * (j * rng.integers(1, 4) / (ny - 2) + rng.random())) * np.exp(
        -((i - p.i_tip_target) / 6.0) ** 2)
    psi = np.clip(s.psi + bump, -1.0, 1.0)
    c = s.c + 0.3 * amp * rng.standard_normal(s.c.shape) * (1 - psi ** 2)
    s.psi[:] = psi
    s.phi[:] = psi
    s.c[:] = c
    fix_ghosts(p, s)
    return s


def fix_ghosts(p, s):
    ny, nx = s.psi.shape
    jmin, jmax = (ny - 2, 1) if p.periodic_j else (1, ny - 2)
    for a in (s.psi, s.phi, s.c):
        a[1:-1, 0] = a[1:-1, 1]
        a[1:-1, -1] = a[1:-1, -2]
        a[0, :] = a[jmin, :]
        a[-1, :] = a[jmax, :]


def maxabs(a, b):
    return float(np.max(np.abs(np.asarray(a, dtype=np.float64) - np.asarray(b, dtype=np.float64))))


# ---- coarse-grid temperature (TFC) fixtures of the reference's own TFC loop
# (tests/golden/make_golden.py gpu_tfc): (grid, steps, pull-back cadence); the
# front starts 5 cells ahead of i_tip_target = 20, so the pull-back of step 0
# shifts the frame
TFC_CASES = {"tfc_64x72": (64, 72, 240, 60), "tfc_256x252": (256, 252, 500, 100)}
TFC_ITIP = 20
TFC_SEED = 29
TFC_T_MARGIN = 8  # coarse columns kept on each side of the phase-field window


def tfc_params(nx, ny, step_pull_back):
    """The TFC harness build (oracle/ref_build.sh): G = 1e7 K/m, V = 0.5 m/s,
    the reference's TCOLD = 2000 K and 50 um coarse domain (the defaults)."""
    p = configs.small(nx, ny, i_tip_target=TFC_ITIP, tfc=1, G=1e7, V=0.5)
    p.step_pull_back = step_pull_back
    return p


def tfc_input(p):
    q = configs.small(p.nx_all, p.ny_all, i_tip_target=TFC_ITIP + 5)
    return pyoracle.initial_planar(q, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, TFC_SEED)


def oracle_tfc_loop(p, d, s0, nsteps):
    """The coarse-temperature loop of fun.cu:431-514 on the oracle: pull_back
    every step_pull_back steps (i_left_end as set_pull_back, fun.cu:693-705),
    the step on the interpolated T_fine, integrate_phi on the (shifted) psi,
    ratio_dt_dtT temperature sub-steps, interpolate_temperature.  Returns
    (state, coarse T, T_fine, pull-back offsets, final i_left_end)."""
    import ctypes as C
    L = pyoracle.lib()
    pr = lambda a: pyoracle._p(np.ascontiguousarray(a))  # noqa: E731
    nT = d.NxT_all * d.NyT_all
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
    return s, T.reshape(d.NyT_all, d.NxT_all), Tf, shifts, ile


def tfc_T_mask(d, cols):
    """The fixture's kept coarse columns, rows 0 .. NyT-1, without the four
    corners (the reference's corner ghost writes race, fun.cu:1571-1577)."""
    m = np.zeros((d.NyT, len(cols)), dtype=bool)
    m[:, :] = True
    for k, c in enumerate(cols):
        if c in (0, d.NxT - 1):
            m[0, k] = m[d.NyT - 1, k] = False
    return m
