"""Named workloads (synthetic inputs) of the coupled phase-field step.

Axes follow the reference: i is the growth axis (contiguous), j is periodic.
The benchmark configurations are written growth-along-y; their y is the
reference's i and their x the reference's j.  Concentrations are the
reference's variable c = Ti mole fraction, so "Ti-10at%Nb" is c = 0.90.

Ti-10Nb phase boundaries come from the exact Ti-Nb evaluator (common tangent
of the liquid and BCC Gibbs energies, fun.cu:1671-1720):
  T_liquidus(c_l = 0.90) = 1974.99160 K, solid in equilibrium c_s = 0.879550
  T_solidus (c_s = 0.90) = 1968.14983 K
tests/test_configs.py re-derives them with the library's evaluator.
"""
from ._abi import Params

C_LIQUID_TI10NB = 0.90
T_LIQUIDUS_TI10NB = 1974.9916030759996
C_SOLID_AT_TLIQ = 0.8795504308633851
T_SOLIDUS_TI10NB = 1968.1498345850491


def default_params(lib=None):
    """constants.hpp parameter set (src/constants.hpp:185-350)."""
    p = Params()
    if lib is not None:
        rc = lib.rs_default_params(p)
        if rc != 0:
            raise RuntimeError("rs_default_params failed")
        return p
    p.nx_all, p.ny_all, p.i_tip_target = 768, 832, 768 - 268
    p.periodic_j, p.tfc, p.one_eps, p.vp_ramp, p.n_orientation = 1, 1, 1, 0, 1
    p.cinf, p.W0, p.S, p.Gamma, p.muk0 = 0.632514105, 0.25, 5.0, 199.0, 0.57
    p.Tmelt, p.T_ref, p.Dl, p.DT = 2161.59, 2118.35, 2.05, 1.1e4
    p.latent_heat, p.molar_weight, p.num_moles, p.cp = 22003.0, 64.418, 93353.43470588748, 40.0
    p.RR, p.v0, p.AA, p.ke = 8.3145, 1.17e-5, 12.0, 0.8146631243899296
    p.dx, p.dt, p.GG, p.Vp = 0.6, 0.0, 10 * 0.001, 1.0
    p.eps1, p.eps2, p.epk1 = 0.06, 0.0, 0.15
    p.delta_initial, p.l_offset_Vp_initial, p.i_offset_history_initial = -1.0, 0.0, 0
    p.ratio_dxT_dx = 10
    for k in range(9):
        p.orientation[k] = 1.0 if k in (0, 4, 8) else 0.0
    p.noise_amplitude, p.seed = 0.0, 0
    p.Tcold, p.length_sample_um = 2000.0, 50.0
    p.total_time_ns = 120.0 * 1000.0
    p.num_fields_output = p.num_tip_output = p.num_check_point_output = 120
    p.step_pull_back = 0
    return p


def _ti10nb(p, n_i, n_j, G_K_per_m, V_m_per_s, T0=T_LIQUIDUS_TI10NB):
    p.nx_all, p.ny_all = n_i, n_j
    p.tfc, p.vp_ramp = 0, 0
    p.dx = 0.8
    p.dt = 0.9 * p.dx * p.dx / 4.0          # 0.9 of the explicit limit dx^2/4
    p.GG = G_K_per_m * 1e-9                  # K/nm
    p.Vp = V_m_per_s
    p.i_tip_target = 16                      # front at y0 = 16 dx
    p.cinf = C_LIQUID_TI10NB                 # melt entering through the pull-back
    deltaT0 = p.Tmelt - p.T_ref
    p.delta_initial = (T0 - p.Tmelt) / deltaT0  # T(i_tip_target) = T0 at t = 0
    return p


def plain_small(lib=None):
    """256x256 (Nx_all x Ny_all) FP64, frozen T, G = 1e6 K/m, V = 0.05 m/s, 500 steps."""
    return _ti10nb(default_params(lib), 256, 256, 1.0e6, 0.05)


def scale(lib=None):
    """2048x2048, G = 5e6 K/m, V = 0.5 m/s, interface noise 0.01, 20000 steps;
    the field precision is the caller's (FP32 bulk or the FP64 exact path).

    The front starts at the solidus isotherm: the c = 0.90 melt ahead of it is
    undercooled by T_liquidus - T_solidus = 6.84 K, so the front grows from
    the first step (about 1.3 m/s, relaxing to about 0.4 m/s after 10^4
    steps) and the moving frame shifts about every thousand steps.

    Output cadence of the reference loop over this run: its 20000 steps are
    total_time, with the reference's num_fields_output = 100 field snapshots
    (old-fun.cu:41-43), so step_fields = 200.
    """
    p = _ti10nb(default_params(lib), 2048, 2048, 5.0e6, 0.5, T0=T_SOLIDUS_TI10NB)
    p.noise_amplitude = 0.01
    p.seed = 20240611
    tau0 = (p.S * p.W0) ** 2 / (p.Gamma * p.muk0)
    p.total_time_ns = (STEPS["scale_fp32"] + 0.5) * tau0 * p.dt
    p.num_fields_output = p.num_tip_output = p.num_check_point_output = 100
    return p


scale_fp32 = scale  # the FP32 bulk configuration of the same workload


def small(n_i, n_j, lib=None, **kw):
    """A small Ti-10Nb grid for parity tests."""
    p = _ti10nb(default_params(lib), n_i, n_j, kw.pop("G", 1.0e6), kw.pop("V", 0.05))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


IC_SEED = 7
STEPS = {"plain_small": 500, "scale_fp32": 20000}


def _tangent(T, cl, cs, iters=12):
    """Common tangent of the liquid and solid Gibbs energies at T (host build of
    the reference evaluator, fun.cu:1671-1720): equal chemical potential
    (Glc = Gsc) and equal intercepts (G - c dG/dc).  Returns (c_liquid, c_solid)."""
    import numpy as np
    from . import lib

    def f(a, b):
        ga = lib.calphad_eval(0, [T], [a])[0] - a * lib.calphad_eval(2, [T], [a])[0]
        gb = lib.calphad_eval(1, [T], [b])[0] - b * lib.calphad_eval(3, [T], [b])[0]
        return np.array([lib.calphad_eval(2, [T], [a])[0] - lib.calphad_eval(3, [T], [b])[0], ga - gb])
    for _ in range(iters):
        r = f(cl, cs)
        h = 1e-7
        J = np.column_stack([(f(cl + h, cs) - r) / h, (f(cl, cs + h) - r) / h])
        dl, ds = np.linalg.solve(J, r)
        cl, cs = cl - dl, cs - ds
    return cl, cs


def phase_boundaries(c0):
    """(T_liquidus, c_solid at T_liquidus, T_solidus) of the melt c_Ti = c0: the
    tangent compositions are followed up in T from the Ti melting point in
    2 K steps (warm-started Newton) to bracket the crossings, then bisected."""
    import math

    # start from the known Ti-10Nb tangent and walk in T both ways (higher T:
    # both tangent compositions drop; the lens closes at the Ti melting point)
    pts = [(T_LIQUIDUS_TI10NB, C_LIQUID_TI10NB, C_SOLID_AT_TLIQ)]
    for step in (1.0, -1.0):
        T, cl, cs = pts[0]
        for _ in range(800):
            T += step
            if T <= 1941.5:
                break
            cl, cs = _tangent(T, cl, cs, iters=6)
            if not (math.isfinite(cl) and math.isfinite(cs)) or not (0.0 < cs < cl < 1.0):
                break
            pts.append((T, cl, cs))
            if (step > 0 and cl < c0 and cs < c0) or (step < 0 and cl > c0 and cs > c0):
                break
    pts.sort()

    def bisect(which):
        for (Ta, la, sa), (Tb, lb, sb) in zip(pts, pts[1:]):
            fa, fb = (la if which == 0 else sa) - c0, (lb if which == 0 else sb) - c0
            if fa >= 0 > fb:
                cl, cs = la, sa
                for _ in range(50):
                    Tm = 0.5 * (Ta + Tb)
                    cl, cs = _tangent(Tm, cl, cs, iters=8)
                    fm = (cl if which == 0 else cs) - c0
                    if fm >= 0:
                        Ta = Tm
                    else:
                        Tb = Tm
                return 0.5 * (Ta + Tb), cl, cs
        raise ValueError(f"no phase boundary found for c0 = {c0}")
    T_liq, _, cs_liq = bisect(0)
    T_sol, _, _ = bisect(1)
    return T_liq, cs_liq, T_sol


def ensemble(n=64, seed=2024, lib=None):
    """The batched-ensemble workload: n Ti-Nb runs, sizes drawn between 256x256
    and 1024x2048 (multiples of 4), V log-uniform in [0.01, 2] m/s, G
    log-uniform in [1e5, 1e7] K/m, x_Nb of the melt uniform in [0.05, 0.20];
    each front starts at its solidus (as the scale workload).  Returns a list
    of (params, c_liquid, c_solid) for rs_initial_planar."""
    import numpy as np
    rng = np.random.default_rng(seed)
    runs = []
    for k in range(n):
        nx = int(rng.integers(64, 257)) * 4
        ny = int(rng.integers(64, 513)) * 4
        V = float(np.exp(rng.uniform(np.log(0.01), np.log(2.0))))
        G = float(np.exp(rng.uniform(np.log(1e5), np.log(1e7))))
        c0 = 1.0 - float(rng.uniform(0.05, 0.20))
        T_liq, cs, T_sol = phase_boundaries(c0)
        p = _ti10nb(default_params(lib), nx, ny, G, V, T0=T_sol)
        p.cinf = c0
        p.seed = seed + k
        runs.append((p, c0, cs))
    return runs


# ---------------------------------------------------------------- 3D variant
# Units of the 3D three-phase model (the reference's TiAg.cu is dimensionless):
# T is an undercooling in units of 1/0.000321787 K (TiAg.cu:52 sets
# 60 * 0.000321787 for 60 K); one model length unit is 50 nm (dx = 1/DXin =
# 0.5 units = 25 nm); one model time unit is 1 ns.  These scales map the
# workload's G and V onto the model; they are this build's choice, not the
# reference's.
T_PER_K = 0.000321787
LENGTH_UNIT_M = 50e-9
TIME_UNIT_S = 1e-9
IC3 = dict(z_front=24.0, amp=0.5, n_alpha=4, cap_radius=30.0, seed=11)
STEPS["peritectic_3d"] = 5000


def peritectic_3d(G_K_per_m=2.0e6, V_m_per_s=0.2, nx=512, ny=512, nz=1024, lib=None):
    """3D three-phase directional solidification on one GPU: 512 x 512 x 1024
    (ghost layers included), the reference model's constants, a frozen
    gradient G moving at V.  The undercooling falls with z (melt above the
    beta front), and T = T_ref at the front plane at step 0."""
    if lib is None:
        from . import lib as _lib
        lib = _lib
    p = lib.default_params3()
    p.nx, p.ny, p.nz = nx, ny, nz
    dx_m = LENGTH_UNIT_M / p.dx_inv
    p.G_T = -G_K_per_m * dx_m * T_PER_K
    p.V_T = V_m_per_s * p.dt * TIME_UNIT_S / dx_m
    p.z_T = IC3["z_front"]
    return p


# ---------------------------------------------------------------- 3D Ti-Nb CALPHAD variant (energy 1)
# The three-phase structure with the Ti-Nb CALPHAD energy of the 2D model; its
# units are the 2D model's: lengths in W = S W0, time in tau0 = W^2 / (Gamma
# muk0), dx = 0.8 W, the coupling lambda = 1 / (2 hh v0) and the solute
# coefficient alpha = Dl / (Gamma muk0 h0 v0) per J/mol, so that in the
# two-phase limit the 3D phase and solute equations are those of the 2D step
# (isotropic).  The two solids are two BCC grains.
IC3_TINB = dict(z_front=24.0, amp=0.5, seed=11)
STEPS["tinb_3d"] = 5000


def tinb_3d(G_K_per_m=2.0e6, V_m_per_s=0.2, x_nb=0.10, nx=512, ny=512, nz=1024, z_front=24.0, lib=None):
    """3D Ti-Nb directional solidification on one GPU (energy 1): nx x ny x nz
    (ghost layers included), melt x_Nb = x_nb, a frozen gradient G moving at V,
    T = the alloy's solidus at the front plane z_front at step 0 (as the 2D
    scale workload).  The three-phase well terms are TiAg.cu's (a2 = 4.43,
    a3 = 6.09, b = 12); they stiffen the phase equations, so dt is 0.45 of the
    explicit diffusive limit dx^2/6 (0.9 of it oscillates where a grain meets
    the melt).  Returns the rs3 parameters; the melt and solid compositions
    are tinb_compositions(x_nb)."""
    if lib is None:
        from . import lib as _lib
        lib = _lib
    p2 = scale()
    d2 = lib.derive(p2)
    p = lib.default_params3()
    p.nx, p.ny, p.nz = nx, ny, nz
    p.energy = 1
    dx = 0.8
    p.dx_inv = p.dy_inv = p.dz_inv = 1.0 / dx
    p.dt = 0.45 * dx * dx / 6.0
    p.lam = 1.0 / (2.0 * d2.hh * p2.v0)
    p.alpha = p2.Dl / (p2.Gamma * p2.muk0) / (d2.h0 * p2.v0)
    p.AA, p.RR = p2.AA, p2.RR
    c0 = 1.0 - x_nb
    p.c_ref = c0
    T_sol = T_SOLIDUS_TI10NB if abs(c0 - C_LIQUID_TI10NB) < 1e-12 else phase_boundaries(c0)[2]
    W_nm = p2.S * p2.W0
    p.T_ref = T_sol
    p.z_T = z_front
    p.G_T = G_K_per_m * dx * W_nm * 1e-9
    p.V_T = V_m_per_s * p.dt * d2.tau0 / (dx * W_nm)
    return p


def tinb_compositions(x_nb=0.10):
    """(c_liquid, c_solid): the melt and the solid of the tangent at its liquidus."""
    c0 = 1.0 - x_nb
    if abs(c0 - C_LIQUID_TI10NB) < 1e-12:
        return C_LIQUID_TI10NB, C_SOLID_AT_TLIQ
    return c0, phase_boundaries(c0)[1]
