"""The 3D oracle's Ti-Nb CALPHAD energy (rs3_params.energy = 1), pinned per
component to the reference:

* its chemical potential is the reference's mu of fun.cu:1443-1452,
  g1 Glc + (1 - g1) Gsc, built from the oracle's Glc and Gsc, which equal the
  reference's compiled host code bit for bit (test_oracle_golden.py);
* in the two-phase limit (no second grain, no triple-junction terms, a
  planar front) one step of the 3D model is one step of the reference's 2D
  CALPHAD model (compute_phi and compute_c_CALPHAD of fun.cu, isotropic), in
  the liquid fraction phi1 = (1 - psi) / 2: the 2D oracle, which is pinned to
  the reference's own kernels, and the 3D oracle follow the same trajectory;
* solute is conserved and the initial state is the documented one."""
import math

import numpy as np
import pytest

import pyoracle
from rapidsolid import _abi, configs

X_NB = 0.10


def params3(nx, ny, nz, **kw):
    p = configs.tinb_3d(nx=nx, ny=ny, nz=nz, lib=_Lib3())
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class _Lib3:
    """configs.tinb_3d's library calls answered by the oracle (no GPU library)."""

    @staticmethod
    def default_params3():
        return pyoracle.default_params3()

    @staticmethod
    def derive(p):
        return pyoracle.derive(p)


def random_fields(p, seed=3):
    rng = np.random.default_rng(seed)
    shape = (p.nz, p.ny, p.nx)
    p1 = rng.uniform(0.0, 1.0, shape)
    p2 = rng.uniform(0.0, 1.0, shape) * (1.0 - p1)
    c = rng.uniform(0.84, 0.96, shape)
    return p1, p2, c


def test_tinb_mu_is_the_reference_mu():
    p = params3(8, 8, 12)
    p1, p2, c = random_fields(p)
    mu = pyoracle.mu3(p, p1, p2, c)
    p2d = configs.scale()
    z = np.arange(p.nz, dtype=np.float64)
    T = p.T_ref + p.G_T * (z - p.z_T)  # step 0
    Tc = np.broadcast_to(T[:, None, None], c.shape)
    glc = pyoracle.calphad(p2d, 2, Tc.ravel(), c.ravel()).reshape(c.shape)
    gsc = pyoracle.calphad(p2d, 3, Tc.ravel(), c.ravel()).reshape(c.shape)
    p3 = 1.0 - p1 - p2
    # Folch-Plapp g of the liquid (TiAg.cu:72)
    g1 = p1 * p1 * 0.25 * (15.0 * (1 - p1) * (1 + p1 - (p3 - p2) * (p3 - p2)) + p1 * (9.0 * (p1 * p1) - 5.0))
    ref = (1.0 - g1) * gsc + g1 * glc
    inner = (slice(1, -1),) * 3
    np.testing.assert_allclose(mu[inner], ref[inner], rtol=1e-14, atol=0)


def two_phase_pair(n_i=96, i0=30.5, nsteps=300):
    """The same planar front in the 2D oracle (N_i x 4, i the growth axis)
    and the 3D oracle (4 x 4 x N_i, z the growth axis, phi2 = 0)."""
    p3 = params3(4, 4, n_i, a1=0.0, a2=0.0, a3=0.0, z_T=30.0)
    p2 = configs._ti10nb(configs.default_params(), n_i, 4, 2.0e6, 0.2, T0=configs.T_SOLIDUS_TI10NB)
    p2.dt = p3.dt
    p2.eps1 = p2.eps2 = p2.epk1 = 0.0
    p2.noise_amplitude = 0.0
    p2.i_tip_target = 30
    d2 = pyoracle.derive(p2)
    cl, cs = configs.tinb_compositions(X_NB)
    i = np.arange(n_i, dtype=np.float64)
    psi = np.tanh((i0 - i) * p2.dx / math.sqrt(2.0))
    psi[0], psi[-1] = psi[1], psi[-2]
    c = cl + (cs - cl) * 0.5 * (1.0 + psi)
    s = pyoracle.State(p2)
    s.psi[:] = psi[None, :]
    s.phi[:] = psi[None, :]
    s.c[:] = c[None, :]
    f = [np.ascontiguousarray(np.broadcast_to(v[:, None, None], (n_i, 4, 4))) for v in
         (0.5 * (1.0 - psi), np.zeros(n_i), c)]
    return p2, d2, s, p3, f


def test_tinb_two_phase_limit_is_the_2d_step():
    p2, d2, s, p3, f = two_phase_pair()
    # the temperature lines agree: T_3D(z, step) = Tmelt + deltaT0 get_delta(i = z)
    assert p3.G_T == pytest.approx(p2.GG * p2.dx * p2.S * p2.W0, rel=1e-14)
    assert p3.V_T == pytest.approx(p2.Vp * p2.dt * d2.tau0 / (p2.dx * p2.S * p2.W0), rel=1e-14)
    assert p3.dt == d2.dt
    # The far end differs by construction: the 2D kernel evaluates the ghost
    # column's chemical potential at the ghost's own temperature
    # (compute_c_CALPHAD, fun.cu:1409-1416 and 1443-1452), which lets solute
    # through the no-flux boundary of a frozen gradient; the 3D model images
    # mu as TiAg.cu's boundaryMu does, so no solute crosses it.  The melt
    # diffuses that difference less than a cell in 300 steps; the comparison
    # stops 8 cells short of the end.
    k = slice(0, p3.nz - 8)
    for n in (1, 300):
        a = pyoracle.run(p2, d2, s, n)
        b = pyoracle.run3(p3, f, n)
        psi3 = 1.0 - 2.0 * b[0][:, 2, 2]
        assert np.abs(b[1]).max() < 1e-15  # the second grain stays at rounding level
        assert np.abs(psi3 - a.psi[2, :])[k].max() < 1e-11, n
        assert np.abs(b[2][:, 2, 2] - a.c[2, :])[k].max() < 1e-12, n
    # and the front moved: a real trajectory, not a fixed point
    assert np.abs(a.psi[2, :] - s.psi[2, :]).max() > 1e-2


def test_tinb_conserves_solute():
    p = params3(12, 8, 24)
    cl, cs = configs.tinb_compositions(X_NB)
    f = pyoracle.initial_grains3(p, 8.0, 0.5, cl, cs, 5)
    m0 = pyoracle.mass3(p, f[2])
    f = pyoracle.run3(p, f, 60)
    assert abs(pyoracle.mass3(p, f[2]) - m0) <= 1e-12 * m0
    assert np.isfinite(f[0]).all() and np.isfinite(f[1]).all()


def test_tinb_initial_grains():
    p = params3(12, 8, 24)
    cl, cs = configs.tinb_compositions(X_NB)
    p1, p2, c = pyoracle.initial_grains3(p, 8.0, 0.5, cl, cs, 5)
    inner = (slice(1, -1), slice(1, -1), slice(1, -1))
    assert set(np.unique(p1[inner])) == {0.0, 1.0}
    assert (p2[:, :, 1:(p.nx - 2) // 2 + 1][p1[:, :, 1:(p.nx - 2) // 2 + 1] == 0.0] == 1.0).all()
    assert (p2[:, :, (p.nx - 2) // 2 + 1:-1] == 0.0).all()
    assert (c[inner][p1[inner] == 1.0] == cl).all() and (c[inner][p1[inner] == 0.0] == cs).all()
    # the front lies within 0.5 of z_front in every column
    zf = (p1[1:-1, 1:-1, 1:-1] == 0.0).sum(0)
    assert zf.min() >= 7 and zf.max() <= 8
