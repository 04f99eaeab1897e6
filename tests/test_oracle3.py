"""The 3D oracle (oracle/rs3_oracle.c) against the reference's own 3D kernels
(TiAg.cu computeMu, boundaryMu*, diffuse, boundary*), whose FP64 outputs on
a seeded 32 x 32 x 20 state are the fixture tests/golden/peri3d_32.npz
(made by tests/golden/make_golden3.py), and the model's own invariants."""
import ctypes as C

import numpy as np
import pytest

import pyoracle
from helpers import golden
from rapidsolid import _abi, configs, lib


def params32():
    p = pyoracle.default_params3()
    p.nx, p.ny, p.nz = 32, 32, 20
    return p


def fixture_input(z):
    ic = z["ic"]
    return dict(z_front=float(ic[0]), amp=float(ic[1]), n_alpha=int(ic[2]), cap_radius=float(ic[3]),
                seed=int(ic[4]))


def test_initial_state_is_the_fixture_input():
    z = golden("peri3d_32.npz")
    f = pyoracle.initial3(params32(), **fixture_input(z))
    for a, n in zip(f, ("phi1", "phi2", "c")):
        assert np.array_equal(a, z[n]), n


def test_mu_matches_reference():
    z = golden("peri3d_32.npz")
    p = params32()
    mu = pyoracle.mu3(p, z["phi1"], z["phi2"], z["c"])
    np.testing.assert_allclose(mu, z["mu0"], rtol=0, atol=1e-15)


@pytest.mark.parametrize("nsteps,tol", [(1, 1e-13), (200, 1e-10)])
def test_steps_match_reference(nsteps, tol):
    """FP64 oracle (no FMA contraction) against the reference kernels (nvcc
    default contraction): one step within 1e-13, 200 steps within 1e-10."""
    z = golden("peri3d_32.npz")
    p = params32()
    f = pyoracle.run3(p, [z["phi1"].copy(), z["phi2"].copy(), z["c"].copy()], nsteps)
    for a, n in zip(f, ("phi1", "phi2", "c")):
        assert np.abs(a - z[f"{n}_{nsteps}"]).max() <= tol, n


def test_solute_is_conserved_and_ghosts_are_images():
    p = params32()
    f = pyoracle.initial3(p, 8.0, 0.5, 2, 5.0, 3)
    m0 = pyoracle.mass3(p, f[2])
    g = pyoracle.run3(p, f, 100)
    assert abs(pyoracle.mass3(p, g[2]) - m0) <= 1e-12 * abs(m0)
    for a in g:
        assert np.array_equal(a[:, :, 0], a[:, :, -2]) and np.array_equal(a[:, :, -1], a[:, :, 1])
        assert np.array_equal(a[:, 0, :], a[:, -2, :]) and np.array_equal(a[:, -1, :], a[:, 1, :])
        assert np.array_equal(a[0], a[1]) and np.array_equal(a[-1], a[-2])


def test_isothermal_gradient_is_the_reference_model():
    """G_T = 0 is TiAg.cu's constant T; a gradient changes the result."""
    p = params32()
    f = pyoracle.initial3(p, 8.0, 0.5, 1, 6.0, 5)
    a = pyoracle.run3(p, [x.copy() for x in f], 5)
    q = params32()
    q.G_T, q.V_T, q.z_T = 0.0, 0.3, 8.0  # a speed without a gradient changes nothing
    b = pyoracle.run3(q, [x.copy() for x in f], 5)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    q.G_T = -1e-3
    c = pyoracle.run3(q, [x.copy() for x in f], 5)
    assert np.abs(c[0] - a[0]).max() > 1e-6


def test_default_params_are_the_reference_constants():
    a, b = lib.default_params3(), pyoracle.default_params3()
    for k, _ in a._fields_:
        assert getattr(a, k) == getattr(b, k), k
    assert a.nx == 512 and a.nz == 128 and a.T_ref == 60.0 * 0.000321787 and a.lam == 30.0
    assert lib.load().rs3_sizeof_params() == C.sizeof(_abi.Params3)


def test_workload_config():
    p = configs.peritectic_3d()
    assert (p.nx, p.ny, p.nz) == (512, 512, 1024)
    assert p.G_T < 0.0 < p.V_T
    # 2e6 K/m over a 25 nm cell, in T units
    assert p.G_T == pytest.approx(-2e6 * 25e-9 * configs.T_PER_K)
