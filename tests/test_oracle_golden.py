"""The CPU oracle pinned against the reference's own compiled code.

Fixtures in tests/golden/ come from tests/golden/make_golden.py, which runs
the reference's routines (old-fun.cu, built by oracle/ref_build.sh).
"""
import numpy as np
import pytest

import pyoracle
from helpers import golden, maxabs
from rapidsolid import configs


def test_calphad_matches_reference_bitwise():
    z = golden("calphad_ref.npz")
    p = configs.default_params()
    for w in range(4):
        o = pyoracle.calphad(p, w, z["T"], z["c"])
        r = z["G"][:, w]
        assert np.array_equal(np.isnan(o), np.isnan(r))
        m = ~np.isnan(r)
        # same expressions, same order, both built without FMA contraction
        assert np.array_equal(o[m], r[m]), f"which={w}"


def test_calphad_covers_branches():
    z = golden("calphad_ref.npz")
    T = z["T"]
    assert (T < 1155).any() and (T >= 4000).any()        # NaN regions
    assert np.isnan(z["G"]).any()
    assert ((T >= 1941.0) & (T < 1941.001)).any()        # Ti kink
    assert (T == 2750.0).any()                           # Nb kink
    c = z["c"]
    assert (c < 1e-8).any() and (1 - c < 1e-8).any()     # guarded log branches


@pytest.mark.parametrize("idx", range(5))
def test_precise_tip_matches_reference(idx):
    z = golden("tip_ref.npz")
    name = str(z["names"][idx])
    ref = z["tips"][idx]
    p = configs.small(64, 64, i_tip_target=24)
    d = pyoracle.derive(p)
    psi = z["psi_" + name]
    assert pyoracle.itip(p, psi) == int(ref[0])
    t = pyoracle.precise_tip(p, d, psi)
    assert (t.i, t.j) == (int(ref[1]), int(ref[2]))
    assert abs(t.x - ref[3]) <= 1e-12 * max(1.0, abs(ref[3]))
    assert abs(t.y - ref[4]) <= 1e-12 * max(1.0, abs(ref[4]))
    assert abs(t.R - ref[5]) <= 1e-9 * max(1.0, abs(ref[5]))


def _have(name):
    import os
    return os.path.exists(os.path.join(pyoracle.HERE, "..", "tests", "golden", name))


@pytest.mark.skipif(not _have("step64.npz"), reason="reference kernel fixtures not generated")
@pytest.mark.parametrize("nsteps", [1, 40])
def test_oracle_step_matches_reference_kernels(nsteps):
    """64x64: pull_back(3) then n steps of the reference's GPU kernels."""
    z = golden("step64.npz")
    p = configs.small(64, 64, i_tip_target=24)
    d = pyoracle.derive(p)
    s = pyoracle.State(p)
    s.c[:] = z["in_c"]
    s.psi[:] = z["in_psi"]
    s.phi[:] = z["in_psi"]
    s = pyoracle.pull_back(p, s, 3)
    s = pyoracle.run(p, d, s, nsteps)
    interior = (slice(1, -1), slice(1, -1))
    for tag, tol in (("nofma", 1e-13), ("fma", 1e-12)):
        for k in ("c", "psi"):
            ref = z[f"{tag}_{nsteps}_{k}"]
            assert maxabs(getattr(s, k)[interior], ref[interior]) <= tol, (tag, k)
            # ghost ring: the reference writes corners from two racing threads;
            # edges are deterministic
            assert maxabs(getattr(s, k)[1:-1, :], ref[1:-1, :]) <= tol
            assert maxabs(getattr(s, k)[:, 1:-1], ref[:, 1:-1]) <= tol


@pytest.mark.skipif(not _have("c1_500.npz"), reason="reference kernel fixtures not generated")
def test_oracle_c1_500_steps_matches_reference_kernels():
    """256x256 Ti-10Nb, frozen T, 500 steps: max |dphi|, |dc| <= 1e-10."""
    z = golden("c1_500.npz")
    p = configs.plain_small()
    d = pyoracle.derive(p)
    s = pyoracle.initial_planar(p, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, int(z["seed"]))
    off = pyoracle.itip(p, s.psi) - p.i_tip_target
    s = pyoracle.pull_back(p, s, off)
    s = pyoracle.run(p, d, s, 500)
    for tag in ("nofma", "fma"):
        for k in ("c", "psi"):
            assert maxabs(getattr(s, k)[1:-1, 1:-1], z[f"{tag}_{k}"][1:-1, 1:-1]) <= 1e-10, (tag, k)
