"""Analytic known-answer properties of the oracle (reference has no tests)."""
import numpy as np
import pytest

import pyoracle
from helpers import perturbed_state, fix_ghosts, maxabs
from rapidsolid import configs


def test_philox_known_answers():
    # Philox4x32-10 known-answer vectors of the Random123 distribution
    assert pyoracle.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert pyoracle.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6,
                                                                   0x6D5451FD]
    assert pyoracle.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == [
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_interpolation_function_identities():
    p = configs.default_params()
    # q(psi) (fun.cu:189): q(-1)=1 liquid, q(1)=0 solid, q(0)=(AA+1)/4
    q = lambda x: 0.5 * p.AA * (1 - x) - 0.25 * (p.AA - 1) * (1 - x) ** 2
    assert q(-1.0) == 1.0 and q(1.0) == 0.0 and q(0.0) == (p.AA + 1) / 4


def test_phi_is_clamped_psi_after_steps():
    p = configs.small(64, 48, i_tip_target=20, G=5e6, V=0.5)
    d = pyoracle.derive(p)
    s = perturbed_state(p, 5, amp=0.3)
    s = pyoracle.run(p, d, s, 30)
    assert np.array_equal(s.phi, np.clip(s.psi, -1.0, 1.0))


def test_flat_isotropic_front_stays_flat():
    """eps = epk = 0 and a j-independent front: every row evolves identically."""
    p = configs.small(48, 40, i_tip_target=18, eps1=0.0, epk1=0.0)
    d = pyoracle.derive(p)
    s = pyoracle.initial_reference(p)
    i = np.arange(p.nx_all)[None, :]
    s.psi[:] = -np.tanh((i - 18.3) * p.dx / np.sqrt(2.0))
    s.phi[:] = s.psi
    s.c[:] = 0.9 - 0.02 * 0.5 * (1 + s.psi)
    s = pyoracle.run(p, d, s, 25)
    assert maxabs(s.psi, s.psi[5:6, :]) == 0.0
    assert maxabs(s.c, s.c[5:6, :]) == 0.0


def test_periodic_shift_commutes_with_step():
    p = configs.small(40, 34, i_tip_target=14)
    d = pyoracle.derive(p)
    s = perturbed_state(p, 9, amp=0.2)
    a = pyoracle.step(p, d, s, 0)
    sh = s.copy()
    k = 7
    for arr in (sh.psi, sh.phi, sh.c):
        arr[1:-1] = np.roll(arr[1:-1], k, axis=0)
    fix_ghosts(p, sh)
    b = pyoracle.step(p, d, sh, 0)
    for name in ("psi", "c"):
        x = np.roll(getattr(a, name)[1:-1], k, axis=0)
        assert maxabs(x, getattr(b, name)[1:-1]) == 0.0


def test_solute_flux_form_conserves_interior_mass():
    """With uniform T and a solid (q=0) boundary layer on both i ends, the flux
    form moves no solute across the ends, so interior mass is conserved to
    rounding."""
    p = configs.small(48, 40, i_tip_target=20, G=0.0)
    d = pyoracle.derive(p)
    s = perturbed_state(p, 3, amp=0.1)
    i = np.arange(p.nx_all)[None, :]
    s.psi[:] = np.where((i < 8) | (i > 40), 1.0, np.clip(s.psi, -1, 1))
    s.psi[:] = np.where((i >= 8) & (i <= 40), np.minimum(s.psi, -0.2 + 0.0 * i), s.psi)
    s.phi[:] = s.psi
    fix_ghosts(p, s)
    m0 = pyoracle.mass(p, s.c)
    s = pyoracle.run(p, d, s, 20)
    assert abs(pyoracle.mass(p, s.c) - m0) / m0 < 1e-13


def test_pull_back_semantics():
    p = configs.small(32, 16, i_tip_target=10)
    s = perturbed_state(p, 1)
    for off in (-3, 0, 4):
        o = pyoracle.pull_back(p, s, off)
        for i in range(p.nx_all):
            src = min(max(i + off, 1), p.nx_all - 2)
            assert np.array_equal(o.psi[:, i], s.psi[:, src])
            if src < p.nx_all - 2:
                assert np.array_equal(o.c[:, i], s.c[:, src])
            else:
                assert np.all(o.c[:, i] == p.cinf)


def test_itip_is_max_column_with_positive_psi():
    p = configs.small(40, 20, i_tip_target=12)
    s = perturbed_state(p, 2, amp=0.3)
    cols = np.where((s.psi > 0).any(axis=0))[0]
    assert pyoracle.itip(p, s.psi) == max(1, cols.max())


def test_temperature_model_relations():
    """Frozen T: T(i_tip_target) = Tmelt + deltaT0 delta_initial = T_liquidus,
    and T rises by GG dx W per cell."""
    p = configs.plain_small()
    d = pyoracle.derive(p)
    lib = pyoracle.lib()
    import ctypes as C
    dlt = lambda i: lib.ro_get_delta(C.byref(p), C.byref(d), i, 0, 0.0)
    T = lambda i: dlt(i) * d.deltaT0 + p.Tmelt
    assert abs(T(p.i_tip_target) - configs.T_LIQUIDUS_TI10NB) < 1e-9
    assert abs((T(100) - T(99)) - p.GG * p.dx * d.W) < 1e-9


def test_solute_log_term_series_identity():
    """Both step kernels replace the solute log term
    L(c) - L(cinf) = log(c/(1-c)) - log(cinf/(1-cinf)) by 2 atanh(s) with
    s = delta / (2 cinf (1-c) + delta), delta = c - cinf, summed as a series
    where |s| < 1/9: FP64 to s^15 (truncation below 3.3e-17 relative), FP32 to
    s^7 (below 2.6e-9).  Checked in extended precision over the whole range."""
    ld = np.longdouble
    cinf = ld(configs.default_params().cinf)
    sA, sB = 2 * cinf * (1 - cinf), 1 - 2 * cinf
    d_hi, d_lo = sA / (9 - sB), -sA / (9 + sB)  # |s| = 1/9 at the ends
    delta = np.linspace(d_lo, d_hi, 20001, dtype=ld)[1:-1]
    c = cinf + delta
    s = delta / (2 * cinf * (1 - c) + delta)
    assert np.abs(s).max() < ld(1) / 9
    # the identity (absolute: the log difference cancels near delta = 0)
    exact = 2 * np.arctanh(s)
    logs = np.log(c / (1 - c)) - np.log(cinf / (1 - cinf))
    assert np.abs(logs - exact).max() < 1e-17
    s2 = s * s

    def series(top):  # s (1 + s^2/3 + ... + s^(2 top)/(2 top + 1))
        p = ld(1) / (2 * top + 1)
        for k in range(top - 1, 0, -1):
            p = p * s2 + ld(1) / (2 * k + 1)
        return 2 * (s + s * s2 * p)

    scale = np.maximum(np.abs(exact), ld(1e-30))
    assert (np.abs(series(7) - exact) / scale).max() < 3.3e-17 + 1e-18
    assert (np.abs(series(3) - exact) / scale).max() < 2.6e-9
    assert (np.abs(series(2) - exact) / scale).max() > 2.6e-9  # one term fewer is not enough
