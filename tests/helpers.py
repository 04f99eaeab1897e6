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
