"""ctypes front end of the CPU FP64 oracle (oracle/lib/librs_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The product never imports it.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "librs_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

sys.path.insert(0, os.path.join(os.path.dirname(HERE), "2d-rapid-solidification_b200"))
from rapidsolid import _abi  # noqa: E402

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.ro_derive.argtypes = [vp, vp]
        L.ro_default_params.argtypes = [vp]
        for n in ("ro_G_Ti_BCC", "ro_G_Ti_Liq", "ro_G_Nb_BCC", "ro_G_Nb_Liq"):
            getattr(L, n).restype = C.c_double
            getattr(L, n).argtypes = [C.c_double]
        for n in ("ro_Gl", "ro_Gs", "ro_Glc", "ro_Gsc"):
            getattr(L, n).restype = C.c_double
            getattr(L, n).argtypes = [vp, C.c_double, C.c_double]
        L.ro_calphad_table.argtypes = [vp, C.c_int, vp, vp, vp, C.c_int64]
        L.ro_get_delta.restype = C.c_double
        L.ro_get_delta.argtypes = [vp, vp, C.c_int, C.c_int, C.c_double]
        L.ro_vp_ramp.restype = C.c_double
        L.ro_vp_ramp.argtypes = [vp, C.c_double]
        L.ro_philox4x32.argtypes = [vp, vp, vp]
        L.ro_step.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, C.c_int64, C.c_int, C.c_double]
        L.ro_pull_back.argtypes = [vp] * 7 + [C.c_int]
        L.ro_itip_all_grain.restype = C.c_int
        L.ro_itip_all_grain.argtypes = [vp, vp]
        L.ro_precise_tip.argtypes = [vp, vp, vp, vp]
        L.ro_mass.restype = C.c_double
        L.ro_mass.argtypes = [vp, vp]
        L.ro_initial.argtypes = [vp, vp, vp, vp]
        L.ro_initial_planar.argtypes = [vp, vp, vp, vp, C.c_double, C.c_double, C.c_uint64]
        L.ro_initial_temperature.argtypes = [vp, vp, vp]
        L.ro_integrate_phi.argtypes = [vp, vp, vp, vp, vp, C.c_int]
        L.ro_compute_temperature.argtypes = [vp, vp, vp, vp, vp, C.c_int64]
        L.ro_interpolate_temperature.argtypes = [vp, vp, vp, vp, C.c_int]
        L.ro_run_steps.argtypes = [vp] * 8 + [C.c_int64, C.c_int64, C.c_int, C.c_double]
        L.ro_run_steps.restype = C.c_int
        L.ro_num_threads.restype = C.c_int
        L.ro3_default_params.argtypes = [vp]
        L.ro3_equilibrium.argtypes = [vp, vp]
        L.ro3_boundary.argtypes = [vp, vp]
        L.ro3_mu.argtypes = [vp] * 5
        L.ro3_step.argtypes = [vp, C.c_int64] + [vp] * 7
        L.ro3_mass.restype = C.c_double
        L.ro3_mass.argtypes = [vp, vp]
        L.ro3_cap_centres.argtypes = [vp, C.c_int, C.c_uint64, vp, vp]
        L.ro3_initial.argtypes = [vp, C.c_double, C.c_double, C.c_int, C.c_double, C.c_uint64, vp, vp, vp]
        L.ro3_initial_grains.argtypes = [vp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint64, vp, vp,
                                         vp]
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.c_void_p)


def derive(p):
    d = _abi.Derived()
    lib().ro_derive(C.byref(p), C.byref(d))
    return d


class State:
    """c, phi, psi (FP64, Ny_all x Nx_all, row j contiguous in i)."""

    def __init__(self, p):
        self.p = p
        shape = (p.ny_all, p.nx_all)
        self.c = np.zeros(shape)
        self.phi = np.zeros(shape)
        self.psi = np.zeros(shape)

    def copy(self):
        s = State(self.p)
        s.c[:] = self.c
        s.phi[:] = self.phi
        s.psi[:] = self.psi
        return s


def initial_planar(p, c_liquid, c_solid, seed):
    s = State(p)
    lib().ro_initial_planar(C.byref(p), _p(s.c), _p(s.phi), _p(s.psi), c_liquid, c_solid, seed)
    return s


def initial_reference(p):
    s = State(p)
    lib().ro_initial(C.byref(p), _p(s.c), _p(s.phi), _p(s.psi))
    return s


def step(p, d, s, step_index, i_offset_history=0, l_offset_Vp=0.0, T_fine=None):
    out = State(p)
    lib().ro_step(C.byref(p), C.byref(d), _p(s.c), _p(s.phi), _p(s.psi), _p(T_fine),
                  _p(out.c), _p(out.phi), _p(out.psi), step_index, i_offset_history, l_offset_Vp)
    return out


def pull_back(p, s, i_offset):
    out = State(p)
    lib().ro_pull_back(C.byref(p), _p(s.c), _p(s.phi), _p(s.psi), _p(out.c), _p(out.phi),
                       _p(out.psi), i_offset)
    return out


def l_offset_increment(p, d, step_index):
    """main.cu:235-236: l_offset_Vp += Vp_ramp(step tau0 dt) dt tau0 / (S W0)."""
    return lib().ro_vp_ramp(C.byref(p), step_index * d.tau0 * d.dt) * d.dt * d.tau0 / (p.S * p.W0)


def run(p, d, s, nsteps, step0=0, i_offset_history=0, l_offset_Vp=0.0):
    """nsteps plain steps (no pull-back), in place on a copy; returns the state."""
    a = s.copy()
    b = State(p)
    lib().ro_run_steps(C.byref(p), C.byref(d), _p(a.c), _p(a.phi), _p(a.psi), _p(b.c), _p(b.phi),
                       _p(b.psi), step0, nsteps, i_offset_history, l_offset_Vp)
    return a


def itip(p, psi):
    return lib().ro_itip_all_grain(C.byref(p), _p(np.ascontiguousarray(psi)))


def precise_tip(p, d, psi):
    t = _abi.Tip()
    lib().ro_precise_tip(C.byref(p), C.byref(d), _p(np.ascontiguousarray(psi)), C.byref(t))
    return t


def mass(p, c):
    return lib().ro_mass(C.byref(p), _p(np.ascontiguousarray(c)))


def calphad(p, which, T, c):
    T = np.ascontiguousarray(T, dtype=np.float64)
    c = np.ascontiguousarray(c, dtype=np.float64)
    out = np.empty_like(T)
    lib().ro_calphad_table(C.byref(p), which, _p(T), _p(c), _p(out), T.size)
    return out


def philox(ctr, key):
    ctr = (C.c_uint32 * 4)(*ctr)
    key = (C.c_uint32 * 2)(*key)
    out = (C.c_uint32 * 4)()
    lib().ro_philox4x32(ctr, key, out)
    return list(out)


def ref_binary(name):
    """Path of a reference harness binary built by oracle/ref_build.sh."""
    return os.path.join(REF_DIR, name)


# ---------------------------------------------------------------- 3D (TiAg.cu)

def default_params3():
    p = _abi.Params3()
    lib().ro3_default_params(C.byref(p))
    return p


def equilibrium3(p):
    """ca, cb, cla, clb at T_ref (TiAg.cu:64-67)."""
    out = np.zeros(4)
    lib().ro3_equilibrium(C.byref(p), _p(out))
    return out


def zeros3(p):
    return np.zeros((p.nz, p.ny, p.nx))


def initial3(p, z_front, amp, n_alpha, cap_radius, seed):
    f = [zeros3(p) for _ in range(3)]
    lib().ro3_initial(C.byref(p), z_front, amp, n_alpha, cap_radius, seed, *[_p(a) for a in f])
    return f


def initial_grains3(p, z_front, amp, c_liquid, c_solid, seed):
    """Two grains under a seeded front, melt above (rs3_initial_grains)."""
    f = [zeros3(p) for _ in range(3)]
    lib().ro3_initial_grains(C.byref(p), z_front, amp, c_liquid, c_solid, seed, *[_p(a) for a in f])
    return f


def boundary3(p, a):
    lib().ro3_boundary(C.byref(p), _p(a))


def mu3(p, phi1, phi2, c):
    mu = zeros3(p)
    lib().ro3_mu(C.byref(p), _p(phi1), _p(phi2), _p(c), _p(mu))
    return mu


def step3(p, step_index, phi1, phi2, c):
    out = [zeros3(p) for _ in range(3)]
    lib().ro3_step(C.byref(p), step_index, _p(phi1), _p(phi2), _p(c), *[_p(a) for a in out], None)
    return out


def run3(p, f, nsteps, step0=0):
    for k in range(nsteps):
        f = step3(p, step0 + k, *f)
    return f


def mass3(p, c):
    return lib().ro3_mass(C.byref(p), _p(c))
