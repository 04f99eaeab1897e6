"""The C-ABI library: loads without a GPU, exports every declared symbol,
struct layouts match, host-side helpers agree with the oracle."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import pyoracle
from helpers import ROOT, golden
from rapidsolid import _abi, configs, lib


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "rs_b200.h")).read()
    return sorted(set(re.findall(r"^(?:int|const char \*|size_t)\s+\*?(rs3?_\w+)\(", txt, flags=re.M)))


def test_library_exports_every_declared_symbol():
    L = lib.load()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s


def test_layouts_and_version():
    L = lib.load()
    assert L.rs_abi_version() == _abi.RS_ABI_VERSION
    assert L.rs_sizeof_params() == C.sizeof(_abi.Params)
    assert L.rs_sizeof_step_args() == C.sizeof(_abi.StepArgs)


def _as_dict(s):
    out = {}
    for k, _ in s._fields_:
        v = getattr(s, k)
        out[k] = list(v) if hasattr(v, "__len__") else v
    return out


def test_default_params_are_constants_hpp():
    a = _as_dict(lib.default_params())
    b = _as_dict(configs.default_params())
    p = _abi.Params()
    pyoracle.lib().ro_default_params(C.byref(p))
    assert a == b == _as_dict(p)
    assert a["Tmelt"] == 2161.59 and a["muk0"] == 0.57 and a["Dl"] == 2.05 and a["v0"] == 1.17e-5


@pytest.mark.parametrize("cfg", ["plain_small", "scale_fp32", "default"])
def test_derive_matches_set_parameters(cfg):
    p = configs.default_params() if cfg == "default" else getattr(configs, cfg)()
    assert _as_dict(lib.derive(p)) == _as_dict(pyoracle.derive(p))


def test_derived_values_of_plain_small():
    d = lib.derive(configs.plain_small())
    assert d.dt == pytest.approx(0.144)
    assert d.step_pull_back == 10082   # 1 W dx / (V dt tau0) at 0.05 m/s


def test_host_calphad_matches_reference():
    z = golden("calphad_ref.npz")
    for w in range(4):
        o = lib.calphad_eval(w, z["T"], z["c"])
        r = z["G"][:, w]
        assert np.array_equal(np.isnan(o), np.isnan(r))
        m = ~np.isnan(r)
        np.testing.assert_allclose(o[m], r[m], rtol=1e-14, atol=1e-9)


def test_errors_are_reported_not_raised():
    L = lib.load()
    assert L.rs_step(None, None, None, None, None) == _abi.RS_E_INVALID
    assert b"null" in L.rs_last_error()
    bad = configs.plain_small()
    bad.n_orientation = 2
    h = C.c_void_p()
    assert L.rs_create(C.byref(bad), C.byref(h)) == _abi.RS_E_UNSUPPORTED
    bad = configs.plain_small()
    bad.nx_all = 4
    assert L.rs_create(C.byref(bad), C.byref(h)) == _abi.RS_E_INVALID
    assert L.rs_calphad_eval(7, None, None, None, 0) == _abi.RS_E_INVALID
    # row bands: frozen temperature only, a non-negative global row offset
    bad = configs.plain_small()
    bad.band, bad.j_offset, bad.tfc = 1, 10, 1
    assert L.rs_create(C.byref(bad), C.byref(h)) == _abi.RS_E_UNSUPPORTED
    bad.tfc, bad.j_offset = 0, -1
    assert L.rs_create(C.byref(bad), C.byref(h)) == _abi.RS_E_INVALID
    # 3D: extents and the x alignment of the tensor maps
    p3 = lib.default_params3()
    p3.nx = 30
    assert L.rs3_create(C.byref(p3), C.byref(h)) == _abi.RS_E_INVALID


def test_phase_boundaries_of_ti10nb():
    """T_liquidus / T_solidus of c_Ti = 0.90 from the common tangent of the
    library's evaluator (Gl, Gs, Glc, Gsc)."""
    def tangent(T, cl=0.9, cs=0.88):
        for _ in range(60):
            f = lambda a, b: np.array([
                lib.calphad_eval(2, [T], [a])[0] - lib.calphad_eval(3, [T], [b])[0],
                (lib.calphad_eval(0, [T], [a])[0] - a * lib.calphad_eval(2, [T], [a])[0]) -
                (lib.calphad_eval(1, [T], [b])[0] - b * lib.calphad_eval(3, [T], [b])[0])])
            r = f(cl, cs)
            h = 1e-7
            J = np.column_stack([(f(cl + h, cs) - r) / h, (f(cl, cs + h) - r) / h])
            dl, ds = np.linalg.solve(J, r)
            cl, cs = cl - dl, cs - ds
        return cl, cs
    cl, cs = tangent(configs.T_LIQUIDUS_TI10NB)
    assert abs(cl - configs.C_LIQUID_TI10NB) < 1e-6
    assert abs(cs - configs.C_SOLID_AT_TLIQ) < 1e-6
    cl, cs = tangent(configs.T_SOLIDUS_TI10NB)
    assert abs(cs - 0.90) < 1e-6


def test_driver_binary_prints_usage():
    """The host driver is built beside the library and starts without a GPU."""
    import subprocess
    drv = os.path.join(os.path.dirname(lib.LIB_PATH), "rs_run")
    r = subprocess.run([drv, "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "usage: rs_run" in r.stdout
