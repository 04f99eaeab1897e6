"""Restart and snapshot files in the reference's layouts (host code)."""
import ctypes as C
import os

import numpy as np
import pytest

from helpers import GOLDEN
from rapidsolid import _abi, configs, lib


def fun_cu_params():
    """The parameter set fun.cu was built with for parameters_ref.txt
    (fun.cu:57-112 macros, -D list of oracle/ref_build.sh)."""
    p = configs.default_params()
    p.nx_all, p.ny_all, p.i_tip_target = 768, 832, 768 - 268
    p.tfc, p.vp_ramp = 1, 1                       # ifTFC 1, if_Vp_ramp true
    p.cinf, p.Gamma, p.muk0, p.Tmelt, p.T_ref = 0.632514105, 199.0, 0.5795, 2750.0, 2161.59
    p.Dl, p.latent_heat, p.molar_weight = 0.9, 22003.0, 64.419
    p.v0, p.num_moles = 1.1088503429118772e-05, 90183.49558101478
    p.total_time_ns, p.Vp, p.GG = 120000.0, 0.6, 0.002
    p.eps1, p.eps2, p.epk1, p.seed = 0.02, 0.001, 0.1, 3
    return p


def test_parameters_file_is_byte_identical_to_the_reference(tmp_path):
    p = fun_cu_params()
    d = lib.derive(p)
    s = _abi.RunState(step=123, i_offset_history=7, l_offset_Vp=0.5, delta=-1.25,
                      i_left_end_initial=d.i_left_end_initial, i_left_end=d.i_left_end_initial)
    out = tmp_path / "parameters.txt"
    lib.write_parameters(out, p, s)
    ref = open(os.path.join(GOLDEN, "parameters_ref.txt"), "rb").read()
    assert out.read_bytes() == ref


def test_parameters_read_like_load_parameters():
    s = lib.read_parameters(os.path.join(GOLDEN, "parameters_ref.txt"), tfc=1)
    ref = open(os.path.join(GOLDEN, "parameters_ref_loaded.txt")).read().split()
    got = [s.step, s.i_offset_history, s.l_offset_Vp, s.delta, s.dt, s.i_left_end_initial, s.i_left_end,
           s.NxT, s.NyT, s.NxT_all, s.NyT_all, s.length_sample, s.dtT, s.ratio_dt_dtT, s.Tcold, s.Thot]
    assert len(ref) == len(got)
    for g, r in zip(got, ref):
        assert float(g) == float(r)


def test_parameters_roundtrip_without_tfc(tmp_path):
    p = configs.plain_small()
    s = _abi.RunState(step=4242, i_offset_history=-3, l_offset_Vp=1.75, delta=-4.3155, gamma0=12.0)
    lib.write_parameters(tmp_path / "p.txt", p, s)
    r = lib.read_parameters(tmp_path / "p.txt", tfc=0)
    assert (r.step, r.i_offset_history, r.l_offset_Vp, r.delta, r.gamma0) == (4242, -3, 1.75, -4.3155, 12.0)
    assert r.dt == pytest.approx(lib.derive(p).dt, rel=1e-5)   # the file carries %g


def test_truncated_parameters_are_an_error(tmp_path):
    text = open(os.path.join(GOLDEN, "parameters_ref.txt")).read()
    (tmp_path / "p.txt").write_text(text[: len(text) // 2])
    with pytest.raises(lib.RsError) as e:
        lib.read_parameters(tmp_path / "p.txt", tfc=1)
    assert e.value.code == _abi.RS_E_IO
    with pytest.raises(lib.RsError):
        lib.read_parameters(tmp_path / "missing.txt", tfc=0)


def test_check_point_layout_and_errors(tmp_path):
    rng = np.random.default_rng(1)
    a = rng.random((40, 64))
    f = tmp_path / "check_point_c.bin"
    lib.write_check_point(f, a)
    # raw FP64, i fastest, Ny_all rows (save_check_point)
    assert f.read_bytes() == a.astype("<f8").tobytes()
    assert np.array_equal(lib.read_check_point(f, 64, 40), a)
    f.write_bytes(f.read_bytes()[:-8])
    with pytest.raises(lib.RsError) as e:
        lib.read_check_point(f, 64, 40)
    assert e.value.code == _abi.RS_E_IO
    with pytest.raises(lib.RsError):
        lib.read_check_point(tmp_path / "nope.bin", 64, 40)


def test_temperature_check_point_uses_the_physical_block(tmp_path):
    L = lib.load()
    NxT, NyT, NxT_all = 10, 6, 16
    T = np.arange(NyT * NxT_all, dtype=np.float64).reshape(NyT, NxT_all)
    f = str(tmp_path / "check_point_temperature.bin").encode()
    lib.check(L.rs_write_check_point_temperature(f, T.ctypes.data, NxT, NyT, NxT_all))
    raw = np.fromfile(f.decode(), dtype=np.float64)
    assert np.array_equal(raw, T[:, :NxT].ravel())
    back = np.zeros_like(T)
    lib.check(L.rs_read_check_point_temperature(f, back.ctypes.data, NxT, NyT, NxT_all))
    assert np.array_equal(back[:, :NxT], T[:, :NxT]) and not back[:, NxT:].any()


def test_field_text_snapshot(tmp_path):
    L = lib.load()
    a = np.array([[0.1, 2.5e-7, -1.0], [1.0 / 3.0, 0.9, 12345678.0]])
    f = tmp_path / "c_0.txt"
    lib.check(L.rs_write_field_text(str(f).encode(), a.ctypes.data, 3, 2, 1, 1))
    expect = "".join("".join("%g\t" % v for v in row) + "\n" for row in a)
    assert f.read_text() == expect
