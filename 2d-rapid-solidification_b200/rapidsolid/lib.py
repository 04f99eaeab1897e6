"""ctypes binding of lib/librsb200.so (the C-ABI of include/rs_b200.h).

Device memory and streams come from PyTorch; every compute call goes through
the CUDA library.  There is no CPU fallback: a missing or unloadable library
raises at load time.
"""
import ctypes as C
import os

import numpy as np

from . import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "lib", "librsb200.so")

_lib = None


class RsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"rs error {code}: {msg}")
        self.code = code


def build():
    """Compile the CUDA library in-tree (nvcc, sm_100a)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", PKG, "-j4"], check=True)


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {PKG}`")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64, sz = C.c_void_p, C.c_int32, C.c_int64, C.c_size_t
    sig = {
        "rs_abi_version": ([], C.c_int),
        "rs_last_error": ([], C.c_char_p),
        "rs_sizeof_params": ([], sz),
        "rs_sizeof_step_args": ([], sz),
        "rs_default_params": ([vp], C.c_int),
        "rs_derive": ([vp, vp], C.c_int),
        "rs_create": ([vp, C.POINTER(vp)], C.c_int),
        "rs_destroy": ([vp], C.c_int),
        "rs_get_derived": ([vp, vp], C.c_int),
        "rs_step": ([vp, vp, vp, vp, vp], C.c_int),
        "rs_pull_back": ([vp, vp, vp, i32, vp], C.c_int),
        "rs_itip": ([vp, vp, vp, vp], C.c_int),
        "rs_precise_tip": ([vp, vp, vp, vp], C.c_int),
        "rs_mass": ([vp, vp, vp, vp], C.c_int),
        "rs_initial": ([vp, vp, vp], C.c_int),
        "rs_initial_planar": ([vp, vp, C.c_double, C.c_double, C.c_uint64, vp], C.c_int),
        "rs_temperature_init": ([vp, vp, vp], C.c_int),
        "rs_temperature_step": ([vp, vp, vp, vp, i64, vp], C.c_int),
        "rs_integrate_phi": ([vp, vp, vp, vp, i32, vp], C.c_int),
        "rs_interpolate_temperature": ([vp, vp, vp, i32, vp], C.c_int),
        "rs_calphad_eval": ([i32, vp, vp, vp, sz], C.c_int),
        "rs_set_option": ([vp, i32, i64], C.c_int),
        "rs_device_status": ([vp, vp], C.c_int),
        "rs_precise_tip_noalloc": ([vp, vp, vp, vp], C.c_int),
        "rs_write_parameters": ([C.c_char_p, vp, vp], C.c_int),
        "rs_read_parameters": ([C.c_char_p, i32, vp], C.c_int),
        "rs_write_check_point": ([C.c_char_p, vp, i32, i32], C.c_int),
        "rs_read_check_point": ([C.c_char_p, vp, i32, i32], C.c_int),
        "rs_write_check_point_temperature": ([C.c_char_p, vp, i32, i32, i32], C.c_int),
        "rs_read_check_point_temperature": ([C.c_char_p, vp, i32, i32, i32], C.c_int),
        "rs_write_field_text": ([C.c_char_p, vp, i32, i32, i32, i32], C.c_int),
        "rs_mlp_sample": ([vp, vp, i64, C.c_uint64, vp, vp, vp], C.c_int),
        "rs_mlp_grad": ([vp, vp, i64, vp, vp, vp, vp, vp], C.c_int),
        "rs_mlp_adam": ([vp, vp, vp, vp, i64, C.c_float, C.c_float, vp], C.c_int),
        "rs_mlp_forward": ([vp, vp, i64, vp, vp, vp], C.c_int),
        "rs_set_surrogate": ([vp, vp, vp], C.c_int),
        "rs_ensemble_create": ([vp, i32, C.POINTER(vp)], C.c_int),
        "rs_ensemble_destroy": ([vp], C.c_int),
        "rs_ensemble_context": ([vp, i32, C.POINTER(vp)], C.c_int),
        "rs_ensemble_bind": ([vp, i32, vp, vp], C.c_int),
        "rs_ensemble_steps": ([vp, i64, vp], C.c_int),
        "rs_ensemble_state": ([vp, i32, vp, vp, vp, vp], C.c_int),
        "rs_host_alloc": ([sz, C.POINTER(vp), C.POINTER(vp)], C.c_int),
        "rs_host_free": ([vp], C.c_int),
        "rs_ensemble_autotune": ([vp, i32, vp, vp, vp], C.c_int),
        "rs_ensemble_set_path": ([vp, i32], C.c_int),
        "rs_surrogate_audit": ([vp, vp, vp, vp, vp, vp], C.c_int),
        "rs3_default_params": ([vp], C.c_int),
        "rs3_sizeof_params": ([], sz),
        "rs3_create": ([vp, C.POINTER(vp)], C.c_int),
        "rs3_destroy": ([vp], C.c_int),
        "rs3_step": ([vp, vp, vp, i64, vp], C.c_int),
        "rs3_mu": ([vp, vp, vp, vp], C.c_int),
        "rs3_mass": ([vp, vp, vp, vp], C.c_int),
        "rs3_initial": ([vp, vp, C.c_double, C.c_double, i32, C.c_double, C.c_uint64, vp], C.c_int),
        "rs3_device_status": ([vp, vp], C.c_int),
        "rs3_c_offset": ([vp, vp], C.c_int),
        "rs3_initial_grains": ([vp, vp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint64, vp], C.c_int),
        "rs3_set_surrogate": ([vp, vp, vp], C.c_int),
        "rs3_surrogate_audit": ([vp, vp, vp, vp, vp, vp], C.c_int),
        "rs_mlp_sample_g": ([vp, vp, i64, C.c_uint64, vp, vp, vp], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    if L.rs_abi_version() != _abi.RS_ABI_VERSION:
        raise RuntimeError("librsb200.so ABI version mismatch: rebuild the library")
    if L.rs_sizeof_params() != C.sizeof(_abi.Params) or L.rs_sizeof_step_args() != C.sizeof(_abi.StepArgs):
        raise RuntimeError("rs_params/rs_step_args layout differs from rapidsolid._abi")
    if L.rs3_sizeof_params() != C.sizeof(_abi.Params3):
        raise RuntimeError("rs3_params layout differs from rapidsolid._abi")
    _lib = L
    return L


def check(rc):
    if rc != 0:
        raise RsError(rc, load().rs_last_error().decode())


def default_params():
    p = _abi.Params()
    check(load().rs_default_params(C.byref(p)))
    return p


def derive(p):
    d = _abi.Derived()
    check(load().rs_derive(C.byref(p), C.byref(d)))
    return d


def calphad_eval(which, T, c):
    """Host Ti-Nb evaluator: which 0 Gl, 1 Gs, 2 Glc, 3 Gsc (numpy float64 arrays)."""
    import numpy as np
    T = np.ascontiguousarray(T, dtype=np.float64)
    c = np.ascontiguousarray(c, dtype=np.float64)
    out = np.empty_like(T)
    check(load().rs_calphad_eval(which, T.ctypes.data, c.ctypes.data, out.ctypes.data, T.size))
    return out


def write_parameters(path, p, state):
    check(load().rs_write_parameters(str(path).encode(), C.byref(p), C.byref(state)))


def read_parameters(path, tfc):
    s = _abi.RunState()
    check(load().rs_read_parameters(str(path).encode(), int(tfc), C.byref(s)))
    return s


def write_check_point(path, field):
    """field: C-contiguous float64 numpy array (Ny_all, Nx_all)."""
    import numpy as np
    a = np.ascontiguousarray(field, dtype=np.float64)
    check(load().rs_write_check_point(str(path).encode(), a.ctypes.data, a.shape[1], a.shape[0]))


def read_check_point(path, nx_all, ny_all):
    import numpy as np
    a = np.empty((ny_all, nx_all))
    check(load().rs_read_check_point(str(path).encode(), a.ctypes.data, nx_all, ny_all))
    return a


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _addr(x):
    """A device-writable address: a tensor's data, or an int (e.g. a
    HostBuffer's device address), or None."""
    if x is None:
        return None
    return x if isinstance(x, int) else x.data_ptr()


class HostBuffer:
    """Mapped page-locked host memory (rs_host_alloc): `host` is a numpy view
    of it, `device` its device address (an int).  A step given
    device + 8 k as mass_out writes its mass into host[k]."""

    def __init__(self, n, dtype=np.float64):
        self.lib = load()
        self.n, self.dtype = n, np.dtype(dtype)
        h, d = C.c_void_p(), C.c_void_p()
        check(self.lib.rs_host_alloc(n * self.dtype.itemsize, C.byref(h), C.byref(d)))
        self._h = h
        self.device = d.value
        self.host = np.ctypeslib.as_array((C.c_byte * (n * self.dtype.itemsize)).from_address(h.value)).view(self.dtype)

    def close(self):
        if self._h:
            self.host = None
            self.lib.rs_host_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _stream(stream):
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


class FieldSet:
    """Device field set: psi and c (and optionally phi) as (ny_all, nx_all) tensors.

    float64 sets hold c; float32 sets hold c - cinf (see include/rs_b200.h).
    """

    def __init__(self, p, dtype, device="cuda", with_phi=False):
        import torch
        shape = (p.ny_all, p.nx_all)
        self.dtype = dtype
        self.psi = torch.zeros(shape, dtype=dtype, device=device)
        self.c = torch.zeros(shape, dtype=dtype, device=device)
        self.phi = torch.zeros(shape, dtype=dtype, device=device) if with_phi else None
        self.precision = _abi.RS_F64 if dtype == torch.float64 else _abi.RS_F32

    def fields(self):
        return _abi.Fields(c=self.c.data_ptr(), psi=self.psi.data_ptr(),
                           phi=None if self.phi is None else self.phi.data_ptr(),
                           precision=self.precision, pitch=0)


class Context:
    """One simulation context (rs_create); owns small device workspaces.
    With handle, wraps a context owned elsewhere (an ensemble run)."""

    def __init__(self, p, handle=None):
        self.lib = load()
        self.p = p
        self._owned = handle is None
        self._h = C.c_void_p()
        if handle is None:
            check(self.lib.rs_create(C.byref(p), C.byref(self._h)))
        else:
            self._h = handle
        self.d = _abi.Derived()
        check(self.lib.rs_get_derived(self._h, C.byref(self.d)))

    def close(self):
        if self._h and self._owned:
            self.lib.rs_destroy(self._h)
        self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_option(self, option, value):
        check(self.lib.rs_set_option(self._h, option, value))

    def device_status(self, stream=None):
        """Raises RsError(RS_E_STATE) if a device-side wait gave up."""
        check(self.lib.rs_device_status(self._h, _stream(stream)))

    # ---- hot path
    def step(self, cur, nxt, step, i_offset_history=0, l_offset_Vp=0.0, pull_back=None,
             T_coarse=None, i_left_end=0, i_left_end_T=0, mass_out=None, itip_out=None, stream=None):
        a = _abi.StepArgs()
        a.step = step
        a.i_offset_history = i_offset_history
        a.pull_back = 0 if pull_back is None else 1
        a.i_offset = 0 if pull_back is None else int(pull_back)
        a.i_left_end = i_left_end
        a.i_left_end_T = i_left_end_T
        a.l_offset_Vp = l_offset_Vp
        a.T_coarse = None if T_coarse is None else T_coarse.data_ptr()
        a.mass_out = _addr(mass_out)
        a.itip_out = _addr(itip_out)
        fc, fn = cur.fields(), nxt.fields()
        check(self.lib.rs_step(self._h, C.byref(fc), C.byref(fn), C.byref(a), _stream(stream)))

    def step_args_ptrs(self, cur, nxt):
        """Prebuilt (cur, next) rs_fields for callers that loop in Python."""
        return cur.fields(), nxt.fields()

    def pull_back(self, cur, nxt, i_offset, stream=None):
        fc, fn = cur.fields(), nxt.fields()
        check(self.lib.rs_pull_back(self._h, C.byref(fc), C.byref(fn), int(i_offset), _stream(stream)))

    def itip(self, fs, out, stream=None):
        f = fs.fields()
        check(self.lib.rs_itip(self._h, C.byref(f), _ptr(out), _stream(stream)))

    def mass(self, fs, out, stream=None):
        f = fs.fields()
        check(self.lib.rs_mass(self._h, C.byref(f), _ptr(out), _stream(stream)))

    def precise_tip(self, fs, out, stream=None):
        """out: a uint8 CUDA tensor of sizeof(rs_tip) bytes."""
        f = fs.fields()
        check(self.lib.rs_precise_tip(self._h, C.byref(f), _ptr(out), _stream(stream)))

    # ---- initial conditions
    def initial(self, fs, stream=None):
        f = fs.fields()
        check(self.lib.rs_initial(self._h, C.byref(f), _stream(stream)))

    def initial_planar(self, fs, c_liquid, c_solid, seed, stream=None):
        f = fs.fields()
        check(self.lib.rs_initial_planar(self._h, C.byref(f), c_liquid, c_solid, seed, _stream(stream)))

    # ---- coarse temperature
    def temperature_init(self, T, stream=None):
        check(self.lib.rs_temperature_init(self._h, _ptr(T), _stream(stream)))

    def temperature_step(self, T, T_next, dphidt, step, stream=None):
        check(self.lib.rs_temperature_step(self._h, _ptr(T), _ptr(T_next), _ptr(dphidt), step, _stream(stream)))

    def integrate_phi(self, cur, nxt, dphidt, i_left_end, stream=None):
        fc, fn = cur.fields(), nxt.fields()
        check(self.lib.rs_integrate_phi(self._h, C.byref(fc), C.byref(fn), _ptr(dphidt), int(i_left_end),
                                        _stream(stream)))

    def set_surrogate(self, w=None, box=None):
        """Use the learned CALPHAD surrogate in the FP32 step (w: RS_MLP_NPARAMS
        float32 device tensor, box: _abi.MlpBox); w None: exact evaluation."""
        check(self.lib.rs_set_surrogate(self._h, None if w is None else _ptr(w),
                                        None if box is None else C.byref(box)))

    def surrogate_audit(self, stream=None):
        """(max |mu'' error|, max |dG error|, fallback cells, audited cells) since the last call."""
        em, eg = C.c_double(), C.c_double()
        nf, na = C.c_int64(), C.c_int64()
        check(self.lib.rs_surrogate_audit(self._h, C.byref(em), C.byref(eg), C.byref(nf), C.byref(na),
                                          _stream(stream)))
        return em.value, eg.value, nf.value, na.value

    def interpolate_temperature(self, T, T_fine, i_left_end, stream=None):
        check(self.lib.rs_interpolate_temperature(self._h, _ptr(T), _ptr(T_fine), int(i_left_end), _stream(stream)))


def tip_from_bytes(buf):
    """rs_tip from a CPU uint8 tensor / bytes."""
    t = _abi.Tip()
    C.memmove(C.byref(t), bytes(buf), C.sizeof(_abi.Tip))
    return t


# the ensemble's stepping paths (include/rs_b200.h RS_ENS_PATHS): three tile
# shapes (output rows of a 128-column tile) x two launch forms x three orders
ENS_SHAPE_ROWS = (16, 8, 32)
ENS_PATHS = 6 * len(ENS_SHAPE_ROWS)


class Ensemble:
    """Batched ensemble of FP32 runs (rs_ensemble_*): one launch steps all runs,
    pull-back-free stretches replay a CUDA graph.  runs: list of _abi.Params."""

    def __init__(self, runs):
        self.lib = load()
        self.params = list(runs)
        arr = (_abi.Params * len(runs))(*runs)
        self._h = C.c_void_p()
        check(self.lib.rs_ensemble_create(arr, len(runs), C.byref(self._h)))
        self.ctx = []
        for r, p in enumerate(self.params):
            h = C.c_void_p()
            check(self.lib.rs_ensemble_context(self._h, r, C.byref(h)))
            self.ctx.append(Context(p, handle=h))
        self.sets = [None] * len(runs)

    def bind(self, run, a, b):
        fa, fb = a.fields(), b.fields()
        check(self.lib.rs_ensemble_bind(self._h, run, C.byref(fa), C.byref(fb)))
        self.sets[run] = (a, b)

    def steps(self, n, stream=None):
        check(self.lib.rs_ensemble_steps(self._h, n, _stream(stream)))

    def state(self, run):
        """(step, i_offset_history, l_offset_Vp, current field set)."""
        st, h, l, cur = C.c_int64(), C.c_int32(), C.c_double(), C.c_int32()
        check(self.lib.rs_ensemble_state(self._h, run, C.byref(st), C.byref(h), C.byref(l), C.byref(cur)))
        return st.value, h.value, l.value, self.sets[run][cur.value]

    def autotune(self, reps=5, stream=None):
        """(path, [mean ms of one step on the ENS_PATHS paths]): path k uses
        the tile shape k // 6 (ENS_SHAPE_ROWS rows by 128 columns); k % 6 =
        0-2 per-step launches (graph replays) with tile orders run by run,
        largest first, interleaved; 3-5 the persistent walk with the same
        orders."""
        ms = (C.c_double * ENS_PATHS)()
        ch = C.c_int32()
        check(self.lib.rs_ensemble_autotune(self._h, reps, ms, C.byref(ch), _stream(stream)))
        return ch.value, list(ms)

    def set_path(self, path):
        """select a stepping path (0 .. ENS_PATHS - 1, as autotune numbers them)"""
        check(self.lib.rs_ensemble_set_path(self._h, path))

    def close(self):
        for c in self.ctx:
            c.close()
        self.ctx = []
        if self._h:
            self.lib.rs_ensemble_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- 3D variant

def default_params3():
    """rs3_params with the constants of the reference's TiAg.cu (512 x 512 x 128, isothermal)."""
    p = _abi.Params3()
    check(load().rs3_default_params(C.byref(p)))
    return p


def c_offset3(p):
    """The offset of c in FP32 3D sets (rs3_c_offset): they hold c - this."""
    v = C.c_double()
    check(load().rs3_c_offset(C.byref(p), C.byref(v)))
    return v.value


class FieldSet3:
    """3D device field set: phi1, phi2, c as (nz, ny, nx) tensors; float32
    sets hold c - c_offset3(p) in c (see include/rs_b200.h)."""

    def __init__(self, p, dtype, device="cuda"):
        import torch
        shape = (p.nz, p.ny, p.nx)
        self.dtype = dtype
        self.phi1 = torch.zeros(shape, dtype=dtype, device=device)
        self.phi2 = torch.zeros(shape, dtype=dtype, device=device)
        self.c = torch.zeros(shape, dtype=dtype, device=device)
        self.precision = _abi.RS_F64 if dtype == torch.float64 else _abi.RS_F32

    def fields(self):
        return _abi.Fields3(phi1=self.phi1.data_ptr(), phi2=self.phi2.data_ptr(), c=self.c.data_ptr(),
                            precision=self.precision, reserved=0)


class Context3:
    """A 3D three-phase context (rs3_create)."""

    def __init__(self, p):
        self.lib = load()
        self.p = p
        self._h = C.c_void_p()
        check(self.lib.rs3_create(C.byref(p), C.byref(self._h)))

    def close(self):
        if self._h:
            self.lib.rs3_destroy(self._h)
        self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, cur, nxt, step, stream=None):
        a, b = cur.fields(), nxt.fields()
        check(self.lib.rs3_step(self._h, C.byref(a), C.byref(b), step, _stream(stream)))

    def mu(self, fs, out, stream=None):
        f = fs.fields()
        check(self.lib.rs3_mu(self._h, C.byref(f), _ptr(out), _stream(stream)))

    def mass(self, fs, out, stream=None):
        f = fs.fields()
        check(self.lib.rs3_mass(self._h, C.byref(f), _ptr(out), _stream(stream)))

    def initial(self, fs, z_front, amp, n_alpha, cap_radius, seed, stream=None):
        f = fs.fields()
        check(self.lib.rs3_initial(self._h, C.byref(f), z_front, amp, n_alpha, cap_radius, seed,
                                   _stream(stream)))

    def device_status(self, stream=None):
        check(self.lib.rs3_device_status(self._h, _stream(stream)))

    def initial_grains(self, fs, z_front, amp, c_liquid, c_solid, seed, stream=None):
        f = fs.fields()
        check(self.lib.rs3_initial_grains(self._h, C.byref(f), z_front, amp, c_liquid, c_solid, seed,
                                          _stream(stream)))

    def set_surrogate(self, w=None, box=None):
        """Energy 1, FP32: the learned CALPHAD surrogate (w: RS_MLP_NPARAMS float32
        device tensor trained on rs_mlp_sample_g samples, box: _abi.MlpBox); None: exact."""
        check(self.lib.rs3_set_surrogate(self._h, None if w is None else _ptr(w),
                                         None if box is None else C.byref(box)))

    def surrogate_audit(self, stream=None):
        """(max |mu'' error|, max |dG error|, fallback cells, audited cells) since the last call."""
        em, eg = C.c_double(), C.c_double()
        nf, na = C.c_int64(), C.c_int64()
        check(self.lib.rs3_surrogate_audit(self._h, C.byref(em), C.byref(eg), C.byref(nf), C.byref(na),
                                           _stream(stream)))
        return em.value, eg.value, nf.value, na.value
