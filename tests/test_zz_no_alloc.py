"""rs_precise_tip_noalloc: the precise tip for hosts that cannot allocate.

Some hosts own all device memory through their own pool allocator, or must
keep cudaMalloc's device-wide synchronisation out of their time loop; they
cannot give the tip tracker the context workspace that rs_create allocates.
The no-allocation entry point keeps its per-row scratch in a static device
array instead.  Here it is called through the C-ABI twice in a row, on two
different fields, and each result is checked against rs_precise_tip (which
uses the context workspace); the second call also shows that the scratch
left over from the first call does not leak into the result.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import pyoracle
from helpers import golden, perturbed_state
from rapidsolid import _abi, configs, lib

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _tip_buffer():
    return torch.zeros(C.sizeof(_abi.Tip), dtype=torch.uint8, device="cuda")


def _noalloc(p, fs, out):
    L = lib.load()
    f = fs.fields()
    rc = L.rs_precise_tip_noalloc(C.byref(p), C.byref(f), C.c_void_p(out.data_ptr()),
                                  C.c_void_p(torch.cuda.current_stream().cuda_stream))
    lib.check(rc)


def _same(a, b):
    assert (a.i, a.j, a.status) == (b.i, b.j, b.status)
    for k in ("x", "y", "R"):
        va, vb = getattr(a, k), getattr(b, k)
        assert abs(va - vb) <= 1e-12 * max(1.0, abs(vb)), k


def test_noalloc_tip_matches_context_tip_twice():
    # field 1: the reference-tracked bump of the tip fixture, FP64 64x64
    z = golden("tip_ref.npz")
    p1 = configs.small(64, 64, i_tip_target=24)
    f1 = lib.FieldSet(p1, torch.float64)
    f1.psi.copy_(torch.from_numpy(z["psi_bump_64_30"]))
    # field 2: an evolved perturbed front, FP32 160x96 (more rows than field 1)
    p2 = configs.small(160, 96, i_tip_target=50, G=5e6, V=0.5)
    d2 = pyoracle.derive(p2)
    s2 = pyoracle.run(p2, d2, perturbed_state(p2, 41, amp=0.7), 40)
    f2 = lib.FieldSet(p2, torch.float32)
    f2.psi.copy_(torch.from_numpy(s2.psi.astype(np.float32)))

    results = []
    for p, fs in ((p1, f1), (p2, f2)):
        ref_out, na_out = _tip_buffer(), _tip_buffer()
        ctx = lib.Context(p)
        ctx.precise_tip(fs, ref_out)
        _noalloc(p, fs, na_out)
        torch.cuda.synchronize()
        ref = lib.tip_from_bytes(ref_out.cpu().numpy().tobytes())
        got = lib.tip_from_bytes(na_out.cpu().numpy().tobytes())
        _same(got, ref)
        results.append(got)
        ctx.close()
    assert (results[0].i, results[0].j) != (results[1].i, results[1].j)


def test_noalloc_tip_rejects_too_many_rows():
    p = configs.small(64, 64, i_tip_target=24)
    fs = lib.FieldSet(p, torch.float64)
    big = configs.small(64, _abi_max_rows() + 2, i_tip_target=24)
    out = _tip_buffer()
    L = lib.load()
    f = fs.fields()
    rc = L.rs_precise_tip_noalloc(C.byref(big), C.byref(f), C.c_void_p(out.data_ptr()), None)
    assert rc == _abi.RS_E_INVALID
    assert b"RS_NOALLOC_TIP_MAX_ROWS" in L.rs_last_error()


def _abi_max_rows():
    import os
    import re
    from helpers import ROOT
    txt = open(os.path.join(ROOT, "include", "rs_b200.h")).read()
    return int(re.search(r"#define RS_NOALLOC_TIP_MAX_ROWS (\d+)", txt).group(1))
