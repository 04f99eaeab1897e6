"""Training of the learned CALPHAD surrogate on the GPU (rs_mlp_* entry points).

The network (3 -> 32 -> 32 -> 2, SiLU) maps (T, c, phi) scaled over a box to
the chemical potential relative to the melt's column value (mu'') and the
driving force Gl - Gs; the training data are evaluated by the exact FP64
evaluator on the GPU (rs_mlp_sample), the gradients by the library's own
backward kernel (rs_mlp_grad) and the update by its Adam kernel
(rs_mlp_adam).  PyTorch only holds the buffers and shuffles the indices.
"""
import ctypes as C
import math

import numpy as np

from . import _abi, configs
from .lib import _ptr, _stream, check, load


def default_box(T_sol=configs.T_SOLIDUS_TI10NB, T_liq=configs.T_LIQUIDUS_TI10NB):
    """T in [T_solidus - 200, T_liquidus + 50] K, x_Nb in [0.001, 0.40]
    (c = x_Ti in [0.60, 0.999]; c -> 1 is left out, where log(1 - c) diverges)."""
    b = _abi.MlpBox()
    b.T_lo, b.T_hi = T_sol - 200.0, T_liq + 50.0
    b.c_lo, b.c_hi = 0.60, 0.999
    b.y_mean[0] = b.y_mean[1] = 0.0
    b.y_scale[0] = b.y_scale[1] = 1.0
    return b


def fitted_box(T_sol=configs.T_SOLIDUS_TI10NB, T_liq=configs.T_LIQUIDUS_TI10NB):
    """A box around the states the Ti-10Nb runs visit: T in [T_solidus - 30,
    T_liquidus + 10] K, c in [0.84, 0.96]; cells outside fall back to the
    exact evaluation."""
    b = default_box(T_sol, T_liq)
    b.T_lo, b.T_hi = T_sol - 30.0, T_liq + 10.0
    b.c_lo, b.c_hi = 0.84, 0.96
    return b


def ensemble_box(params):
    """A box over every run of an ensemble: T from 200 K below the lowest
    front temperature (each run starts at its solidus) to 80 K above the
    highest, c = x_Ti in [0.60, 0.999] (x_Nb <= 0.40, as the wide box)."""
    Ts = [p.Tmelt + p.delta_initial * (p.Tmelt - p.T_ref) for p in params]
    b = default_box()
    b.T_lo, b.T_hi = min(Ts) - 200.0, max(Ts) + 80.0
    return b


def init_weights(seed=0):
    """Glorot-uniform weights, zero biases, as a float32 numpy vector."""
    rng = np.random.default_rng(seed)
    w = np.zeros(_abi.RS_MLP_NPARAMS, dtype=np.float32)
    H = 32

    def glorot(n_out, n_in):
        a = math.sqrt(6.0 / (n_in + n_out))
        return rng.uniform(-a, a, size=(n_out, n_in)).astype(np.float32)
    o = 0
    w[o:o + H * 3] = glorot(H, 3).ravel(); o += H * 3 + H
    w[o:o + H * H] = glorot(H, H).ravel(); o += H * H + H
    w[o:o + 2 * H] = glorot(2, H).ravel()
    return w


def sample(p, box, n, seed, stream=None, g_input=False):
    """n samples over the box: (T, c, phi) inputs of the 2D model, or with
    g_input (T, c, g) of the 3D model's energy 1 (rs_mlp_sample_g)."""
    import torch
    x = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    y = torch.empty((n, 2), dtype=torch.float32, device="cuda")
    fn = load().rs_mlp_sample_g if g_input else load().rs_mlp_sample
    check(fn(C.byref(p), C.byref(box), n, seed, _ptr(x), _ptr(y), _stream(stream)))
    return x, y


def grad(box, w, x, y, stream=None):
    """(gradient, loss) of sum |out - scaled y|^2 over the samples."""
    import torch
    g = torch.zeros(_abi.RS_MLP_NPARAMS, dtype=torch.float32, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    check(load().rs_mlp_grad(C.byref(box), _ptr(w), x.shape[0], _ptr(x), _ptr(y), _ptr(g), _ptr(loss),
                             _stream(stream)))
    return g, loss


def forward(box, w, x, stream=None):
    import torch
    out = torch.empty((x.shape[0], 2), dtype=torch.float32, device="cuda")
    check(load().rs_mlp_forward(C.byref(box), _ptr(w), x.shape[0], _ptr(x), _ptr(out), _stream(stream)))
    return out


def train(p, box=None, n_samples=1 << 20, epochs=20, batch=4096, lr=3e-3, seed=1, verbose=False, g_input=False):
    """Returns (weights float32 cuda tensor, box with output scaling, history).
    g_input: the 3D model's inputs (T, c, g), p a 2D parameter set whose cinf
    is the 3D context's c_ref."""
    import torch
    L = load()
    box = default_box() if box is None else box
    x, y = sample(p, box, n_samples, seed, g_input=g_input)
    ym, ys = y.double().mean(0), y.double().std(0)
    for q in range(2):
        box.y_mean[q], box.y_scale[q] = float(ym[q]), float(ys[q])
    w = torch.from_numpy(init_weights(seed)).cuda()
    m, v = torch.zeros_like(w), torch.zeros_like(w)
    g = torch.zeros_like(w)
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    st = _stream(None)
    t, hist = 0, []
    nb = n_samples // batch
    for ep in range(epochs):
        perm = torch.randperm(n_samples, device="cuda", generator=gen)
        xs, ysh = x[perm].contiguous(), y[perm].contiguous()
        loss.zero_()
        lr_ep = lr * 0.5 * (1.0 + math.cos(math.pi * ep / epochs))  # cosine schedule
        for b in range(nb):
            xb, yb = xs[b * batch:(b + 1) * batch], ysh[b * batch:(b + 1) * batch]
            g.zero_()
            check(L.rs_mlp_grad(C.byref(box), _ptr(w), batch, _ptr(xb), _ptr(yb), _ptr(g), _ptr(loss), st))
            t += 1
            check(L.rs_mlp_adam(_ptr(w), _ptr(g), _ptr(m), _ptr(v), t, lr_ep, 1.0 / batch, st))
        mse = loss.item() / (nb * batch * 2)
        hist.append(mse)
        if verbose:
            print(f"epoch {ep}: scaled mse {mse:.3e}", flush=True)
    return w, box, hist


def errors(box, w, x, y):
    """Max and RMS absolute error of the raw outputs (mu'', dG) in J/mol."""
    out = forward(box, w, x)
    e = (out.double() - y.double()).abs()
    return e.max(0).values.tolist(), e.pow(2).mean(0).sqrt().tolist()
