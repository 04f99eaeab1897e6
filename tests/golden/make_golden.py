"""Generates the golden fixtures of tests/golden/ from the reference's own code.

The reference ships no tests or golden vectors, so its own routines, compiled
by oracle/ref_build.sh from the reference sources (old-fun.cu, constants.hpp
parameter set), are run on seeded inputs and their raw FP64 outputs kept:

  python tests/golden/make_golden.py cpu        # host routines, runs anywhere
      calphad_ref.npz   Gl, Gs, Glc, Gsc on a (T, c) grid (fun.cu:1628-1720)
      tip_ref.npz       get_itip_all_grain + get_precise_tip on psi fields
      parameters_ref.txt  save_parameters of fun.cu (its own -D list) after
                        set_parameters, step 123, i_offset_history 7,
                        l_offset_Vp 0.5, delta -1.25 (fun.cu:1984-2202)
      parameters_ref_loaded.txt  the fields load_parameters sets from it
  python tests/golden/make_golden.py gpu OUT    # reference kernels, needs a GPU
      OUT/step64.npz    64x64: pull_back(3) then 1 and 40 steps, plus the
                        nofma build (fun.cu kernels with -fmad=false)
      OUT/c1_500.npz    256x256 Ti-10Nb: pull_back(auto) then 500 steps
  python tests/golden/make_golden.py gpu_tfc OUT  # reference TFC loop, needs a GPU
      OUT/tfc_64x72.npz, OUT/tfc_256x252.npz   the reference's main() loop with
                        its production coarse-grid temperature (ifTFC 1,
                        fun.cu:431-514): pull-backs at a fixed cadence, the
                        three step kernels on the interpolated T_fine,
                        integrate_phi, ratio_dt_dtT x compute_temperature,
                        interpolate_temperature (fun.cu:1494-1608)

The inputs are built with the oracle's initial-condition routines (seeded), so
the fixtures record inputs by seed, not by value.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "2d-rapid-solidification_b200"))
sys.path.insert(0, os.path.dirname(HERE))
import pyoracle  # noqa: E402
from helpers import TFC_CASES, TFC_SEED, TFC_T_MARGIN, tfc_input, tfc_params  # noqa: E402
from rapidsolid import configs  # noqa: E402


def calphad_grid():
    T = np.concatenate([np.linspace(1150.0, 3100.0, 40), [1155.0, 1300.0, 1940.999, 1941.0, 2749.999,
                                                          2750.0, 3999.0, 4000.0, 1100.0, 298.0]])
    c = np.array([0.0, 1e-9, 1e-8, 2e-8, 1e-6, 0.01, 0.1, 0.3, 0.5, 0.632514105, 0.7, 0.8795504308633851,
                  0.9, 0.95, 0.99, 1 - 2e-8, 1 - 1e-8, 1 - 1e-9, 1.0])
    TT, CC = np.meshgrid(T, c, indexing="ij")
    return TT.ravel().copy(), CC.ravel().copy()


def run_calphad(binary):
    T, c = calphad_grid()
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.bin")
        fout = os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            np.array([float(T.size)]).tofile(f)
            T.tofile(f)
            c.tofile(f)
        subprocess.run([binary, "calphad", fin, fout], check=True)
        out = np.fromfile(fout, dtype=np.float64).reshape(-1, 4)
    return T, c, out


def tip_fields():
    """psi fields on which the reference's tip routines are evaluated."""
    fields = {}
    p64 = configs.small(64, 64, i_tip_target=24)
    d64 = pyoracle.derive(p64)
    s = pyoracle.initial_reference(p64)
    fields["ref_ic_64"] = s.psi.copy()
    s2 = pyoracle.initial_planar(p64, 0.90, configs.C_SOLID_AT_TLIQ, 11)
    fields["planar_64"] = s2.psi.copy()
    # a bump: tanh front with a Gaussian protrusion, not centred on the tip row
    i = np.arange(64)[None, :]
    j = np.arange(64)[:, None]
    i0 = 24 + 6.0 * np.exp(-((j - 37.3) / 5.0) ** 2)
    fields["bump_64"] = -np.tanh((i - i0) * 0.8 / np.sqrt(2.0))
    # the bump after 30 oracle steps
    sb = pyoracle.State(p64)
    sb.psi[:] = fields["bump_64"]
    sb.phi[:] = np.clip(sb.psi, -1, 1)
    sb.c[:] = 0.90 - (0.90 - configs.C_SOLID_AT_TLIQ) * 0.5 * (1 + sb.phi)
    fields["bump_64_30"] = pyoracle.run(p64, d64, sb, 30).psi.copy()
    # periodic wrap: protrusion across the j boundary
    i0w = 24 + 5.0 * np.exp(-((np.minimum(np.abs(j - 1.5), 62 - np.abs(j - 1.5))) / 4.0) ** 2)
    fields["wrap_64"] = -np.tanh((i - i0w) * 0.8 / np.sqrt(2.0))
    return fields


def run_tip(binary, psi):
    with tempfile.TemporaryDirectory() as td:
        f = os.path.join(td, "psi.bin")
        np.ascontiguousarray(psi, dtype=np.float64).tofile(f)
        r = subprocess.run([binary, "tip", f], check=True, capture_output=True, text=True)
    vals = r.stdout.strip().splitlines()[-1].split()
    return [float(v) for v in vals]


def make_cpu():
    b = pyoracle.ref_binary("ref_harness_64")
    T, c, out = run_calphad(b)
    np.savez_compressed(os.path.join(HERE, "calphad_ref.npz"), T=T, c=c, G=out)
    fields = tip_fields()
    names = sorted(fields)
    tips = np.array([run_tip(b, fields[n]) for n in names])
    np.savez_compressed(os.path.join(HERE, "tip_ref.npz"), names=np.array(names), tips=tips,
                        **{"psi_" + n: fields[n] for n in names})
    with tempfile.TemporaryDirectory() as td:
        subprocess.run([pyoracle.ref_binary("ref_params_harness"), "save", "123", "7", "0.5", "-1.25"], check=True,
                       cwd=td, capture_output=True)
        with open(os.path.join(td, "parameters.txt"), "rb") as f:
            data = f.read()
        loaded = subprocess.run([pyoracle.ref_binary("ref_params_harness"), "load"], check=True, cwd=td,
                                capture_output=True, text=True).stdout.strip().splitlines()[-1]
    with open(os.path.join(HERE, "parameters_ref.txt"), "wb") as f:
        f.write(data)
    # what load_parameters sets from that file: step, i_offset_history_initial,
    # l_offset_Vp_initial, delta_initial, dt, i_left_end_initial, i_left_end,
    # NxT, NyT, NxT_all, NyT_all, length_sample, dtT, ratio_dt_dtT, Tcold, Thot
    with open(os.path.join(HERE, "parameters_ref_loaded.txt"), "w") as f:
        f.write(loaded + "\n")
    print("wrote calphad_ref.npz, tip_ref.npz, parameters_ref.txt")


def write_state(d, s):
    os.makedirs(d, exist_ok=True)
    for k in ("c", "phi", "psi"):
        getattr(s, k).astype(np.float64).tofile(os.path.join(d, k + ".bin"))


def read_state(d, shape):
    return {k: np.fromfile(os.path.join(d, k + ".bin"), dtype=np.float64).reshape(shape)
            for k in ("c", "phi", "psi")}


def run_steps(binary, s, nsteps, dt, delta_initial, pull, offset, td, tag):
    din = os.path.join(td, tag + "_in")
    dout = os.path.join(td, tag + "_out")
    write_state(din, s)
    os.makedirs(dout, exist_ok=True)
    subprocess.run([binary, "step", din, dout, str(nsteps), repr(dt), repr(delta_initial), str(pull),
                    str(offset)], check=True)
    return read_state(dout, s.c.shape)


def make_gpu(out_dir):
    os.makedirs(out_dir, exist_ok=True)
    p64 = configs.small(64, 64, i_tip_target=24)
    d64 = pyoracle.derive(p64)
    s64 = pyoracle.initial_planar(p64, 0.90, configs.C_SOLID_AT_TLIQ, 3)
    res = {"in_c": s64.c, "in_psi": s64.psi, "dt": d64.dt, "delta_initial": p64.delta_initial}
    with tempfile.TemporaryDirectory() as td:
        for binname, tag in (("ref_harness_64", "fma"), ("ref_harness_64_nofma", "nofma")):
            b = pyoracle.ref_binary(binname)
            for n in (1, 40):
                r = run_steps(b, s64, n, d64.dt, p64.delta_initial, 1, 3, td, f"{tag}{n}")
                for k in ("c", "psi"):
                    res[f"{tag}_{n}_{k}"] = r[k]
    np.savez_compressed(os.path.join(out_dir, "step64.npz"), **res)

    p = configs.plain_small()
    d = pyoracle.derive(p)
    s = pyoracle.initial_planar(p, configs.C_LIQUID_TI10NB, configs.C_SOLID_AT_TLIQ, configs.IC_SEED)
    res = {"dt": d.dt, "delta_initial": p.delta_initial, "seed": configs.IC_SEED}
    with tempfile.TemporaryDirectory() as td:
        for binname, tag in (("ref_harness_256", "fma"), ("ref_harness_256_nofma", "nofma")):
            r = run_steps(pyoracle.ref_binary(binname), s, 500, d.dt, p.delta_initial, 1, "auto", td, tag)
            for k in ("c", "psi"):
                res[f"{tag}_{k}"] = r[k]
    np.savez_compressed(os.path.join(out_dir, "c1_500.npz"), **res)
    print("wrote", out_dir)


def tfc_window(d, ile, nx):
    """Coarse columns kept in a fixture: the phase-field window (integrate_phi's
    iT1 .. iTn, fun.cu:1502-1503) with a margin, and both boundary strips."""
    iT1, iTn = ile // 10, (ile + nx - 3) // 10
    lo, hi = max(iT1 - TFC_T_MARGIN, 0), min(iTn + TFC_T_MARGIN + 1, d.NxT)
    return list(range(0, 4)) + list(range(lo, hi)) + list(range(d.NxT - 4, d.NxT))


def make_gpu_tfc(out_dir):
    import re
    os.makedirs(out_dir, exist_ok=True)
    for name, (nx, ny, nsteps, spb) in TFC_CASES.items():
        p = tfc_params(nx, ny, spb)
        d = pyoracle.derive(p)
        s = tfc_input(p)
        res = {}
        for tag, suffix in (("fma", ""), ("nofma", "_nofma")):
            with tempfile.TemporaryDirectory() as td:
                din, dout = os.path.join(td, "in"), os.path.join(td, "out")
                write_state(din, s)
                os.makedirs(dout, exist_ok=True)
                r = subprocess.run([pyoracle.ref_binary(f"ref_harness_{name}{suffix}"), "tfc", din, dout,
                                    str(nsteps), repr(d.dt), repr(p.delta_initial), str(spb)], check=True,
                                   capture_output=True, text=True)
                log = r.stdout
                out = read_state(dout, s.c.shape)
                T = np.fromfile(os.path.join(dout, "T.bin"), dtype=np.float64).reshape(d.NyT_all, d.NxT_all)
                Tf = np.fromfile(os.path.join(dout, "T_fine.bin"), dtype=np.float64).reshape(s.c.shape)
            geo = re.search(r"NxT (\d+) NyT (\d+) NxT_all (\d+) NyT_all (\d+) ratio_dt_dtT (\d+) "
                            r"i_left_end_initial (-?\d+)", log).groups()
            offsets = [int(v) for v in re.findall(r"i_offset (-?\d+) i_left_end", log)]
            ile = int(re.findall(r"i_left_end (-?\d+)", log)[-1])
            cols = tfc_window(d, ile, nx)
            res.update({f"{tag}_c": out["c"], f"{tag}_psi": out["psi"], f"{tag}_T": T[:, cols],
                        f"{tag}_T_fine": Tf, f"{tag}_offsets": np.array(offsets), f"{tag}_i_left_end": ile,
                        f"{tag}_T_cols": np.array(cols), f"{tag}_geometry": np.array([int(v) for v in geo])})
            print(name, tag, "offsets", offsets, "i_left_end", ile)
        np.savez_compressed(os.path.join(out_dir, name + ".npz"), nsteps=nsteps, step_pull_back=spb,
                            seed=TFC_SEED, dt=d.dt, **res)
    print("wrote", out_dir)


if __name__ == "__main__":
    if sys.argv[1] == "cpu":
        make_cpu()
    elif sys.argv[1] == "gpu":
        make_gpu(sys.argv[2])
    elif sys.argv[1] == "gpu_tfc":
        make_gpu_tfc(sys.argv[2])
    else:
        raise SystemExit("usage: make_golden.py cpu | gpu OUT_DIR | gpu_tfc OUT_DIR")
