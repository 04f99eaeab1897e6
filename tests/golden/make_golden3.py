"""Generates the 3D fixture of tests/golden/ from the reference's own kernels.

The reference's 3D three-phase model (multi/peritectic_multiGPU/TiAg.cu) ships
no tests.  oracle/ref_build.sh compiles its kernels (computeMu, boundaryMu*,
diffuse, boundary*) at 32 x 32 x 20 into oracle/_ref/ref3_harness_32; this
script runs them (a GPU is needed) on a seeded input and keeps the raw FP64
outputs:

  python tests/golden/make_golden3.py OUT
      OUT/peri3d_32.npz   input (the oracle's seeded initial state: beta
                          front at z = 8 +- 0.5, one alpha cap of base radius
                          6, seed 5), mu of the input, the fields after 1 and
                          after 200 reference steps
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
import pyoracle  # noqa: E402

IC = dict(z_front=8.0, amp=0.5, n_alpha=1, cap_radius=6.0, seed=5)


def params32():
    p = pyoracle.default_params3()
    p.nx, p.ny, p.nz = 32, 32, 20
    return p


def run_reference(binary, fields, nsteps):
    with tempfile.TemporaryDirectory() as td:
        din, dout = os.path.join(td, "in"), os.path.join(td, "out")
        os.makedirs(din)
        os.makedirs(dout)
        for name, a in zip(("phi1", "phi2", "c"), fields):
            a.tofile(os.path.join(din, name + ".bin"))
        subprocess.run([binary, "step", din, dout, str(nsteps)], check=True)
        shape = fields[0].shape
        return {n: np.fromfile(os.path.join(dout, n + ".bin"), dtype=np.float64).reshape(shape)
                for n in ("phi1", "phi2", "c", "mu0")}


def main(out_dir):
    p = params32()
    f = pyoracle.initial3(p, **IC)
    binary = pyoracle.ref_binary("ref3_harness_32")
    r1 = run_reference(binary, f, 1)
    r200 = run_reference(binary, f, 200)
    os.makedirs(out_dir, exist_ok=True)
    np.savez_compressed(os.path.join(out_dir, "peri3d_32.npz"),
                        phi1=f[0], phi2=f[1], c=f[2], mu0=r1["mu0"],
                        phi1_1=r1["phi1"], phi2_1=r1["phi2"], c_1=r1["c"],
                        phi1_200=r200["phi1"], phi2_200=r200["phi2"], c_200=r200["c"],
                        ic=np.array([IC["z_front"], IC["amp"], IC["n_alpha"], IC["cap_radius"], IC["seed"]]))


if __name__ == "__main__":
    main(sys.argv[1])
