"""The oracle's coarse-grid temperature loop (TFC, the reference's production
mode ifTFC 1) against the reference's own TFC kernels: fixtures of
tests/golden/make_golden.py gpu_tfc, which ran the reference's main() loop
body (pull_back, compute_phi, compute_psi, compute_c_CALPHAD on T_fine,
integrate_phi, compute_temperature, interpolate_temperature; fun.cu:431-514,
1494-1608), built with and without FMA contraction.

The coupled loop (latent heat of the moving front into the coarse T, which
drives the front) amplifies rounding: the reference's own FMA and no-FMA
builds differ after the 500-step run by 2.3e-10 in psi and 3.6e-10 K in T.
The oracle stays within psi 5e-9, c 1e-10, T 1e-8 K of both builds
(measured: psi 1.8e-9, c 5.4e-12, T 3.0e-9 K); interior cells, the ghost
corners, which the reference writes from two racing threads, and the corner
cells of the coarse grid left out."""
import pytest

import pyoracle
from helpers import TFC_CASES, golden, maxabs, oracle_tfc_loop, tfc_input, tfc_params, tfc_T_mask


@pytest.mark.parametrize("name", sorted(TFC_CASES))
def test_oracle_tfc_loop_matches_reference_kernels(name):
    z = golden(name + ".npz")
    nx, ny, nsteps, spb = TFC_CASES[name]
    p = tfc_params(nx, ny, spb)
    d = pyoracle.derive(p)
    s, T, Tf, shifts, ile = oracle_tfc_loop(p, d, tfc_input(p), nsteps)
    assert any(shifts), shifts  # the frame moved inside the run
    for tag in ("fma", "nofma"):
        geo = list(z[f"{tag}_geometry"])
        assert geo == [d.NxT, d.NyT, d.NxT_all, d.NyT_all, d.ratio_dt_dtT, d.i_left_end_initial]
        assert list(z[f"{tag}_offsets"]) == shifts and int(z[f"{tag}_i_left_end"]) == ile
        assert maxabs(s.psi[1:-1, 1:-1], z[f"{tag}_psi"][1:-1, 1:-1]) <= 5e-9
        assert maxabs(s.c[1:-1, 1:-1], z[f"{tag}_c"][1:-1, 1:-1]) <= 1e-10
        cols = list(z[f"{tag}_T_cols"])
        m = tfc_T_mask(d, cols)
        assert maxabs(T[:d.NyT, cols][m], z[f"{tag}_T"][:d.NyT][m]) <= 1e-8  # K
        assert maxabs(Tf[1:-1, 1:-1], z[f"{tag}_T_fine"][1:-1, 1:-1]) <= 1e-8
