"""ctypes mirror of the C-ABI structures declared in include/rs_b200.h.

The layouts here must match the header field for field; the library exports
rs_sizeof_params()/rs_sizeof_step_args() and the tests compare them.
"""
import ctypes as C

RS_ABI_VERSION = 9
RS_MLP_NPARAMS = 1250
RS_OPT_TMA = 1
RS_OPT_WAIT_LIMIT = 2
RS_OPT_PIPELINE = 3
RS_OK = 0
RS_E_INVALID = -1
RS_E_CUDA = -2
RS_E_UNSUPPORTED = -3
RS_E_STATE = -4
RS_E_IO = -5
RS_F64 = 0
RS_F32 = 1


class Params(C.Structure):
    """rs_params — run parameters (reference constants.hpp names in comments)."""
    _fields_ = [
        ("nx_all", C.c_int32), ("ny_all", C.c_int32), ("i_tip_target", C.c_int32),
        ("periodic_j", C.c_int32), ("tfc", C.c_int32), ("one_eps", C.c_int32),
        ("vp_ramp", C.c_int32), ("n_orientation", C.c_int32),
        ("cinf", C.c_double), ("W0", C.c_double), ("S", C.c_double), ("Gamma", C.c_double),
        ("muk0", C.c_double), ("Tmelt", C.c_double), ("T_ref", C.c_double), ("Dl", C.c_double),
        ("DT", C.c_double), ("latent_heat", C.c_double), ("molar_weight", C.c_double),
        ("num_moles", C.c_double), ("cp", C.c_double), ("RR", C.c_double), ("v0", C.c_double),
        ("AA", C.c_double), ("ke", C.c_double),
        ("dx", C.c_double), ("dt", C.c_double), ("GG", C.c_double), ("Vp", C.c_double),
        ("eps1", C.c_double), ("eps2", C.c_double), ("epk1", C.c_double),
        ("delta_initial", C.c_double), ("l_offset_Vp_initial", C.c_double),
        ("i_offset_history_initial", C.c_int32), ("ratio_dxT_dx", C.c_int32),
        ("orientation", C.c_double * 9),
        ("noise_amplitude", C.c_double), ("seed", C.c_uint64),
        ("Tcold", C.c_double), ("length_sample_um", C.c_double),
        ("total_time_ns", C.c_double), ("num_fields_output", C.c_int32),
        ("num_tip_output", C.c_int32), ("num_check_point_output", C.c_int32),
        ("step_pull_back", C.c_int32), ("j_offset", C.c_int32), ("band", C.c_int32),
    ]


class Derived(C.Structure):
    """rs_derived — quantities set_parameters derives (fun.cu:1984-2058)."""
    _fields_ = [
        ("tau0", C.c_double), ("deltaT0", C.c_double), ("a1", C.c_double), ("W", C.c_double),
        ("hh", C.c_double), ("h0", C.c_double), ("dt", C.c_double), ("dtT", C.c_double),
        ("length_sample", C.c_double), ("Thot", C.c_double),
        ("total_step", C.c_int64),
        ("step_fields", C.c_int32), ("step_tip", C.c_int32), ("step_check_point", C.c_int32),
        ("step_pull_back", C.c_int32), ("ratio_dt_dtT", C.c_int32), ("NxT", C.c_int32),
        ("NyT", C.c_int32), ("NxT_all", C.c_int32), ("NyT_all", C.c_int32),
        ("i_left_end_initial", C.c_int32),
    ]


class Fields(C.Structure):
    """rs_fields — one device field set (psi, c; phi optional)."""
    _fields_ = [("c", C.c_void_p), ("psi", C.c_void_p), ("phi", C.c_void_p),
                ("precision", C.c_int32), ("pitch", C.c_int32)]


class StepArgs(C.Structure):
    """rs_step_args — per-step scalars passed by value in the reference."""
    _fields_ = [
        ("step", C.c_int64), ("i_offset_history", C.c_int32), ("pull_back", C.c_int32),
        ("i_offset", C.c_int32), ("i_left_end", C.c_int32), ("i_left_end_T", C.c_int32),
        ("reserved", C.c_int32), ("l_offset_Vp", C.c_double), ("T_coarse", C.c_void_p),
        ("mass_out", C.c_void_p), ("itip_out", C.c_void_p),
    ]


class Tip(C.Structure):
    """rs_tip — precise tip (reference TIP struct, fun.cu:2612-2622)."""
    _fields_ = [("i", C.c_int32), ("j", C.c_int32), ("status", C.c_int32),
                ("reserved", C.c_int32), ("x", C.c_double), ("y", C.c_double),
                ("R", C.c_double)]


class RunState(C.Structure):
    """rs_run_state — dynamic state recorded in parameters.txt."""
    _fields_ = [
        ("step", C.c_int64), ("i_offset_history", C.c_int32), ("i_left_end_initial", C.c_int32),
        ("i_left_end", C.c_int32), ("ratio_dt_dtT", C.c_int32), ("NxT", C.c_int32), ("NyT", C.c_int32),
        ("NxT_all", C.c_int32), ("NyT_all", C.c_int32), ("l_offset_Vp", C.c_double), ("delta", C.c_double),
        ("dt", C.c_double), ("dtT", C.c_double), ("length_sample", C.c_double), ("Tcold", C.c_double),
        ("Thot", C.c_double), ("gamma0", C.c_double), ("gamma1", C.c_double), ("path_input", C.c_char_p),
    ]


class MlpBox(C.Structure):
    """rs_mlp_box — training box and output scaling of the CALPHAD surrogate."""
    _fields_ = [("T_lo", C.c_double), ("T_hi", C.c_double), ("c_lo", C.c_double), ("c_hi", C.c_double),
                ("y_mean", C.c_double * 2), ("y_scale", C.c_double * 2)]


class Params3(C.Structure):
    """rs3_params — the 3D three-phase model (TiAg.cu macro names in comments)."""
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("z_chunk", C.c_int32),
        ("dt", C.c_double),                                   # DT
        ("dx_inv", C.c_double), ("dy_inv", C.c_double), ("dz_inv", C.c_double),  # DXin ..
        ("a1", C.c_double), ("a2", C.c_double), ("a3", C.c_double), ("b", C.c_double),
        ("lam", C.c_double), ("alpha", C.c_double), ("Da", C.c_double), ("Db", C.c_double),
        ("A1", C.c_double), ("A2", C.c_double), ("B11", C.c_double), ("B12", C.c_double),
        ("B21", C.c_double), ("B22", C.c_double),
        ("T_ref", C.c_double), ("G_T", C.c_double), ("V_T", C.c_double), ("z_T", C.c_double),
        # energy 0: TiAg.cu's grand potentials; 1: Ti-Nb CALPHAD (AA, RR, c_ref apply)
        ("energy", C.c_int32), ("reserved", C.c_int32),
        ("AA", C.c_double), ("RR", C.c_double), ("c_ref", C.c_double),
    ]


class Fields3(C.Structure):
    """rs3_fields — one 3D device field set (phi1, phi2, c)."""
    _fields_ = [("phi1", C.c_void_p), ("phi2", C.c_void_p), ("c", C.c_void_p),
                ("precision", C.c_int32), ("reserved", C.c_int32)]
