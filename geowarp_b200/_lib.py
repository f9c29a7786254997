"""ctypes binding of the C ABI declared in include/geowarp_b200.h.

The product path has no fallback: if the shared library is missing or fails to
load, importing the engine raises.  Structures mirror the C structs field by
field; every call's status is checked and turned into a GeoWarpError.
"""
import ctypes as C
import os

from .build import LIB

# ---------------------------------------------------------------- constants (include/geowarp_b200.h)
GW_OK, GW_EINVAL, GW_ECUDA, GW_ENOCONV, GW_EBREAKDOWN, GW_ENAN, GW_ERANGE, GW_EMODEL = 0, -1, -2, -3, -4, -5, -6, -7
KIND_SOLID2D, KIND_COUPLED2D, KIND_COUPLED3D = 0, 1, 2
MODEL_HENCKY, MODEL_J2, MODEL_NEOHOOKEAN, MODEL_LINEAR, MODEL_DP, MODEL_NORSAND = range(6)
PREC_F64, PREC_F32 = 0, 1
PRECOND_DIAG, PRECOND_BLOCK = 0, 1
KRYLOV_BICGSTAB, KRYLOV_CG, KRYLOV_GMRES = 0, 1, 2
(TUNE_PARTICLE_BLOCK, TUNE_ADJOINT_BLOCK, TUNE_ROW_WARPS, TUNE_MG_COARSE, TUNE_MG_ONE_SWEEP, TUNE_MG_SWEEPS,
 TUNE_MG_OMEGA, TUNE_GS_CANCEL, TUNE_MG_TAIL, TUNE_MG_BF16, TUNE_MG_FINE_SWEEPS, TUNE_GMRES_STALL,
 TUNE_COUNT) = range(13)


class GeoWarpError(RuntimeError):
    def __init__(self, code, where, msg):
        super().__init__(f"{where}: {msg} (status {code})")
        self.code = code


class Grid(C.Structure):
    _fields_ = [("dim", C.c_int32), ("kind", C.c_int32), ("nf", C.c_int32), ("n_grid", C.c_int32 * 3),
                ("n_nodes", C.c_int32), ("pad0", C.c_int32),
                ("h", C.c_double * 3), ("inv_h", C.c_double * 3), ("h_nodes", C.c_double * 3),
                ("domain_min", C.c_double * 3), ("domain_max", C.c_double * 3)]


class Material(C.Structure):
    _fields_ = [("model", C.c_int32), ("dp_tension_cutoff", C.c_int32),
                ("youngs_modulus", C.c_double), ("poisson_ratio", C.c_double), ("kappa", C.c_double),
                ("friction_angle", C.c_double), ("dilation_angle", C.c_double), ("cohesion", C.c_double),
                ("shape_factor", C.c_double),
                ("ns_kappa", C.c_double), ("ns_tilde_lambda", C.c_double), ("ns_M", C.c_double),
                ("ns_N", C.c_double), ("ns_beta", C.c_double), ("ns_vc0", C.c_double), ("ns_p0", C.c_double),
                ("ns_v0", C.c_double), ("ns_h", C.c_double), ("ns_shear_modulus", C.c_double),
                ("ns_eps_v0", C.c_double), ("dp_tip_tangent", C.c_double)]


class Step(C.Structure):
    _fields_ = [("current_step", C.c_double), ("total_steps", C.c_double), ("gravity_mag", C.c_double),
                ("point_load", C.c_double * 3), ("traction", C.c_double * 3),
                ("p_vol", C.c_double), ("p_rho", C.c_double), ("PPD", C.c_double),
                ("dt", C.c_double), ("phi_initial", C.c_double), ("mobility", C.c_double), ("lp0", C.c_double),
                ("has_footing", C.c_int32), ("footing_stable", C.c_int32),
                ("footing_min", C.c_double * 2), ("footing_max", C.c_double * 2),
                ("footing_initial_height", C.c_double), ("footing_incr_disp", C.c_double),
                ("penalty_factor", C.c_double), ("gravity_full", C.c_int32), ("mobility_law", C.c_int32)]


class Particles(C.Structure):
    _fields_ = [("n", C.c_int32), ("pad0", C.c_int32),
                ("x", C.c_void_p), ("x0", C.c_void_p), ("lp", C.c_void_p),
                ("F_old", C.c_void_p), ("F_new", C.c_void_p), ("b_old", C.c_void_p), ("b_new", C.c_void_p),
                ("sigma", C.c_void_p), ("pressure", C.c_void_p), ("pi_old", C.c_void_p), ("pi_new", C.c_void_p),
                ("ext_flag", C.c_void_p), ("trac_flag", C.c_void_p), ("pbc_flag", C.c_void_p), ("E", C.c_void_p)]


class Bsr(C.Structure):
    _fields_ = [("n_rows", C.c_int32), ("nf", C.c_int32), ("nnzb", C.c_int32), ("mask_words", C.c_int32),
                ("row_ptr", C.c_void_p), ("cols", C.c_void_p), ("row2node", C.c_void_p), ("node2row", C.c_void_p),
                ("stencil", C.c_void_p), ("vals", C.c_void_p)]


MG_MAX_LEVELS = 20


class MgPlan(C.Structure):
    _fields_ = [("levels", C.c_int32), ("dense_n", C.c_int32), ("n_rows", C.c_int32 * MG_MAX_LEVELS),
                ("nnzb", C.c_int32 * MG_MAX_LEVELS), ("nf", C.c_int32), ("fine_n_rows", C.c_int32),
                ("fine_nnzb", C.c_int32), ("lag", C.c_int32), ("workspace", C.c_void_p),
                ("row_ptr", C.c_void_p), ("cols", C.c_void_p), ("last_iters", C.c_int32), ("pad0", C.c_int32)]


class Adjoint(C.Structure):
    _fields_ = [("x", C.c_void_p), ("lp", C.c_void_p), ("F", C.c_void_p), ("b", C.c_void_p), ("E", C.c_void_p)]


P = C.c_void_p
I32 = C.c_int32
I64 = C.c_int64
PI32 = C.POINTER(C.c_int32)
PD = C.POINTER(C.c_double)

# name -> (restype, argtypes)
SIGNATURES = {
    "gw_version": (C.c_int, []),
    "gw_status_string": (C.c_char_p, [C.c_int]),
    "gw_read_device_status": (C.c_int, [PI32, P]),
    "gw_guard_read": (C.c_int, [PI32, C.POINTER(C.c_int64), P]),
    "gw_guard_site_name": (C.c_char_p, [I32]),
    "gw_sort_workspace_bytes": (I64, [I32]),
    "gw_cell_sort": (C.c_int, [C.POINTER(Grid), C.POINTER(Particles), P, P, P, P]),
    "gw_p2g_activate": (C.c_int, [C.POINTER(Grid), C.POINTER(Particles), P, P, P, P, P]),
    "gw_touched_nodes": (C.c_int, [C.POINTER(Grid), P, P, P]),
    "gw_compact_rows": (C.c_int, [C.POINTER(Grid), P, P, P, P, P, PI32, P, P]),
    "gw_scan_workspace_bytes": (I64, [I32]),
    "gw_pattern_count": (C.c_int, [C.POINTER(Grid), P, P, P, I32, P, P, PI32, P, P]),
    "gw_pattern_fill": (C.c_int, [C.POINTER(Grid), C.POINTER(Bsr), P, P]),
    "gw_mass_assemble": (C.c_int, [C.POINTER(Grid), C.POINTER(Particles), P, C.POINTER(Step), C.POINTER(Bsr), P, P]),
    "gw_mass_lumped_solve": (C.c_int, [C.POINTER(Bsr), P, P, P]),
    "gw_set_nodal_pressure": (C.c_int, [C.POINTER(Grid), P, I32, P, P, P, P, P, P]),
    "gw_assemble": (C.c_int, [C.POINTER(Grid), C.POINTER(Material), C.POINTER(Step), C.POINTER(Particles), P, P, P, P,
                              C.POINTER(Bsr), I32, P, P, P]),
    "gw_assemble_workspace_bytes": (I64, [C.POINTER(Grid), I32, I32]),
    "gw_assemble_sorted": (C.c_int, [C.POINTER(Grid), C.POINTER(Material), C.POINTER(Step), C.POINTER(Particles), P,
                                     P, P, P, P, C.POINTER(Bsr), I32, P, P, P, I64, P]),
    "gw_krylov_workspace_bytes": (I64, [I32, I32, I32]),
    "gw_bsr_krylov_solve": (C.c_int, [C.POINTER(Bsr), I32, I32, I32, P, P, C.c_double, I32, P, PI32, PD, P]),
    "gw_krylov_static_max_unknowns": (I64, []),
    "gw_bsr_krylov_solve_static": (C.c_int, [C.POINTER(Bsr), I32, I32, I32, P, P, C.c_double, I32, PI32, PD, P]),
    "gw_gmres_workspace_bytes": (I64, [I32, I32, I32]),
    "gw_gmres_mg_workspace_bytes": (I64, [C.POINTER(Grid), I32, I32, I32]),
    "gw_mg_plan_build": (C.c_int, [C.POINTER(Grid), C.POINTER(Bsr), P, I64, C.POINTER(MgPlan), P]),
    "gw_bsr_gmres_mg_solve": (C.c_int, [C.POINTER(Grid), C.POINTER(Bsr), I32, C.POINTER(MgPlan), P, P, C.c_double, I32,
                                        I32, P, I64, PI32, PD, P]),
    "gw_gmres_last_reorths": (I32, []),
    "gw_gmres_last_stalled": (I32, []),
    "gw_bsr_gmres_solve": (C.c_int, [C.POINTER(Bsr), I32, I32, P, P, C.c_double, I32, I32, P, PI32, PD, P]),
    "gw_bsr_spmv": (C.c_int, [C.POINTER(Bsr), I32, P, P, P]),
    "gw_bsr_spmv_t": (C.c_int, [C.POINTER(Bsr), I32, P, P, P]),
    "gw_norm2": (C.c_int, [P, I32, P, P, P]),
    "gw_apply_increment": (C.c_int, [C.POINTER(Bsr), P, P, P]),
    "gw_predict_increment": (C.c_int, [C.POINTER(Bsr), P, P, P, P]),
    "gw_g2p": (C.c_int, [C.POINTER(Grid), C.POINTER(Step), C.POINTER(Particles), P, P, P]),
    "gw_return_map": (C.c_int, [C.POINTER(Material), I32, P, P, P, P, P, P, P, P]),
    "gw_profile_enable": (C.c_int, [I32]),
    "gw_profile_count": (C.c_int, []),
    "gw_launch_count": (I64, []),
    "gw_tune_set": (C.c_int, [I32, I32]),
    "gw_tune_get": (I32, [I32]),
    "gw_profile_reset": (C.c_int, []),
    "gw_profile_read": (C.c_int, [I32, PD, C.POINTER(C.c_int64), PD]),
    "gw_profile_name": (C.c_char_p, [I32]),
    "gw_bsr_transpose": (C.c_int, [C.POINTER(Grid), C.POINTER(Bsr), I32, P, P]),
    "gw_adjoint_g2p": (C.c_int, [C.POINTER(Grid), C.POINTER(Material), C.POINTER(Step), C.POINTER(Particles), P, P,
                                 P, C.POINTER(Bsr), C.POINTER(Adjoint), C.POINTER(Adjoint), P, P]),
    "gw_adjoint_residual": (C.c_int, [C.POINTER(Grid), C.POINTER(Material), C.POINTER(Step), C.POINTER(Particles),
                                      P, P, P, C.POINTER(Bsr), P, C.POINTER(Adjoint), P]),
}

_lib = None


def load(path=None):
    """Load the shared library (raises if it is missing).  The environment
    variable GEOWARP_B200_LIB names another build of it (a variant compiled for
    an A/B timing); the default is the in-tree library."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or os.environ.get("GEOWARP_B200_LIB") or LIB
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: run geowarp_b200.build.build() (the engine has no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(code, where):
    if code != GW_OK:
        msg = load().gw_status_string(code)
        raise GeoWarpError(code, where, msg.decode() if msg else "")
    return code


def call(name, *args):
    return check(getattr(load(), name)(*args), name)


def exported_symbols():
    return list(SIGNATURES)
