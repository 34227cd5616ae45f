"""ctypes binding of libdmffb200.so (the C ABI declared in include/dmffb200.h).

The shared library is built in-tree by ``dmff_b200/csrc/build.sh`` (or ``__graft_entry__.build``).
There is no CPU fallback: importing the engine without the library raises immediately.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdmffb200.so")

DMFFB_OK = 0
DMFFB_BAD_ARG = 1
DMFFB_OOM = 2
DMFFB_CUDA_ERROR = 3
DMFFB_NOT_CONVERGED = 4
DMFFB_NEIGHBOR_OVERFLOW = 5
DMFFB_NONFINITE = 6
DMFFB_CUFFT_ERROR = 7
DMFFB_SCRATCH_TOO_SMALL = 8
DMFFB_TIMEOUT = 9
NOALLOC_MAX_ATOMS = 65536

DMFFB_FP32 = 0
DMFFB_FP64 = 1
DMFFB_SOLVER_CG = 0
DMFFB_SOLVER_REFERENCE = 1

# every function the header declares (checked by the CPU test suite)
EXPORTED = [
    "dmffb_admp_create", "dmffb_admp_reconfigure", "dmffb_destroy", "dmffb_last_error", "dmffb_admp_set_params",
    "dmffb_admp_compute", "dmffb_admp_compute_host", "dmffb_admp_field", "dmffb_admp_multipole_grads",
    "dmffb_build_neighbors", "dmffb_admp_build_neighbors", "dmffb_engine_pairs", "dmffb_get_timings", "dmffb_set_timing",
    "dmffb_set_profiling", "dmffb_get_kernel_stats", "dmffb_get_counters", "dmffb_build_neighbors_noalloc",
    "dmffb_disp_create", "dmffb_disp_set_params", "dmffb_disp_compute", "dmffb_disp_param_grads", "dmffb_disp_set_param_grads",
    "dmffb_classical_create", "dmffb_classical_set_params", "dmffb_classical_set_terms",
    "dmffb_classical_set_param_grads", "dmffb_classical_compute", "dmffb_classical_param_grads",
    "dmffb_classical_set_cell_pass",
    "dmffb_set_graphs", "dmffb_set_fused_fft", "dmffb_fused_fft_active", "dmffb_set_persistent_cg", "dmffb_persistent_cg_blocks", "dmffb_set_cg_wait_limit", "dmffb_get_cg_phase_times", "dmffb_admp_backward", "dmffb_admp_param_grads_host", "dmffb_admp_set_param_grads", "dmffb_admp_set_zero_guess", "dmffb_admp_param_grads", "dmffb_server_create", "dmffb_server_submit", "dmffb_server_wait", "dmffb_server_clock",
    "dmffb_request_footprint", "dmffb_server_prewarm", "dmffb_server_destroy", "dmffb_md_force_create",
    "dmffb_md_force_execute", "dmffb_md_force_last_result", "dmffb_md_force_dipoles", "dmffb_md_force_destroy",
    "dmffb_pairwise_create", "dmffb_pairwise_set_params", "dmffb_pairwise_set_param_grads", "dmffb_pairwise_compute",
    "dmffb_pairwise_param_grads",
]
DMFFB_SR_TT_QQ, DMFFB_SR_SLATER_DISP, DMFFB_SR_SLATER, DMFFB_SR_TT_QQ_C6 = 0, 1, 2, 3
DMFFB_SR_QEQ_GAUSS3, DMFFB_SR_QEQ_GAUSS2 = 4, 5
SR_NPARAM = {0: 2, 1: 4, 2: 2, 3: 4, 4: 2, 5: 2}

DMFFB_COUL_NONE = 0
DMFFB_COUL_PME = 1
DMFFB_COUL_RF = 2
DMFFB_COUL_NOCUTOFF = 3
DMFFB_TERM_BOND = 0
DMFFB_TERM_ANGLE = 1
DMFFB_TERM_TORSION = 2

KERNEL_CLASSES = ["prepare", "pair_full", "pair_field", "pair_matvec", "spread", "fft", "conv", "gather_full",
                  "gather_field", "self_frames", "vector", "neighbors", "matvec_coef", "pair_full_scaled",
                  "pair_field_scaled", "param_grads", "bonded", "fft_conv", "cg_persistent"]


class AdmpDesc(ctypes.Structure):
    _fields_ = [
        ("n_atoms", ctypes.c_int32),
        ("lmax", ctypes.c_int32),
        ("lpol", ctypes.c_int32),
        ("lpme", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("rc", ctypes.c_double),
        ("kappa", ctypes.c_double),
        ("K", ctypes.c_int32 * 3),
        ("axis_types", ctypes.POINTER(ctypes.c_int32)),
        ("axis_indices", ctypes.POINTER(ctypes.c_int32)),
        ("n_cov", ctypes.c_int64),
        ("cov_rows", ctypes.POINTER(ctypes.c_int32)),
        ("mscales", ctypes.c_double * 6),
        ("pscales", ctypes.c_double * 6),
        ("dscales", ctypes.c_double * 6),
        ("solver", ctypes.c_int32),
        ("cg_tol", ctypes.c_double),
        ("max_iter", ctypes.c_int32),
        ("steps_pol", ctypes.c_int32),
    ]


class AdmpResult(ctypes.Structure):
    _fields_ = [
        ("energy", ctypes.c_double),
        ("e_real", ctypes.c_double),
        ("e_recip", ctypes.c_double),
        ("e_self", ctypes.c_double),
        ("e_pol", ctypes.c_double),
        ("box_grad", ctypes.c_double * 9),
        ("n_iter", ctypes.c_int32),
        ("converged", ctypes.c_int32),
        ("residual_rms", ctypes.c_double),
        ("n_pairs", ctypes.c_int64),
    ]


class AdmpCotangent(ctypes.Structure):
    _fields_ = [
        ("pos", ctypes.c_void_p),
        ("box", ctypes.c_double * 9),
        ("Q_local", ctypes.c_void_p),
        ("pol", ctypes.c_void_p),
        ("thole", ctypes.c_void_p),
    ]


class AdmpSecond(ctypes.Structure):
    _fields_ = [
        ("pos", ctypes.c_void_p),
        ("box", ctypes.c_double * 9),
        ("Q_local", ctypes.c_void_p),
        ("pol", ctypes.c_void_p),
        ("thole", ctypes.c_void_p),
        ("n_iter", ctypes.c_int32),
        ("residual_rms", ctypes.c_double),
        ("step", ctypes.c_double),
    ]


class MdContext(ctypes.Structure):
    _fields_ = [
        ("posq", ctypes.c_void_p),
        ("posq_double", ctypes.c_int32),
        ("force_buffer", ctypes.c_void_p),
        ("atom_index", ctypes.c_void_p),
        ("num_atoms", ctypes.c_int32),
        ("padded_num_atoms", ctypes.c_int32),
        ("box_nm", ctypes.c_double * 9),
        ("stream", ctypes.c_void_p),
    ]


class PairwiseDesc(ctypes.Structure):
    _fields_ = [
        ("n_atoms", ctypes.c_int32),
        ("kind", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("rc", ctypes.c_double),
        ("n_cov", ctypes.c_int64),
        ("cov_rows", ctypes.POINTER(ctypes.c_int32)),
        ("mscales", ctypes.c_double * 6),
        ("sign", ctypes.c_double),
    ]


class PairwiseResult(ctypes.Structure):
    _fields_ = [
        ("energy", ctypes.c_double),
        ("box_grad", ctypes.c_double * 9),
        ("n_pairs", ctypes.c_int64),
    ]


class DispDesc(ctypes.Structure):
    _fields_ = [
        ("n_atoms", ctypes.c_int32),
        ("pmax", ctypes.c_int32),
        ("lpme", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("rc", ctypes.c_double),
        ("kappa", ctypes.c_double),
        ("K", ctypes.c_int32 * 3),
        ("n_cov", ctypes.c_int64),
        ("cov_rows", ctypes.POINTER(ctypes.c_int32)),
        ("mscales", ctypes.c_double * 6),
        ("tt_damping", ctypes.c_int32),
    ]


class DispResult(ctypes.Structure):
    _fields_ = [
        ("energy", ctypes.c_double),
        ("e_real", ctypes.c_double),
        ("e_recip", ctypes.c_double),
        ("e_self", ctypes.c_double),
        ("e_sr", ctypes.c_double),
        ("box_grad", ctypes.c_double * 9),
        ("box_grad_sr", ctypes.c_double * 9),
        ("n_pairs", ctypes.c_int64),
    ]


class ClassicalDesc(ctypes.Structure):
    _fields_ = [
        ("n_atoms", ctypes.c_int32),
        ("n_types", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("coulomb", ctypes.c_int32),
        ("pbc", ctypes.c_int32),
        ("rc", ctypes.c_double),
        ("kappa", ctypes.c_double),
        ("K", ctypes.c_int32 * 3),
        ("eps_solvent", ctypes.c_double),
        ("n_cov", ctypes.c_int64),
        ("cov_rows", ctypes.POINTER(ctypes.c_int32)),
        ("mscales_coul", ctypes.c_double * 6),
        ("mscales_lj", ctypes.c_double * 6),
    ]


class ClassicalResult(ctypes.Structure):
    _fields_ = [
        ("energy", ctypes.c_double),
        ("e_coul_real", ctypes.c_double),
        ("e_coul_recip", ctypes.c_double),
        ("e_coul_self", ctypes.c_double),
        ("e_lj", ctypes.c_double),
        ("e_bond", ctypes.c_double),
        ("e_angle", ctypes.c_double),
        ("e_torsion", ctypes.c_double),
        ("box_grad", ctypes.c_double * 9),
        ("n_pairs", ctypes.c_int64),
    ]


class ServerDesc(ctypes.Structure):
    _fields_ = [
        ("n_slots", ctypes.c_int32),
        ("capacity_atoms", ctypes.c_int32),
        ("hbm_budget_bytes", ctypes.c_int64),
        ("lmax", ctypes.c_int32),
        ("lpol", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("mscales", ctypes.c_double * 6),
        ("pscales", ctypes.c_double * 6),
        ("dscales", ctypes.c_double * 6),
        ("solver", ctypes.c_int32),
        ("cg_tol", ctypes.c_double),
        ("max_iter", ctypes.c_int32),
        ("use_graphs", ctypes.c_int32),
    ]


class Request(ctypes.Structure):
    _fields_ = [
        ("n_atoms", ctypes.c_int32),
        ("pos", ctypes.c_void_p),
        ("box", ctypes.c_double * 9),
        ("axis_types", ctypes.c_void_p),
        ("axis_indices", ctypes.c_void_p),
        ("n_cov", ctypes.c_int64),
        ("cov_rows", ctypes.c_void_p),
        ("Q_local", ctypes.c_void_p),
        ("pol", ctypes.c_void_p),
        ("thole", ctypes.c_void_p),
        ("rc", ctypes.c_double),
        ("kappa", ctypes.c_double),
        ("K", ctypes.c_int32 * 3),
        ("t_arrival", ctypes.c_double),
        ("forces_out", ctypes.c_void_p),
        ("energy", ctypes.c_double),
        ("box_grad", ctypes.c_double * 9),
        ("n_iter", ctypes.c_int32),
        ("status", ctypes.c_int32),
        ("slot", ctypes.c_int32),
        ("done", ctypes.c_int32),
        ("t_start", ctypes.c_double),
        ("t_done", ctypes.c_double),
        ("footprint_bytes", ctypes.c_int64),
    ]


# C struct name of each ctypes mirror (layout checked against the header by the CPU tests)
STRUCTS = {"dmffb_admp_desc": AdmpDesc, "dmffb_admp_result": AdmpResult, "dmffb_admp_cotangent": AdmpCotangent,
           "dmffb_admp_second": AdmpSecond, "dmffb_md_context": MdContext, "dmffb_pairwise_desc": PairwiseDesc,
           "dmffb_pairwise_result": PairwiseResult, "dmffb_disp_desc": DispDesc,
           "dmffb_disp_result": DispResult, "dmffb_classical_desc": ClassicalDesc,
           "dmffb_classical_result": ClassicalResult, "dmffb_server_desc": ServerDesc, "dmffb_request": Request}

_lib = None


def load():
    """Load the engine library; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libdmffb200.so not found at {LIB_PATH}; build it with dmff_b200/csrc/build.sh")
    lib = ctypes.CDLL(LIB_PATH)
    vp, i32, i64, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    P = ctypes.POINTER
    lib.dmffb_admp_create.argtypes = [P(AdmpDesc), P(vp)]
    lib.dmffb_admp_create.restype = ctypes.c_int
    lib.dmffb_admp_reconfigure.argtypes = [vp, P(AdmpDesc)]
    lib.dmffb_destroy.argtypes = [vp]
    lib.dmffb_destroy.restype = None
    lib.dmffb_last_error.argtypes = [vp]
    lib.dmffb_last_error.restype = ctypes.c_char_p
    lib.dmffb_admp_set_params.argtypes = [vp, vp, vp, vp]
    lib.dmffb_admp_compute.argtypes = [vp, vp, vp, vp, vp, i64, vp, vp, P(AdmpResult)]
    lib.dmffb_admp_compute_host.argtypes = [vp, vp, vp, vp, i64, vp, vp, P(AdmpResult)]
    lib.dmffb_admp_field.argtypes = [vp, vp, vp, vp, vp, i64, vp, vp]
    lib.dmffb_admp_multipole_grads.argtypes = [vp, vp, vp, vp]
    lib.dmffb_admp_set_param_grads.argtypes = [vp, i32]
    lib.dmffb_admp_set_zero_guess.argtypes = [vp, i32]
    lib.dmffb_admp_param_grads.argtypes = [vp, vp, vp, vp, vp, vp]
    lib.dmffb_admp_backward.argtypes = [vp, vp, P(AdmpCotangent), P(AdmpSecond)]
    lib.dmffb_admp_param_grads_host.argtypes = [vp, vp, vp, vp]
    lib.dmffb_build_neighbors.argtypes = [vp, vp, vp, vp, dbl, vp, i64, P(i64)]
    lib.dmffb_admp_build_neighbors.argtypes = [vp, vp, vp, vp]
    lib.dmffb_engine_pairs.argtypes = [vp, vp, vp, i64, P(i64)]
    lib.dmffb_get_timings.argtypes = [vp, P(dbl), i32]
    lib.dmffb_set_timing.argtypes = [vp, i32]
    lib.dmffb_set_profiling.argtypes = [vp, i32]
    lib.dmffb_get_kernel_stats.argtypes = [vp, P(dbl), P(i64), i32]
    lib.dmffb_get_counters.argtypes = [vp, P(i64), i32]
    lib.dmffb_build_neighbors_noalloc.argtypes = [vp, vp, i32, vp, dbl, vp, vp, vp, vp, i64, P(i64)]
    lib.dmffb_disp_create.argtypes = [P(DispDesc), P(vp)]
    lib.dmffb_disp_set_params.argtypes = [vp, vp, vp, vp, vp]
    lib.dmffb_disp_compute.argtypes = [vp, vp, vp, vp, vp, i64, vp, vp, P(DispResult)]
    lib.dmffb_disp_param_grads.argtypes = [vp, vp, vp, vp]
    lib.dmffb_disp_set_param_grads.argtypes = [vp, i32]
    lib.dmffb_classical_create.argtypes = [P(ClassicalDesc), P(vp)]
    lib.dmffb_classical_set_params.argtypes = [vp, vp, vp, vp, vp]
    lib.dmffb_classical_set_terms.argtypes = [vp, i32, i64, vp, vp]
    lib.dmffb_classical_set_param_grads.argtypes = [vp, i32]
    lib.dmffb_classical_set_cell_pass.argtypes = [vp, i32]
    lib.dmffb_classical_compute.argtypes = [vp, vp, vp, vp, vp, i64, vp, P(ClassicalResult)]
    lib.dmffb_classical_param_grads.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]
    lib.dmffb_set_graphs.argtypes = [vp, i32]
    lib.dmffb_set_fused_fft.argtypes = [vp, i32]
    lib.dmffb_fused_fft_active.argtypes = [vp]
    lib.dmffb_set_persistent_cg.argtypes = [vp, i32]
    lib.dmffb_persistent_cg_blocks.argtypes = [vp]
    lib.dmffb_set_cg_wait_limit.argtypes = [vp, ctypes.c_double, i32]
    lib.dmffb_get_cg_phase_times.argtypes = [vp, vp, i32]
    lib.dmffb_server_create.argtypes = [P(ServerDesc), P(vp)]
    lib.dmffb_server_submit.argtypes = [vp, P(Request)]
    lib.dmffb_server_wait.argtypes = [vp, dbl]
    lib.dmffb_server_prewarm.argtypes = [vp, P(Request), i32]
    lib.dmffb_server_destroy.argtypes = [vp]
    lib.dmffb_server_clock.argtypes = [vp]
    lib.dmffb_request_footprint.argtypes = [i32, dbl, P(i32), dbl, i32]
    lib.dmffb_md_force_create.argtypes = [P(AdmpDesc), vp, vp, vp, P(vp)]
    lib.dmffb_md_force_execute.argtypes = [vp, P(MdContext), i32, P(dbl)]
    lib.dmffb_md_force_last_result.argtypes = [vp, P(AdmpResult)]
    lib.dmffb_md_force_dipoles.argtypes = [vp, vp, vp]
    lib.dmffb_md_force_destroy.argtypes = [vp]
    lib.dmffb_pairwise_create.argtypes = [P(PairwiseDesc), P(vp)]
    lib.dmffb_pairwise_set_params.argtypes = [vp, vp]
    lib.dmffb_pairwise_set_param_grads.argtypes = [vp, i32]
    lib.dmffb_pairwise_compute.argtypes = [vp, vp, vp, vp, vp, i64, vp, P(PairwiseResult)]
    lib.dmffb_pairwise_param_grads.argtypes = [vp, vp, vp]
    for name in EXPORTED:
        if name not in ("dmffb_destroy", "dmffb_last_error", "dmffb_server_destroy", "dmffb_server_clock",
                        "dmffb_request_footprint", "dmffb_md_force_destroy"):
            getattr(lib, name).restype = ctypes.c_int
    lib.dmffb_server_destroy.restype = None
    lib.dmffb_md_force_destroy.restype = None
    lib.dmffb_server_clock.restype = dbl
    lib.dmffb_request_footprint.restype = i64
    _lib = lib
    return lib


class EngineError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"dmffb status {status}: {msg}")
        self.status = status
