"""ctypes binding of libamigo_b200.so (the C ABI in include/amigo_b200.h).

The library is built in-tree by ``python -m amigo_b200.build``.  Importing
this module never falls back to another implementation: a missing library
raises immediately.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libamigo_b200.so")

AB_OK = 0
AB_ERR = {
    -1: "bad argument",
    -2: "CUDA runtime error",
    -3: "not factored",
    -4: "unsupported option",
    -5: "non-finite pivot in the factorization",
    -6: "workspace capacity",
}

_i = ctypes.c_int
_d = ctypes.c_double
_vp = ctypes.c_void_p
_ip = ctypes.POINTER(ctypes.c_int)
_dp = ctypes.POINTER(ctypes.c_double)


class IpmProblem(ctypes.Structure):
    _fields_ = [("n", _i), ("np", _i), ("nc", _i), ("pidx", _vp),
                ("cidx", _vp), ("lbx", _vp), ("ubx", _vp), ("lbh", _vp),
                ("mu_inst", _vp), ("pinst", _vp), ("vinst", _vp),
                ("ninst", _i), ("poff", _vp), ("coff", _vp)]


class IpmState(ctypes.Structure):
    _fields_ = [("xlam", _vp), ("zl", _vp), ("zu", _vp), ("sl", _vp),
                ("su", _vp)]


class Simp2DStruct(ctypes.Structure):
    """Mirror of ab_simp2d (include/amigo_b200.h)."""
    _fields_ = ([(k, _i) for k in ("n", "nnz", "nelems", "nnodes", "u0", "rt0",
                                   "re0", "s_index", "lam0", "mu0", "nu_index")]
                + [("color_ptr", _i * 5)]
                + [(k, _vp) for k in ("color_elems", "ev", "fv", "epos", "fpos",
                                      "vpos", "spos", "fixed", "fixed_zero_pos",
                                      "fixed_diag_pos", "load_idx", "load_val",
                                      "K0", "A")]
                + [(k, _i) for k in ("nfixed", "nfixed_zero", "nload")]
                + [(k, _d) for k in ("Bq", "vcoef", "volfrac", "E0", "Emin",
                                     "penalty")])


class Simp3DStruct(ctypes.Structure):
    """Mirror of ab_simp3d (include/amigo_b200.h)."""
    _fields_ = ([(k, _i) for k in ("n", "nnz", "nelems", "nnodes", "u0", "rt0",
                                   "re0", "s_index", "lam0", "mu0", "nu_index")]
                + [("color_ptr", _i * 9)]
                + [(k, _vp) for k in ("color_elems", "ev", "fv", "epos", "fpos",
                                      "vpos", "spos", "fixed", "fixed_zero_pos",
                                      "fixed_diag_pos", "load_idx", "load_val",
                                      "K0", "A")]
                + [(k, _i) for k in ("nfixed", "nfixed_zero", "nload")]
                + [(k, _d) for k in ("Bq", "vcoef", "volfrac", "E0", "Emin",
                                     "penalty")])


class CartPoleStruct(ctypes.Structure):
    """Mirror of ab_cartpole (include/amigo_b200.h)."""
    _fields_ = ([(k, _i) for k in ("n", "nnz", "N")]
                + [(k, _d) for k in ("h", "M", "m", "l", "g")]
                + [(k, _vp) for k in ("iv", "ipos", "bv", "bpos", "h_iv", "m_iv")]
                + [("nbc", _i), ("ninst", _i), ("inst_iv", _vp)])


class BctlStruct(ctypes.Structure):
    """Mirror of ab_bctl (include/amigo_b200.h): device arrays of ninst."""
    DOUBLES = ("mu", "nu", "dw", "dc", "dwf", "dcf", "dw_last", "alpha", "az",
               "phi0", "dphi", "ratio", "ratio_old", "nrm", "e0")
    INTS = ("live", "pending", "search", "on", "its", "n_ic", "retire",
            "np_each", "nc_each", "n_each")
    _fields_ = ([("ninst", _i)] + [(k, _vp) for k in DOUBLES]
                + [(k, _vp) for k in INTS] + [("flags", _vp)])


class BctlOpts(ctypes.Structure):
    """Mirror of ab_bctl_opts."""
    NAMES = ("tol", "mu_min", "kappa_eps", "kappa_mu", "theta_mu", "dw_first",
             "dw_min", "dw_max", "kw_plus_first", "kw_plus", "kw_minus", "dc",
             "kappa_c", "armijo")
    _fields_ = [(k, _d) for k in NAMES] + [("max_iter", _i)]


BCTL_RETIRED, BCTL_LIVE, BCTL_IC_PENDING, BCTL_REFINING, BCTL_STALLED, \
    BCTL_SEARCHING, BCTL_MISMATCH = range(7)
BCTL_NFLAGS = 8

_BC = ctypes.POINTER(BctlStruct)
_BO = ctypes.POINTER(BctlOpts)

# name -> (restype, argtypes)
_SIGS = {
    "ab_bctl_clear_flags": (_i, [_BC, _vp]),
    "ab_bctl_converge_barrier": (_i, [_BC, _BO, _vp, _vp]),
    "ab_bctl_ic_begin": (_i, [_BC, _vp]),
    "ab_bctl_shift_diag": (_i, [_BC, _i, _vp, _vp, _vp, _vp, _vp]),
    "ab_bctl_ic_step": (_i, [_BC, _BO, _vp, _vp]),
    "ab_bctl_ic_end": (_i, [_BC, _vp]),
    "ab_bctl_ic_check": (_i, [_BC, _vp, _vp]),
    "ab_bctl_refine_init": (_i, [_BC, _vp, _vp]),
    "ab_bctl_refine_step": (_i, [_BC, _vp, _i, _vp]),
    "ab_bctl_refine_stalled": (_i, [_BC, _vp]),
    "ab_bctl_mask_update": (_i, [_BC, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "ab_bctl_ls_begin": (_i, [_BC, _vp, _vp, _vp]),
    "ab_bctl_ls_test": (_i, [_BC, _BO, _vp, _vp, _vp]),
    "ab_bctl_end": (_i, [_BC, _vp]),
    "ab_ldl_inertia_device": (_i, [_vp, ctypes.POINTER(_vp)]),
    "ab_ldl_set_solve_queue": (_i, [_vp, _i]),
    "ab_ldl_solve_status": (_i, [_vp, _vp]),
    "ab_ldl_autotune": (_i, [_vp, _vp, _i, _vp, _vp]),
    "ab_ldl_apply_tuning": (_i, [_vp, _vp]),
    "ab_ldl_create": (_i, [_i, _ip, _ip, _i, _i, _d, _d, _d, ctypes.POINTER(_vp)]),
    "ab_ldl_analyze": (_i, [_i, _ip, _ip, _i, ctypes.POINTER(_vp)]),
    "ab_ldl_destroy": (_i, [_vp]),
    "ab_ldl_mem_estimate": (_i, [_vp, _i, _d, _i, ctypes.POINTER(ctypes.c_longlong)]),
    "ab_ldl_symbolic_sizes": (_i, [_vp, _ip, _ip]),
    "ab_ldl_symbolic_arrays": (_i, [_vp, _ip, _ip, _ip, _ip, _ip, _ip, _ip]),
    "ab_ldl_factor": (_i, [_vp, _vp, _vp]),
    "ab_ldl_inertia": (_i, [_vp, _vp, _ip, _ip]),
    "ab_ldl_solve": (_i, [_vp, _vp, _i, _i, _vp]),
    "ab_ldl_stats": (_i, [_vp, _vp, _dp, _dp, _ip, _ip, _ip]),
    "ab_ldl_node_pivots": (_i, [_vp, _vp, _ip, _ip]),
    "ab_ldl_batch_create": (_i, [_i, _ip, ctypes.POINTER(_ip), ctypes.POINTER(_ip),
                                 _i, _i, _d, _d, _d, ctypes.POINTER(_vp)]),
    "ab_ldl_batch_inertia": (_i, [_vp, _vp, _ip, _ip]),
    "ab_ldl_batch_sizes": (_i, [_vp, _ip, _ip, ctypes.POINTER(ctypes.c_longlong)]),
    "ab_ipm_residual": (_i, [ctypes.POINTER(IpmProblem), ctypes.POINTER(IpmState),
                             _d, _vp, _vp, _vp, _vp]),
    "ab_ipm_diagonal": (_i, [ctypes.POINTER(IpmProblem), ctypes.POINTER(IpmState),
                             _vp, _vp]),
    "ab_ipm_bound_dual_step": (_i, [ctypes.POINTER(IpmProblem),
                                    ctypes.POINTER(IpmState), _d, _vp, _vp,
                                    _vp, _vp]),
    "ab_ipm_max_step": (_i, [ctypes.POINTER(IpmProblem), ctypes.POINTER(IpmState),
                             _d, _vp, _vp, _vp, _vp, _vp, _vp]),
    "ab_ipm_max_step_noalloc": (_i, [ctypes.POINTER(IpmProblem),
                                     ctypes.POINTER(IpmState), _d, _vp, _vp,
                                     _vp, _vp, _vp, _vp]),
    "ab_ipm_apply_step": (_i, [ctypes.POINTER(IpmProblem), ctypes.POINTER(IpmState),
                               _d, _d, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                               _vp]),
    "ab_ipm_reductions": (_i, [ctypes.POINTER(IpmProblem), ctypes.POINTER(IpmState),
                               _d, _vp, _vp, _vp]),
    "ab_ipm_barrier_dphi": (_i, [ctypes.POINTER(IpmProblem),
                                 ctypes.POINTER(IpmState), _d, _vp, _vp, _vp,
                                 _vp]),
    "ab_ipm_reset_bound_multipliers": (_i, [ctypes.POINTER(IpmProblem),
                                            ctypes.POINTER(IpmState), _d, _d,
                                            _vp, _vp, _vp]),
    "ab_ipm_affine_start_point": (_i, [ctypes.POINTER(IpmProblem),
                                       ctypes.POINTER(IpmState), _d, _vp, _vp,
                                       _vp, _vp, _vp]),
    "ab_ipm_barrier_dphi_kkt": (_i, [ctypes.POINTER(IpmProblem),
                                     ctypes.POINTER(IpmState), _vp, _vp, _vp,
                                     _vp, _vp]),
    "ab_ipm_relax_bounds": (_i, [_i, _vp, _vp, _vp, _vp, _d, _d, _vp]),
    "ab_ipm_initialize": (_i, [ctypes.POINTER(IpmProblem), _vp, _vp, _vp, _vp,
                               _vp, _d, _d, _vp]),
    "ab_ipm_seg_reduce": (_i, [ctypes.POINTER(IpmProblem), ctypes.POINTER(IpmState),
                               _d, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "ab_ipm_apply_step_seg": (_i, [ctypes.POINTER(IpmProblem),
                                   ctypes.POINTER(IpmState), _vp, _vp, _vp, _vp,
                                   _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "ab_ipm_refine_init": (_i, [ctypes.POINTER(IpmProblem), ctypes.POINTER(IpmState),
                                _d, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "ab_ipm_refine_residual": (_i, [ctypes.POINTER(IpmProblem),
                                    ctypes.POINTER(IpmState), _d, _vp, _vp, _vp,
                                    _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "ab_ipm_refine_update": (_i, [ctypes.POINTER(IpmProblem),
                                  ctypes.POINTER(IpmState), _vp, _vp, _vp, _vp,
                                  _vp, _vp, _vp]),
    "ab_ipm_refine_init_seg": (_i, [ctypes.POINTER(IpmProblem),
                                    ctypes.POINTER(IpmState), _vp, _vp, _vp,
                                    _vp, _vp, _vp, _vp]),
    "ab_ipm_refine_residual_seg": (_i, [ctypes.POINTER(IpmProblem),
                                        ctypes.POINTER(IpmState), _vp, _vp,
                                        _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                        _vp, _vp]),
    "ab_ipm_refine_update_seg": (_i, [ctypes.POINTER(IpmProblem),
                                      ctypes.POINTER(IpmState), _vp, _vp, _vp,
                                      _vp, _vp, _vp, _vp, _vp]),
    "ab_launch_count": (ctypes.c_longlong, []),
    "ab_ldl_set_wide_threshold": (_i, [_vp, ctypes.c_longlong]),
    "ab_ldl_set_cluster_threshold": (_i, [_vp, ctypes.c_longlong]),
    "ab_ldl_set_panel_mode": (_i, [_vp, _i, _i]),
    "ab_ldl_set_precision": (_i, [_vp, _i]),
    "ab_ldl_set_tensor_cores": (_i, [_vp, _i]),
    "ab_ldl_set_panel_cache": (_i, [_vp, _i]),
    "ab_tc_syrk_tf32x3": (_i, [_i, _i, _vp, _i, _vp, _i, _vp, _i, _vp, _vp]),
    "ab_csr_add_diagonal": (_i, [_i, _vp, _vp, _vp, _vp]),
    "ab_vec_absmax_gather": (_i, [_i, _vp, _vp, _vp, _vp]),
    "ab_ipm_constraint_scale": (_i, [_i, _i, _vp, _vp, _vp, _d, _d, _vp, _vp,
                                     _vp, _vp]),
    "ab_csr_scale_symmetric": (_i, [_i, _vp, _vp, _vp, _vp, _vp]),
    "ab_vec_scale_gather": (_i, [_i, _vp, _vp, _vp, _i, _vp]),
    "ab_ipm_initialize_slacks": (_i, [_i, _vp, _vp, _vp, _vp, _vp]),
    "ab_ipm_dual_residual_vector": (_i, [_i, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "ab_vec_copy_gather": (_i, [_i, _vp, _vp, _vp, _vp]),
    "ab_csr_matvec": (_i, [_i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "ab_cartpole_gradient": (_i, [ctypes.POINTER(CartPoleStruct), _vp, _d, _vp, _vp]),
    "ab_cartpole_hessian": (_i, [ctypes.POINTER(CartPoleStruct), _vp, _d, _vp, _vp]),
    "ab_cartpole_objective": (_i, [ctypes.POINTER(CartPoleStruct), _vp, _vp, _vp]),
    "ab_simp3d_gradient": (_i, [ctypes.POINTER(Simp3DStruct), _vp, _d, _vp, _vp]),
    "ab_simp3d_hessian": (_i, [ctypes.POINTER(Simp3DStruct), _vp, _d, _vp, _vp]),
    "ab_simp2d_gradient": (_i, [ctypes.POINTER(Simp2DStruct), _vp, _d, _vp, _vp]),
    "ab_simp2d_hessian": (_i, [ctypes.POINTER(Simp2DStruct), _vp, _d, _vp, _vp]),
}

_lib = None


def exported_symbols():
    """Names of every entry point the binding declares."""
    return sorted(_SIGS)


def lib():
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                "libamigo_b200.so is not built (run python -m amigo_b200.build); "
                "there is no fallback implementation")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class AmigoB200Error(RuntimeError):
    def __init__(self, name, code):
        super().__init__("%s failed: %s (%d)" % (name, AB_ERR.get(code, "error"), code))
        self.code = code


def check(name, code):
    if code < 0:
        raise AmigoB200Error(name, code)
    return code


def call(name, *args):
    return check(name, getattr(lib(), name)(*args))
