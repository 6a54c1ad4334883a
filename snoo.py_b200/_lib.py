"""ctypes binding of ``libsnoopy_b200.so`` (the C ABI declared in ``include/snoopy_b200.h``).

There is no fallback: importing the compute entry points without the built library, or
calling them without a CUDA device, raises.
"""

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsnoopy_b200.so")

_c_i32 = ctypes.c_int32
_c_i64 = ctypes.c_int64
_c_f64 = ctypes.c_double
_vp = ctypes.c_void_p
_pp = ctypes.POINTER(ctypes.c_void_p)


class SnpError(RuntimeError):
    """A status other than SNP_OK from the native library."""

    def __init__(self, status, message):
        super().__init__(f"{message} (status {status})")
        self.status = status


# parts of the two-phase curl-curl assembly's element records (SNP_TERMS_* in the header)
TERMS_K, TERMS_DK, TERMS_J, TERMS_F, TERMS_RHS = 1, 2, 4, 8, 16

STATUS = {0: "SNP_OK", 1: "SNP_BAD_ARG", 2: "SNP_CUDA_ERROR", 3: "SNP_NOT_CONVERGED", 4: "SNP_NAN_DETECTED",
          5: "SNP_ZERO_PIVOT", 6: "SNP_NO_MEMORY"}


class SolveOpts(ctypes.Structure):
    _fields_ = [("mode", _c_i32), ("tol", _c_f64), ("cg_maxiter", _c_i64), ("max_newton", _c_i32),
                ("cg_rtol", _c_f64), ("precision", _c_i32), ("verbose", _c_i32), ("line_search", _c_i32),
                ("res_ref", _c_f64)]


class SolveStats(ctypes.Structure):
    _fields_ = [("newton_iterations", _c_i32), ("cg_iterations", _c_i64), ("res0", _c_f64), ("res", _c_f64),
                ("t_assemble_ms", _c_f64), ("t_krylov_ms", _c_f64), ("t_total_ms", _c_f64), ("status", _c_i32),
                ("kernel_launches", _c_i64), ("residual_evals", _c_i32), ("start_dropped", _c_i32),
                ("galerkin_steps", _c_i32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchInfo(ctypes.Structure):
    _fields_ = [("problems", _c_i32), ("dofs", _c_i64), ("elements", _c_i64), ("pass1_block", _c_i32),
                ("asm_waves", _c_i32), ("graph", _c_i32), ("tuned_pass1_us", _c_f64 * 3), ("tuned_asm_us", _c_f64 * 2)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["tuned_pass1_us"] = list(self.tuned_pass1_us)
        d["tuned_asm_us"] = list(self.tuned_asm_us)
        return d


# name -> argtypes (every function returns int32 status unless listed in _RESTYPES)
_SIGS = {
    "snp_last_error": [],
    "snp_version": [],
    "snp_pattern_create": [_vp, _c_i64, _c_i32, _c_i32, _vp, _pp],
    "snp_pattern_info": [_vp, ctypes.POINTER(_c_i32), ctypes.POINTER(_c_i64), ctypes.POINTER(_c_i64),
                         ctypes.POINTER(_c_i32)],
    "snp_pattern_arrays": [_vp, _pp, _pp, _pp],
    "snp_pattern_diag": [_vp, _pp],
    "snp_pattern_destroy": [_vp],
    "snp_curlcurl_assemble": [_vp, _c_i64, _c_i64, _vp, _vp, _vp, _vp, _vp, _c_i32, _vp, _vp, _c_i32, _vp, _vp,
                              _c_i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "snp_curlcurl_assemble_diluted": [_vp, _c_i64, _c_i64, _vp, _vp, _vp, _vp, _vp, _c_i32, _vp, _vp, _vp, _c_i32,
                                      _vp, _vp, _c_i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "snp_curlcurl_assemble_f32": [_vp, _c_i64, _c_i64, _vp, _vp, _vp, _vp, _vp, _c_i32, _vp, _vp, _c_i32, _vp, _vp,
                                  _c_i32, _vp, _vp, _vp, _vp],
    "snp_curlcurl_terms_stride": [_c_i32, ctypes.POINTER(_c_i32)],
    "snp_curlcurl_rows_supported": [_vp, ctypes.POINTER(_c_i32)],
    "snp_curlcurl_terms": [_vp, _c_i64, _c_i64, _vp, _vp, _vp, _vp, _vp, _c_i32, _vp, _vp, _vp, _c_i32, _vp, _vp,
                           _c_i32, _vp, _vp, _vp, _c_i32, _vp, _vp],
    "snp_curlcurl_rows": [_vp, _vp, _c_i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "snp_solver_set_krylov": [_vp, _c_i32, _c_i32],
    "snp_curlcurl_rhs_red": [_c_i64, _vp, _vp, _vp, _vp, _vp, _c_i32, _vp, _vp, _c_i32, _vp, _vp, _c_i32, _vp, _vp,
                             _vp, _vp],
    "snp_gradgrad_assemble": [_vp, _c_i64, _c_i64, _vp, _vp, _vp, _vp, _c_i32, _vp, _c_i32, _c_i32, _c_i32, _vp, _vp,
                              _c_f64, _c_f64, _vp, _vp, _vp, _vp],
    "snp_b_hcurl": [_c_i64, _vp, _vp, _vp, _vp, _vp, _c_i32, _vp, _vp, _c_i32, _vp, _vp, _vp, _vp],
    "snp_quad_points": [_c_i64, _vp, _vp, _vp, _c_i32, _vp, _vp],
    "snp_b_at_elements": [_c_i64, _vp, _vp, _vp, _vp, _vp, _vp, _c_i32, _vp, _c_i32, _vp, _vp, _vp],
    "snp_rhs_grad_potential": [_c_i64, _vp, _vp, _vp, _vp, _vp, _c_i32, _vp, _vp, _c_i32, _vp, _vp, _vp],
    "snp_biot_savart": [_vp, _c_i64, _vp, _c_i64, _c_f64, _c_f64, _vp, _vp],
    "snp_spmv": [_c_i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "snp_pcg": [_c_i32, _vp, _vp, _vp, _vp, _vp, _vp, _c_f64, _c_f64, _c_i64, ctypes.POINTER(_c_i64),
                ctypes.POINTER(_c_f64), _vp],
    "snp_pcg_noalloc": [_c_i32, _vp, _vp, _vp, _vp, _vp, _vp, _c_f64, _c_f64, _c_i64, ctypes.POINTER(_c_i64),
                        ctypes.POINTER(_c_f64), _vp],
    "snp_solver_create": [_c_i32, _vp, _c_i64, _vp, _c_i32, _vp, _vp, _c_i32, _vp, _vp, _pp],
    "snp_solver_add_material": [_vp, _vp, _vp, _vp, _c_i64, _c_i32, _vp, _vp, _vp],
    "snp_solver_set_rhs": [_vp, _vp],
    "snp_solver_finalize": [_vp],
    "snp_solver_solve": [_vp, _vp, ctypes.POINTER(SolveOpts), ctypes.POINTER(SolveStats)],
    "snp_solver_assemble": [_vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "snp_solver_pattern": [_vp, _pp],
    "snp_solver_jacobian_apply": [_vp, ctypes.c_int, _vp, _vp, _vp],
    "snp_solver_reduced_system": [_vp, ctypes.c_int, _vp, ctypes.c_int32, ctypes.c_int64, _vp, _vp, _vp, _vp],
    "snp_solver_set_galerkin_basis": [_vp, _vp, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32],
    "snp_solver_set_block_jacobi": [_vp, _vp],
    "snp_spd_solve": [ctypes.c_int32, _vp, _vp, _vp],
    "snp_solver_block_jacobi_export": [_vp, ctypes.c_int, _vp, _vp, _vp],
    "snp_solver_precond_apply": [_vp, ctypes.c_int, _vp, _vp, ctypes.POINTER(ctypes.c_int32), _vp],
    "snp_solver_jacobian_layout": [_vp, ctypes.POINTER(ctypes.c_int)],
    "snp_solver_assemble_tensors": [_vp, _vp, ctypes.c_int, _vp, _vp],
    "snp_solver_set_nodes": [_vp, _vp, _vp],
    "snp_solver_solve_many": [_vp, _c_i32, _vp, _vp, _vp, _c_i32, _vp],
    "snp_basis_combine": [_c_i32, _vp, _c_i32, _c_i64, _vp, _c_i32, _vp, _vp, _c_i64, _vp],
    "snp_batch_create": [_vp, _c_i32, _pp],
    "snp_batch_solve": [_vp, _vp, _vp, _vp, _vp],
    "snp_batch_tune": [_vp, _c_i32],
    "snp_batch_get_info": [_vp, _vp],
    "snp_batch_destroy": [_vp],
    "snp_solver_set_source": [_vp, _c_i32, _vp, _vp],
    "snp_solver_set_dilution": [_vp, _c_i32, _vp, _vp],
    "snp_mesh_index_create": [_vp, _c_i64, _vp, _c_i64, _vp, _vp],
    "snp_mesh_index_info": [_vp, _vp, _vp, _vp, _vp],
    "snp_mesh_index_locate": [_vp, _vp, _c_i64, ctypes.c_double, _vp, _vp, _vp],
    "snp_mesh_index_nodal_average": [_vp, _vp, _c_i32, _vp, _vp, _vp],
    "snp_mesh_index_interpolate": [_vp, _c_i64, _vp, _vp, _vp, _c_i32, _c_i32, _vp, _vp, _vp],
    "snp_mesh_index_destroy": [_vp],
    "snp_gemm_bf16": [_c_i32, _c_i32, _c_i32, _vp, _c_i32, _vp, _c_i32, _vp, _c_i32, _vp, _c_i32, _vp, _c_i32, _vp,
                      _vp],
    "snp_gelu_backward": [_c_i64, _vp, _vp, _vp, _vp, _vp],
    "snp_transpose_bf16": [_c_i32, _c_i32, _vp, _c_i32, _vp, _c_i32, _vp],
    "snp_col_sum": [_c_i32, _c_i32, _vp, _c_i32, _vp, _vp],
    "snp_adam_step": [_c_i64, _vp, _vp, _vp, _vp, _vp, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                      ctypes.c_float, _c_i32, _vp],
    "snp_f32_to_bf16": [_c_i64, _vp, _vp, _vp],
    "snp_mse_grad": [_c_i64, _vp, _vp, ctypes.c_float, _vp, _vp, _vp],
    "snp_solver_destroy": [_vp],
}
_RESTYPES = {"snp_last_error": ctypes.c_char_p, "snp_version": ctypes.c_int}

EXPORTED = tuple(_SIGS)

_lib = None


def load(path=LIB_PATH):
    """Load the library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} not found: build it with `python snoo.py_b200/build_ext.py` "
                          "(or __graft_entry__.build())")
    L = ctypes.CDLL(path)
    for name, args in _SIGS.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, ctypes.c_int)
    _lib = L
    return L


def check(rc):
    if rc != 0:
        msg = load().snp_last_error().decode(errors="replace")
        raise SnpError(rc, f"{STATUS.get(rc, rc)}: {msg}")


def call(name, *args):
    """Call ``name`` and raise SnpError on a failing status."""
    check(getattr(load(), name)(*args))


def require_cuda():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("snoopy_b200 needs a CUDA device: the kernels are sm_100a CUDA with no CPU path")
    load()


def ptr(t):
    """Device pointer of a torch tensor (None for None)."""
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr())


def stream_ptr(stream=None):
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)
