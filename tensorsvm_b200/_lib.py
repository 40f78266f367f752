"""ctypes binding of the C ABI in include/tensorsvm.h (libtensorsvm_b200.so).

This mirrors, one to one, the entry points a ctypes user of the library binds; the product
path is the CUDA library itself.  Loading fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libtensorsvm_b200.so")
CLI_PATH = os.path.join(_HERE, "bin", "tensorsvm-train")

# tsvm_status
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_CUDA = 2
ERR_OUT_OF_MEMORY = 3
ERR_NOT_SPD = 4
ERR_UNSUPPORTED = 5
ERR_NO_DEVICE = 6
ERR_TIMEOUT = 7
WARN_ILL_CONDITIONED = 8
WARN_MAX_ITER = 9
ERR_SKETCH = 10
ERR_IO = 11
ERR_COMM = 12

KERNEL_LINEAR = 0
KERNEL_RBF = 2
PREC_FP32 = 0
PREC_BF16 = 1
PREC_FP16 = 2
PREC_BF16_FAST = 3
PREC_FP16_FAST = 4
SKETCH_GLIBC = 0
SKETCH_USER = 1
SKETCH_PHILOX = 2

# every symbol include/tensorsvm.h and include/tensorsvm_testing.h declare
EXPORTS = [
    "tsvm_status_string", "tsvm_create", "tsvm_destroy", "tsvm_set_stream",
    "tsvm_ipm_default_options",
    "tsvm_factor", "tsvm_linear_factor", "tsvm_ipm", "tsvm_bias", "tsvm_bias_noalloc",
    "tsvm_train", "tsvm_kernel_launches", "tsvm_ipm_batched", "tsvm_hypergrad",
    "tsvm_decision_values", "tsvm_predict", "tsvm_kernel_residual", "tsvm_train_residual",
    "tsvm_read_libsvm", "tsvm_free", "tsvm_write_model", "tsvm_read_model", "tsvm_free_model",
    "tsvm_set_comm", "tsvm_factor_rows", "tsvm_set_sketch_seed", "tsvm_factor_batched",
    "tsvm_set_factor_keep",
]
TEST_EXPORTS = [
    "tsvm_test_rand_stream", "tsvm_test_sketch", "tsvm_test_kermatmul", "tsvm_test_chol",
    "tsvm_test_potrs", "tsvm_test_eig", "tsvm_test_gram", "tsvm_test_syrk_mixed",
    "tsvm_test_grid_barrier", "tsvm_test_fail_alloc", "tsvm_test_sketch_philox",
    "tsvm_test_kprod", "tsvm_test_kermatmul_half", "tsvm_test_kermatmul_cols",
    "tsvm_test_kermatmul_half_cols", "tsvm_test_eig_batched",
]


# int (*allreduce)(void *user, void *buf, int64_t count, int32_t dtype, int32_t op, void *stream)
ALLREDUCE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p)


class Comm(ctypes.Structure):
    _fields_ = [("rank", ctypes.c_int32), ("world", ctypes.c_int32),
                ("allreduce", ALLREDUCE_FN), ("user", ctypes.c_void_p)]


class FactorProblem(ctypes.Structure):
    _fields_ = [("X", ctypes.c_void_p), ("y", ctypes.c_void_p), ("n", ctypes.c_int64),
                ("gamma", ctypes.c_double), ("Z", ctypes.c_void_p)]


class IpmProblem(ctypes.Structure):
    _fields_ = [("Z", ctypes.c_void_p), ("y", ctypes.c_void_p), ("n", ctypes.c_int64),
                ("C", ctypes.c_double), ("alpha_out", ctypes.c_void_p),
                ("xi_out", ctypes.c_void_p)]


class BatchInfo(ctypes.Structure):
    _fields_ = [("units", ctypes.c_int32), ("unit_rows", ctypes.c_int32),
                ("graph_used", ctypes.c_int32), ("iters_max", ctypes.c_int32),
                ("ms_total", ctypes.c_double), ("ms_autotune", ctypes.c_double)]


class HypergradResult(ctypes.Structure):
    _fields_ = [("loss", ctypes.c_double), ("dloss_dlog_gamma", ctypes.c_double),
                ("dloss_dlog_C", ctypes.c_double), ("n_free_bias", ctypes.c_int32),
                ("ms", ctypes.c_double), ("factor_reused", ctypes.c_int32)]


class ModelView(ctypes.Structure):
    _fields_ = [("kernel", ctypes.c_int32), ("d", ctypes.c_int32), ("nsv", ctypes.c_int64),
                ("sv", ctypes.c_void_p), ("coef", ctypes.c_void_p), ("rho", ctypes.c_double),
                ("gamma", ctypes.c_double)]


class FactorInfo(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int64), ("d", ctypes.c_int32), ("k", ctypes.c_int32),
                ("k_padded", ctypes.c_int32), ("realk", ctypes.c_int32),
                ("precision", ctypes.c_int32),
                ("eig_max", ctypes.c_double), ("eig_min", ctypes.c_double),
                ("ms_sketch", ctypes.c_double), ("ms_pass1", ctypes.c_double),
                ("ms_ortho", ctypes.c_double), ("ms_pass2", ctypes.c_double),
                ("ms_project", ctypes.c_double), ("ms_total", ctypes.c_double),
                ("ms_kermatmul_kernel", ctypes.c_double), ("flops_kermatmul", ctypes.c_double)]


class IpmOptions(ctypes.Structure):
    _fields_ = [("max_iter", ctypes.c_int32), ("tol", ctypes.c_double),
                ("rel_gap_tol", ctypes.c_double), ("precision", ctypes.c_int32),
                ("refine_sweeps", ctypes.c_int32), ("kernel", ctypes.c_int32),
                ("verbose", ctypes.c_int32)]


class IpmStats(ctypes.Structure):
    _fields_ = [("iters", ctypes.c_int32), ("status", ctypes.c_int32),
                ("mu", ctypes.c_double), ("norm_rd", ctypes.c_double),
                ("norm_rp", ctypes.c_double), ("cond_d", ctypes.c_double),
                ("pobj", ctypes.c_double), ("dobj", ctypes.c_double),
                ("rel_gap", ctypes.c_double), ("ms_total", ctypes.c_double),
                ("ms_syrk", ctypes.c_double), ("ms_factor", ctypes.c_double),
                ("ms_streams", ctypes.c_double), ("t_rel_gap_1e6_ms", ctypes.c_double),
                ("mixed_syrk", ctypes.c_int32), ("syrk_retries", ctypes.c_int32),
                ("exact_rows_max", ctypes.c_int32), ("exact_rows_mean", ctypes.c_double),
                ("refine_res_max", ctypes.c_double)]


_lib = None


def load() -> ctypes.CDLL:
    """Load libtensorsvm_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"tensorsvm CUDA library not built: {LIB_PATH} (run `make`)")
    lib = ctypes.CDLL(LIB_PATH)
    P, I32, I64, D = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    lib.tsvm_status_string.restype = ctypes.c_char_p
    lib.tsvm_status_string.argtypes = [ctypes.c_int]
    lib.tsvm_create.restype = ctypes.c_int
    lib.tsvm_create.argtypes = [ctypes.POINTER(P), ctypes.c_int]
    lib.tsvm_destroy.restype = ctypes.c_int
    lib.tsvm_destroy.argtypes = [P]
    lib.tsvm_set_stream.restype = ctypes.c_int
    lib.tsvm_set_stream.argtypes = [P, P]
    lib.tsvm_ipm_default_options.restype = None
    lib.tsvm_ipm_default_options.argtypes = [ctypes.POINTER(IpmOptions)]
    lib.tsvm_factor.restype = ctypes.c_int
    lib.tsvm_factor.argtypes = [P, P, P, I64, I32, D, I32, I32, I32, P, P, I32,
                                ctypes.POINTER(FactorInfo)]
    lib.tsvm_set_factor_keep.restype = ctypes.c_int
    lib.tsvm_set_factor_keep.argtypes = [P, I32]
    lib.tsvm_set_sketch_seed.restype = ctypes.c_int
    lib.tsvm_set_sketch_seed.argtypes = [P, ctypes.c_uint64]
    lib.tsvm_factor_batched.restype = ctypes.c_int
    lib.tsvm_factor_batched.argtypes = [P, ctypes.POINTER(FactorProblem), I32, I32, I32, I32,
                                        I32, I32, ctypes.POINTER(FactorInfo)]
    lib.tsvm_set_comm.restype = ctypes.c_int
    lib.tsvm_set_comm.argtypes = [P, ctypes.POINTER(Comm)]
    lib.tsvm_factor_rows.restype = ctypes.c_int
    lib.tsvm_factor_rows.argtypes = [P, P, P, I64, I32, I64, I64, D, I32, I32, I32, P, P, I32,
                                     ctypes.POINTER(FactorInfo)]
    lib.tsvm_linear_factor.restype = ctypes.c_int
    lib.tsvm_linear_factor.argtypes = [P, P, P, I64, I32, P, I32]
    lib.tsvm_ipm.restype = ctypes.c_int
    lib.tsvm_ipm.argtypes = [P, P, I32, P, I64, I32, D, ctypes.POINTER(IpmOptions), P, P, P,
                             ctypes.POINTER(D), ctypes.POINTER(IpmStats)]
    lib.tsvm_bias.restype = ctypes.c_int
    lib.tsvm_bias.argtypes = [P, P, I32, P, P, I64, I32, D, ctypes.POINTER(D), ctypes.POINTER(D),
                              ctypes.POINTER(I32), ctypes.POINTER(I32)]
    lib.tsvm_bias_noalloc.restype = ctypes.c_int
    lib.tsvm_bias_noalloc.argtypes = [P, I32, P, P, I64, I32, D, P, P]
    lib.tsvm_train.restype = ctypes.c_int
    lib.tsvm_train.argtypes = [P, P, P, I64, I32, I32, D, D, I32, I32, ctypes.POINTER(IpmOptions),
                               P, ctypes.POINTER(D), ctypes.POINTER(FactorInfo),
                               ctypes.POINTER(IpmStats)]
    lib.tsvm_ipm_batched.restype = ctypes.c_int
    lib.tsvm_ipm_batched.argtypes = [P, ctypes.POINTER(IpmProblem), I32, I32, I32,
                                     ctypes.POINTER(IpmOptions), ctypes.POINTER(IpmStats),
                                     ctypes.POINTER(BatchInfo)]
    lib.tsvm_hypergrad.restype = ctypes.c_int
    lib.tsvm_hypergrad.argtypes = [P, P, P, I64, I32, P, P, I64, D, D, I32, I32, P, P, P, D, D,
                                   ctypes.POINTER(HypergradResult), P]
    MV = ctypes.POINTER(ModelView)
    PD = ctypes.POINTER(D)
    PP = ctypes.POINTER(P)
    PI64 = ctypes.POINTER(I64)
    for name, res, args in [
        ("tsvm_decision_values", ctypes.c_int, [P, MV, P, I64, P]),
        ("tsvm_predict", ctypes.c_int, [P, MV, P, I64, P]),
        ("tsvm_kernel_residual", ctypes.c_int, [P, P, P, I64, I32, D, P, I32, I32, PD, PD]),
        ("tsvm_train_residual", ctypes.c_int, [P, PD, PD]),
        ("tsvm_read_libsvm", ctypes.c_int, [ctypes.c_char_p, I32, I32, PP, PP, PI64, PI64, PI64,
                                            PI64]),
        ("tsvm_free", None, [P]),
        ("tsvm_write_model", ctypes.c_int, [ctypes.c_char_p, I32, P, P, P, I64, I32, D, D, D, I32,
                                            I32, I32, PI64, PI64]),
        ("tsvm_read_model", ctypes.c_int, [ctypes.c_char_p, MV, ctypes.POINTER(I32),
                                           ctypes.POINTER(I32)]),
        ("tsvm_free_model", None, [MV]),
    ]:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    lib.tsvm_kernel_launches.restype = ctypes.c_int64
    lib.tsvm_kernel_launches.argtypes = [P]
    # test hooks (include/tensorsvm_testing.h)
    for name, args in {
        "tsvm_test_rand_stream": [P, I64, P],
        "tsvm_test_sketch": [P, I64, P],
        "tsvm_test_kermatmul": [P, P, P, I64, I32, D, P, I32, P, I32, I32],
        "tsvm_test_kermatmul_half": [P, P, P, I64, I32, D, P, I32, P, P, I32, I32],
        "tsvm_test_kermatmul_cols": [P, P, P, I64, I32, D, P, I32, I32, P, I32, I32],
        "tsvm_test_eig_batched": [P, P, I32, I32, P, P, P],
        "tsvm_test_kermatmul_half_cols": [P, P, P, I64, I32, D, P, I32, I32, P, P, I32, I32],
        "tsvm_test_sketch_philox": [P, ctypes.c_uint64, I64, P],
        "tsvm_test_kprod": [P, P, I64, P, I64, I32, D, P, I32, P, I32, I32],
        "tsvm_test_chol": [P, P, I32, ctypes.POINTER(I32)],
        "tsvm_test_potrs": [P, P, I32, P, I32, I32],
        "tsvm_test_eig": [P, P, I32, P, P, ctypes.POINTER(I32)],
        "tsvm_test_gram": [P, P, I64, P, I64, I64, I32, I32, I32, P, P],
        "tsvm_test_syrk_mixed": [P, P, I32, I64, I32, P, D, I32, P, ctypes.POINTER(I32)],
        "tsvm_test_grid_barrier": [P, I32, I32, I64, ctypes.POINTER(I32)],
        "tsvm_test_fail_alloc": [P, I32],
    }.items():
        fn = getattr(lib, name)
        fn.restype = ctypes.c_int
        fn.argtypes = args
    _lib = lib
    return lib


class TsvmError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        msg = load().tsvm_status_string(status).decode()
        super().__init__(f"{where}: {msg} (status {status})")


def check(status: int, where: str, allow=()) -> int:
    if status != OK and status not in allow:
        raise TsvmError(status, where)
    return status


def default_options(**kw) -> IpmOptions:
    o = IpmOptions()
    load().tsvm_ipm_default_options(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class Context:
    """Owns a tsvm_context (one CUDA device, one stream)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        self.handle = ctypes.c_void_p()
        check(self.lib.tsvm_create(ctypes.byref(self.handle), device), "tsvm_create")

    def close(self):
        if self.handle:
            self.lib.tsvm_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_factor_keep(self, on: bool) -> None:
        """Keep each factor's state for tsvm_hypergrad (tsvm_set_factor_keep)."""
        check(self.lib.tsvm_set_factor_keep(self.handle, 1 if on else 0), "tsvm_set_factor_keep")

    def set_stream(self, stream_handle: int) -> None:
        """Issue all work on the given cudaStream_t (e.g. torch.cuda.Stream().cuda_stream)."""
        check(self.lib.tsvm_set_stream(self.handle, ctypes.c_void_p(stream_handle)), "tsvm_set_stream")

    @property
    def launches(self) -> int:
        return int(self.lib.tsvm_kernel_launches(self.handle))
