"""ctypes declarations of include/b2p_pdhg.h and include/b2p_mlp.h, and the
loader of libb2p_pdhg.so.

The library is built in-tree (``make -C optimized-gpu-accelerator_b200``).
There is no fallback: if the shared library is missing, ``load()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libb2p_pdhg.so")

B2P_OK = 0
ERRORS = {1: "invalid argument", 2: "CUDA error", 3: "no usable sm_100 device", 4: "out of memory",
          5: "size beyond maximum"}
STATUS_NAMES = {0: "NotSolved", 1: "Optimal", 5: "TimeLimit", 6: "IterationLimit"}
PRECISION_FP64 = 0
PRECISION_MIXED = 1
KERNELS_AUTO, KERNELS_FUSED, KERNELS_RESIDENT = 0, 1, 2
SCHEDULE_AUTO, SCHEDULE_BINNED, SCHEDULE_TILED, SCHEDULE_TUNED = 0, 1, 2, 3
MULTI_AUTO, MULTI_GRID, MULTI_CTA = 0, 1, 2
CTA_LAYOUT_AUTO, CTA_LAYOUT_CSR = 0, 1
CTA_AUTO, CTA_GENERAL, CTA_OWNER1, CTA_OWNER2 = 0, 1, 2, 3

dptr = C.POINTER(C.c_double)
iptr = C.POINTER(C.c_int32)


class B2pLp(C.Structure):
    _fields_ = [("num_rows", C.c_int32), ("num_cols", C.c_int32), ("start", iptr), ("index", iptr),
                ("value", dptr), ("col_cost", dptr), ("col_lower", dptr), ("col_upper", dptr),
                ("row_lower", dptr), ("row_upper", dptr), ("obj_offset", C.c_double)]


class B2pCase(C.Structure):
    _fields_ = [("cost", dptr), ("col_lower", dptr), ("col_upper", dptr), ("row_lower", dptr),
                ("row_upper", dptr)]


class B2pOptions(C.Structure):
    _fields_ = [("tolerance", C.c_double), ("max_iterations", C.c_int64), ("check_every", C.c_int32),
                ("ruiz_iterations", C.c_int32), ("pock_chambolle", C.c_int32),
                ("rescale_objective_and_bounds", C.c_int32), ("reflection", C.c_double),
                ("log_interval", C.c_int32), ("device", C.c_int32), ("time_limit", C.c_double),
                ("cancel_flag", C.POINTER(C.c_int32)), ("precision", C.c_int32), ("use_graphs", C.c_int32),
                ("lanes_per_row_a", C.c_int32), ("lanes_per_row_at", C.c_int32), ("short_row_rounds", C.c_int32),
                ("kernel_mode", C.c_int32), ("spmv_schedule", C.c_int32), ("multi_form", C.c_int32),
                ("cta_smem_limit", C.c_int32), ("cta_threads", C.c_int32), ("cta_kernel", C.c_int32),
                ("batch_variant", C.c_int32), ("batch_no_compaction", C.c_int32),
                ("cta_layout", C.c_int32), ("pad_options", C.c_int32)]


class B2pStats(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("restarts", C.c_int32), ("pad0", C.c_int32),
                ("primal_residual", C.c_double), ("dual_residual", C.c_double), ("gap", C.c_double),
                ("primal_weight", C.c_double), ("setup_seconds", C.c_double), ("solve_seconds", C.c_double),
                ("kernel_seconds", C.c_double), ("transfer_seconds", C.c_double), ("bytes_uploaded", C.c_int64),
                ("bytes_downloaded", C.c_int64), ("kernel_launches", C.c_int64), ("spectral_norm", C.c_double),
                ("prepare_seconds", C.c_double), ("upload_seconds", C.c_double), ("graph_seconds", C.c_double),
                ("lanes_per_row_a", C.c_int32), ("lanes_per_row_at", C.c_int32), ("kernel_mode", C.c_int32),
                ("resident_blocks", C.c_int32), ("resident_smem_bytes", C.c_int64), ("precision_used", C.c_int32),
                ("batch_compactions", C.c_int32), ("fp32_iterations", C.c_int64), ("schedule_a", C.c_int32),
                ("schedule_at", C.c_int32), ("autotune_seconds", C.c_double), ("streaming_a", C.c_int32),
                ("streaming_at", C.c_int32), ("multi_form", C.c_int32), ("cta_threads", C.c_int32),
                ("cta_smem_bytes", C.c_int64), ("cta_lps_smem", C.c_int32), ("cta_lps_vectors", C.c_int32),
                ("cta_owned_per_thread", C.c_int32), ("tile_rows_at", C.c_int32),
                ("cases_per_thread_at", C.c_int32), ("cases_per_thread_a", C.c_int32),
                ("warp_rows_at", C.c_int32), ("warp_rows_a", C.c_int32),
                ("tile_rows_a", C.c_int32), ("cta_sliced", C.c_int32)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_ if not f.startswith("pad")}


class B2pSafeBound(C.Structure):
    _fields_ = [("bound", C.c_double), ("infinite_terms", C.c_int32), ("pad0", C.c_int32),
                ("max_dual_infeasibility", C.c_double), ("row_projection", C.c_double),
                ("cost_perturbation", C.c_double)]


class B2pResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("pad0", C.c_int32), ("iterations", C.c_int64),
                ("objective", C.c_double), ("dual_objective", C.c_double), ("relative_kkt", C.c_double)]


class B2pCertTolerances(C.Structure):
    _fields_ = [("primal_feasibility", C.c_double), ("dual_feasibility", C.c_double), ("relative_gap", C.c_double)]


class B2pCertificate(C.Structure):
    _fields_ = [("accepted", C.c_int32), ("used_implied_bounds", C.c_int32), ("primal_objective", C.c_double),
                ("safe_dual_bound", C.c_double), ("certified_gap", C.c_double),
                ("max_primal_violation", C.c_double), ("max_col_violation", C.c_double),
                ("max_row_violation", C.c_double), ("max_dual_violation", C.c_double),
                ("cost_perturbation", C.c_double), ("infinite_terms", C.c_int32), ("worst_row", C.c_int32)]


class B2pMlpTrainOptions(C.Structure):
    _fields_ = [("epochs", C.c_int32), ("batch", C.c_int32), ("lr", C.c_float), ("lr_final", C.c_float),
                ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float), ("weight_decay", C.c_float),
                ("seed", C.c_uint64)]


fptr = C.POINTER(C.c_float)
u16ptr = C.c_void_p

# Every symbol the headers declare, with its ctypes signature.
SIGNATURES = {
    "b2p_default_options": (None, [C.POINTER(B2pOptions)]),
    "b2p_solve_pdhg": (C.c_int, [C.POINTER(B2pLp), C.POINTER(B2pOptions), dptr, dptr, C.POINTER(B2pResult),
                                 C.POINTER(B2pStats)]),
    "b2p_solve_pdhg_batch": (C.c_int, [C.POINTER(B2pLp), C.POINTER(B2pCase), C.c_int32, C.POINTER(B2pOptions),
                                       dptr, dptr, C.POINTER(B2pResult), C.POINTER(B2pStats)]),
    "b2p_solve_pdhg_multi": (C.c_int, [C.POINTER(B2pLp), C.c_int32, C.POINTER(B2pOptions), C.POINTER(dptr),
                                       C.POINTER(dptr), C.POINTER(dptr), C.POINTER(dptr), C.POINTER(B2pResult),
                                       C.POINTER(B2pStats)]),
    "b2p_solve_pdhg_multi_warm": (C.c_int, [C.POINTER(B2pLp), C.c_int32, C.POINTER(B2pOptions), C.POINTER(dptr),
                                            C.POINTER(dptr), dptr, C.POINTER(dptr), C.POINTER(dptr), dptr,
                                            C.POINTER(B2pResult), C.POINTER(B2pStats)]),
    "b2p_engine_set_start": (C.c_int, [C.c_void_p, dptr, dptr, C.c_double]),
    "b2p_gpu_available": (C.c_int, []),
    "b2p_gpu_info_json": (C.c_int, [C.c_char_p, C.c_size_t]),
    "b2p_last_error": (C.c_char_p, []),
    "b2p_engine_create": (C.c_int, [C.POINTER(B2pLp), C.POINTER(B2pCase), C.c_int32, C.POINTER(B2pOptions),
                                    C.POINTER(C.c_void_p)]),
    "b2p_engine_solve": (C.c_int, [C.c_void_p, C.POINTER(B2pResult), C.POINTER(B2pStats)]),
    "b2p_engine_fetch": (C.c_int, [C.c_void_p, dptr, dptr]),
    "b2p_engine_destroy": (C.c_int, [C.c_void_p]),
    "b2p_engine_set_profiling": (C.c_int, [C.c_void_p, C.c_int32]),
    "b2p_engine_kernel_times": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_int64), dptr]),
    "b2p_engine_kernel_bytes": (C.c_int, [C.c_void_p, C.c_int32, dptr]),
    "b2p_csr_spmv": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, iptr, iptr, dptr, dptr, dptr]),
    "b2p_safe_dual_bound": (C.c_int, [C.POINTER(B2pLp), C.POINTER(B2pCase), C.c_int32, dptr,
                                      C.POINTER(B2pSafeBound)]),
    "b2p_implied_bounds": (C.c_int, [C.POINTER(B2pLp), C.POINTER(B2pCase), C.c_int32, dptr, dptr]),
    "b2p_certify_lp": (C.c_int, [C.POINTER(B2pLp), C.POINTER(B2pCase), C.c_int32, dptr, dptr,
                                 C.POINTER(B2pCertTolerances), C.POINTER(B2pCertificate)]),
    "b2p_kkt_residual": (C.c_int, [C.POINTER(B2pLp), C.POINTER(B2pCase), C.c_int32, dptr, dptr, dptr]),
    "b2p_kkt_residual_noalloc": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p]),
    # include/b2p_mlp.h
    "b2p_mlp_default_train_options": (B2pMlpTrainOptions, []),
    "b2p_mlp_create": (C.c_int, [iptr, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    "b2p_mlp_destroy": (C.c_int, [C.c_void_p]),
    "b2p_mlp_num_params": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "b2p_mlp_set_params": (C.c_int, [C.c_void_p, fptr]),
    "b2p_mlp_get_params": (C.c_int, [C.c_void_p, fptr]),
    "b2p_mlp_forward": (C.c_int, [C.c_void_p, fptr, C.c_int64, fptr]),
    "b2p_mlp_forward_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]),
    "b2p_mlp_loss_grad": (C.c_int, [C.c_void_p, fptr, fptr, C.c_int32, dptr, fptr]),
    "b2p_mlp_train": (C.c_int, [C.c_void_p, fptr, fptr, C.c_int64, C.POINTER(B2pMlpTrainOptions), fptr]),
    "b2p_mlp_gemm_bf16": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, u16ptr, C.c_int64, C.c_int64, u16ptr,
                                    C.c_int64, C.c_int64, C.c_float, C.c_void_p, C.c_int32, u16ptr, C.c_int64,
                                    C.c_void_p, C.c_int64, u16ptr, C.c_int64, C.c_void_p]),
    "b2p_mlp_gemm_bf16_time": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, u16ptr, C.c_int64, C.c_int64, u16ptr,
                                         C.c_int64, C.c_int64, C.c_void_p, C.c_int64, C.c_int32, dptr]),
}

_lock = threading.Lock()
_lib = None


class B2pError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{ERRORS.get(code, 'error')} ({code}): {message}")
        self.code = code


def load():
    """Load libb2p_pdhg.so (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `make -C optimized-gpu-accelerator_b200` "
                "(the PDHG engine has no CPU fallback)")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(rc: int) -> None:
    if rc != B2P_OK:
        raise B2pError(rc, load().b2p_last_error().decode(errors="replace"))
