"""ctypes binding of ``libartefact_b200.so`` (the C ABI in include/artefact_b200.h).

The library is the only compute path: importing this module raises if it is
missing, and every solver call goes to the CUDA kernels it contains.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libartefact_b200.so"

ART_OK = 0
ART_ERR_INVALID_ARGUMENT = -1
ART_ERR_INVALID_DATA = -2
ART_ERR_CUDA = -3
ART_ERR_DECODE = -4
ART_ERR_UNSUPPORTED = -5

ART_COEF_F32 = 0
ART_COEF_I16 = 1
ART_INIT_DECODED = 0
ART_INIT_SCALAR_COMPAT = 1
ART_INIT_LEARNED = 2


class ArtChannel(C.Structure):
    _fields_ = [
        ("rounded_px_w", C.c_uint32),
        ("rounded_px_h", C.c_uint32),
        ("block_w", C.c_uint32),
        ("block_h", C.c_uint32),
        ("samp_h", C.c_uint32),
        ("samp_v", C.c_uint32),
        ("coef_type", C.c_uint32),
        ("reserved", C.c_uint32),
        ("dct_coefs", C.c_void_p),
        ("quant_table", C.POINTER(C.c_float)),
    ]


class ArtOptions(C.Structure):
    _fields_ = [
        ("init_mode", C.c_uint32),
        ("device", C.c_int32),
        ("step_iterations", C.c_uint32),
        ("tail_iterations", C.c_uint32),
        ("tail_step_iterations", C.c_uint32),
        ("step_decay", C.c_float),
        ("reserved", C.c_uint32 * 2),
    ]


class ArtImage(C.Structure):
    _fields_ = [
        ("nchannel", C.c_uint32),
        ("max_rounded_px_w", C.c_uint32),
        ("max_rounded_px_h", C.c_uint32),
        ("out_pitch", C.c_uint32),
        ("channels", C.POINTER(ArtChannel)),
        ("weight", C.c_float),
        ("pweight", C.c_float * 3),
        ("out_planes", C.POINTER(C.c_void_p)),
    ]


class ArtProcessImage(C.Structure):
    _fields_ = [
        ("nchannel", C.c_uint32),
        ("real_w", C.c_uint32),
        ("real_h", C.c_uint32),
        ("reserved", C.c_uint32),
        ("channels", C.POINTER(ArtChannel)),
        ("weight", C.c_float * 3),
        ("pweight", C.c_float * 3),
        ("rgb_out", C.c_void_p),
    ]


class ArtTuneResult(C.Structure):
    _fields_ = [
        ("variant", C.c_uint32), ("strip_rows", C.c_uint32), ("proj_warps", C.c_uint32),
        ("candidates", C.c_uint32), ("best_ms", C.c_float), ("heuristic_ms", C.c_float),
        ("heuristic_variant", C.c_uint32), ("heuristic_strip_rows", C.c_uint32),
    ]


class ArtTuneCandidate(C.Structure):
    _fields_ = [("variant", C.c_uint32), ("strip_rows", C.c_uint32), ("proj_warps", C.c_uint32), ("ms", C.c_float)]


class ArtCnnConv(C.Structure):
    _fields_ = [
        ("B", C.c_int32), ("H", C.c_int32), ("W", C.c_int32),
        ("cin", C.c_int32), ("ck", C.c_int32), ("n", C.c_int32), ("n_store", C.c_int32),
        ("x", C.c_void_p), ("wpack", C.c_void_p), ("bias", C.c_void_p),
        ("out", C.c_void_p), ("out_cstride", C.c_int32), ("out_coff", C.c_int32),
        ("out_f32", C.c_void_p), ("f32_cstride", C.c_int32),
        ("mask", C.c_void_p), ("mask_cstride", C.c_int32),
        ("relu", C.c_int32), ("accumulate", C.c_int32),
        ("err", C.c_void_p),
        ("pool_out", C.c_void_p), ("up2", C.c_int32), ("tile_rows", C.c_int32), ("f32_channels", C.c_int32),
    ]


class ArtCnnWgrad(C.Structure):
    _fields_ = [
        ("B", C.c_int32), ("H", C.c_int32), ("W", C.c_int32), ("cout", C.c_int32), ("cin", C.c_int32),
        ("dy", C.c_void_p), ("x", C.c_void_p), ("dw", C.c_void_p), ("accumulate", C.c_int32),
        ("workspace", C.c_void_p), ("workspace_bytes", C.c_int64), ("err", C.c_void_p),
    ]


class ArtError(RuntimeError):
    """Raised when a C ABI call returns a negative status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code
        self.message = message


EXPORTS = {
    "art_last_error": (C.c_char_p, []),
    "art_version": (C.c_char_p, []),
    "art_compute": (C.c_int32, [C.c_uint32, C.POINTER(ArtChannel), C.c_float, C.POINTER(C.c_float), C.c_uint32,
                                C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(C.c_void_p), C.POINTER(ArtOptions)]),
    "art_context_create": (C.c_int32, [C.c_int32, C.POINTER(C.c_void_p)]),
    "art_context_destroy": (None, [C.c_void_p]),
    "art_context_compute": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(ArtChannel), C.c_float,
                                        C.POINTER(C.c_float), C.c_uint32, C.c_uint32, C.c_uint32,
                                        C.POINTER(C.c_void_p), C.POINTER(ArtOptions)]),
    "art_context_compute_device": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(ArtChannel), C.c_float,
                                               C.POINTER(C.c_float), C.c_uint32, C.c_uint32, C.c_uint32,
                                               C.POINTER(C.c_void_p), C.c_uint32, C.POINTER(ArtOptions),
                                               C.c_void_p]),
    "art_context_process": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(ArtChannel), C.POINTER(C.c_float),
                                        C.POINTER(C.c_float), C.POINTER(C.c_uint32), C.c_int32, C.c_uint32,
                                        C.c_uint32, C.c_void_p, C.POINTER(ArtOptions)]),
    "art_solve_noalloc": (C.c_int32, [C.c_uint32, C.POINTER(ArtChannel), C.c_float, C.POINTER(C.c_float),
                                      C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_void_p), C.c_uint32,
                                      C.c_void_p]),
    "art_context_compute_batch": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(ArtImage), C.c_uint32,
                                              C.POINTER(ArtOptions)]),
    "art_context_compute_batch_device": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(ArtImage), C.c_uint32,
                                                     C.POINTER(ArtOptions), C.c_void_p]),
    "art_context_process_batch": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(ArtProcessImage), C.c_uint32,
                                              C.c_int32, C.POINTER(ArtOptions)]),
    "art_context_autotune": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                         C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32),
                                         C.POINTER(C.c_uint32)]),
    "art_context_autotune_batch": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(ArtImage), C.c_uint32,
                                               C.POINTER(ArtTuneResult)]),
    "art_context_last_tune": (C.c_int32, [C.c_void_p, C.POINTER(ArtTuneResult)]),
    "art_context_tune_candidates": (C.c_int32, [C.c_void_p, C.POINTER(ArtTuneCandidate), C.c_uint32,
                                                C.POINTER(C.c_uint32)]),
    "art_context_tune_cache": (C.c_int32, [C.c_void_p, C.c_char_p, C.c_int32]),
    "art_context_synchronize": (C.c_int32, [C.c_void_p]),
    "art_context_set_warm_start": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "art_context_set_joint_warm_start": (C.c_int32, [C.c_void_p, C.c_void_p]),
    "art_context_evaluate": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(C.c_double)]),
    "art_context_set_timing": (C.c_int32, [C.c_void_p, C.c_int32]),
    "art_context_last_timing": (C.c_int32, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                            C.POINTER(C.c_float), C.POINTER(C.c_uint32)]),
    "art_jpeg_decode": (C.c_int32, [C.c_char_p, C.c_size_t, C.POINTER(C.c_void_p)]),
    "art_jpeg_free": (None, [C.c_void_p]),
    "art_jpeg_info": (C.c_int32, [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                  C.POINTER(C.c_uint32)]),
    "art_jpeg_channel": (C.c_int32, [C.c_void_p, C.c_uint32, C.POINTER(ArtChannel)]),
    "art_net_num_params": (C.c_int64, []),
    "art_net_create": (C.c_int32, [C.c_int32, C.c_void_p, C.c_int64, C.POINTER(C.c_void_p)]),
    "art_net_destroy": (None, [C.c_void_p]),
    "art_net_params": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int64]),
    "art_net_gradients": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int64]),
    "art_net_predict": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_void_p, C.c_int32, C.c_int32,
                                    C.c_int32, C.c_void_p, C.c_void_p]),
    "art_net_predict_joint": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_void_p, C.c_int32,
                                          C.c_int64, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                                          C.c_void_p, C.c_void_p]),
    "art_net_train_step_joint": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_void_p, C.c_int32,
                                             C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32,
                                             C.c_int32, C.c_float, C.POINTER(C.c_float), C.c_void_p]),
    "art_net_set_loss": (C.c_int32, [C.c_void_p, C.c_float]),
    "art_net_set_joint_loss": (C.c_int32, [C.c_void_p, C.c_float]),
    "art_net_set_objective": (C.c_int32, [C.c_void_p, C.c_float, C.c_float, C.c_float, C.c_int32]),
    "art_net_train_step": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_void_p, C.c_void_p,
                                       C.c_int32, C.c_int32, C.c_int32, C.c_float, C.POINTER(C.c_float),
                                       C.c_void_p]),
    "art_cnn_conv3x3": (C.c_int32, [C.POINTER(ArtCnnConv), C.c_void_p]),
    "art_cnn_wgrad3x3": (C.c_int32, [C.POINTER(ArtCnnWgrad), C.c_void_p]),
    "art_cnn_pack_weights": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                         C.c_int32, C.c_void_p, C.c_void_p]),
    "art_cnn_pool2": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                  C.c_void_p, C.c_void_p]),
    "art_cnn_upsample2": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                                      C.c_int32, C.c_int32, C.c_void_p]),
    "art_cnn_downsum2_mask": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                                          C.c_void_p, C.c_void_p]),
    "art_cnn_unpool_add_mask": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                            C.c_void_p, C.c_int32, C.c_int32, C.c_void_p]),
    "art_cnn_bias_grad": (C.c_int32, [C.c_void_p, C.c_int64, C.c_int32, C.c_void_p, C.c_int64, C.c_void_p,
                                      C.c_int32, C.c_void_p]),
    "art_cnn_features": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int64, C.c_void_p, C.c_int32, C.c_int32,
                                     C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]),
    "art_cnn_residual": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32,
                                     C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]),
    "art_cnn_wait_selftest": (C.c_int32, [C.c_void_p, C.c_int64, C.c_void_p]),
    "art_cnn_adam": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_float, C.c_float,
                                 C.c_float, C.c_float, C.c_int32, C.c_void_p]),
}

_lib = None


def lib() -> C.CDLL:
    """Load the native library (building it first when ART_AUTOBUILD=1)."""
    global _lib
    if _lib is not None:
        return _lib
    if os.environ.get("ART_AUTOBUILD") == "1":
        from . import build as _build

        _build.build()
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m artefact_b200.build` "
            "(there is no CPU fallback for the solver)")
    handle = C.CDLL(str(LIB_PATH))
    for name, (res, args) in EXPORTS.items():
        fn = getattr(handle, name)
        fn.restype = res
        fn.argtypes = args
    _lib = handle
    return handle


def check(rc: int) -> None:
    if rc != ART_OK:
        msg = lib().art_last_error().decode("utf-8", "replace")
        raise ArtError(rc, msg)
