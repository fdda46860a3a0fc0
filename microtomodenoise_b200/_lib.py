"""ctypes binding of the C ABI in include/inlm.h (libinlm.so, built in-tree).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libinlm.so")

INLM_OK = 0
ERRORS = {
    -1: "INLM_ERR_ARG",
    -2: "INLM_ERR_CUDA",
    -3: "INLM_ERR_NODEVICE",
    -4: "INLM_ERR_NOMEM",
    -5: "INLM_ERR_STATE",
    -6: "INLM_ERR_TIMEOUT",
    -7: "INLM_ERR_UNSUPPORTED",
    -8: "INLM_ERR_IO",
}
NOISE_MODES = {"z-adaptive": 0, "auto": 0, "global": 1, "manual": 2, "semimanual": 3}
PRECISIONS = {"f32": 0, "f16": 1, "f16_df32": 2, "f32_fma": 3}

# Every entry point include/inlm.h declares.
EXPORTS = (
    "inlm_default_params", "inlm_last_error", "inlm_denoiser_create", "inlm_denoiser_destroy",
    "inlm_set_sigma", "inlm_run_iteration", "inlm_get_result", "inlm_run_iteration_device",
    "inlm_get_result_device", "inlm_denoise", "inlm_set_stream", "inlm_filter_kernel_ms",
    "inlm_describe", "inlm_noise_create", "inlm_noise_destroy", "inlm_noise_estimate",
    "inlm_noise_samples", "inlm_noise_patchstd", "inlm_geometry", "inlm_noise_draw_samples",
    "inlm_kernel_launches", "inlm_noise_em_noalloc",
    "inlm_tile_grid", "inlm_set_offset_plan",
    "inlm_proposal_create", "inlm_proposal_destroy", "inlm_proposal_n_params",
    "inlm_proposal_set_params", "inlm_proposal_get_params", "inlm_proposal_logits",
    "inlm_proposal_set_tensor_cores",
    "inlm_proposal_train", "inlm_proposal_select", "inlm_attach_proposal", "inlm_proposal_stats",
    "inlm_weight_map", "inlm_net_input",
    "inlm_autotune", "inlm_select_tile_form", "inlm_batch_create", "inlm_batch_destroy", "inlm_batch_run",
    "inlm_batch_describe", "inlm_stream_denoise", "inlm_set_result",
    "inlm_tiff_shape", "inlm_tiff_read", "inlm_tiff_write_sequence",
    "inlm_get_result_slices", "inlm_set_result_slices", "inlm_noise_patchstd_slab",
    "inlm_noise_estimate_from_patchstd", "inlm_rgb_denoise", "inlm_tiff_read_rgb",
    "inlm_tiff_write_rgb", "inlm_attach_proposal_grouped", "inlm_attach_proposal_ex", "inlm_proposal_select_grouped",
    "inlm_stream_denoise_grouped", "inlm_denoise_multi", "inlm_device_count",
    "inlm_blocks_create", "inlm_blocks_destroy", "inlm_blocks_slab_depth", "inlm_blocks_set_sigma",
    "inlm_blocks_run_iteration", "inlm_blocks_attach_proposal", "inlm_stream_denoise_ex",
    "inlm_proposal_schedule", "inlm_stream_denoise_sched", "inlm_blocks_proposal_schedule", "inlm_device_memory", "inlm_debug_fail_allocation",
    "inlm_debug_live_allocations", "inlm_debug_wait_expiry", "inlm_denoise_f64_blocks",
)


class InlmColorParams(C.Structure):
    _fields_ = [
        ("stabilize_variance", C.c_int),
        ("independent_channels", C.c_int),
        ("average_channelsigma", C.c_int),
    ]


RGB_ITERATION_FN = C.CFUNCTYPE(None, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p)


class InlmParams(C.Structure):
    _fields_ = [
        ("alpha", C.c_float),
        ("maxiterations", C.c_int),
        ("nslices", C.c_int),
        ("search_radius", C.c_int * 3),
        ("patch_radius", C.c_int * 3),
        ("beta", C.c_float),
        ("z_anisotropy", C.c_float),
        ("noise_mode", C.c_int),
        ("zwindow", C.c_int),
        ("sigma", C.c_float * 2),
        ("n_samples", C.c_uint64),
        ("noise_patchsize", C.c_int),
        ("stds_from_mean", C.c_float),
        ("continuous_estimate", C.c_int),
        ("circular_mask_diameter", C.c_int),
        ("noise_seed", C.c_uint),
        ("device_id", C.c_int),
        ("precision", C.c_int),
        ("weight_table", C.c_int),
    ]


class InlmError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        self.code = code
        super().__init__(f"{where}: {ERRORS.get(code, code)}: {msg}")


_lib = None


def load(path: str = "") -> C.CDLL:
    """Loads libinlm.so once (the in-tree build, or the file INLM_LIB names);
    raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or os.environ.get("INLM_LIB", LIB_PATH)
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python -m microtomodenoise_b200.build` "
            "(the package has no CPU fallback)")
    L = C.CDLL(path)
    vp = C.c_void_p
    L.inlm_last_error.restype = C.c_char_p
    L.inlm_default_params.argtypes = [C.POINTER(InlmParams)]
    L.inlm_default_params.restype = None
    L.inlm_denoiser_create.argtypes = [C.c_int * 3, C.POINTER(InlmParams), C.POINTER(vp)]
    L.inlm_denoiser_destroy.argtypes = [vp]
    L.inlm_set_sigma.argtypes = [vp, vp]
    L.inlm_run_iteration.argtypes = [vp, C.c_int, vp]
    L.inlm_get_result.argtypes = [vp, vp]
    L.inlm_run_iteration_device.argtypes = [vp, C.c_int, vp]
    L.inlm_get_result_device.argtypes = [vp, vp]
    L.inlm_denoise.argtypes = [vp, vp, vp, C.c_int, vp, vp]
    L.inlm_set_stream.argtypes = [vp, vp]
    L.inlm_filter_kernel_ms.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_int)]
    L.inlm_describe.argtypes = [vp, C.c_char_p, C.c_size_t]
    L.inlm_noise_create.argtypes = [C.c_int * 3, C.c_uint64, C.c_int, C.c_uint, C.c_int,
                                    C.POINTER(vp)]
    L.inlm_noise_destroy.argtypes = [vp]
    L.inlm_noise_estimate.argtypes = [vp, C.POINTER(InlmParams), vp, C.c_int, vp]
    L.inlm_noise_samples.argtypes = [vp, vp, C.c_uint64, C.POINTER(C.c_uint64)]
    L.inlm_noise_patchstd.argtypes = [vp, vp, C.c_uint64]
    L.inlm_geometry.argtypes = [C.POINTER(InlmParams), C.c_int, vp, C.POINTER(C.c_int), vp, vp,
                                C.POINTER(C.c_int), vp]
    L.inlm_noise_draw_samples.argtypes = [C.c_int * 3, C.c_uint64, C.c_int, C.c_int, C.c_uint, vp]
    L.inlm_kernel_launches.argtypes = [vp, C.POINTER(C.c_uint64)]
    L.inlm_tile_grid.argtypes = [vp, C.c_int * 3, C.c_int * 3]
    L.inlm_set_offset_plan.argtypes = [vp, vp, vp, vp, C.c_int, C.c_int]
    L.inlm_noise_em_noalloc.argtypes = [vp, vp, C.c_int64, vp, C.c_int, vp, vp]
    L.inlm_proposal_create.argtypes = [C.c_int, C.c_int, C.POINTER(vp)]
    L.inlm_proposal_destroy.argtypes = [vp]
    L.inlm_proposal_n_params.argtypes = [vp, C.POINTER(C.c_int64)]
    L.inlm_proposal_set_params.argtypes = [vp, vp, C.c_int64]
    L.inlm_proposal_get_params.argtypes = [vp, vp, C.c_int64]
    L.inlm_proposal_logits.argtypes = [vp, vp, vp, C.c_int * 3, vp]
    L.inlm_proposal_set_tensor_cores.argtypes = [vp, C.c_int]
    L.inlm_proposal_train.argtypes = [vp, C.c_int, vp, vp, vp, vp, C.c_float,
                                      C.POINTER(C.c_double), vp]
    L.inlm_proposal_select.argtypes = [vp, vp, vp, C.c_int * 3, C.c_int, C.c_float, vp, vp,
                                       C.POINTER(C.c_int)]
    L.inlm_attach_proposal.argtypes = [vp, vp, C.c_int, C.c_float]
    L.inlm_attach_proposal_grouped.argtypes = [vp, vp, C.c_int, C.c_float, C.c_int]
    L.inlm_attach_proposal_ex.argtypes = [vp, vp, C.c_int, C.c_float, C.c_float, C.c_int]
    L.inlm_proposal_select_grouped.argtypes = [vp, vp, vp, C.c_int * 3, C.c_int, C.c_int, C.c_float,
                                               vp, vp, C.POINTER(C.c_int)]
    L.inlm_proposal_stats.argtypes = [vp, C.c_int64 * 5]
    L.inlm_weight_map.argtypes = [vp, vp]
    L.inlm_net_input.argtypes = [vp, vp, vp]
    L.inlm_autotune.argtypes = [vp, C.c_char_p, C.c_size_t]
    L.inlm_select_tile_form.argtypes = [vp, C.c_int]
    L.inlm_batch_create.argtypes = [C.c_int, vp, vp, C.POINTER(vp)]
    L.inlm_batch_destroy.argtypes = [vp]
    L.inlm_batch_run.argtypes = [vp, vp, vp, C.c_int, C.POINTER(C.c_float)]
    L.inlm_batch_describe.argtypes = [vp, C.c_char_p, C.c_size_t]
    L.inlm_stream_denoise.argtypes = [C.c_int * 3, C.POINTER(InlmParams), vp, vp, C.c_int, vp,
                                      C.c_int, C.c_float, vp, vp, vp]
    L.inlm_set_result.argtypes = [vp, C.c_int, vp, vp]
    L.inlm_device_count.argtypes = [C.POINTER(C.c_int)]
    L.inlm_debug_fail_allocation.argtypes = [C.c_int64]
    L.inlm_debug_live_allocations.argtypes = [C.POINTER(C.c_int64)]
    L.inlm_debug_wait_expiry.argtypes = [vp, C.c_int64]
    L.inlm_denoise_f64_blocks.argtypes = [C.c_int * 3, C.POINTER(InlmParams), vp, C.c_int, vp, C.c_int, vp,
                                          C.c_int, C.c_int * 3, vp]
    L.inlm_device_memory.argtypes = [C.c_int, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
    L.inlm_blocks_create.argtypes = [C.c_int * 3, C.POINTER(InlmParams), C.c_int, vp, C.c_int, C.POINTER(vp)]
    L.inlm_blocks_destroy.argtypes = [vp]
    L.inlm_blocks_slab_depth.argtypes = [vp, C.POINTER(C.c_int)]
    L.inlm_blocks_set_sigma.argtypes = [vp, vp]
    L.inlm_blocks_attach_proposal.argtypes = [vp, vp, C.c_int, C.c_float, C.c_float, C.c_int]
    L.inlm_stream_denoise_ex.argtypes = [C.c_int * 3, C.POINTER(InlmParams), vp, vp, C.c_int, vp, C.c_int,
                                         C.c_float, C.c_float, C.c_int, vp, vp, vp]
    L.inlm_proposal_schedule.argtypes = [vp, C.c_int, vp, vp]
    L.inlm_blocks_proposal_schedule.argtypes = [vp, C.c_int, vp, vp]
    L.inlm_stream_denoise_sched.argtypes = [C.c_int * 3, C.POINTER(InlmParams), vp, vp, C.c_int, vp, C.c_int,
                                            vp, vp, C.c_float, C.c_int, vp, vp, vp]
    L.inlm_blocks_run_iteration.argtypes = [vp, C.c_int, vp, vp, vp]
    L.inlm_denoise_multi.argtypes = [C.c_int * 3, C.POINTER(InlmParams), vp, vp, C.c_int, vp, vp, vp]
    L.inlm_stream_denoise_grouped.argtypes = [C.c_int * 3, C.POINTER(InlmParams), vp, vp, C.c_int, vp,
                                              C.c_int, C.c_float, C.c_int, vp, vp, vp]
    L.inlm_tiff_shape.argtypes = [C.c_char_p, C.c_int * 3, C.POINTER(C.c_int)]
    L.inlm_tiff_read.argtypes = [C.c_char_p, C.c_int, C.c_int, vp, C.c_uint64]
    L.inlm_tiff_write_sequence.argtypes = [vp, C.c_int * 3, C.c_int, C.c_char_p, C.c_char_p, C.c_int]
    L.inlm_get_result_slices.argtypes = [vp, C.c_int, C.c_int, vp, C.c_int]
    L.inlm_set_result_slices.argtypes = [vp, C.c_int, C.c_int, vp, C.c_int]
    L.inlm_noise_patchstd_slab.argtypes = [vp, C.POINTER(InlmParams), vp, C.c_int, C.c_int, C.c_int,
                                           vp, C.c_uint64]
    L.inlm_noise_estimate_from_patchstd.argtypes = [vp, C.POINTER(InlmParams), vp, C.c_uint64, vp]
    L.inlm_rgb_denoise.argtypes = [C.c_int, C.c_int, C.POINTER(InlmParams), C.POINTER(InlmColorParams),
                                   vp, vp, vp, vp, vp, vp, RGB_ITERATION_FN, vp, C.c_float * 3,
                                   C.c_float * 3]
    L.inlm_tiff_read_rgb.argtypes = [C.c_char_p, C.c_int * 2, vp, vp, vp, C.c_uint64]
    L.inlm_tiff_write_rgb.argtypes = [C.c_char_p, C.c_char_p, vp, vp, vp, C.c_int, C.c_int]
    for name in EXPORTS:
        if name not in ("inlm_last_error", "inlm_default_params"):
            getattr(L, name).restype = C.c_int
    _lib = L
    return L


def check(rc: int, where: str) -> None:
    if rc != INLM_OK:
        msg = _lib.inlm_last_error().decode(errors="replace") if _lib else ""
        raise InlmError(rc, where, msg)
