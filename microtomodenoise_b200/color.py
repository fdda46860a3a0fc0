"""The colour (2D RGB) path of iterNLM (Color/color_denoising.h): one image at
a time, Anscombe-stabilised channels, one joint weight per search offset from
the mean of the channels' patch distances (or one weight per channel), on the
GPU through inlm_rgb_denoise.

    planes = read_rgb("photo.tif")                      # three (ny, nx) float planes
    out, s_first, s_last = rgb_denoise(planes, DenoiseParameters(...), ColorParameters())
    save_rgb(out, "outdir", "photo_denoised")           # 8-bit RGB TIFF
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Callable, Optional, Sequence

import numpy as np

from . import _lib


@dataclass
class ColorParameters:
    """protocol::DenoiseParameters::Color (denoise_parameters.h:65-69)."""

    stabilize_variance: bool = True    # --nopoisson turns the Anscombe transform off
    independent_channels: bool = False  # --independent
    average_channelsigma: bool = True   # --noaverage keeps one sigma per channel

    def to_c(self) -> _lib.InlmColorParams:
        return _lib.InlmColorParams(int(self.stabilize_variance), int(self.independent_channels),
                                    int(self.average_channelsigma))


def read_rgb(path: str):
    """An 8- or 16-bit RGB(A) TIFF as three float32 (ny, nx) planes."""
    L = _lib.load()
    shape = (C.c_int * 2)()
    _lib.check(L.inlm_tiff_read_rgb(os.fsencode(path), shape, None, None, None, 0), "tiff_read_rgb")
    nx, ny = shape[0], shape[1]
    planes = [np.empty((ny, nx), np.float32) for _ in range(3)]
    _lib.check(L.inlm_tiff_read_rgb(os.fsencode(path), shape, planes[0].ctypes.data,
                                    planes[1].ctypes.data, planes[2].ctypes.data, nx * ny),
               "tiff_read_rgb")
    return planes


def save_rgb(planes: Sequence[np.ndarray], directory: str, name: str) -> None:
    """directory/<name>.tif, 8-bit RGB, each value as (uint8) min(255, v)."""
    r, g, b = (np.ascontiguousarray(a, np.float32) for a in planes)
    ny, nx = r.shape
    _lib.check(_lib.load().inlm_tiff_write_rgb(os.fsencode(directory), name.encode(), r.ctypes.data,
                                               g.ctypes.data, b.ctypes.data, nx, ny),
               "tiff_write_rgb")


def rgb_denoise(planes: Sequence[np.ndarray], params, color: Optional[ColorParameters] = None,
                on_iteration: Optional[Callable[[int, list], None]] = None):
    """Whole colour job for one image; returns (final planes, sigma_first,
    sigma_last). on_iteration(iter, planes) receives each iteration's planes
    as the reference saves them (and makes the job match the reference run
    that saves every iteration)."""
    color = color or ColorParameters()
    r, g, b = (np.ascontiguousarray(a, np.float32) for a in planes)
    ny, nx = r.shape
    out = [np.empty((ny, nx), np.float32) for _ in range(3)]
    cp = params.to_c()
    s_first, s_last = (C.c_float * 3)(), (C.c_float * 3)()
    n = nx * ny

    def _cb(it, pr, pg, pb, _user):
        arrs = [np.ctypeslib.as_array(C.cast(q, C.POINTER(C.c_float)), shape=(n,)).reshape(ny, nx).copy()
                for q in (pr, pg, pb)]
        on_iteration(int(it), arrs)

    cb = _lib.RGB_ITERATION_FN(_cb) if on_iteration else _lib.RGB_ITERATION_FN()
    rc = _lib.load().inlm_rgb_denoise(nx, ny, C.byref(cp), C.byref(color.to_c()), r.ctypes.data,
                                      g.ctypes.data, b.ctypes.data, out[0].ctypes.data,
                                      out[1].ctypes.data, out[2].ctypes.data, cb, None, s_first,
                                      s_last)
    _lib.check(rc, "rgb_denoise")
    return out, np.array(s_first[:], np.float32), np.array(s_last[:], np.float32)
