"""TIFF sequence IO of the iterNLM driver (hdcom::HdCommunication,
Geometry/hdcommunication.cpp), through the library's own uncompressed TIFF
reader and writer (libtiff is not needed). Stacks are numpy arrays (nz, ny, nx).

    shape = stack_shape(path)               # GetFilelist_And_ImageSequenceDimensions
    vol = read_stack(path, first, last)     # GetTif_unknowndim_32bit / Get3DTifSequence_32bitPointer
    save_stack(vol, outdir, "denoised", z0, as_16bit)  # SaveTifSequence_32bit / _as16bit
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib


def stack_shape(path: str):
    """(nz, ny, nx) of a slice directory or multi-page file, and its samples
    per pixel."""
    shape = (C.c_int * 3)()
    spp = C.c_int(0)
    _lib.check(_lib.load().inlm_tiff_shape(os.fsencode(path), shape, C.byref(spp)), "tiff_shape")
    return (shape[2], shape[1], shape[0]), spp.value


def read_stack(path: str, first_slice: int = -1, last_slice: int = -1) -> np.ndarray:
    """Slices first..last (inclusive, clamped; -1, -1 = all) as float32."""
    (nz, ny, nx), _ = stack_shape(path)
    z0, z1 = 0, nz - 1
    if first_slice != -1 or last_slice != -1:
        z0 = max(0, first_slice)
        z1 = nz - 1 if last_slice == -1 else min(nz - 1, last_slice)
    out = np.empty((max(0, z1 - z0 + 1), ny, nx), np.float32)
    rc = _lib.load().inlm_tiff_read(os.fsencode(path), int(first_slice), int(last_slice),
                                    out.ctypes.data, out.size)
    _lib.check(rc, "tiff_read")
    return out


def save_stack(image: np.ndarray, directory: str, name: str = "denoised", z0: int = 0,
               as_16bit: bool = False) -> None:
    """Writes directory/<name><z0+i:04d>.tif for each slice i."""
    img = np.ascontiguousarray(image, dtype=np.float32)
    if img.ndim == 2:
        img = img[None]
    shape = (C.c_int * 3)(img.shape[2], img.shape[1], img.shape[0])
    rc = _lib.load().inlm_tiff_write_sequence(img.ctypes.data, shape, int(z0), os.fsencode(directory),
                                              name.encode(), int(bool(as_16bit)))
    _lib.check(rc, "tiff_write_sequence")
