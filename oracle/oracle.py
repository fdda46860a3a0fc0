"""TEST INFRASTRUCTURE ONLY — ctypes bindings to the two CPU oracles.

* ``Port``: this project's plain-C restatement (oracle/inlm_oracle.c), built by
  ``make -C oracle port``. Travels with the repository; it is the checker on
  machines where the reference sources are absent.
* ``Reference``: the reference's own CPU filter and noise estimator compiled
  from its unmodified sources (oracle/_ref/libiternlm_ref.so, built by
  ``make -C oracle ref`` where the reference tree exists). Used to pin the port
  and as the timed CPU baseline.
* ``ReferenceGPU``: the reference's own GPU class (Denoiser/iternlm_gpu.cu)
  compiled unmodified for sm_100a (oracle/_ref/libiternlm_gpu_ref.so, built by
  ``make -C oracle ref_gpu``): the reference GPU kernel timed beside the
  product. Its expf weights and its generic-kernel fall-through make it differ
  from the CPU reference, so it is a timing baseline, not a checker.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module. The product (microtomodenoise_b200) never does.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "libinlm_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libiternlm_ref.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libiternlm_gpu_ref.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


@dataclass
class FilterParams:
    """Filter knobs of protocol::DenoiseParameters (denoise_parameters.h:11-20)."""

    search_radius: tuple = (10, 10, 10)
    patch_radius: tuple = (1, 1, 1)
    nslices: int = 11
    beta: float = 1.0
    z_anisotropy: float = 1.0


class _CParams(C.Structure):
    _fields_ = [
        ("search_radius", C.c_int * 3),
        ("patch_radius", C.c_int * 3),
        ("nslices", C.c_int),
        ("beta", C.c_float),
        ("z_anisotropy", C.c_float),
    ]


def _cparams(p: FilterParams) -> _CParams:
    c = _CParams()
    for i in range(3):
        c.search_radius[i] = int(p.search_radius[i])
        c.patch_radius[i] = int(p.patch_radius[i])
    c.nslices = int(p.nslices)
    c.beta = float(p.beta)
    c.z_anisotropy = float(p.z_anisotropy)
    return c


def _shape3(vol: np.ndarray):
    nz, ny, nx = vol.shape
    return (C.c_int * 3)(nx, ny, nz)


class Port:
    """The plain-C restatement."""

    def __init__(self, path: str = PORT_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle port`")
        L = self.lib = C.CDLL(path)
        L.ora_search_offsets.restype = C.c_int
        L.ora_search_offsets.argtypes = [C.POINTER(_CParams), _i32p, _i32p, _i32p, C.c_int]
        L.ora_patch_taps.restype = C.c_int
        L.ora_patch_taps.argtypes = [C.POINTER(_CParams), _i32p, _i32p, _i32p, C.c_int]
        L.ora_distweight.restype = C.c_int
        L.ora_distweight.argtypes = [C.POINTER(_CParams), C.c_int, _f32p, C.c_int]
        L.ora_filter_weights.restype = C.c_int
        L.ora_filter_weights.argtypes = [C.POINTER(_CParams), C.c_int, _f32p, C.c_int,
                                         C.POINTER(C.c_int)]
        L.ora_padding.argtypes = [C.POINTER(_CParams), C.c_int * 3]
        L.ora_pad_reflective.argtypes = [_f32p, C.c_int * 3, C.c_int * 3, _f32p]
        L.ora_filter_f32.argtypes = [_f32p, _f32p, C.c_int * 3, C.POINTER(_CParams), _f32p, _f32p]
        L.ora_denoise_f32.argtypes = [_f32p, C.c_int * 3, C.POINTER(_CParams), _f32p, C.c_int,
                                      _f32p, C.c_void_p]
        L.ora_denoise_f64.argtypes = [_f32p, C.c_int * 3, C.POINTER(_CParams), _f32p, C.c_int,
                                      _f64p]
        L.ora_filter_f64.argtypes = [_f64p, _f64p, C.c_int * 3, C.POINTER(_CParams), _f64p, _f64p]
        L.ora_filter_f32_voxels.argtypes = [_f32p, _f32p, C.c_int * 3, C.POINTER(_CParams), _f32p,
                                            C.c_int64, _i64p, _f32p]
        L.ora_denoise_f64_plan.argtypes = [_f32p, C.c_int * 3, C.POINTER(_CParams), _f32p, C.c_int,
                                           C.c_int * 3,
                                           np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS"),
                                           C.c_longlong, _f64p]
        L.ora_weight_mass_f64.argtypes = [_f32p, C.c_int * 3, C.POINTER(_CParams), _f32p,
                                          C.c_int * 3, _f64p]
        L.ora_sigma_to_mult.argtypes = [_f32p, C.c_int, C.c_float, _f32p]
        L.ora_srand.argtypes = [C.c_void_p, C.c_uint]
        L.ora_rand.restype = C.c_int
        L.ora_rand.argtypes = [C.c_void_p]
        L.ora_draw_samples.argtypes = [C.c_int * 3, C.c_int64, C.c_int, C.c_int, C.c_uint, _i64p]
        L.ora_patchstd.argtypes = [_f32p, C.c_int * 3, _i64p, C.c_int64, C.c_int, _f32p]
        L.ora_create2clusters_f32.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _f32p]
        L.ora_create2clusters_f64acc.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _f32p]
        L.ora_zwindows.argtypes = [_i64p, C.c_int64, C.c_int * 3, C.c_int, _i32p, _i32p]
        L.ora_fill_empty_slices.argtypes = [_f32p, _f32p, C.c_int]
        L.ora_noise_from_patchstd.argtypes = [_f32p, _i64p, C.c_int64, C.c_int * 3, C.c_int,
                                              C.c_int, C.c_float, C.c_int, _f32p]
        L.ora_filter_rgb.argtypes = [C.c_void_p * 3, C.c_void_p * 3, C.c_int, C.c_int,
                                     C.POINTER(_CParams), C.c_float * 3, C.c_int, C.c_void_p * 3]
        L.ora_anscombe.argtypes = [_f32p, C.c_int64, C.c_int]

    # ---- geometry ----
    def padding(self, p: FilterParams):
        out = (C.c_int * 3)()
        self.lib.ora_padding(C.byref(_cparams(p)), out)
        return tuple(out)

    def search_offsets(self, p: FilterParams) -> np.ndarray:
        cp = _cparams(p)
        n = self.lib.ora_search_offsets(C.byref(cp), np.zeros(1, np.int32), np.zeros(1, np.int32),
                                        np.zeros(1, np.int32), 0)
        dx, dy, dz = (np.zeros(n, np.int32) for _ in range(3))
        self.lib.ora_search_offsets(C.byref(cp), dx, dy, dz, n)
        return np.stack([dx, dy, dz], 1)

    def patch_taps(self, p: FilterParams) -> np.ndarray:
        cp = _cparams(p)
        n = self.lib.ora_patch_taps(C.byref(cp), np.zeros(1, np.int32), np.zeros(1, np.int32),
                                    np.zeros(1, np.int32), 0)
        dx, dy, dz = (np.zeros(n, np.int32) for _ in range(3))
        self.lib.ora_patch_taps(C.byref(cp), dx, dy, dz, n)
        return np.stack([dx, dy, dz], 1)

    def distweight(self, p: FilterParams, nz_padded: int) -> np.ndarray:
        w = np.zeros(4096, np.float32)
        n = self.lib.ora_distweight(C.byref(_cparams(p)), nz_padded, w, 4096)
        return w[:n].copy()

    def filter_weights(self, p: FilterParams, nz_padded: int):
        w = np.zeros(4096, np.float32)
        spec = C.c_int(0)
        n = self.lib.ora_filter_weights(C.byref(_cparams(p)), nz_padded, w, 4096, C.byref(spec))
        return w[:n].copy(), bool(spec.value)

    def pad_reflective(self, vol: np.ndarray, pad) -> np.ndarray:
        vol = np.ascontiguousarray(vol, np.float32)
        nz, ny, nx = vol.shape
        out = np.empty((nz + 2 * pad[2], ny + 2 * pad[1], nx + 2 * pad[0]), np.float32)
        self.lib.ora_pad_reflective(vol.ravel(), _shape3(vol), (C.c_int * 3)(*pad), out.ravel())
        return out

    # ---- filter ----
    def denoise_f32(self, raw: np.ndarray, p: FilterParams, sigmas: np.ndarray,
                    all_iters: bool = False):
        raw = np.ascontiguousarray(raw, np.float32)
        sig = np.ascontiguousarray(np.atleast_2d(sigmas), np.float32)
        n_iter = sig.shape[0]
        assert sig.shape[1] == raw.shape[0]
        out = np.empty_like(raw)
        allbuf = np.empty((n_iter,) + raw.shape, np.float32) if all_iters else None
        self.lib.ora_denoise_f32(raw.ravel(), _shape3(raw), C.byref(_cparams(p)), sig.ravel(),
                                 n_iter, out.ravel(),
                                 allbuf.ctypes.data if all_iters else None)
        return allbuf if all_iters else out

    def denoise_f64_plan(self, raw: np.ndarray, p: FilterParams, sigmas: np.ndarray, tile_xyz,
                         keep: np.ndarray) -> np.ndarray:
        """FP64 filter with per-tile offset subsets (keep: n_tiles x S bool, or
        n_iter x n_tiles x S for a subset per iteration)."""
        raw = np.ascontiguousarray(raw, np.float32)
        sig = np.ascontiguousarray(np.atleast_2d(sigmas), np.float32)
        out = np.empty(raw.shape, np.float64)
        keep = np.ascontiguousarray(keep, np.uint8)
        stride = keep[0].size if keep.ndim == 3 else 0
        if keep.ndim == 3:
            assert keep.shape[0] == sig.shape[0]
        self.lib.ora_denoise_f64_plan(raw.ravel(), _shape3(raw), C.byref(_cparams(p)), sig.ravel(),
                                      sig.shape[0], (C.c_int * 3)(*tile_xyz), keep.ravel(), stride,
                                      out.ravel())
        return out

    def weight_mass_f64(self, prev: np.ndarray, p: FilterParams, sigma: np.ndarray,
                        tile_xyz=(8, 8, 8)) -> np.ndarray:
        """Per-tile offset weight mass of one iteration (n_tiles x S, rows sum to 1)."""
        prev = np.ascontiguousarray(prev, np.float32)
        nz, ny, nx = prev.shape
        nt = -(-nx // tile_xyz[0]) * -(-ny // tile_xyz[1]) * -(-nz // tile_xyz[2])
        S = len(self.search_offsets(p))
        out = np.empty((nt, S), np.float64)
        self.lib.ora_weight_mass_f64(prev.ravel(), _shape3(prev), C.byref(_cparams(p)),
                                     np.ascontiguousarray(sigma, np.float32),
                                     (C.c_int * 3)(*tile_xyz), out.ravel())
        return out

    def sigma_to_mult(self, sigma, beta: float = 1.0) -> np.ndarray:
        sigma = np.ascontiguousarray(sigma, np.float32)
        out = np.empty_like(sigma)
        self.lib.ora_sigma_to_mult(sigma, len(sigma), beta, out)
        return out

    def filter_voxels(self, raw_pad: np.ndarray, prev_pad: np.ndarray, shape_zyx, p: FilterParams,
                      sigma: np.ndarray, voxels: np.ndarray) -> np.ndarray:
        """One FP32 filter iteration at selected unpadded linear voxel indices."""
        nz, ny, nx = shape_zyx
        mult = self.sigma_to_mult(sigma, p.beta)
        vox = np.ascontiguousarray(voxels, np.int64)
        out = np.empty(len(vox), np.float32)
        self.lib.ora_filter_f32_voxels(np.ascontiguousarray(raw_pad, np.float32).ravel(),
                                       np.ascontiguousarray(prev_pad, np.float32).ravel(),
                                       (C.c_int * 3)(nx, ny, nz), C.byref(_cparams(p)), mult,
                                       len(vox), vox, out)
        return out

    def denoise_f64(self, raw: np.ndarray, p: FilterParams, sigmas: np.ndarray) -> np.ndarray:
        raw = np.ascontiguousarray(raw, np.float32)
        sig = np.ascontiguousarray(np.atleast_2d(sigmas), np.float32)
        out = np.empty(raw.shape, np.float64)
        self.lib.ora_denoise_f64(raw.ravel(), _shape3(raw), C.byref(_cparams(p)), sig.ravel(),
                                 sig.shape[0], out.ravel())
        return out

    def denoise_f64_blocks(self, raw: np.ndarray, p: FilterParams, sigmas: np.ndarray,
                           corners, size) -> list:
        """The FP64 full-search result of the last iteration on sub-blocks of
        a volume, without filtering the whole volume: iteration k runs on the
        block grown by (n_iter - k) x the filter's reach (its padding) per
        side, clipped to the volume, from iteration k-1 on that box grown by
        one reach; positions outside the volume take the reference's
        reflective rule (-i below 0, 2n-i-2 above n-1). corners: (z, y, x)
        lower corners; size: (dz, dy, dx). Returns one float64 array per
        block. Same arithmetic as ora_denoise_f64 (ora_filter_f64 on crops)."""
        raw = np.ascontiguousarray(raw, np.float32)
        sig = np.ascontiguousarray(np.atleast_2d(sigmas), np.float32)
        n_iter = sig.shape[0]
        pad = self.padding(p)[::-1]  # (z, y, x)
        shp = raw.shape
        cp = _cparams(p)
        beta = float(np.float32(p.beta))
        s64 = sig.astype(np.float64)
        mults = [-1.0 / (s64[k] * s64[k] * beta) for k in range(n_iter)]  # as ora_denoise_f64

        def mirror(i, n):
            i = np.asarray(i)
            for _ in range(64):
                i = np.where(i < 0, -i, i)
                i = np.where(i > n - 1, 2 * n - i - 2, i)
            return i

        out = []
        for c in corners:
            boxes = []  # iteration k's box (lo, hi) per axis, k = 1..n_iter
            for k in range(1, n_iter + 1):
                g = n_iter - k
                boxes.append([(max(0, c[a] - g * pad[a]), min(shp[a], c[a] + size[a] + g * pad[a]))
                              for a in range(3)])
            prev = None  # iterate k-1 on boxes[k-2]
            for k in range(n_iter):
                box = boxes[k]
                idx = [mirror(np.arange(lo - pad[a], hi + pad[a]), shp[a]) for a, (lo, hi) in enumerate(box)]
                raw_pad = raw[np.ix_(*idx)].astype(np.float64)
                if k == 0:
                    prev_pad = raw_pad
                else:
                    pb = boxes[k - 1]
                    rel = [ix - pb[a][0] for a, ix in enumerate(idx)]
                    for a in range(3):
                        assert rel[a].min() >= 0 and rel[a].max() < pb[a][1] - pb[a][0], "box too small"
                    prev_pad = prev[np.ix_(*rel)]
                inner = [hi - lo for lo, hi in box]
                res = np.empty(inner, np.float64)
                m = np.ascontiguousarray(mults[k][box[0][0]:box[0][1]])
                self.lib.ora_filter_f64(np.ascontiguousarray(raw_pad).ravel(),
                                        np.ascontiguousarray(prev_pad).ravel(),
                                        (C.c_int * 3)(inner[2], inner[1], inner[0]), C.byref(cp), m,
                                        res.ravel())
                prev = res
            lo = [c[a] - boxes[-1][a][0] for a in range(3)]
            out.append(prev[lo[0]:lo[0] + size[0], lo[1]:lo[1] + size[1], lo[2]:lo[2] + size[2]].copy())
        return out

    # ---- colour path ----
    def filter_rgb(self, raw3, prev3, p: FilterParams, mult3, independent: bool = False):
        """One three-channel 2D iteration (filterslice_3channels); raw3 / prev3:
        three (ny, nx) planes; p with z radii 0 and nslices 1."""
        raw3 = [np.ascontiguousarray(a, np.float32) for a in raw3]
        prev3 = [np.ascontiguousarray(a, np.float32) for a in prev3]
        ny, nx = raw3[0].shape
        out = [np.empty((ny, nx), np.float32) for _ in range(3)]
        ptr = lambda arrs: (C.c_void_p * 3)(*[a.ctypes.data for a in arrs])
        self.lib.ora_filter_rgb(ptr(raw3), ptr(prev3), nx, ny, C.byref(_cparams(p)),
                                (C.c_float * 3)(*[float(m) for m in mult3]), int(bool(independent)),
                                ptr(out))
        return out

    def anscombe(self, v: np.ndarray, inverse: bool = False) -> np.ndarray:
        out = np.ascontiguousarray(v, np.float32).copy()
        self.lib.ora_anscombe(out.ravel(), out.size, int(bool(inverse)))
        return out

    # ---- noise ----
    def rand_sequence(self, seed: int, n: int) -> np.ndarray:
        st = C.create_string_buffer(256)
        self.lib.ora_srand(st, seed)
        return np.array([self.lib.ora_rand(st) for _ in range(n)], np.int64)

    def draw_samples(self, shape_zyx, n_samples: int, patchsize: int = 15, mask: int = 0,
                     seed: int = 0) -> np.ndarray:
        nz, ny, nx = shape_zyx
        out = np.empty(n_samples, np.int64)
        self.lib.ora_draw_samples((C.c_int * 3)(nx, ny, nz), n_samples, patchsize, mask, seed, out)
        return out

    def patchstd(self, vol: np.ndarray, samples: np.ndarray, patchsize: int = 15) -> np.ndarray:
        vol = np.ascontiguousarray(vol, np.float32)
        samples = np.ascontiguousarray(samples, np.int64)
        out = np.empty(len(samples), np.float32)
        self.lib.ora_patchstd(vol.ravel(), _shape3(vol), samples, len(samples), patchsize, out)
        return out

    def create2clusters(self, values: np.ndarray, first: int = -1, last: int = -1,
                        f64acc: bool = False):
        values = np.ascontiguousarray(values, np.float32)
        out = np.zeros(2, np.float32)
        fn = self.lib.ora_create2clusters_f64acc if f64acc else self.lib.ora_create2clusters_f32
        fn(values, len(values), first, last, out)
        return float(out[0]), float(out[1])

    def zwindows(self, samples: np.ndarray, shape_zyx, windowsize: int):
        nz, ny, nx = shape_zyx
        st = np.zeros(nz, np.int32)
        en = np.zeros(nz, np.int32)
        self.lib.ora_zwindows(np.ascontiguousarray(samples, np.int64), len(samples),
                              (C.c_int * 3)(nx, ny, nz), windowsize, st, en)
        return st, en

    def noise_from_patchstd(self, patchstd, samples, shape_zyx, mode: str, zwindow: int = 100,
                            stds_from_mean: float = 1.0, f64acc: bool = False) -> np.ndarray:
        nz, ny, nx = shape_zyx
        sig = np.zeros(nz, np.float32)
        self.lib.ora_noise_from_patchstd(np.ascontiguousarray(patchstd, np.float32),
                                         np.ascontiguousarray(samples, np.int64), len(samples),
                                         (C.c_int * 3)(nx, ny, nz),
                                         0 if mode == "global" else 1, zwindow,
                                         stds_from_mean, int(f64acc), sig)
        return sig

    def noise_estimate(self, vol, mode="global", n_samples=100000, patchsize=15, zwindow=100,
                       stds_from_mean=1.0, mask=0, seed=0, f64acc=False, samples=None):
        if samples is None:
            samples = self.draw_samples(vol.shape, n_samples, patchsize, mask, seed)
        ps = self.patchstd(vol, samples, patchsize)
        return self.noise_from_patchstd(ps, samples, vol.shape, mode, zwindow, stds_from_mean,
                                        f64acc)


class _RefParams(C.Structure):
    _fields_ = _CParams._fields_


class _RefNoiseParams(C.Structure):
    _fields_ = [
        ("mode", C.c_char_p),
        ("zwindow", C.c_int),
        ("sigma", C.c_float * 2),
        ("stds_from_mean", C.c_float),
        ("circular_mask_diameter", C.c_int),
    ]


class _RefRgbParams(C.Structure):
    _fields_ = [
        ("alpha", C.c_float),
        ("maxiterations", C.c_int),
        ("mode", C.c_char_p),
        ("sigma", C.c_float * 2),
        ("n_samples", C.c_ulonglong),
        ("patchsize", C.c_int),
        ("stds_from_mean", C.c_float),
        ("continuous_estimate", C.c_int),
        ("circular_mask_diameter", C.c_int),
        ("seed", C.c_uint),
        ("stabilize_variance", C.c_int),
        ("independent_channels", C.c_int),
        ("average_channelsigma", C.c_int),
        ("keep_iterations", C.c_int),
    ]


def reference_available() -> bool:
    return os.path.exists(REF_SO)


def reference_gpu_available() -> bool:
    return os.path.exists(REF_GPU_SO)


class ReferenceGPU:
    """The reference's own GPU class, whole-stack path (iternlm_gpu.cu:1651-1728)
    on device 0, driven as the reference driver drives it."""

    def __init__(self, path: str = REF_GPU_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref_gpu`")
        L = self.lib = C.CDLL(path)
        L.ref_gpu_run.restype = C.c_int
        L.ref_gpu_run.argtypes = [C.c_int * 3, C.c_int, C.c_int, C.c_int, C.c_float, _f32p, _f32p,
                                  C.c_int, C.c_void_p, _f64p]

    def denoise(self, raw: np.ndarray, patch_radius: int, search_radius: int, sigmas: np.ndarray,
                nslices: int = 11, beta: float = 1.0, want_result: bool = True):
        """Runs len(sigmas) iterations; returns (result or None, ms per
        Run_GaussianNoise call). Raises if the stack does not fit in one pass."""
        raw = np.ascontiguousarray(raw, np.float32)
        sig = np.ascontiguousarray(np.atleast_2d(sigmas), np.float32)
        iters = sig.shape[0]
        out = np.empty_like(raw) if want_result else None
        ms = np.zeros(iters, np.float64)
        rc = self.lib.ref_gpu_run(_shape3(raw), patch_radius, search_radius, nslices, beta, raw.ravel(),
                                  sig.ravel(), iters, out.ctypes.data if want_result else None, ms)
        if rc != 0:
            raise RuntimeError(f"reference GPU run failed: {rc}")
        return out, ms


class Reference:
    """The reference's own CPU implementation (unmodified sources)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref`")
        L = self.lib = C.CDLL(path)
        L.ref_denoise.restype = C.c_double
        L.ref_denoise.argtypes = [_f32p, C.c_int * 3, C.POINTER(_RefParams), _f32p, C.c_int,
                                  _f32p, C.c_void_p, C.c_int]
        L.ref_tables.restype = C.c_int
        L.ref_tables.argtypes = [C.c_int * 3, C.POINTER(_RefParams), _i64p, C.POINTER(C.c_int),
                                 _i64p, C.POINTER(C.c_int), _f32p, C.c_int]
        L.ref_pad_reflective.argtypes = [_f32p, C.c_int * 3, C.c_int * 6, _f32p]
        L.ref_noise_create.restype = C.c_void_p
        L.ref_noise_create.argtypes = [C.c_int * 3, C.c_ulonglong, C.c_int, C.c_uint]
        L.ref_noise_estimate.restype = C.c_int
        L.ref_noise_estimate.argtypes = [C.c_void_p, _f32p, C.POINTER(_RefNoiseParams), _f32p]
        L.ref_noise_samples.restype = C.c_longlong
        L.ref_noise_samples.argtypes = [C.c_void_p, _i64p, C.c_longlong]
        L.ref_noise_sigma1.restype = C.c_float
        L.ref_noise_sigma1.argtypes = [C.c_void_p]
        L.ref_noise_destroy.argtypes = [C.c_void_p]
        L.ref_patchstd.argtypes = [_f32p, C.c_int * 3, _i64p, C.c_longlong, C.c_int, _f32p]
        L.ref_create2clusters.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _f32p]
        L.ref_rgb_job.restype = C.c_int
        L.ref_rgb_job.argtypes = [_f32p, _f32p, _f32p, C.c_int, C.c_int, C.POINTER(_RefParams),
                                  C.POINTER(_RefRgbParams), _f32p, _f32p, _f32p, C.c_void_p,
                                  C.c_float * 3, C.c_float * 3]

    def denoise(self, raw: np.ndarray, p: FilterParams, sigmas: np.ndarray, n_threads: int = 0,
                all_iters: bool = False):
        """Returns (result, seconds inside Run_GaussianNoise)."""
        raw = np.ascontiguousarray(raw, np.float32)
        sig = np.ascontiguousarray(np.atleast_2d(sigmas), np.float32)
        out = np.empty_like(raw)
        allbuf = np.empty((sig.shape[0],) + raw.shape, np.float32) if all_iters else None
        cp = _RefParams.from_buffer_copy(_cparams(p))
        secs = self.lib.ref_denoise(raw.ravel(), _shape3(raw), C.byref(cp), sig.ravel(),
                                    sig.shape[0], out.ravel(),
                                    allbuf.ctypes.data if all_iters else None, n_threads)
        return (allbuf if all_iters else out), secs

    def tables(self, p: FilterParams, shape_padded_xyz):
        cp = _RefParams.from_buffer_copy(_cparams(p))
        mx = 40000
        s = np.zeros(mx, np.int64)
        q = np.zeros(mx, np.int64)
        w = np.zeros(mx, np.float32)
        ns, nq = C.c_int(0), C.c_int(0)
        rc = self.lib.ref_tables((C.c_int * 3)(*shape_padded_xyz), C.byref(cp), s, C.byref(ns), q,
                                 C.byref(nq), w, mx)
        assert rc == 0
        return s[:ns.value].copy(), q[:nq.value].copy(), w[:nq.value].copy()

    def pad_reflective(self, vol: np.ndarray, pad) -> np.ndarray:
        vol = np.ascontiguousarray(vol, np.float32)
        nz, ny, nx = vol.shape
        out = np.empty((nz + 2 * pad[2], ny + 2 * pad[1], nx + 2 * pad[0]), np.float32)
        p6 = (C.c_int * 6)(pad[0], pad[1], pad[2], pad[0], pad[1], pad[2])
        self.lib.ref_pad_reflective(vol.ravel(), _shape3(vol), p6, out.ravel())
        return out

    def noise_session(self, shape_zyx, n_samples=100000, patchsize=15, seed=0):
        return _RefNoiseSession(self, shape_zyx, n_samples, patchsize, seed)

    def patchstd(self, vol, samples, patchsize=15):
        vol = np.ascontiguousarray(vol, np.float32)
        out = np.empty(len(samples), np.float32)
        self.lib.ref_patchstd(vol.ravel(), _shape3(vol), np.ascontiguousarray(samples, np.int64),
                              len(samples), patchsize, out)
        return out

    def create2clusters(self, values, first=-1, last=-1):
        values = np.ascontiguousarray(values, np.float32)
        out = np.zeros(2, np.float32)
        self.lib.ref_create2clusters(values, len(values), first, last, out)
        return float(out[0]), float(out[1])

    def rgb_job(self, rgb, p: FilterParams, alpha=0.5, maxiterations=4, mode="global",
                sigma=(0.0, 0.0), n_samples=2048, patchsize=15, stds_from_mean=1.0,
                continuous=False, mask=0, seed=0, stabilize=True, independent=False,
                average=True, keep_iterations=True):
        """The colour driver's job on one image (color_denoising.h:19-150) with
        the reference's own transforms, noise estimate and three-channel
        filter. rgb: three (ny, nx) planes. Returns (final planes, per-iteration
        saved planes or None, sigma_first, sigma_last)."""
        r, g, b = (np.ascontiguousarray(a, np.float32) for a in rgb)
        ny, nx = r.shape
        cp = _RefRgbParams(alpha, maxiterations, mode.encode(), (C.c_float * 2)(*sigma), n_samples,
                           patchsize, stds_from_mean, int(continuous), mask, seed, int(stabilize),
                           int(independent), int(average), int(keep_iterations))
        rp = _RefParams(*[getattr(_cparams(p), f) for f, _ in _CParams._fields_])
        out = [np.empty((ny, nx), np.float32) for _ in range(3)]
        its = np.empty((maxiterations, 3, ny, nx), np.float32) if keep_iterations else None
        s0, s1 = (C.c_float * 3)(), (C.c_float * 3)()
        self.lib.ref_rgb_job(r, g, b, nx, ny, C.byref(rp), C.byref(cp), out[0], out[1], out[2],
                             its.ctypes.data if its is not None else None, s0, s1)
        return out, its, np.array(s0[:], np.float32), np.array(s1[:], np.float32)


class _RefNoiseSession:
    def __init__(self, ref: Reference, shape_zyx, n_samples, patchsize, seed):
        self.ref = ref
        nz, ny, nx = shape_zyx
        self.nz = nz
        self.h = ref.lib.ref_noise_create((C.c_int * 3)(nx, ny, nz), n_samples, patchsize, seed)
        self.n_samples = n_samples

    def estimate(self, vol, mode="global", zwindow=100, sigma=(0.0, 0.0), stds_from_mean=1.0,
                 mask=0) -> np.ndarray:
        np_ = _RefNoiseParams()
        np_.mode = mode.encode()
        np_.zwindow = zwindow
        np_.sigma[0], np_.sigma[1] = sigma
        np_.stds_from_mean = stds_from_mean
        np_.circular_mask_diameter = mask
        out = np.zeros(self.nz, np.float32)
        self.ref.lib.ref_noise_estimate(self.h, np.ascontiguousarray(vol, np.float32).ravel(),
                                        C.byref(np_), out)
        return out

    def samples(self) -> np.ndarray:
        out = np.zeros(self.n_samples, np.int64)
        n = self.ref.lib.ref_noise_samples(self.h, out, self.n_samples)
        return out[:n]

    def sigma1(self) -> float:
        return self.ref.lib.ref_noise_sigma1(self.h)

    def close(self):
        if self.h:
            self.ref.lib.ref_noise_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
