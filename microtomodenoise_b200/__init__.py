"""iterNLM on B200: the iterative 3D nonlocal-means filter and the two-cluster
noise estimators of iternlm/microtomodenoise (iterNLM_v0.3), as hand-written
sm_100a CUDA kernels behind a C ABI (include/inlm.h).

The Python classes mirror the reference's C++ call surface:

* ``DenoiseParameters``  <- protocol::DenoiseParameters (denoise_parameters.h:9-74)
* ``IterativeNLM_GPU``   <- denoise::IterativeNLM_GPU (Denoiser/iternlm_gpu.h:20-56)
* ``NoiseLevel``         <- noise::NoiseLevel (Noise/noiselevel.h:14-46)
* ``denoise()``          <- the iterNLM driver's sigma0/sigma1 schedule and loop
                            (main.cpp:327-545), run on the device

Volumes are numpy float32 arrays of shape (nz, ny, nx) (x fastest), or device
pointers (ints) for the ``*_device`` forms. Everything runs in libinlm.so; if
it is missing, importing this package's GPU classes raises.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Tuple

import numpy as np

from . import _lib
from ._lib import InlmError, InlmParams, NOISE_MODES, PRECISIONS

__all__ = ["DenoiseParameters", "IterativeNLM_GPU", "NoiseLevel", "Batch", "denoise",
           "denoise_multi", "denoise_f64_blocks", "stream_denoise", "Blocks", "InlmError"]


@dataclass
class DenoiseParameters:
    """Knobs and defaults of protocol::DenoiseParameters (denoise_parameters.h:11-73)
    that the GPU path uses, plus the device-side additions."""

    alpha: float = 0.5
    maxiterations: int = 4
    nslices: int = 11
    radius_searchspace: Tuple[int, int, int] = (10, 10, 10)
    radius_patchspace: Tuple[int, int, int] = (1, 1, 1)
    beta: float = 1.0
    z_anisotropy: float = 1.0
    # NoiseLevel
    noise_mode: str = "z-adaptive"
    zwindow: int = 100
    sigma: Tuple[float, float] = (0.0, 0.0)
    n_samples: int = 100000
    patchsize: int = 15
    stds_from_mean: float = 1.0
    continuous_estimate: bool = False
    circular_mask_diameter: int = 0
    noise_seed: int = 0
    # GPU
    deviceID: int = 0
    precision: str = "f32"
    weight_table: str = "cpu"   # "cpu" = the reference CPU filter's table, "distweight"

    def to_c(self) -> InlmParams:
        p = InlmParams()
        _lib.load().inlm_default_params(C.byref(p))
        p.alpha = self.alpha
        p.maxiterations = self.maxiterations
        p.nslices = self.nslices
        for i in range(3):
            p.search_radius[i] = int(self.radius_searchspace[i])
            p.patch_radius[i] = int(self.radius_patchspace[i])
        p.beta = self.beta
        p.z_anisotropy = self.z_anisotropy
        if self.noise_mode not in NOISE_MODES:
            raise ValueError(f"unknown noise mode {self.noise_mode!r}")
        p.noise_mode = NOISE_MODES[self.noise_mode]
        p.zwindow = self.zwindow
        p.sigma[0], p.sigma[1] = float(self.sigma[0]), float(self.sigma[1])
        p.n_samples = int(self.n_samples)
        p.noise_patchsize = int(self.patchsize)
        p.stds_from_mean = self.stds_from_mean
        p.continuous_estimate = int(bool(self.continuous_estimate))
        p.circular_mask_diameter = int(self.circular_mask_diameter)
        p.noise_seed = int(self.noise_seed) & 0xFFFFFFFF
        p.device_id = int(self.deviceID)
        p.precision = PRECISIONS[self.precision]
        p.weight_table = 0 if self.weight_table == "cpu" else 1
        return p


def _shape_c(shape_zyx) -> "C.Array":
    nz, ny, nx = shape_zyx
    return (C.c_int * 3)(int(nx), int(ny), int(nz))


def _f32c(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


class IterativeNLM_GPU:
    """denoise::IterativeNLM_GPU on one B200.

    configure_device(shape, params) allocates and builds the tables;
    set_sigma(sigma); Run_GaussianNoise(iter, instack); get_result();
    free_device(). Shapes are (nz, ny, nx).
    """

    def __init__(self):
        self._h = C.c_void_p(None)
        self.shape = None
        self.n_parallelslices = 0
        self.resumed = False

    def configure_device(self, shape_zyx, params: DenoiseParameters) -> int:
        L = _lib.load()
        cp = params.to_c()
        rc = L.inlm_denoiser_create(_shape_c(shape_zyx), C.byref(cp), C.byref(self._h))
        if rc == -3:
            return -1  # no GPU, as the reference reports it (iternlm_gpu.cu:1444)
        _lib.check(rc, "configure_device")
        self.shape = tuple(int(s) for s in shape_zyx)
        self.n_parallelslices = self.shape[0]
        return self.n_parallelslices

    def _need(self):
        if not self._h:
            raise InlmError(-5, "IterativeNLM_GPU", "configure_device first")

    def set_sigma(self, sigma: np.ndarray) -> None:
        self._need()
        s = _f32c(sigma)
        assert s.shape == (self.shape[0],)
        _lib.check(_lib.load().inlm_set_sigma(self._h, s.ctypes.data), "set_sigma")

    def Run_GaussianNoise(self, iteration: int, instack: Optional[np.ndarray] = None) -> None:
        self._need()
        ptr = None
        if iteration == 1:
            if instack is None:
                raise ValueError("iteration 1 needs the raw stack")
            instack = _f32c(instack)
            assert instack.shape == self.shape
            ptr = instack.ctypes.data
        _lib.check(_lib.load().inlm_run_iteration(self._h, int(iteration), ptr),
                   "Run_GaussianNoise")

    def Run_GaussianNoise_device(self, iteration: int, raw_dev_ptr: Optional[int] = None) -> None:
        self._need()
        _lib.check(_lib.load().inlm_run_iteration_device(self._h, int(iteration), raw_dev_ptr),
                   "Run_GaussianNoise_device")

    def get_result(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        self._need()
        if out is None:
            out = np.empty(self.shape, np.float32)
        _lib.check(_lib.load().inlm_get_result(self._h, out.ctypes.data), "get_result")
        return out

    def set_result(self, iteration: int, result: np.ndarray,
                   instack: Optional[np.ndarray] = None) -> None:
        """--resume: installs a finished iteration read back from disk in place
        of computing it (iternlm_gpu.cu:1665-1697); iteration 1 also needs the
        raw stack, which is prepared as a computed iteration 1 would."""
        self._need()
        result = _f32c(result)
        assert result.shape == self.shape
        ptr = None
        if iteration == 1:
            if instack is None:
                raise ValueError("iteration 1 needs the raw stack")
            instack = _f32c(instack)
            assert instack.shape == self.shape
            ptr = instack.ctypes.data
        _lib.check(_lib.load().inlm_set_result(self._h, int(iteration), result.ctypes.data, ptr),
                   "set_result")

    def get_result_device(self, out_dev_ptr: int) -> None:
        self._need()
        _lib.check(_lib.load().inlm_get_result_device(self._h, out_dev_ptr), "get_result_device")

    def denoise(self, raw, on_device: bool = False, out=None):
        """Whole job (noise estimates + all iterations) on the device.
        Returns (result, sigma0, sigma1)."""
        self._need()
        nz = self.shape[0]
        s0 = np.zeros(nz, np.float32)
        s1 = np.zeros(nz, np.float32)
        if on_device:
            rc = _lib.load().inlm_denoise(self._h, raw, out, 1, s0.ctypes.data, s1.ctypes.data)
            _lib.check(rc, "denoise")
            return out, s0, s1
        raw = _f32c(raw)
        if out is None:
            out = np.empty(self.shape, np.float32)
        rc = _lib.load().inlm_denoise(self._h, raw.ctypes.data, out.ctypes.data, 0,
                                      s0.ctypes.data, s1.ctypes.data)
        _lib.check(rc, "denoise")
        return out, s0, s1

    def set_stream(self, stream_ptr: int) -> None:
        self._need()
        _lib.check(_lib.load().inlm_set_stream(self._h, stream_ptr), "set_stream")

    def filter_kernel_ms(self):
        """(average ms, launches) of the filter kernel since the last call."""
        self._need()
        ms = C.c_double(0)
        n = C.c_int(0)
        _lib.check(_lib.load().inlm_filter_kernel_ms(self._h, C.byref(ms), C.byref(n)),
                   "filter_kernel_ms")
        return ms.value, n.value

    def describe(self) -> str:
        self._need()
        buf = C.create_string_buffer(512)
        _lib.check(_lib.load().inlm_describe(self._h, buf, 512), "describe")
        return buf.value.decode()

    def autotune(self) -> str:
        """Chooses the tiled FP32 kernel configuration by timing (results unchanged)."""
        self._need()
        buf = C.create_string_buffer(512)
        _lib.check(_lib.load().inlm_autotune(self._h, buf, 512), "autotune")
        return buf.value.decode()

    def select_tile_form(self, form: str = "auto") -> str:
        """Plain FP32 kernel family: "auto", "tile" (the tiled kernels without
        warp specialisation), "column" (the column form, patch radius 1) or
        "ws" (the warp-specialised kernel). Results do not change; returns
        describe()."""
        self._need()
        code = {"auto": 0, "tile": 1, "column": 2, "ws": 3}[form]
        _lib.check(_lib.load().inlm_select_tile_form(self._h, code), "select_tile_form")
        return self.describe()

    def n_search_offsets(self) -> int:
        """Number of search offsets S of the configured geometry."""
        self._need()
        return int(self.describe().split(" S=")[1].split()[0])

    def tile_grid(self):
        """(tile shape {x,y,z}, tile counts {x,y,z}) of the filter kernel."""
        self._need()
        ts, tc = (C.c_int * 3)(), (C.c_int * 3)()
        _lib.check(_lib.load().inlm_tile_grid(self._h, ts, tc), "tile_grid")
        return tuple(ts), tuple(tc)

    def attach_proposal(self, net, k=256, min_mass: float = 0.95, tiles_x: int = 1,
                        rel_mass=0.0) -> None:
        """Evaluates only each 8^3 tile's top-k offsets predicted by `net` (a
        proposal.ProposalNet), or every offset where the predicted kept mass
        is below min_mass, or below rel_mass x its mean over the volume.
        tiles_x = 4 ranks one list per 4 tiles along x (32 x 8 x 8 blocks, the
        full-width kernel). k and rel_mass may be per-iteration sequences
        (inlm_proposal_schedule: iteration i uses entry min(i, n) - 1; k 0 =
        full search that iteration). net=None returns to full search. FP16
        form only."""
        self._need()
        h = net._h if net is not None else None
        ks, rels = _schedule(k, rel_mass)
        _lib.check(_lib.load().inlm_attach_proposal_ex(self._h, h, max(int(ks.max()), 1), float(min_mass),
                                                       float(rels[-1]), int(tiles_x)), "attach_proposal")
        if net is not None and len(ks) > 1:
            _lib.check(_lib.load().inlm_proposal_schedule(self._h, len(ks), ks.ctypes.data, rels.ctypes.data),
                       "proposal_schedule")
        self._proposal = net  # keep the network alive while attached

    def proposal_stats(self) -> dict:
        """Last iteration: tiles, fallback tiles, offsets evaluated, full-search
        cost (CTAs x S) and S."""
        self._need()
        st = (C.c_int64 * 5)()
        _lib.check(_lib.load().inlm_proposal_stats(self._h, st), "proposal_stats")
        t, fb, ev, full, S = (int(v) for v in st)
        return dict(tiles=t, fallback_tiles=fb, offsets_evaluated=ev, full_search=full, S=S,
                    fraction_evaluated=ev / max(full, 1))

    def weight_map(self, map_dev_ptr: int) -> None:
        """Per-8^3-tile weight mass of every search offset of the last
        iteration (device array of tiles x S floats)."""
        self._need()
        _lib.check(_lib.load().inlm_weight_map(self._h, map_dev_ptr), "weight_map")

    def net_input(self, vol_dev_ptr: int, scale_dev_ptr: int) -> None:
        """The last iteration's previous iterate (nz*ny*nx floats) and per-slice
        scale (nz floats), as the proposal network reads them."""
        self._need()
        _lib.check(_lib.load().inlm_net_input(self._h, vol_dev_ptr, scale_dev_ptr), "net_input")

    def free_device(self) -> None:
        if self._h:
            _lib.load().inlm_denoiser_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.free_device()
        except Exception:
            pass


class NoiseLevel:
    """noise::NoiseLevel(n_samples, patchsize, shape) on the device.

    get_noiselevel(stack, params) returns the per-slice sigma (nz floats).
    Sample positions are drawn on the first call from params.noise_seed (the
    reference seeds with time(NULL)) and reused afterwards.
    """

    def __init__(self, n_samples: int, patchsize: int, shape_zyx, seed: int = 0,
                 device: int = 0):
        self.shape = tuple(int(s) for s in shape_zyx)
        self._h = C.c_void_p(None)
        _lib.check(_lib.load().inlm_noise_create(_shape_c(shape_zyx), int(n_samples), int(patchsize),
                                                 int(seed) & 0xFFFFFFFF, int(device),
                                                 C.byref(self._h)), "NoiseLevel")
        self.n_samples = int(n_samples)

    def get_noiselevel(self, stack, params: DenoiseParameters, on_device: bool = False) -> np.ndarray:
        cp = params.to_c()
        out = np.zeros(self.shape[0], np.float32)
        if on_device:
            ptr = stack
        else:
            stack = _f32c(stack)
            assert stack.shape == self.shape
            ptr = stack.ctypes.data
        _lib.check(_lib.load().inlm_noise_estimate(self._h, C.byref(cp), ptr, int(on_device),
                                                   out.ctypes.data), "get_noiselevel")
        if params.noise_mode == "semimanual":
            params.sigma = (params.sigma[0], float(cp.sigma[1]))
        return out

    def samples(self) -> np.ndarray:
        out = np.zeros(self.n_samples, np.int64)
        n = C.c_uint64(0)
        _lib.check(_lib.load().inlm_noise_samples(self._h, out.ctypes.data, self.n_samples,
                                                  C.byref(n)), "samples")
        return out[: n.value]

    def patchstd(self) -> np.ndarray:
        out = np.zeros(self.n_samples, np.float32)
        _lib.check(_lib.load().inlm_noise_patchstd(self._h, out.ctypes.data, self.n_samples),
                   "patchstd")
        return out

    def close(self):
        if self._h:
            _lib.load().inlm_noise_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many volumes of different sizes and radii filtered together: one
    persistent kernel per iteration over all their tiles, the whole schedule
    replayed as a CUDA graph (inlm_batch_*). Plain FP32 filter; every volume's
    result equals its single-volume run."""

    def __init__(self, shapes_zyx, params):
        L = _lib.load()
        n = len(shapes_zyx)
        if isinstance(params, DenoiseParameters):
            params = [params] * n
        assert len(params) == n
        self.shapes = [tuple(int(v) for v in s) for s in shapes_zyx]
        sh = (C.c_int * (3 * n))()
        for i, (nz, ny, nx) in enumerate(self.shapes):
            sh[3 * i:3 * i + 3] = [nx, ny, nz]
        ps = (InlmParams * n)(*[p.to_c() for p in params])
        self._h = C.c_void_p(None)
        _lib.check(L.inlm_batch_create(n, sh, ps, C.byref(self._h)), "batch_create")
        self.n = n
        self.last_ms = None

    def run(self, raws, outs=None, on_device: bool = False):
        """raws: list of float32 arrays (host) or device pointers (on_device)."""
        n = self.n
        if on_device:
            rp = (C.c_void_p * n)(*raws)
            op = (C.c_void_p * n)(*outs)
        else:
            raws = [_f32c(r) for r in raws]
            for r, s in zip(raws, self.shapes):
                assert r.shape == s
            if outs is None:
                outs = [np.empty(s, np.float32) for s in self.shapes]
            rp = (C.c_void_p * n)(*[r.ctypes.data for r in raws])
            op = (C.c_void_p * n)(*[o.ctypes.data for o in outs])
        ms = C.c_float(0)
        _lib.check(_lib.load().inlm_batch_run(self._h, rp, op, int(on_device), C.byref(ms)),
                   "batch_run")
        self.last_ms = ms.value
        return outs

    def describe(self) -> str:
        buf = C.create_string_buffer(8192)
        _lib.check(_lib.load().inlm_batch_describe(self._h, buf, 8192), "batch_describe")
        return buf.value.decode()

    def close(self):
        if self._h:
            _lib.load().inlm_batch_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _schedule(k, rel_mass):
    """Per-iteration (k, rel_mass) arrays from scalars or sequences (the
    shorter one repeats its last entry)."""
    ks = np.atleast_1d(np.asarray(k, np.int32))
    rels = np.atleast_1d(np.asarray(rel_mass, np.float32))
    n = max(len(ks), len(rels))
    ks = np.ascontiguousarray(np.concatenate([ks, np.full(n - len(ks), ks[-1], np.int32)]))
    rels = np.ascontiguousarray(np.concatenate([rels, np.full(n - len(rels), rels[-1], np.float32)]))
    return ks, rels


def stream_denoise(raw: np.ndarray, params: DenoiseParameters, slab_depth: int = 64,
                   net=None, k=256, min_mass: float = 0.95, out: Optional[np.ndarray] = None,
                   tiles_x: int = 1, rel_mass=0.0):
    """The denoise schedule for a host-resident volume, filtered in z-slabs
    (inlm_stream_denoise_sched; tiles_x, rel_mass and per-iteration k /
    rel_mass sequences as IterativeNLM_GPU.attach_proposal, the relative
    threshold's mean taken per sub-volume). Returns (result, sigma0, sigma1,
    stats) with stats = {ms, h2d_bytes, d2h_bytes, slabs, halo, slab_depth}."""
    raw = _f32c(raw)
    if out is None:
        out = np.empty(raw.shape, np.float32)
    nz = raw.shape[0]
    s0 = np.zeros(nz, np.float32)
    s1 = np.zeros(nz, np.float32)
    st = np.zeros(6, np.float64)
    cp = params.to_c()
    ks, rels = _schedule(k, rel_mass)
    rc = _lib.load().inlm_stream_denoise_sched(_shape_c(raw.shape), C.byref(cp), raw.ctypes.data,
                                               out.ctypes.data, int(slab_depth),
                                               net._h if net is not None else None, len(ks), ks.ctypes.data,
                                               rels.ctypes.data, float(min_mass), int(tiles_x), s0.ctypes.data,
                                               s1.ctypes.data, st.ctypes.data)
    _lib.check(rc, "stream_denoise")
    keys = ("ms", "h2d_bytes", "d2h_bytes", "slabs", "halo", "slab_depth")
    return out, s0, s1, dict(zip(keys, st.tolist()))


class Blocks:
    """One iteration at a time over host-resident volumes (inlm_blocks_*, the
    host-RAM Run_GaussianNoise_GPUBlocks): z-slabs of slab_depth slices on one
    device, or the stack split over several device_ids. The caller sets sigma
    before iterations and estimates the noise itself."""

    def __init__(self, shape_zyx, params: DenoiseParameters, device_ids=(0,), slab_depth: int = 64):
        self.shape = tuple(int(v) for v in shape_zyx)
        ids = np.ascontiguousarray(device_ids, np.int32)
        cp = params.to_c()
        self._h = C.c_void_p(None)
        _lib.check(_lib.load().inlm_blocks_create(_shape_c(self.shape), C.byref(cp), len(ids), ids.ctypes.data,
                                                  int(slab_depth), C.byref(self._h)), "blocks_create")
        self._net = None

    def attach_proposal(self, net, k, min_mass: float = 0.0, tiles_x: int = 4, rel_mass=0.0):
        """k and rel_mass: scalars or per-iteration sequences (as
        IterativeNLM_GPU.attach_proposal)."""
        ks, rels = _schedule(k, rel_mass)
        _lib.check(_lib.load().inlm_blocks_attach_proposal(self._h, net._h, max(int(ks.max()), 1), float(min_mass),
                                                           float(rels[-1]), int(tiles_x)), "blocks_attach_proposal")
        if len(ks) > 1:
            _lib.check(_lib.load().inlm_blocks_proposal_schedule(self._h, len(ks), ks.ctypes.data, rels.ctypes.data),
                       "blocks_proposal_schedule")
        self._net = net

    def set_sigma(self, sigma) -> None:
        s = _f32c(sigma)
        _lib.check(_lib.load().inlm_blocks_set_sigma(self._h, s.ctypes.data), "blocks_set_sigma")

    def run_iteration(self, it: int, raw: np.ndarray, prev: Optional[np.ndarray], out: np.ndarray) -> None:
        _lib.check(_lib.load().inlm_blocks_run_iteration(self._h, int(it), raw.ctypes.data,
                                                         prev.ctypes.data if prev is not None else None,
                                                         out.ctypes.data), "blocks_run_iteration")

    def close(self) -> None:
        if self._h:
            _lib.load().inlm_blocks_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def denoise_multi(raw: np.ndarray, params: DenoiseParameters, device_ids, out: Optional[np.ndarray] = None):
    """The denoise schedule on a host-resident stack split in z over the GPUs
    device_ids (inlm_denoise_multi; ids may repeat). Returns (result, sigma0,
    sigma1), equal to denoise()'s."""
    raw = _f32c(raw)
    if out is None:
        out = np.empty(raw.shape, np.float32)
    nz = raw.shape[0]
    s0 = np.zeros(nz, np.float32)
    s1 = np.zeros(nz, np.float32)
    ids = np.ascontiguousarray(device_ids, np.int32)
    cp = params.to_c()
    rc = _lib.load().inlm_denoise_multi(_shape_c(raw.shape), C.byref(cp), raw.ctypes.data, out.ctypes.data,
                                        len(ids), ids.ctypes.data, s0.ctypes.data, s1.ctypes.data)
    _lib.check(rc, "denoise_multi")
    return out, s0, s1


def denoise_f64_blocks(raw, params: DenoiseParameters, sigmas: np.ndarray, corners, size,
                       shape=None) -> list:
    """FP64 full-search result of the last of len(sigmas) iterations on
    size = (dz, dy, dx) blocks at the (z, y, x) corners of a volume, on the GPU
    (inlm_denoise_f64_blocks): the precision reference of the FP16 and learned
    forms. raw: a host array, or a device pointer with shape=(nz, ny, nx).
    sigmas: (n_iter, nz). Returns one float64 (dz, dy, dx) array per block."""
    on_device = not isinstance(raw, np.ndarray)
    if not on_device:
        raw = _f32c(raw)
        shape = raw.shape
    sig = np.ascontiguousarray(np.atleast_2d(sigmas), np.float32)
    cxyz = np.ascontiguousarray([[c[2], c[1], c[0]] for c in corners], np.int32)
    sz = (C.c_int * 3)(int(size[2]), int(size[1]), int(size[0]))
    out = np.empty((len(corners),) + tuple(size), np.float64)
    cp = params.to_c()
    rc = _lib.load().inlm_denoise_f64_blocks(_shape_c(shape), C.byref(cp), raw if on_device else raw.ctypes.data,
                                             int(on_device), sig.ctypes.data, sig.shape[0], cxyz.ctypes.data,
                                             len(corners), sz, out.ctypes.data)
    _lib.check(rc, "denoise_f64_blocks")
    return list(out)


def denoise(raw: np.ndarray, params: Optional[DenoiseParameters] = None):
    """Runs the iterNLM schedule on one GPU; returns (result, sigma0, sigma1)."""
    params = params or DenoiseParameters()
    g = IterativeNLM_GPU()
    rc = g.configure_device(raw.shape, params)
    if rc < 0:
        raise InlmError(-3, "denoise", "no CUDA device")
    try:
        return g.denoise(raw)
    finally:
        g.free_device()
