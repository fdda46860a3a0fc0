"""Multi-GPU z-slab sharding of the whole iterNLM job: one process per GPU,
torch.distributed (NCCL over NVLink, or gloo) for the two exchanges the job
has, the library for everything else.

The reference splits a stack in z across ``n_gpus`` in
``IterativeNLM_GPU::Run_GaussianNoise_GPUBlocks`` (Denoiser/iternlm_gpu.cu:
1732-2115) and estimates the noise on the host (Noise/noiselevel.cpp:9-95).
Here rank r owns slices [z0_r, z1_r) (multiples of 8, so 8^3 tiles line up
with the unsharded volume) and filters them as a sub-volume with ``halo``
slices of each neighbour on either side:

* after every iteration the ranks swap the ``halo`` boundary slices of their
  own results (P2P send/recv); the next iteration then reads its neighbours'
  current slices, so every owned voxel sees exactly the previous iterate the
  unsharded job sees. The raw halos are swapped once.
* a noise estimate draws the same sample positions on every rank (same seed
  and full-stack shape); each rank measures the patch std of the samples in
  its own slices, one sum all-reduce gives every rank all of them, and the
  two-cluster EM runs replicated.

Owned results are therefore identical to the single-GPU job, bit for bit in
the FP32 form. Requirements: every slab at least ``halo`` slices deep.

    job = ZSlabJob(full_shape_zyx, params, group=None)   # default process group
    out_own, sigma0, sigma1 = job.run(raw_own)           # raw_own: this rank's slices
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Tuple

import numpy as np

from . import _lib

BLOCK = 8  # z granularity of slab boundaries (the 8^3 tile of the FP16 / learned forms)


def slab_bounds(nz: int, world: int, block: int = BLOCK) -> List[Tuple[int, int]]:
    """[z0, z1) per rank: nz split into ``block``-slice units, as evenly as
    possible, lower ranks taking the remainder."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    units = -(-nz // block)
    if units < world:
        raise ValueError(f"{nz} slices give {units} units of {block}: fewer than {world} ranks")
    base, extra = divmod(units, world)
    out, u = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((min(nz, u * block), min(nz, (u + n) * block)))
        u += n
    return out


def halo_depth(params, proposal: bool = False) -> int:
    """Slices of each neighbour a rank keeps: the filter's z padding
    (min(nslices/2, search_z) + patch_z, iternlm_prepare.cpp) rounded up to a
    multiple of 8, and at least 16 with a learned proposal (its network sees
    a 16-slice neighbourhood of each tile)."""
    pz = min(params.nslices // 2, int(params.radius_searchspace[2])) + int(params.radius_patchspace[2])
    h = -(-max(pz, 1) // BLOCK) * BLOCK
    return max(h, 16) if proposal else h


class TorchExchange:
    """The two collectives of the sharded job on a torch.distributed group:
    neighbour halo swaps (P2P) and a sum all-reduce of the patch stds.
    Tensors travel on ``device`` (a CUDA device for NCCL, CPU for gloo)."""

    def __init__(self, group=None, device=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist, self.group = torch, dist, group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        if device is None:
            device = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
        self.device = torch.device(device)

    def _global(self, r: int) -> int:
        return r if self.group is None else self.dist.get_global_rank(self.group, r)

    def swap(self, send_lo, send_hi, recv_lo_shape, recv_hi_shape):
        """Sends send_lo to rank-1 and send_hi to rank+1 and returns what they
        sent back (None where there is no neighbour)."""
        torch, dist = self.torch, self.dist
        ops, recv_lo, recv_hi = [], None, None
        if self.rank > 0:
            recv_lo = torch.empty(recv_lo_shape, dtype=torch.float32, device=self.device)
            ops.append(dist.P2POp(dist.isend, self._as_tensor(send_lo), self._global(self.rank - 1),
                                  self.group))
            ops.append(dist.P2POp(dist.irecv, recv_lo, self._global(self.rank - 1), self.group))
        if self.rank < self.world - 1:
            recv_hi = torch.empty(recv_hi_shape, dtype=torch.float32, device=self.device)
            ops.append(dist.P2POp(dist.isend, self._as_tensor(send_hi), self._global(self.rank + 1),
                                  self.group))
            ops.append(dist.P2POp(dist.irecv, recv_hi, self._global(self.rank + 1), self.group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        return recv_lo, recv_hi

    def allreduce_sum(self, values: np.ndarray) -> np.ndarray:
        t = self.torch.from_numpy(np.ascontiguousarray(values, np.float32)).to(self.device)
        self.dist.all_reduce(t, group=self.group)
        return t.cpu().numpy()

    def _as_tensor(self, x):
        torch = self.torch
        if isinstance(x, np.ndarray):
            x = torch.from_numpy(np.ascontiguousarray(x, np.float32))
        return x.to(self.device).contiguous()


class CudaSlabBackend:
    """One rank's share on its GPU: a denoiser over the rank's sub-volume
    (own slices plus halos) and a noise handle over the full stack's shape.
    Halos move as torch CUDA tensors on the denoiser's stream."""

    def __init__(self, full_shape_zyx, params, z0: int, z1: int, halo: int, proposal=None):
        import torch
        from . import IterativeNLM_GPU
        self.torch = torch
        nz, ny, nx = (int(s) for s in full_shape_zyx)
        self.full = (nz, ny, nx)
        self.params = params
        self.z0, self.z1 = z0, z1
        self.a, self.b = max(0, z0 - halo), min(nz, z1 + halo)
        self.lo, self.own = z0 - self.a, z1 - z0
        self.hi = self.b - z1
        self.dev = torch.device("cuda", int(params.deviceID))
        # one stream for the denoiser and for every torch op on its buffers
        self.stream = torch.cuda.Stream(device=self.dev)
        self.g = IterativeNLM_GPU()
        self.g.configure_device((self.b - self.a, ny, nx), params)
        self.g.set_stream(self.stream.cuda_stream)
        if proposal is not None:
            self.g.attach_proposal(*proposal)
        self.raw = torch.empty((self.b - self.a, ny, nx), dtype=torch.float32, device=self.dev)
        self.buf = torch.empty((self.own, ny, nx), dtype=torch.float32, device=self.dev)
        L = _lib.load()
        self.L = L
        self.cp = params.to_c()
        self.noise = C.c_void_p(None)
        shape = (C.c_int * 3)(nx, ny, nz)
        _lib.check(L.inlm_noise_create(shape, int(params.n_samples), int(params.patchsize),
                                       self.cp.noise_seed, self.cp.device_id, C.byref(self.noise)),
                   "noise_create")

    # raw sub-volume: own slices from the caller, halos from the neighbours
    def set_raw(self, raw_own, raw_lo, raw_hi) -> None:
        r = self.raw
        with self.torch.cuda.stream(self.stream):
            r[self.lo:self.lo + self.own].copy_(
                self.torch.as_tensor(np.ascontiguousarray(raw_own, np.float32)))
            if self.lo:
                r[:self.lo].copy_(raw_lo[-self.lo:])
            if self.hi:
                r[self.lo + self.own:].copy_(raw_hi[:self.hi])
        self.stream.synchronize()

    def result_edges(self, h: int):
        """The first and last h owned result slices (device tensors, complete
        on return, so any stream may send them)."""
        t = self.torch
        with t.cuda.stream(self.stream):
            lo = t.empty((h,) + self.full[1:], dtype=t.float32, device=self.dev)
            hi = t.empty_like(lo)
        _lib.check(self.L.inlm_get_result_slices(self.g._h, self.lo, h, lo.data_ptr(), 1), "get_slices")
        _lib.check(self.L.inlm_get_result_slices(self.g._h, self.lo + self.own - h, h, hi.data_ptr(), 1),
                   "get_slices")
        self.stream.synchronize()
        return lo, hi

    def set_halos(self, recv_lo, recv_hi) -> None:
        keep = []
        with self.torch.cuda.stream(self.stream):
            if self.lo:
                src = recv_lo[-self.lo:].to(self.dev).contiguous()
                keep.append(src)
                _lib.check(self.L.inlm_set_result_slices(self.g._h, 0, self.lo, src.data_ptr(), 1),
                           "set_slices")
            if self.hi:
                src = recv_hi[:self.hi].to(self.dev).contiguous()
                keep.append(src)
                _lib.check(self.L.inlm_set_result_slices(self.g._h, self.lo + self.own, self.hi,
                                                         src.data_ptr(), 1), "set_slices")
        self.stream.synchronize()  # the sources may be freed after this

    def patchstd(self, source: str) -> np.ndarray:
        n = C.c_uint64(0)
        self.L.inlm_noise_samples(self.noise, None, 0, C.byref(n))
        if source == "raw":
            slab = self.raw[self.lo:self.lo + self.own]
        else:
            _lib.check(self.L.inlm_get_result_slices(self.g._h, self.lo, self.own, self.buf.data_ptr(), 1),
                       "get_slices")
            slab = self.buf
        self.stream.synchronize()  # the noise handle runs on its own stream
        count = max(int(n.value), int(self.params.n_samples))
        out = np.zeros(count, np.float32)
        _lib.check(self.L.inlm_noise_patchstd_slab(self.noise, C.byref(self.cp), slab.data_ptr(), 1,
                                                   self.z0, self.own, out.ctypes.data, count),
                   "noise_patchstd_slab")
        self.L.inlm_noise_samples(self.noise, None, 0, C.byref(n))
        return out[:n.value]

    def sigma(self, patchstd: Optional[np.ndarray]) -> np.ndarray:
        sig = np.zeros(self.full[0], np.float32)
        ps = None if patchstd is None else np.ascontiguousarray(patchstd, np.float32)
        _lib.check(self.L.inlm_noise_estimate_from_patchstd(
            self.noise, C.byref(self.cp), None if ps is None else ps.ctypes.data,
            0 if ps is None else ps.size, sig.ctypes.data), "noise_estimate_from_patchstd")
        self.params.sigma = (float(self.cp.sigma[0]), float(self.cp.sigma[1]))
        return sig

    def set_sigma(self, sigma_full: np.ndarray) -> None:
        self.g.set_sigma(np.ascontiguousarray(sigma_full[self.a:self.b], np.float32))

    def iterate(self, it: int) -> None:
        self.g.Run_GaussianNoise_device(it, self.raw.data_ptr() if it == 1 else None)

    def result_own(self) -> np.ndarray:
        out = np.empty((self.own,) + self.full[1:], np.float32)
        _lib.check(self.L.inlm_get_result_slices(self.g._h, self.lo, self.own, out.ctypes.data, 0),
                   "get_slices")
        return out

    def close(self) -> None:
        if self.noise:
            self.L.inlm_noise_destroy(self.noise)
            self.noise = C.c_void_p(None)
        self.g.free_device()


class ZSlabJob:
    """The driver's schedule (main.cpp:327-545: sigma0 on raw, iteration 1,
    sigma1 on its result blended with alpha, iterations 2.., re-estimates
    under continuous_estimate) over z-slabs, one per rank."""

    def __init__(self, full_shape_zyx, params, group=None, exchange=None, backend_factory=None,
                 proposal=None):
        self.full = tuple(int(s) for s in full_shape_zyx)
        self.params = params
        self.ex = exchange if exchange is not None else TorchExchange(group)
        self.bounds = slab_bounds(self.full[0], self.ex.world)
        self.halo = halo_depth(params, proposal is not None)
        for (z0, z1) in self.bounds:
            if self.ex.world > 1 and z1 - z0 < self.halo:
                raise ValueError(f"slab {z0}..{z1 - 1} is shallower than the halo of {self.halo} slices")
        self.z0, self.z1 = self.bounds[self.ex.rank]
        make = backend_factory or (lambda *a: CudaSlabBackend(*a, proposal=proposal))
        self.be = make(self.full, params, self.z0, self.z1, self.halo)

    def _swap_results(self) -> None:
        h = min(self.halo, self.z1 - self.z0)
        lo, hi = self.be.result_edges(h)
        shp = (h,) + self.full[1:]
        r_lo, r_hi = self.ex.swap(lo, hi, shp, shp)
        self.be.set_halos(r_lo, r_hi)

    def _estimate(self, source: str) -> np.ndarray:
        if self.params.noise_mode == "manual":
            return self.be.sigma(None)
        ps = self.be.patchstd(source)
        return self.be.sigma(self.ex.allreduce_sum(ps))

    def run(self, raw_own: np.ndarray):
        """raw_own: this rank's slices [z0, z1) of the raw stack (host).
        Returns (this rank's result slices, sigma0, sigma1) as host arrays,
        sigma1 being the estimate on iteration 1's result before the alpha
        blend (zeros for a single iteration), as inlm_denoise reports it."""
        self.load(raw_own)
        s0, s1 = self.run_loaded()
        return self.be.result_own(), s0, s1

    def load(self, raw_own: np.ndarray) -> None:
        """Puts this rank's raw slices, and its neighbours' raw halo slices,
        on its GPU (the first exchange of the job)."""
        raw_own = np.ascontiguousarray(raw_own, np.float32)
        assert raw_own.shape == (self.z1 - self.z0,) + self.full[1:], raw_own.shape
        h = min(self.halo, self.z1 - self.z0)
        shp = (h,) + self.full[1:]
        lo, hi = raw_own[:h], raw_own[-h:]
        r_lo, r_hi = self.ex.swap(lo, hi, shp, shp)
        self.be.set_raw(raw_own, r_lo, r_hi)

    def run_loaded(self):
        """The whole schedule on the raw volume load() put on the GPU; the
        result stays there (result_own() copies it out). Returns (sigma0,
        sigma1)."""
        p = self.params
        s0 = self._estimate("raw")
        self.be.set_sigma(s0)
        self.be.iterate(1)
        s1 = np.zeros_like(s0)
        if p.maxiterations > 1:
            self._swap_results()
            s1 = self._estimate("result")
            self.be.set_sigma(self._blend(s0, s1))
        for it in range(2, p.maxiterations + 1):
            self.be.iterate(it)
            if it < p.maxiterations:
                self._swap_results()
            if p.continuous_estimate and p.maxiterations > it + 1:
                self.be.set_sigma(self._blend(s0, self._estimate("result")))
        # sigma1 as inlm_denoise reports it: the pre-blend estimate on iteration 1's result
        return s0, s1

    def _blend(self, s0, s1):
        a = np.float32(self.params.alpha)
        return (a * s0 + (np.float32(1) - a) * s1).astype(np.float32)

    def close(self) -> None:
        self.be.close()
