"""Multi-GPU z-slab sharding (microtomodenoise_b200.sharded), host logic on
the CPU: two and three gloo ranks run the sharded schedule with a per-rank
compute stand-in built from the oracle, and their owned slices must equal the
unsharded job bit for bit. This covers the slab split, the halo swaps after
every iteration, the raw halos, the sample ownership and the patch-std
all-reduce, the per-slab sigma slicing and the sigma schedule. The CUDA
backend itself runs in test_sharded_gpu.py."""
from __future__ import annotations

import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from microtomodenoise_b200 import DenoiseParameters, synth
from microtomodenoise_b200.sharded import ZSlabJob, halo_depth, slab_bounds


class OracleSlabBackend:
    """One rank's share computed by the oracle (CPU): the same interface as
    sharded.CudaSlabBackend, for the host-logic tests only."""

    def __init__(self, full, params, z0, z1, halo):
        from oracle.oracle import FilterParams, Port
        self.port = Port()
        self.full, self.params = full, params
        nz, ny, nx = full
        self.z0, self.z1 = z0, z1
        self.a, self.b = max(0, z0 - halo), min(nz, z1 + halo)
        self.lo, self.own, self.hi = z0 - self.a, z1 - z0, self.b - z1
        self.fp = FilterParams(search_radius=params.radius_searchspace,
                               patch_radius=params.radius_patchspace, nslices=params.nslices)
        self.pad = self.port.padding(self.fp)
        self.samples = self.port.draw_samples(full, params.n_samples, params.patchsize,
                                              params.circular_mask_diameter, params.noise_seed)
        self.ncalls = 0
        self.res = None

    @staticmethod
    def _np(x):
        return x.numpy() if hasattr(x, "numpy") else np.asarray(x)

    def set_raw(self, raw_own, raw_lo, raw_hi):
        parts = []
        if self.lo:
            parts.append(self._np(raw_lo)[-self.lo:])
        parts.append(raw_own)
        if self.hi:
            parts.append(self._np(raw_hi)[:self.hi])
        self.raw = np.ascontiguousarray(np.concatenate(parts), np.float32)

    def result_edges(self, h):
        own = self.res[self.lo:self.lo + self.own]
        return own[:h].copy(), own[-h:].copy()

    def set_halos(self, recv_lo, recv_hi):
        if self.lo:
            self.res[:self.lo] = self._np(recv_lo)[-self.lo:]
        if self.hi:
            self.res[self.lo + self.own:] = self._np(recv_hi)[:self.hi]

    def patchstd(self, source):
        vol = self.raw if source == "raw" else self.res
        own = np.ascontiguousarray(vol[self.lo:self.lo + self.own])
        plane = self.full[1] * self.full[2]
        i0, i1 = np.searchsorted(self.samples, [self.z0 * plane, self.z1 * plane])
        out = np.zeros(len(self.samples), np.float32)
        if i1 > i0:
            out[i0:i1] = self.port.patchstd(own, self.samples[i0:i1] - self.z0 * plane,
                                            self.params.patchsize)
        return out

    def sigma(self, ps):
        p = self.params
        if p.noise_mode == "manual":
            v = p.sigma[1 if self.ncalls else 0]
            self.ncalls += 1
            return np.full(self.full[0], v, np.float32)
        self.ncalls += 1
        return self.port.noise_from_patchstd(ps, self.samples, self.full, p.noise_mode, p.zwindow,
                                             p.stds_from_mean, f64acc=True)

    def set_sigma(self, s):
        self.sig = np.ascontiguousarray(s[self.a:self.b], np.float32)

    def iterate(self, it):
        prev = self.raw if it == 1 else self.res
        shape = self.raw.shape
        rp = self.port.pad_reflective(self.raw, self.pad)
        pp = self.port.pad_reflective(prev, self.pad)
        vox = np.arange(int(np.prod(shape)), dtype=np.int64)
        self.res = self.port.filter_voxels(rp, pp, shape, self.fp, self.sig, vox).reshape(shape)

    def result_own(self):
        return self.res[self.lo:self.lo + self.own].copy()

    def close(self):
        pass


class LocalExchange:
    """A world of one: no neighbours, the all-reduce is the identity."""
    rank, world = 0, 1

    def swap(self, *a):
        return None, None

    def allreduce_sum(self, v):
        return v


def _params(**kw):
    base = dict(radius_searchspace=(2, 2, 2), radius_patchspace=(1, 1, 1), nslices=5,
                maxiterations=3, n_samples=3000, patchsize=7, noise_seed=11)
    base.update(kw)
    return DenoiseParameters(**base)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, vol, params, q):
    import torch.distributed as dist
    from microtomodenoise_b200.sharded import TorchExchange
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        ex = TorchExchange(device="cpu")
        job = ZSlabJob(vol.shape, params, exchange=ex, backend_factory=OracleSlabBackend)
        out, s0, s1 = job.run(vol[job.z0:job.z1])
        q.put((rank, job.z0, job.z1, out, s0, s1))
    except Exception as e:  # reported to the parent
        q.put((rank, "error", repr(e)))
    finally:
        dist.destroy_process_group()


def _run_world(world, vol, params):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, vol, params, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
    for r in res:
        assert r[1] != "error", r
    return sorted(res, key=lambda r: r[0])


def _unsharded(vol, params):
    job = ZSlabJob(vol.shape, params, exchange=LocalExchange(), backend_factory=OracleSlabBackend)
    return job.run(vol)


def test_slab_bounds_and_halo():
    assert slab_bounds(64, 2) == [(0, 32), (32, 64)]
    assert slab_bounds(60, 3) == [(0, 24), (24, 48), (48, 60)]
    assert slab_bounds(17, 2) == [(0, 16), (16, 17)]
    with pytest.raises(ValueError):
        slab_bounds(16, 3)
    p = _params(radius_searchspace=(5, 5, 5), radius_patchspace=(2, 2, 2), nslices=11)
    assert halo_depth(p) == 8          # min(11/2, 5) + 2 = 7 -> 8
    assert halo_depth(p, proposal=True) == 16
    p = _params(radius_searchspace=(7, 7, 7), radius_patchspace=(3, 3, 3), nslices=21)
    assert halo_depth(p) == 16         # min(10, 7) + 3 = 10 -> 16


def test_oracle_backend_unsharded_matches_schedule(port):
    """The stand-in's one-iteration steps reproduce the oracle's own job."""
    vol = synth.spheres_volume((16, 24, 24), n_spheres=4, rmin=2, rmax=6, seed=1)
    prm = _params(noise_mode="global")
    out, s0, s1 = _unsharded(vol, prm)
    from oracle.oracle import FilterParams
    fp = FilterParams(search_radius=(2, 2, 2), patch_radius=(1, 1, 1), nslices=5)
    blend = (np.float32(0.5) * s0 + np.float32(0.5) * s1).astype(np.float32)
    want = port.denoise_f32(vol, fp, np.stack([s0, blend, blend]))
    assert np.array_equal(out, want)


@pytest.mark.parametrize("world,mode", [(2, "global"), (2, "z-adaptive"), (3, "manual")])
def test_sharded_equals_unsharded(world, mode):
    vol = synth.spheres_volume((48, 24, 26), n_spheres=6, rmin=2, rmax=7, seed=3)
    prm = _params(noise_mode=mode, zwindow=10, sigma=(0.05, 0.04))
    ref_out, ref_s0, ref_s1 = _unsharded(vol, prm)
    res = _run_world(world, vol, prm)
    bounds = slab_bounds(48, world)
    for rank, z0, z1, out, s0, s1 in res:
        assert (z0, z1) == bounds[rank]
        assert np.array_equal(s0, ref_s0) and np.array_equal(s1, ref_s1)
        assert np.array_equal(out, ref_out[z0:z1]), (rank, np.abs(out - ref_out[z0:z1]).max())


def test_sharded_continuous_estimate():
    vol = synth.spheres_volume((32, 22, 22), n_spheres=5, rmin=2, rmax=6, seed=5)
    prm = _params(noise_mode="global", continuous_estimate=True, maxiterations=4)
    ref_out, _, ref_s1 = _unsharded(vol, prm)
    for rank, z0, z1, out, s0, s1 in _run_world(2, vol, prm):
        assert np.array_equal(s1, ref_s1)
        assert np.array_equal(out, ref_out[z0:z1])


def test_thin_slabs_rejected():
    prm = _params(radius_searchspace=(7, 7, 7), radius_patchspace=(3, 3, 3), nslices=21)

    class Two(LocalExchange):
        world = 2
    with pytest.raises(ValueError, match="halo"):
        ZSlabJob((24, 16, 16), prm, exchange=Two(), backend_factory=OracleSlabBackend)
