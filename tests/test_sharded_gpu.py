"""Multi-GPU z-slab sharding with the CUDA backend: two ranks (processes,
gloo for the exchange) each filter their slab plus halos with the library on
a GPU; their owned slices must equal the single-GPU job (inlm_denoise) bit
for bit in the FP32, FP16 and learned forms. With one GPU both ranks share
it: their kernels never wait on each other (all exchange is host-side), so
this is two ordinary processes on one device."""
from __future__ import annotations

import multiprocessing as mp
import socket

import numpy as np
import pytest

from microtomodenoise_b200 import DenoiseParameters, IterativeNLM_GPU, synth

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _net(S):
    from microtomodenoise_b200.proposal import ProposalNet
    from test_proposal_gpu import rand_params
    net = ProposalNet(S)
    net.set_params(rand_params(S, 12))
    return net


def _rank_main(rank, world, port, vol, params, learned, q):
    import torch
    import torch.distributed as dist
    from microtomodenoise_b200.sharded import TorchExchange, ZSlabJob
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        prop = (_net(learned[0]), learned[1], 0.0) if learned else None
        job = ZSlabJob(vol.shape, params, exchange=TorchExchange(device="cpu"), proposal=prop)
        out, s0, s1 = job.run(vol[job.z0:job.z1])
        q.put((rank, job.z0, job.z1, job.halo, out, s0, s1))
        job.close()
        if prop:
            prop[0].close()
    except Exception as e:
        q.put((rank, "error", repr(e)))
    finally:
        dist.destroy_process_group()


def _run(vol, params, world=2, learned=None):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, vol, params, learned, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=600) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
    for r in res:
        assert r[1] != "error", r
    return sorted(res, key=lambda r: r[0])


def _single(vol, params, learned=None):
    g = IterativeNLM_GPU()
    g.configure_device(vol.shape, params)
    net = None
    if learned:
        net = _net(learned[0])
        g.attach_proposal(net, learned[1], 0.0)
    out, s0, s1 = g.denoise(vol)
    g.free_device()
    if net:
        net.close()
    return out, s0, s1


@pytest.mark.parametrize("mode,prec", [("z-adaptive", "f32"), ("global", "f16"), ("manual", "f32")])
def test_sharded_equals_single_gpu(gpu, mode, prec):
    vol = synth.small_case((48, 40, 56), seed=31)
    p = DenoiseParameters(radius_patchspace=(2, 2, 2), radius_searchspace=(3, 3, 3),
                          noise_mode=mode, zwindow=10, sigma=(0.06, 0.05), noise_seed=7,
                          n_samples=20000, precision=prec)
    want, w0, w1 = _single(vol, p)
    for rank, z0, z1, halo, out, s0, s1 in _run(vol, p):
        assert np.array_equal(s0, w0) and np.array_equal(s1, w1)
        assert np.array_equal(out, want[z0:z1]), (rank, float(np.abs(out - want[z0:z1]).max()))


def test_sharded_learned_proposal(gpu, port):
    from oracle.oracle import FilterParams
    vol = synth.small_case((64, 40, 48), seed=8)
    p = DenoiseParameters(radius_patchspace=(1, 1, 1), radius_searchspace=(3, 3, 3),
                          noise_mode="global", noise_seed=2, n_samples=20000, precision="f16")
    S = len(port.search_offsets(FilterParams(search_radius=(3, 3, 3), patch_radius=(1, 1, 1))))
    want, _, _ = _single(vol, p, (S, 40))
    res = _run(vol, p, learned=(S, 40))
    assert res[0][3] >= 16
    for rank, z0, z1, halo, out, s0, s1 in res:
        assert np.array_equal(out, want[z0:z1])
