"""z-slab streaming of host-resident volumes: every form must equal the
in-memory schedule (inlm_denoise) bit for bit, whatever the slab depth,
because each slab is filtered as a sub-volume whose halo covers every value
its voxels read (and, for the FP16 and learned forms, whose tiles sit where
the whole volume's do)."""
import numpy as np
import pytest

from microtomodenoise_b200 import DenoiseParameters, IterativeNLM_GPU, stream_denoise, synth

pytestmark = pytest.mark.gpu


def in_memory(raw, p, net=None, k=0, min_mass=0.0, tiles_x=1):
    g = IterativeNLM_GPU()
    g.configure_device(raw.shape, p)
    if net is not None:
        g.attach_proposal(net, k, min_mass, tiles_x=tiles_x)
    out, s0, s1 = g.denoise(raw)
    g.free_device()
    return out, s0, s1


@pytest.mark.parametrize("mode,slab,prec", [
    ("z-adaptive", 8, "f32"), ("global", 16, "f32"), ("manual", 24, "f32"),
    ("z-adaptive", 8, "f16"), ("global", 64, "f16"),
])
def test_stream_equals_in_memory(gpu, mode, slab, prec):
    raw = synth.small_case((44, 40, 56), seed=21)
    p = DenoiseParameters(radius_patchspace=(2, 2, 2), radius_searchspace=(3, 3, 3),
                          noise_mode=mode, zwindow=10, sigma=(0.06, 0.05), noise_seed=3,
                          precision=prec)
    want, w0, w1 = in_memory(raw, p)
    got, s0, s1, st = stream_denoise(raw, p, slab_depth=slab)
    print(mode, prec, st)
    assert st["slabs"] == -(-44 // st["slab_depth"])
    if mode != "manual":
        assert np.array_equal(s0, w0) and np.array_equal(s1, w1)
    assert np.array_equal(got, want)


def test_stream_continuous_estimate(gpu):
    raw = synth.small_case((30, 36, 40), seed=4)
    p = DenoiseParameters(radius_patchspace=(1, 1, 1), radius_searchspace=(2, 2, 2),
                          noise_mode="global", continuous_estimate=True, noise_seed=9)
    want, _, _ = in_memory(raw, p)
    got, _, _, _ = stream_denoise(raw, p, slab_depth=8)
    assert np.array_equal(got, want)


def test_stream_learned_proposal(gpu, port):
    from microtomodenoise_b200.proposal import ProposalNet
    from oracle.oracle import FilterParams
    from test_proposal_gpu import rand_params
    raw = synth.small_case((48, 40, 48), seed=8)
    p = DenoiseParameters(radius_patchspace=(1, 1, 1), radius_searchspace=(3, 3, 3),
                          noise_mode="global", noise_seed=2, precision="f16")
    S = len(port.search_offsets(FilterParams(search_radius=(3, 3, 3), patch_radius=(1, 1, 1))))
    net = ProposalNet(S)
    net.set_params(rand_params(S, 12))
    want, _, _ = in_memory(raw, p, net, 40, 0.0)
    got, _, _, st = stream_denoise(raw, p, slab_depth=8, net=net, k=40, min_mass=0.0)
    assert st["halo"] >= 16
    assert np.array_equal(got, want)
    net.close()


def test_stream_grouped_proposal(gpu, port):
    """Per-32x8x8-block lists: slabs split z only, so the streamed job equals
    the in-memory one with the same grouping."""
    from microtomodenoise_b200.proposal import ProposalNet
    from oracle.oracle import FilterParams
    from test_proposal_gpu import rand_params
    raw = synth.small_case((48, 40, 72), seed=8)
    p = DenoiseParameters(radius_patchspace=(1, 1, 1), radius_searchspace=(3, 3, 3),
                          noise_mode="global", noise_seed=2, precision="f16")
    S = len(port.search_offsets(FilterParams(search_radius=(3, 3, 3), patch_radius=(1, 1, 1))))
    net = ProposalNet(S)
    net.set_params(rand_params(S, 12))
    want, _, _ = in_memory(raw, p, net, 40, 0.0, tiles_x=4)
    got, _, _, st = stream_denoise(raw, p, slab_depth=16, net=net, k=40, min_mass=0.0, tiles_x=4)
    assert np.array_equal(got, want)
    net.close()


def test_blocks_with_grouped_proposal_equal_in_memory(gpu, port):
    """The per-iteration engine (inlm_blocks_*) with a learned proposal and
    one list per 32x8x8 block: every iteration equals the in-memory FP16
    learned form's, given the same sigma; with the relative fallback on, a
    whole volume in one slab gives the in-memory result too (one mean over
    the same lists)."""
    from microtomodenoise_b200 import Blocks
    from microtomodenoise_b200.proposal import ProposalNet
    from oracle.oracle import FilterParams
    from test_proposal_gpu import rand_params
    raw = synth.small_case((48, 40, 72), seed=13)
    p = DenoiseParameters(radius_patchspace=(1, 1, 1), radius_searchspace=(3, 3, 3), precision="f16")
    S = len(port.search_offsets(FilterParams(search_radius=(3, 3, 3), patch_radius=(1, 1, 1))))
    net = ProposalNet(S)
    net.set_params(rand_params(S, 14))
    sig = [np.full(48, 0.06, np.float32), np.full(48, 0.05, np.float32), np.full(48, 0.05, np.float32)]
    for slab, rel in ((16, 0.0), (48, 0.9)):
        g = IterativeNLM_GPU()
        g.configure_device(raw.shape, p)
        g.attach_proposal(net, 40, 0.0, tiles_x=4, rel_mass=rel)
        want = []
        for it, s in enumerate(sig):
            g.set_sigma(s)
            g.Run_GaussianNoise(it + 1, raw if it == 0 else None)
            want.append(g.get_result())
        g.free_device()
        b = Blocks(raw.shape, p, slab_depth=slab)
        b.attach_proposal(net, 40, 0.0, tiles_x=4, rel_mass=rel)
        prev = None
        for it, s in enumerate(sig):
            b.set_sigma(s)
            out = np.empty_like(raw)
            b.run_iteration(it + 1, raw, prev, out)
            assert np.array_equal(out, want[it]), f"slab {slab}, iteration {it + 1}"
            prev = out
        b.close()
    net.close()
