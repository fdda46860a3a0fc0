"""GPU parity of the FP32 filter against the reference CPU filter.

The bar is bit-exactness: the device kernels round every product and sum the
way the reference's g++ -O3 build does, in the reference's order.
  * golden fixtures (reference output, every shape the reference specialises,
    generic shapes, anisotropy, clipped z search),
  * the plain-C oracle on odd sizes and partial tiles,
  * the 128x128x64 workload against the reference's own sha256 per iterate,
  * the 512^3 workload at sampled voxels (one iteration at a time).
"""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

from microtomodenoise_b200 import DenoiseParameters, IterativeNLM_GPU, InlmError, synth
from oracle.oracle import FilterParams

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from cases import FILTER_CASES  # noqa: E402

pytestmark = pytest.mark.gpu


def run_gpu(raw, pr, sr, sigmas, nslices=11, aniso=1.0, weight_table="cpu", form="auto"):
    g = IterativeNLM_GPU()
    dp = DenoiseParameters(radius_patchspace=pr, radius_searchspace=sr, nslices=nslices,
                           z_anisotropy=aniso, weight_table=weight_table)
    assert g.configure_device(raw.shape, dp) == raw.shape[0]
    if form != "auto":
        g.select_tile_form(form)
    outs = []
    for it in range(sigmas.shape[0]):
        g.set_sigma(sigmas[it])
        g.Run_GaussianNoise(it + 1, raw if it == 0 else None)
        outs.append(g.get_result())
    desc = g.describe()
    g.free_device()
    return np.stack(outs), desc


@pytest.mark.parametrize("case", FILTER_CASES, ids=[c[0] for c in FILTER_CASES])
def test_filter_bit_exact_vs_reference_golden(gpu, golden_filter, case):
    name, pr, sr, nsl, an = case
    got, desc = run_gpu(golden_filter["raw"], pr, sr, golden_filter["sigmas"], nsl, an)
    want = golden_filter[name]
    if not np.array_equal(got, want):
        d = np.abs(got - want)
        pytest.fail(f"{name} [{desc}]: {np.count_nonzero(d)} voxels differ, max {d.max():.3g}")
    spec = name.split("_")[0] in ("p111", "p112", "p113", "p221", "p222", "p331", "p332", "p333")
    if spec and nsl // 2 >= pr[2]:
        assert desc.startswith(("nlm_tile_f32", "nlm_tile_ws_f32", "nlm_column_f32")), desc


@pytest.mark.parametrize("shape,pr,sr", [
    ((9, 19, 41), (2, 2, 2), (3, 4, 2)),
    ((13, 9, 70), (2, 2, 1), (5, 5, 5)),
    ((17, 23, 37), (3, 3, 3), (3, 3, 3)),
    ((20, 40, 48), (2, 2, 2), (5, 5, 5)),
    ((11, 17, 33), (1, 1, 1), (5, 5, 5)),
    ((24, 33, 40), (2, 2, 2), (7, 7, 7)),   # raw box too large: raw from global memory
    ((18, 30, 45), (3, 3, 3), (4, 4, 4)),   # raw from global memory at patch radius 3
])
def test_warp_specialised_form_bit_exact(gpu, port, shape, pr, sr):
    """The warp-specialised kernel (producer warps form the squared
    differences into a ring of shared-memory buffers, consumer warps the patch
    sums, weights and sums; mbarrier hand-off) equals the oracle bit for bit
    over two iterations, with the raw box staged and with raw read from global
    memory, at odd sizes and partial tiles."""
    raw = synth.small_case(shape, seed=sum(shape))
    sig = np.stack([np.full(shape[0], 0.07, np.float32),
                    np.linspace(0.03, 0.08, shape[0], dtype=np.float32)])
    got, desc = run_gpu(raw, pr, sr, sig, form="ws")
    assert desc.startswith("nlm_tile_ws_f32"), desc
    want = port.denoise_f32(raw, FilterParams(search_radius=sr, patch_radius=pr), sig, all_iters=True)
    if not np.array_equal(got, want):
        d = np.abs(got - want)
        pytest.fail(f"[{desc}]: {np.count_nonzero(d)} voxels differ, max {d.max():.3g}")


@pytest.mark.parametrize("shape,pr,sr", [
    ((5, 7, 9), (1, 1, 1), (2, 2, 2)),
    ((11, 17, 33), (1, 1, 1), (5, 5, 5)),
    ((9, 19, 41), (2, 2, 2), (3, 4, 2)),
    ((13, 9, 70), (2, 2, 1), (5, 5, 5)),
    ((17, 23, 37), (3, 3, 3), (3, 3, 3)),
    ((8, 8, 8), (3, 3, 2), (2, 2, 2)),
    ((3, 40, 40), (1, 1, 1), (4, 4, 4)),     # nz smaller than the z halo: repeated reflection
    ((20, 12, 12), (1, 1, 3), (7, 7, 7)),    # padding larger than the axis
])
def test_filter_bit_exact_vs_oracle_odd_sizes(gpu, port, shape, pr, sr):
    raw = synth.small_case(shape, seed=sum(shape))
    sig = np.stack([np.full(shape[0], 0.07, np.float32),
                    np.linspace(0.03, 0.08, shape[0], dtype=np.float32)])
    got, desc = run_gpu(raw, pr, sr, sig)
    want = port.denoise_f32(raw, FilterParams(search_radius=sr, patch_radius=pr), sig, all_iters=True)
    assert np.array_equal(got, want), desc


@pytest.mark.parametrize("shape,pr,sr", [((20, 40, 48), (1, 1, 1), (10, 10, 10)),
                                         ((18, 33, 45), (2, 2, 2), (7, 7, 7)),
                                         ((16, 24, 40), (1, 1, 2), (9, 9, 9)),
                                         ((9, 30, 37), (1, 1, 1), (10, 10, 10))])
def test_raw_slab_bit_exact(gpu, port, shape, pr, sr):
    """Search radii whose whole raw box does not fit beside the prev box stage
    raw as a slab of TZ + 1 planes per pair of z offsets, restaged as the
    z-major offsets move on: bit-identical to the reference like every form
    (nz = 9: a volume shallower than the slab's reach)."""
    raw = synth.small_case(shape, seed=sum(shape) + 3)
    sig = np.stack([np.full(shape[0], 0.06, np.float32),
                    np.linspace(0.03, 0.08, shape[0], dtype=np.float32)])
    got, desc = run_gpu(raw, pr, sr, sig, form="tile")
    assert "raw_slab" in desc, desc
    want = port.denoise_f32(raw, FilterParams(search_radius=sr, patch_radius=pr), sig, all_iters=True)
    assert np.array_equal(got, want), desc


@pytest.mark.parametrize("shape,pr,sr,nsl", [
    ((5, 7, 9), (1, 1, 1), (2, 2, 2), 11),
    ((20, 40, 48), (1, 1, 1), (10, 10, 10), 11),   # the reference's default geometry
    ((17, 23, 70), (1, 1, 1), (4, 5, 3), 11),
    ((3, 40, 40), (1, 1, 1), (4, 4, 4), 11),       # fewer planes than the CTA depth and the z halo
    ((33, 9, 31), (1, 1, 1), (3, 3, 7), 15),       # two CTA layers in z, partial x and y tiles
    ((16, 24, 40), (1, 1, 2), (6, 6, 6), 11),
    ((12, 30, 33), (1, 1, 3), (3, 3, 3), 11),
])
def test_column_form_bit_exact(gpu, port, shape, pr, sr, nsl):
    """The column form (patch radius 1 in x and y: a warp per z plane, each
    thread 8 voxels along y, no barrier in the offset loop, raw from global
    memory) equals the oracle and the tiled kernel bit for bit."""
    raw = synth.small_case(shape, seed=sum(shape) + 5)
    sig = np.stack([np.full(shape[0], 0.05, np.float32),
                    np.linspace(0.03, 0.08, shape[0], dtype=np.float32)])
    got, desc = run_gpu(raw, pr, sr, sig, nslices=nsl, form="column")
    assert desc.startswith("nlm_column_f32"), desc
    tile, desc_t = run_gpu(raw, pr, sr, sig, nslices=nsl, form="tile")
    assert desc_t.startswith("nlm_tile_f32"), desc_t
    want = port.denoise_f32(raw, FilterParams(search_radius=sr, patch_radius=pr, nslices=nsl), sig,
                            all_iters=True)
    assert np.array_equal(got, want), desc
    assert np.array_equal(tile, want), desc_t


@pytest.mark.parametrize("pr,sr", [((1, 1, 1), (2, 2, 2)), ((2, 2, 2), (3, 3, 3))])
def test_nan_input_propagates_as_the_oracle(gpu, port, pr, sr):
    """NaN voxels: a NaN distance fails the Pade cutoff and weighs 0, a NaN
    raw value poisons the sums it enters; the NaN positions and every finite
    value equal the oracle's (pinned to the reference build on the same
    case)."""
    rng = np.random.default_rng(11 + sum(pr))
    raw = rng.random((12, 21, 37), dtype=np.float32)
    raw[5, 10, 18] = np.nan
    raw[0, 0, 3] = np.nan
    sig = np.full((2, 12), 0.3, np.float32)
    got, desc = run_gpu(raw, pr, sr, sig)
    want = port.denoise_f32(raw, FilterParams(search_radius=sr, patch_radius=pr), sig, all_iters=True)
    assert np.array_equal(np.isnan(got), np.isnan(want)), desc
    assert np.array_equal(got[~np.isnan(got)], want[~np.isnan(want)]), desc


def test_distweight_table_and_generic_kernel(gpu, port):
    raw = synth.small_case((12, 16, 20), seed=4)
    sig = np.full((2, 12), 0.06, np.float32)
    # weight_table="distweight" uses setup_distweight for the specialised shapes too
    got, _ = run_gpu(raw, (2, 2, 2), (2, 2, 2), sig, weight_table="distweight")
    p = FilterParams(search_radius=(2, 2, 2), patch_radius=(2, 2, 2))
    ref_cpu = port.denoise_f32(raw, p, sig, all_iters=True)
    assert not np.array_equal(got, ref_cpu)          # different table, different result
    rel = np.abs(got - ref_cpu) / np.abs(ref_cpu)
    assert rel.max() < 1e-3


def test_sigma_zero_and_constant_volume(gpu, port):
    raw = np.full((6, 10, 12), 0.25, np.float32)
    sig = np.full((1, 6), 0.05, np.float32)
    got, _ = run_gpu(raw, (1, 1, 1), (2, 2, 2), sig)
    want = port.denoise_f32(raw, FilterParams(search_radius=(2, 2, 2), patch_radius=(1, 1, 1)), sig)
    assert np.array_equal(got[0], want)
    assert np.max(np.abs(got[0] - 0.25)) < 1e-6
    # sigma 0: every weight is cut off (or NaN) and the raw value comes back
    raw2 = synth.small_case((6, 10, 12), seed=1)
    got0, _ = run_gpu(raw2, (1, 1, 1), (2, 2, 2), np.zeros((1, 6), np.float32))
    want0 = port.denoise_f32(raw2, FilterParams(search_radius=(2, 2, 2), patch_radius=(1, 1, 1)),
                             np.zeros((1, 6), np.float32))
    assert np.array_equal(got0[0], want0)


def test_call_order_errors(gpu):
    g = IterativeNLM_GPU()
    g.configure_device((6, 20, 20), DenoiseParameters(radius_searchspace=(2, 2, 2)))
    with pytest.raises(InlmError):
        g.Run_GaussianNoise(1, np.zeros((6, 20, 20), np.float32))   # sigma not set
    g.set_sigma(np.full(6, 0.1, np.float32))
    with pytest.raises(InlmError):
        g.Run_GaussianNoise(2)                                      # iteration 1 first
    g.Run_GaussianNoise(1, np.zeros((6, 20, 20), np.float32))
    g.Run_GaussianNoise(2)
    g.free_device()
    with pytest.raises(InlmError):
        IterativeNLM_GPU().configure_device((1, 20, 20), DenoiseParameters(radius_searchspace=(2, 2, 2)))


def test_device_pointer_forms(gpu, port):
    torch = pytest.importorskip("torch")
    raw = synth.small_case((10, 24, 40), seed=9)
    sig = np.full(10, 0.06, np.float32)
    g = IterativeNLM_GPU()
    g.configure_device(raw.shape, DenoiseParameters(radius_searchspace=(3, 3, 3)))
    g.set_sigma(sig)
    t_raw = torch.from_numpy(raw).cuda()
    t_out = torch.empty_like(t_raw)
    torch.cuda.synchronize()
    g.Run_GaussianNoise_device(1, t_raw.data_ptr())
    g.get_result_device(t_out.data_ptr())
    got = t_out.cpu().numpy()
    want = port.denoise_f32(raw, FilterParams(search_radius=(3, 3, 3), patch_radius=(1, 1, 1)), sig[None])
    assert np.array_equal(got, want)
    ms, n = g.filter_kernel_ms()
    assert n == 1 and ms > 0
    g.free_device()


def test_config1_workload_matches_reference_sha(gpu):
    import make_golden
    cfg = json.load(open(os.path.join(HERE, "golden", "config1.json")))
    vol = make_golden.config1_volume()
    if make_golden.sha(vol) != cfg["input_sha256"]:
        pytest.skip("synthetic generator produced a different volume on this machine")
    sigmas = np.array([cfg["sigma0"]] + [cfg["sigma1"]] * 3, np.float32)
    got, desc = run_gpu(vol, (1, 1, 1), (5, 5, 5), sigmas)
    for i in range(4):
        if make_golden.sha(got[i]) != cfg["iterate_sha256"][i]:
            vals = got[i].ravel()[cfg["sample_index"]]
            d = np.abs(vals - np.array(cfg["sample_values"][i], np.float32))
            pytest.fail(f"iterate {i + 1} differs from the reference [{desc}]; sampled max diff {d.max()}")


@pytest.mark.slow
def test_512_cube_p2s5_sampled_voxels(gpu, port):
    """The 512^3 grain-pack workload: two iterations on the GPU, 3000 random
    voxels of each recomputed by the oracle from the same inputs."""
    vol = synth.grain_pack_volume((512, 512, 512), seed=0)
    nz = vol.shape[0]
    p = FilterParams(search_radius=(5, 5, 5), patch_radius=(2, 2, 2))
    sig = np.stack([np.linspace(0.05, 0.06, nz, dtype=np.float32),
                    np.full(nz, 0.045, np.float32)])
    got, desc = run_gpu(vol, (2, 2, 2), (5, 5, 5), sig)
    pad = port.padding(p)
    raw_pad = port.pad_reflective(vol, pad)
    rng = np.random.default_rng(0)
    vox = rng.integers(0, vol.size, 3000)
    # iteration 1: prev = raw
    w1 = port.filter_voxels(raw_pad, raw_pad, vol.shape, p, sig[0], vox)
    assert np.array_equal(got[0].ravel()[vox], w1), desc
    # iteration 2 from the GPU's first iterate
    prev_pad = port.pad_reflective(got[0], pad)
    w2 = port.filter_voxels(raw_pad, prev_pad, vol.shape, p, sig[1], vox)
    assert np.array_equal(got[1].ravel()[vox], w2), desc
    # size-independent properties on the whole output
    assert np.isfinite(got).all()
    assert got.min() >= vol.min() - 1e-6 and got.max() <= vol.max() + 1e-6  # convex combination


@pytest.mark.parametrize("pr,sr,shape", [((1, 1, 1), (3, 3, 3), (24, 40, 56)),
                                         ((2, 2, 2), (3, 3, 3), (20, 33, 47)),
                                         ((3, 3, 3), (2, 2, 2), (16, 40, 40)),
                                         ((2, 2, 1), (4, 4, 4), (24, 48, 48)),
                                         ((1, 1, 2), (3, 3, 3), (20, 36, 40)),   # column form
                                         ((2, 2, 2), (7, 7, 7), (18, 40, 44))])  # search radius 7
def test_fused_form_tolerance(gpu, port, pr, sr, shape):
    """precision="f32_fma": the tiled kernel with fused multiply-adds, a
    Horner Pade and a fast division. Tolerance, written here: relative error
    against the reference CPU filter at most 1e-4 on all but 1e-4 of the
    voxels (a weight whose argument lands within rounding of the Pade cutoff
    can switch between ~0.025 and 0, which moves that voxel further), and at
    most 1e-5 for the median voxel."""
    vol = synth.small_case(shape, seed=1)
    sig = np.full(shape[0], 0.05, np.float32)
    want = port.denoise_f32(vol, FilterParams(sr, pr), np.stack([sig, sig]))
    g = IterativeNLM_GPU()
    g.configure_device(shape, DenoiseParameters(radius_patchspace=pr, radius_searchspace=sr,
                                                precision="f32_fma"))
    g.set_sigma(sig)
    g.Run_GaussianNoise(1, vol)
    g.Run_GaussianNoise(2)
    got = g.get_result()
    assert "fused" in g.describe()
    g.free_device()
    rel = np.abs(got.astype(np.float64) - want) / np.maximum(np.abs(want.astype(np.float64)), 1e-6)
    assert float((rel > 1e-4).mean()) <= 1e-4, rel.max()
    assert float(np.median(rel)) <= 1e-5


@pytest.mark.parametrize("shape,pr,sr", [
    ((20, 40, 48), (2, 2, 2), (5, 5, 5)),   # raw box staged
    ((18, 33, 45), (2, 2, 2), (7, 7, 7)),   # raw from global memory
    ((17, 23, 37), (3, 3, 3), (3, 3, 3)),
])
def test_fused_warp_specialised_equals_fused_tile(gpu, shape, pr, sr):
    """The fused FP32 form on the warp-specialised kernel performs the fused
    tile kernel's operations per voxel in the same order: equal bit for bit
    over two iterations (and so within the fused form's tolerance above)."""
    vol = synth.small_case(shape, seed=sum(shape) + 7)
    sig = np.stack([np.full(shape[0], 0.06, np.float32),
                    np.linspace(0.03, 0.08, shape[0], dtype=np.float32)])
    outs = {}
    for form in ("ws", "tile"):
        g = IterativeNLM_GPU()
        g.configure_device(shape, DenoiseParameters(radius_patchspace=pr, radius_searchspace=sr,
                                                    precision="f32_fma"))
        desc = g.select_tile_form(form)
        assert "fused" in desc and (desc.startswith("nlm_tile_ws_f32") == (form == "ws")), desc
        res = []
        for it in range(2):
            g.set_sigma(sig[it])
            g.Run_GaussianNoise(it + 1, vol if it == 0 else None)
            res.append(g.get_result())
        g.free_device()
        outs[form] = np.stack(res)
    assert np.array_equal(outs["ws"], outs["tile"])
