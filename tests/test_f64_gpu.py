"""The FP64 full-search form on sub-blocks (inlm_denoise_f64_blocks), the
precision reference of the FP16 and learned forms at full volume sizes,
against the oracle's FP64 restatement of the reference filter
(oracle/inlm_oracle.c ora_filter_f64, iternlm_cpu.cpp:795-834 in double):
equal bit for bit, blocks on faces, edges, corners and inside, host and
device input."""
import numpy as np
import pytest

from microtomodenoise_b200 import DenoiseParameters, denoise_f64_blocks, synth
from oracle.oracle import FilterParams

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pr,sr", [((2, 2, 2), (3, 3, 3)), ((1, 1, 1), (5, 5, 2)), ((3, 3, 1), (2, 2, 2)),
                                   ((2, 2, 1), (3, 3, 2))])
def test_fp64_blocks_equal_the_fp64_oracle(gpu, port, pr, sr):
    torch = pytest.importorskip("torch")
    vol = synth.small_case((20, 34, 40), seed=11)
    rng = np.random.default_rng(1)
    sig = rng.uniform(0.03, 0.08, (3, 20)).astype(np.float32)
    corners = [(0, 0, 0), (14, 27, 32), (7, 13, 16), (0, 27, 5)]
    size = (6, 7, 8)
    want = port.denoise_f64_blocks(vol, FilterParams(search_radius=sr, patch_radius=pr), sig, corners, size)
    dp = DenoiseParameters(radius_patchspace=pr, radius_searchspace=sr)
    got = denoise_f64_blocks(vol, dp, sig, corners, size)
    dev = torch.from_numpy(vol).cuda()
    got_dev = denoise_f64_blocks(dev.data_ptr(), dp, sig, corners, size, shape=vol.shape)
    for c, g, gd, w in zip(corners, got, got_dev, want):
        assert np.array_equal(g, w), f"block at {c}: max diff {np.abs(g - w).max()}"
        assert np.array_equal(gd, w), f"block at {c} (device input)"


def test_fp64_blocks_track_the_fp32_reference_filter(gpu, port):
    """Four iterations at patch radius 2, search radius 5: the FP64 blocks stay
    within 1e-5 relative of the reference's FP32 filter (the oracle's FP32
    restatement, bit-exact to the reference build)."""
    vol = synth.grain_pack_volume((40, 48, 56), seed=3)
    sig = np.full((4, 40), 0.1, np.float32)
    corners = [(0, 0, 0), (24, 32, 40), (12, 16, 20)]
    size = (16, 16, 16)
    got = denoise_f64_blocks(vol, DenoiseParameters(radius_patchspace=(2, 2, 2), radius_searchspace=(5, 5, 5)),
                             sig, corners, size)
    f32 = port.denoise_f32(vol, FilterParams(search_radius=(5, 5, 5), patch_radius=(2, 2, 2)), sig)
    for (z, y, x), g in zip(corners, got):
        w = f32[z:z + 16, y:y + 16, x:x + 16].astype(np.float64)
        assert np.max(np.abs(g - w) / np.maximum(np.abs(w), 1e-3)) < 1e-5
