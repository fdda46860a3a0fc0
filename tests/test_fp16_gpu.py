"""FP16-storage form: accuracy against the FP64 oracle (same geometry, table,
Pade weight and cutoff, all in double), and per-tile offset plans.

Tolerances: PSNR >= 50 dB against the FP64 result and at most 0.2% of voxels
off by more than 3e-3. The reference weight jumps from ~0.025 to 0 at the
Pade cutoff, so FP16 rounding of a squared difference occasionally flips one
weight of a voxel; such voxels move by up to ~0.1 after two iterations, and
the max-abs error is reported rather than bounded.
"""
import numpy as np
import pytest

from microtomodenoise_b200 import DenoiseParameters, IterativeNLM_GPU, _lib, synth
from oracle.oracle import FilterParams

pytestmark = pytest.mark.gpu


def psnr(a, b, peak=1.0):
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return float("inf") if mse == 0 else 10 * np.log10(peak * peak / mse)


def check_close(got, ref, what):
    err = np.abs(got - ref)
    frac = float(np.mean(err > 3e-3))
    p = psnr(got, ref)
    print(f"{what}: max-abs {err.max():.3g}, PSNR vs FP64 {p:.1f} dB, outliers {frac:.2e}")
    assert p >= 50.0, (what, p)
    assert frac <= 2e-3, (what, frac)


def run(raw, pr, sr, sigmas, precision, plan=None):
    g = IterativeNLM_GPU()
    g.configure_device(raw.shape, DenoiseParameters(radius_patchspace=pr, radius_searchspace=sr,
                                                    precision=precision))
    if plan is not None:
        start, count, offs = (np.ascontiguousarray(v, np.int32) for v in plan)
        _lib.check(_lib.load().inlm_set_offset_plan(g._h, start.ctypes.data, count.ctypes.data,
                                                    offs.ctypes.data, len(offs), 0), "plan")
    outs = []
    for it in range(sigmas.shape[0]):
        g.set_sigma(sigmas[it])
        g.Run_GaussianNoise(it + 1, raw if it == 0 else None)
        outs.append(g.get_result())
    desc = g.describe()
    g.free_device()
    return np.stack(outs), desc


def tile_grid(shape_zyx):
    """8^3 tile counts (x, y, z): plans hold one offset list per 8^3 tile."""
    nz, ny, nx = shape_zyx
    return (-(-nx // 8), -(-ny // 8), -(-nz // 8))


@pytest.mark.parametrize("precision", ["f16", "f16_df32"])
@pytest.mark.parametrize("pr,sr,shape", [((1, 1, 1), (3, 3, 3), (12, 30, 40)),
                                         ((2, 2, 2), (5, 5, 5), (16, 24, 64)),
                                         ((3, 3, 3), (2, 2, 2), (9, 17, 33))])
def test_fp16_form_vs_fp64_oracle(gpu, port, precision, pr, sr, shape):
    vol = synth.small_case(shape, seed=7)
    sig = np.stack([np.full(shape[0], 0.06, np.float32), np.full(shape[0], 0.05, np.float32)])
    got, desc = run(vol, pr, sr, sig, precision)
    # the column form at patch radius 1, the tile kernel elsewhere
    assert desc.startswith("nlm_column_fast" if pr == (1, 1, 1) else "nlm_tile_fast"), desc
    ref = port.denoise_f64(vol, FilterParams(search_radius=sr, patch_radius=pr), sig)
    check_close(got[-1], ref, desc)


@pytest.mark.parametrize("precision", ["f16", "f16_df32"])
@pytest.mark.parametrize("shape,pr", [((12, 20, 40), (1, 1, 1)), ((21, 27, 70), (1, 1, 1)),
                                      ((19, 24, 40), (1, 1, 3))])
def test_plan_with_every_offset_equals_full_search(gpu, shape, pr, precision):
    """Per-tile plans listing every offset (the one-tile-per-CTA kernel)
    equal the full search, which at patch radius 1 runs the column form:
    both round every voxel as the 32-wide tile kernel does (a 21-plane
    volume: column CTAs of 16 planes over tiles of 8)."""
    vol = synth.small_case(shape, seed=2)
    sig = np.stack([np.full(shape[0], 0.06, np.float32),
                    np.linspace(0.04, 0.08, shape[0], dtype=np.float32)])
    full, dfull = run(vol, pr, (2, 2, 2), sig, precision)
    assert dfull.startswith("nlm_column_fast"), dfull
    S = 32  # search radius 2 (nslices 11): 32 offsets
    n = int(np.prod(tile_grid(vol.shape)))
    plan = (np.arange(n) * S, np.full(n, S), np.tile(np.arange(S), n))
    got, desc = run(vol, pr, (2, 2, 2), sig, precision, plan)
    assert "plan=per-tile" in desc and "tx=8" in desc
    # the one-tile-per-CTA kernel rounds every voxel as the full-search kernel does
    assert np.array_equal(got, full)


def test_plan_subsets_vs_fp64_oracle(gpu, port):
    vol = synth.small_case((16, 24, 64), seed=4)
    p = FilterParams(search_radius=(3, 3, 3), patch_radius=(1, 1, 1))
    S = len(port.search_offsets(p))
    tiles = tile_grid(vol.shape)
    n = int(np.prod(tiles))
    rng = np.random.default_rng(1)
    keep = np.zeros((n, S), bool)
    start, count, offs = [], [], []
    for t in range(n):
        k = int(rng.integers(1, S + 1))
        sel = np.sort(rng.choice(S, k, replace=False))
        keep[t, sel] = True
        start.append(len(offs))
        count.append(k)
        offs.extend(sel.tolist())
    sig = np.stack([np.full(vol.shape[0], 0.07, np.float32)] * 2)
    got, _ = run(vol, (1, 1, 1), (3, 3, 3), sig, "f16", (start, count, offs))
    ref = port.denoise_f64_plan(vol, p, sig, (8, 8, 8), keep)
    check_close(got[-1], ref, "plan")


def test_plan_rejects_bad_ranges(gpu):
    vol = synth.small_case((8, 16, 32), seed=1)
    g = IterativeNLM_GPU()
    g.configure_device(vol.shape, DenoiseParameters(radius_searchspace=(2, 2, 2), precision="f16"))
    L = _lib.load()
    start = np.zeros(1, np.int32)
    count = np.array([1000], np.int32)  # more than S
    offs = np.zeros(1000, np.int32)
    assert L.inlm_set_offset_plan(g._h, start.ctypes.data, count.ctypes.data, offs.ctypes.data,
                                  1000, 0) == -1
    g.free_device()
