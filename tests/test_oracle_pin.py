"""Pins the plain-C oracle (oracle/inlm_oracle.c) to the reference.

Against the golden fixtures (generated from the reference's own CPU build,
tests/golden/make_golden.py) everywhere, and against that build itself
(oracle/_ref) where it is present. All comparisons are bit-exact.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from cases import FILTER_CASES, TABLE_CASES  # noqa: E402

from oracle.oracle import FilterParams  # noqa: E402


@pytest.mark.parametrize("seed", [0, 1, 7, 12345, 2**31 + 7, 4294967295])
def test_glibc_rand_restatement(port, seed):
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(ctypes.c_uint(seed))
    expect = np.array([libc.rand() for _ in range(1000)], np.int64)
    assert np.array_equal(port.rand_sequence(seed, 1000), expect)


@pytest.mark.parametrize("case", FILTER_CASES, ids=[c[0] for c in FILTER_CASES])
def test_port_filter_matches_golden(port, golden_filter, case):
    name, pr, sr, nsl, an = case
    p = FilterParams(search_radius=sr, patch_radius=pr, nslices=nsl, z_anisotropy=an)
    got = port.denoise_f32(golden_filter["raw"], p, golden_filter["sigmas"], all_iters=True)
    assert np.array_equal(got, golden_filter[name])


@pytest.mark.parametrize("i", range(len(TABLE_CASES)))
def test_port_tables_match_golden(port, golden_tables, i):
    prm = golden_tables[f"c{i}_params"]
    pr, sr, nsl, ps = tuple(prm[0:3]), tuple(prm[3:6]), int(prm[6]), tuple(prm[7:10])
    p = FilterParams(search_radius=sr, patch_radius=pr, nslices=nsl)
    so = port.search_offsets(p)
    po = port.patch_taps(p)
    nsl_ = ps[0] * ps[1]
    assert np.array_equal(so[:, 2] * nsl_ + so[:, 1] * ps[0] + so[:, 0], golden_tables[f"c{i}_search"])
    assert np.array_equal(po[:, 2] * nsl_ + po[:, 1] * ps[0] + po[:, 0], golden_tables[f"c{i}_patch"])
    assert np.array_equal(port.distweight(p, ps[2]), golden_tables[f"c{i}_weights"])


def test_reference_tap_counts(port):
    # float32 geometry: 115 taps at radius 3 (not the 123 a double test gives)
    counts = {(1, 1, 1): 7, (1, 1, 2): 9, (1, 1, 3): 11, (2, 2, 1): 15, (2, 2, 2): 33,
              (3, 3, 1): 31, (3, 3, 2): 73, (3, 3, 3): 115}
    for pr, n in counts.items():
        assert len(port.patch_taps(FilterParams(patch_radius=pr))) == n
    s = {3: 114, 5: 514, 7: 1326, 10: 3102}
    for r, n in s.items():
        assert len(port.search_offsets(FilterParams(search_radius=(r, r, r)))) == n


@pytest.mark.parametrize("mode", ["global", "z-adaptive"])
@pytest.mark.parametrize("mask", [0, 60])
def test_port_noise_matches_golden(port, golden_noise, mode, mask):
    import make_golden
    vol = make_golden.noise_volume()
    assert make_golden.sha(vol) == str(golden_noise["vol_sha"])
    key = f"{mode}_m{mask}"
    samp = port.draw_samples(vol.shape, 20000, 15, mask, 7)
    assert np.array_equal(samp, golden_noise[key + "_samples"].astype(np.int64))
    ps = port.patchstd(vol, samp)
    assert np.array_equal(ps, golden_noise[key + "_patchstd"])
    s1 = port.noise_from_patchstd(ps, samp, vol.shape, mode, zwindow=20)
    assert np.array_equal(s1, golden_noise[key + "_sigma1"])
    vol2 = vol * np.float32(0.8)
    s2 = port.noise_from_patchstd(port.patchstd(vol2, samp), samp, vol.shape, mode, zwindow=20)
    assert np.array_equal(s2, golden_noise[key + "_sigma2"])
    # the FP64-accumulating EM (device arithmetic) stays within 2e-5 relative
    s64 = port.noise_from_patchstd(ps, samp, vol.shape, mode, zwindow=20, f64acc=True)
    assert np.max(np.abs(s64 / s1 - 1)) < 2e-5


def test_port_pad_matches_reference(port, reference):
    rng = np.random.default_rng(5)
    vol = rng.random((7, 9, 11), dtype=np.float32)
    for pad in [(1, 1, 1), (3, 2, 5), (12, 9, 8)]:   # pads larger than the axis reflect repeatedly
        assert np.array_equal(port.pad_reflective(vol, pad), reference.pad_reflective(vol, pad))


@pytest.mark.parametrize("pr", [(1, 1, 1), (2, 2, 2), (3, 3, 1), (2, 1, 3), (1, 1, 0)])
def test_port_filter_matches_reference_build(port, reference, pr):
    rng = np.random.default_rng(sum(pr))
    raw = rng.random((9, 13, 17), dtype=np.float32)
    sr = (2, 3, 2) if pr[2] else (2, 3, 0)
    p = FilterParams(search_radius=sr, patch_radius=pr)
    sig = np.full((2, 9), 0.3, np.float32)
    got = port.denoise_f32(raw, p, sig, all_iters=True)
    want, _ = reference.denoise(raw, p, sig, n_threads=2, all_iters=True)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("pr", [(1, 1, 1), (2, 2, 2)])
def test_port_filter_matches_reference_build_with_nan_input(port, reference, pr):
    """NaN voxels (e.g. masked regions) propagate through the restatement as
    through the reference: a NaN distance fails the Pade cutoff test and
    weighs 0, a NaN raw value poisons every sum it enters. Same positions,
    same finite values."""
    rng = np.random.default_rng(11 + sum(pr))
    raw = rng.random((9, 13, 17), dtype=np.float32)
    raw[4, 6, 8] = np.nan
    raw[0, 0, 3] = np.nan
    p = FilterParams(search_radius=(2, 2, 2), patch_radius=pr)
    sig = np.full((2, 9), 0.3, np.float32)
    got = port.denoise_f32(raw, p, sig, all_iters=True)
    want, _ = reference.denoise(raw, p, sig, n_threads=2, all_iters=True)
    assert np.array_equal(np.isnan(got), np.isnan(want))
    assert np.isnan(want).any() and (~np.isnan(want)).any()
    assert np.array_equal(got[~np.isnan(got)], want[~np.isnan(want)])


def test_port_em_matches_reference_build(port, reference):
    rng = np.random.default_rng(3)
    v = np.concatenate([rng.normal(0.05, 0.005, 3000), rng.normal(0.2, 0.03, 1000)]).astype(np.float32)
    v[::97] = 0.0   # zero-variance samples are excluded
    for first, last in [(-1, -1), (100, 2500), (3000, 3999)]:
        assert port.create2clusters(v, first, last) == reference.create2clusters(v, first, last)


def test_f64_oracle_close_to_f32(port, golden_filter):
    p = FilterParams(search_radius=(3, 3, 3), patch_radius=(1, 1, 1))
    raw = golden_filter["raw"]
    sig = golden_filter["sigmas"]
    f32 = port.denoise_f32(raw, p, sig)
    f64 = port.denoise_f64(raw, p, sig)
    rel = np.abs(f32 - f64) / np.maximum(np.abs(f64), 1e-6)
    assert np.median(rel) < 1e-6


def test_reference_gpu_build_loads_and_exports():
    """The reference GPU class build (oracle/Makefile ref_gpu, where the
    reference tree exists) loads without a GPU and exports its driver entry."""
    from oracle.oracle import REF_GPU_SO, reference_gpu_available
    if not reference_gpu_available():
        pytest.skip("reference GPU build absent")
    lib = ctypes.CDLL(REF_GPU_SO)
    assert hasattr(lib, "ref_gpu_run")


def test_fp64_blocks_equal_the_whole_volume_fp64(port):
    """The FP64 sub-block oracle (iterations on shrinking boxes) gives the
    whole-volume FP64 result on every block, edges and corners included."""
    from microtomodenoise_b200 import synth
    vol = synth.small_case((20, 34, 40), seed=11)
    p = FilterParams(search_radius=(3, 3, 2), patch_radius=(2, 2, 1))
    rng = np.random.default_rng(0)
    sig = rng.uniform(0.03, 0.08, (3, 20)).astype(np.float32)
    want = port.denoise_f64(vol, p, sig)
    size = (6, 7, 8)
    corners = [(0, 0, 0), (14, 27, 32), (7, 13, 16), (0, 27, 5)]
    got = port.denoise_f64_blocks(vol, p, sig, corners, size)
    for c, g in zip(corners, got):
        w = want[c[0]:c[0] + size[0], c[1]:c[1] + size[1], c[2]:c[2] + size[2]]
        assert np.array_equal(g, w), f"block at {c}"
