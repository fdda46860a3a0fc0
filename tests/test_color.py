"""The colour path's oracle on the CPU: the plain-C restatement of the
three-channel filter and the Anscombe transforms, run through the colour
driver's schedule (Color/color_denoising.h:19-150), must reproduce the
reference's own run (tests/golden/rgb_small.npz, made by
tests/golden/make_golden.py from oracle/_ref) bit for bit given the sigma
schedule; and the RGB TIFF reader / writer must agree with Pillow."""
from __future__ import annotations

import os

import numpy as np
import pytest

from oracle.oracle import FilterParams

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

import sys  # noqa: E402
sys.path.insert(0, GOLDEN)
from make_golden import RGB_CASES  # noqa: E402


@pytest.fixture(scope="module")
def golden_rgb():
    return np.load(os.path.join(GOLDEN, "rgb_small.npz"))


def port_rgb_job(port, img, case, sigmas):
    """The colour schedule with the port's pieces and a given sigma per
    iteration (three values each)."""
    sr, pr, iters, mode, sig, indep, stab, avg, cont, keep = case
    p = FilterParams(search_radius=(sr[0], sr[1], 0), patch_radius=(pr[0], pr[1], 0), nslices=1)
    raw = [port.anscombe(c) if stab else c.copy() for c in img]
    prev, saved = raw, []
    for it in range(iters):
        s = np.asarray(sigmas[it], np.float32)
        mult = [np.float32(-1) / (s[c] * s[c] * np.float32(1)) for c in range(3)]
        res = port.filter_rgb(raw, prev, p, mult, indep)
        if keep:
            if stab:
                res = [port.anscombe(c, inverse=True) for c in res]
            saved.append(np.stack(res))
            if stab:
                res = [port.anscombe(c) for c in res]
        prev = res
    final = [port.anscombe(c, inverse=True) for c in prev] if stab else prev
    return np.stack(final), saved


def manual_sigmas(case):
    _, _, iters, _, sig, *_ = case
    s0 = np.full(3, sig[0], np.float32)
    blend = (np.float32(0.5) * s0 + np.float32(0.5) * np.full(3, sig[1], np.float32)).astype(np.float32)
    return [s0] + [blend] * (iters - 1)


@pytest.mark.parametrize("name", ["manual_joint", "manual_indep_raw"])
def test_port_matches_reference_manual(port, golden_rgb, name):
    case = RGB_CASES[name]
    img = list(golden_rgb["image"])
    final, saved = port_rgb_job(port, img, case, manual_sigmas(case))
    assert np.array_equal(final, golden_rgb[name + "/final"])
    if saved:
        assert np.array_equal(np.stack(saved), golden_rgb[name + "/iterations"])


@pytest.mark.parametrize("name", ["global_joint", "semimanual"])
def test_port_matches_reference_given_sigma(port, golden_rgb, name):
    """Estimated sigma without --continuous: iteration 1 runs at the first
    estimate, later ones at the blended value the reference reports last."""
    case = RGB_CASES[name]
    iters = case[2]
    sig = [golden_rgb[name + "/sigma_first"]] + [golden_rgb[name + "/sigma_last"]] * (iters - 1)
    final, saved = port_rgb_job(port, list(golden_rgb["image"]), case, sig)
    assert np.array_equal(final, golden_rgb[name + "/final"])
    assert np.array_equal(np.stack(saved), golden_rgb[name + "/iterations"])


def test_port_pinned_to_live_reference(port, reference):
    """Same as the golden check, against the reference build when present."""
    from make_golden import rgb_image
    img = rgb_image()
    case = RGB_CASES["manual_joint"]
    p = FilterParams(search_radius=(4, 4, 0), patch_radius=(1, 1, 0), nslices=1)
    fin, its, _, _ = reference.rgb_job(img, p, maxiterations=3, mode="manual", sigma=(1.2, 0.9))
    final, saved = port_rgb_job(port, img, case, manual_sigmas(case))
    assert np.array_equal(final, np.stack(fin)) and np.array_equal(np.stack(saved), its)


def test_rgb_tiff_io_against_pillow(tmp_path):
    PIL = pytest.importorskip("PIL.Image")
    from microtomodenoise_b200 import color
    rng = np.random.default_rng(1)
    img = rng.integers(0, 256, (30, 41, 3), dtype=np.uint8)
    PIL.fromarray(img).save(tmp_path / "a.tif")
    planes = color.read_rgb(str(tmp_path / "a.tif"))
    assert all(np.array_equal(planes[c], img[..., c].astype(np.float32)) for c in range(3))
    PIL.fromarray(np.dstack([img, np.full((30, 41), 7, np.uint8)])).save(tmp_path / "rgba.tif")
    assert all(np.array_equal(a, b) for a, b in zip(color.read_rgb(str(tmp_path / "rgba.tif")), planes))
    vals = [p * np.float32(1.01) - np.float32(0.2) for p in planes]
    vals[0][0, 0], vals[1][0, 0], vals[2][0, 0] = np.nan, 300.0, -0.3
    color.save_rgb(vals, str(tmp_path / "o"), "x")
    im = PIL.open(tmp_path / "o" / "x.tif")
    assert im.mode == "RGB"
    want = np.stack([np.where(np.isnan(v), 255, np.where(v < 255, v, 255)) for v in vals], -1)
    assert np.array_equal(np.array(im), np.where(want > 0, want, 0).astype(np.uint8))
