"""CPU checks of the proposal oracle itself (no GPU): its gradients against
finite differences, its top-k tie rule and per-tile plans, and the FP64
plan / weight-mass restatements against the plain FP64 filter."""
import numpy as np

from microtomodenoise_b200 import synth
from oracle import proposal_oracle as po
from oracle.oracle import FilterParams


def test_gradients_match_finite_differences():
    S = 12
    rng = np.random.default_rng(0)
    lay = po.layout(S)
    params = rng.standard_normal(lay["total"]) * 0.3
    vol = rng.random((6, 9, 11)).astype(np.float32)
    scale = np.linspace(5, 8, 6).astype(np.float32)
    nt = int(np.prod(po.levels(vol.shape)[3]))
    t = rng.random((nt, S))
    t /= t.sum(axis=1, keepdims=True)
    ex = [(vol, scale, t)]
    _, g = po.loss_and_grad(params, ex, S, rounded=False)
    idx = np.concatenate([rng.choice(lay["total"], 30, replace=False),
                          [lay["b1"][0], lay["w1"][0] + 5, lay["bh"][0] + 3, lay["b4"][0] + 2]])
    for i in idx:
        e = 1e-6
        pp, pm = params.copy(), params.copy()
        pp[i] += e
        pm[i] -= e
        fd = (po.loss_and_grad(pp, ex, S, rounded=False)[0] -
              po.loss_and_grad(pm, ex, S, rounded=False)[0]) / (2 * e)
        assert abs(fd - g[i]) <= 1e-5 * (abs(g[i]) + 1e-3 * np.abs(g).max()), i


def test_bf16_round_ties_to_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.14159], np.float32)
    r = po.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6
    assert r[3] == -2.5 and abs(r[4] - 3.140625) < 1e-7


def test_tf32_truncation_and_mode():
    """tf32_trunc keeps sign, exponent and the top 10 mantissa bits (rounds
    toward zero); the oracle's tf32 mode moves the logits of a small case by
    about that rounding and leaves layer 1 and the head in FP64."""
    x = np.array([1.0 + 2 ** -10, 1.0 + 2 ** -11 + 2 ** -12, -(1.0 + 2 ** -10 + 2 ** -11), 3.0e-8],
                 np.float32)
    t = po.tf32_trunc(x)
    assert t[0] == 1.0 + 2 ** -10 and t[1] == 1.0 and t[2] == -(1.0 + 2 ** -10)
    assert abs(t[3]) <= abs(float(x[3])) and abs(t[3] - float(x[3])) <= 2 ** -10 * abs(float(x[3]))
    S = 8
    rng = np.random.default_rng(1)
    params = rng.standard_normal(po.layout(S)["total"]) * 0.3
    vol = rng.random((10, 12, 14)).astype(np.float32)
    scale = np.full(10, 6.0, np.float32)
    a = po.forward(params, vol, scale, S)
    b = po.forward(params, vol, scale, S, tf32=True)
    d = np.abs(a - b).max() / np.abs(a).max()
    assert 0 < d < 1e-2


def test_select_ties_and_fallback():
    logits = np.array([[0.0, 1.0, 1.0, 1.0, 0.5], [5.0, 0.0, 0.0, 0.0, 0.0]])
    keep, pm, fb = po.select(logits, 2, 0.0)
    assert keep[0].tolist() == [False, True, True, False, False]
    assert keep[1].tolist() == [True, True, False, False, False]
    keep, pm, fb = po.select(logits, 2, 0.9)
    assert fb.tolist() == [True, False] and keep[0].all()


def test_plans_per_tile():
    keep = np.zeros((3, 6), bool)
    keep[0, [0, 2]] = True
    keep[2, [5, 1]] = True
    assert po.plans(keep) == [[0, 2], [], [1, 5]]


def test_plan_oracle_keep_all_is_full_search(port):
    vol = synth.small_case((6, 10, 12), seed=1)
    p = FilterParams(search_radius=(2, 2, 2), patch_radius=(1, 1, 1))
    S = len(port.search_offsets(p))
    sig = np.full((2, 6), 0.06, np.float32)
    nt = 1 * 2 * 2
    full = port.denoise_f64(vol, p, sig)
    assert np.array_equal(port.denoise_f64_plan(vol, p, sig, (8, 8, 8), np.ones((nt, S), bool)), full)
    per_iter = np.ones((2, nt, S), bool)
    assert np.array_equal(port.denoise_f64_plan(vol, p, sig, (8, 8, 8), per_iter), full)
    per_iter[1, :, S // 2:] = False
    assert not np.array_equal(port.denoise_f64_plan(vol, p, sig, (8, 8, 8), per_iter), full)


def test_weight_mass_rows_and_flat_limit(port):
    vol = synth.small_case((9, 12, 20), seed=2)
    p = FilterParams(search_radius=(2, 2, 2), patch_radius=(1, 1, 1))
    S = len(port.search_offsets(p))
    m = port.weight_mass_f64(vol, p, np.full(9, 0.05, np.float32))
    assert m.shape == (2 * 2 * 3, S)
    assert np.allclose(m.sum(axis=1), 1.0)
    # huge sigma: every weight ~1, uniform mass
    m2 = port.weight_mass_f64(vol, p, np.full(9, 1e4, np.float32))
    assert np.allclose(m2, 1.0 / S, atol=1e-6)
