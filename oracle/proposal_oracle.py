"""FP64 CPU restatement of the learned search-offset proposal network.

TEST INFRASTRUCTURE ONLY: the checker for the device kernels of
microtomodenoise_b200/csrc/proposal.cu (forward, soft-target cross-entropy
loss, backward, top-k selection and per-tile plans). Nothing in the product
imports it. The network has no counterpart in the reference; what it prunes
is the search loop of Denoiser/iternlm_cpu.cpp:758-843.

Network (channels-last, x fastest, arrays indexed [z, y, x, c]):
  L1  input d_t(o) = scale[2 oz] * (v(2o + t) - v(2o)) over the 27 taps t of a
      3^3 window (reflective halo of one voxel), 1 -> 16 channels, ReLU;
  L2  3^3 conv stride 2, L3 3^3 conv stride 2, L4 3^3 conv stride 1, all
      16 -> 16 with zero padding, ReLU;
  head  logits[tile, k] = bh[k] + sum_c Wh[k, c] a4[tile, c];
  loss  sum_tiles inv_n * sum_k t_k (logsumexp(l) - l_k)   (targets per tile
        sum to 1 or 0; inv_n = 1 / number of tiles).
Weight blocks are rounded to BF16 (round to nearest even) before use;
biases are not.

tf32=True restates the tensor-core path of layers 2-4
(microtomodenoise_b200/csrc/proposal_tc.cu): the tensor core reads each FP32
activation (the A operand of the forward convs) and each FP32 output gradient
(the A operand of the input-gradient convs) as TF32, keeping the sign, the
exponent and the top 10 mantissa bits (the low 13 bits dropped, i.e. rounded
toward zero); BF16 weights are exact in TF32, products accumulate in FP32.
Weight gradients stay on the CUDA cores (full FP32 operands).
"""
from __future__ import annotations

import numpy as np

C = 16
TAPS = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]


def layout(S: int) -> dict:
    """Offsets and shapes of the flat parameter vector (same order as the C ABI)."""
    blocks = [("w1", (27, C)), ("b1", (C,)), ("w2", (27, C, C)), ("b2", (C,)),
              ("w3", (27, C, C)), ("b3", (C,)), ("w4", (27, C, C)), ("b4", (C,)),
              ("wh", (S, C)), ("bh", (S,))]
    out, o = {}, 0
    for name, shape in blocks:
        n = int(np.prod(shape))
        out[name] = (o, shape)
        o += n
    out["total"] = o
    return out


def bf16_round(a) -> np.ndarray:
    """float32 -> nearest bfloat16 (ties to even), returned as float32."""
    u = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)


def tf32_trunc(a) -> np.ndarray:
    """Value -> float32 (nearest) -> TF32 by dropping the low 13 mantissa bits."""
    u = np.asarray(a, np.float32).view(np.uint32) & np.uint32(0xFFFFE000)
    return u.view(np.float32).astype(np.float64)


def unpack(params: np.ndarray, S: int, rounded: bool = True) -> dict:
    lay = layout(S)
    p = {}
    for name, val in lay.items():
        if name == "total":
            continue
        o, shape = val
        v = np.asarray(params[o:o + int(np.prod(shape))]).reshape(shape)
        if rounded:
            v = np.asarray(v, np.float32)
            if name.startswith("w"):
                v = bf16_round(v)
        p[name] = np.asarray(v, np.float64)
    return p


def levels(shape_zyx):
    lv = [tuple(int(s) for s in shape_zyx)]
    for _ in range(3):
        lv.append(tuple((s + 1) // 2 for s in lv[-1]))
    return lv


def _l1_inputs(vol, scale):
    """d[t, z, y, x] for the level-1 grid."""
    v = np.pad(np.asarray(vol, np.float64), 1, mode="reflect")  # mirror, no edge repeat
    lv = levels(vol.shape)
    nz, ny, nx = lv[1]
    cz, cy, cx = np.arange(nz) * 2 + 1, np.arange(ny) * 2 + 1, np.arange(nx) * 2 + 1
    centre = v[np.ix_(cz, cy, cx)]
    s = np.asarray(scale, np.float64)[np.arange(nz) * 2][:, None, None]
    d = np.empty((27, nz, ny, nx))
    for t, (dz, dy, dx) in enumerate(TAPS):
        d[t] = s * (v[np.ix_(cz + dz, cy + dy, cx + dx)] - centre)
    return d


def _conv(a, W, b, stride, lo):
    """a: [z, y, x, Cin] -> pre-activation [lo..., Cout] (zero padding)."""
    li = a.shape[:3]
    pad = np.zeros(tuple(max(li[i] + 2, stride * (lo[i] - 1) + 3) for i in range(3)) + (a.shape[3],))
    pad[1:1 + li[0], 1:1 + li[1], 1:1 + li[2]] = a
    out = np.broadcast_to(b, tuple(lo) + (W.shape[2],)).copy()
    for t, (dz, dy, dx) in enumerate(TAPS):
        sl = pad[1 + dz: 1 + dz + stride * lo[0]: stride,
                 1 + dy: 1 + dy + stride * lo[1]: stride,
                 1 + dx: 1 + dx + stride * lo[2]: stride]
        out += np.einsum("zyxi,io->zyxo", sl, W[t])
    return out


def _conv_back(a, W, g, stride):
    """Gradients of _conv: returns (dW, db, da) for pre-activation gradient g."""
    li = a.shape[:3]
    lo = g.shape[:3]
    shp = tuple(max(li[i] + 2, stride * (lo[i] - 1) + 3) for i in range(3)) + (a.shape[3],)
    pad = np.zeros(shp)
    pad[1:1 + li[0], 1:1 + li[1], 1:1 + li[2]] = a
    dpad = np.zeros(shp)
    dW = np.zeros_like(W)
    for t, (dz, dy, dx) in enumerate(TAPS):
        idx = (slice(1 + dz, 1 + dz + stride * lo[0], stride),
               slice(1 + dy, 1 + dy + stride * lo[1], stride),
               slice(1 + dx, 1 + dx + stride * lo[2], stride))
        dW[t] = np.einsum("zyxi,zyxo->io", pad[idx], g)
        dpad[idx] += np.einsum("zyxo,io->zyxi", g, W[t])
    db = g.sum(axis=(0, 1, 2))
    da = dpad[1:1 + li[0], 1:1 + li[1], 1:1 + li[2]]
    return dW, db, da


def forward(params, vol, scale, S, cache=False, rounded=True, tf32=False):
    """Returns logits [tiles, S] (tiles in (z, y, x) order) and optionally the
    cache. rounded=False skips the BF16 rounding (finite-difference checks);
    tf32=True: the tensor-core operand rounding of layers 2-4."""
    p = unpack(params, S, rounded)
    lv = levels(vol.shape)
    op = tf32_trunc if tf32 else (lambda a: a)
    d = _l1_inputs(vol, scale)
    z1 = np.einsum("tzyx,tc->zyxc", d, p["w1"]) + p["b1"]
    a1 = np.maximum(z1, 0)
    z2 = _conv(op(a1), p["w2"], p["b2"], 2, lv[2])
    a2 = np.maximum(z2, 0)
    z3 = _conv(op(a2), p["w3"], p["b3"], 2, lv[3])
    a3 = np.maximum(z3, 0)
    z4 = _conv(op(a3), p["w4"], p["b4"], 1, lv[3])
    a4 = np.maximum(z4, 0)
    h = a4.reshape(-1, C)
    logits = h @ p["wh"].T + p["bh"]
    if cache:
        return logits, dict(p=p, d=d, a1=a1, a2=a2, a3=a3, a4=a4, h=h)
    return logits


def softmax(logits):
    m = logits.max(axis=1, keepdims=True)
    e = np.exp(logits - m)
    return e / e.sum(axis=1, keepdims=True)


def loss_and_grad(params, examples, S, rounded=True, tf32=False):
    """examples: list of (vol, scale, target[tiles, S]). Returns (loss, grad)
    with respect to the weights as used (BF16-rounded unless rounded=False);
    tf32=True: the tensor-core operand rounding of layers 2-4 in the forward
    pass and in the input gradients."""
    lay = layout(S)
    n_tiles = sum(int(np.prod(levels(v.shape)[3])) for v, _, _ in examples)
    inv_n = 1.0 / n_tiles
    grad = np.zeros(lay["total"])
    loss = 0.0
    for vol, scale, target in examples:
        logits, c = forward(params, vol, scale, S, cache=True, rounded=rounded, tf32=tf32)
        op = tf32_trunc if tf32 else (lambda a: a)
        p = c["p"]
        t = np.asarray(target, np.float64).reshape(logits.shape)
        T = t.sum(axis=1, keepdims=True)
        m = logits.max(axis=1, keepdims=True)
        lse = m + np.log(np.exp(logits - m).sum(axis=1, keepdims=True))
        loss += inv_n * float((T * lse - (t * logits).sum(axis=1, keepdims=True)).sum())
        g = (softmax(logits) * T - t) * inv_n                  # dL/dlogits
        gwh = g.T @ c["h"]
        gbh = g.sum(axis=0)
        dh = g @ p["wh"]
        g4 = (dh * (c["h"] > 0)).reshape(c["a4"].shape)
        def back(a, w, g, stride):
            dW, db, da = _conv_back(a, w, g, stride)
            if tf32:  # the input gradient reads g as TF32
                da = _conv_back(a, w, op(g), stride)[2]
            return dW, db, da

        dW4, db4, da3 = back(c["a3"], p["w4"], g4, 1)
        g3 = da3 * (c["a3"] > 0)
        dW3, db3, da2 = back(c["a2"], p["w3"], g3, 2)
        g2 = da2 * (c["a2"] > 0)
        dW2, db2, da1 = back(c["a1"], p["w2"], g2, 2)
        g1 = da1 * (c["a1"] > 0)
        dW1 = np.einsum("tzyx,zyxc->tc", c["d"], g1)
        db1 = g1.sum(axis=(0, 1, 2))
        for name, val in (("w1", dW1), ("b1", db1), ("w2", dW2), ("b2", db2), ("w3", dW3),
                          ("b3", db3), ("w4", dW4), ("b4", db4), ("wh", gwh), ("bh", gbh)):
            o, shape = lay[name]
            grad[o:o + val.size] += val.ravel()
    return loss, grad


def select(logits, k, min_mass):
    """Top-k per tile (ties: lower offset index first); tiles whose predicted
    kept mass is below min_mass keep every offset. Returns (keep[tiles, S],
    pred_mass[tiles], fallback[tiles])."""
    n, S = logits.shape
    k = max(1, min(k, S))
    keep = np.zeros((n, S), bool)
    pm = np.zeros(n)
    prob = softmax(np.asarray(logits, np.float64))
    for i in range(n):
        order = sorted(range(S), key=lambda j: (-float(logits[i, j]), j))
        keep[i, order[:k]] = True
        pm[i] = prob[i, keep[i]].sum()
    fb = ~(pm >= min_mass)
    keep[fb] = True
    return keep, pm, fb


def plans(keep):
    """Per-8^3-tile plan lists (kept offsets in ascending order) from keep flags."""
    return [np.nonzero(row)[0].tolist() for row in np.asarray(keep, bool)]
