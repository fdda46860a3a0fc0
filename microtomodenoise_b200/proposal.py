"""Learned search-offset proposal: network handle, training data and training.

The network (4 conv layers of 16 channels with 3^3 kernels, BF16 weights,
FP32 accumulation, a linear head with a softmax over the search offsets per
8^3 tile) and its training kernels live in libinlm.so (csrc/proposal.cu);
this module drives them through the C ABI. Device buffers are torch tensors
(plumbing only); every computation is one of the library's kernels.

Training data: for seeded synthetic volumes, the FP16-form denoiser runs the
iterNLM schedule (noise estimate, iteration 1, blended sigma, iterations
2..n) and after every iteration records the network input (the iterate the
filter read and its per-slice scale) and the target, the per-tile weight
mass of every search offset under full search (inlm_weight_map).

    python -m microtomodenoise_b200.proposal --pr 2 --sr 5 --volumes 64 --out weights.npz
"""
from __future__ import annotations

import argparse
import ctypes as C
import os
import time
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import DenoiseParameters, IterativeNLM_GPU, NoiseLevel, _lib, synth
from ._lib import InlmError

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS_DIR = os.path.join(HERE, "weights")

C16 = 16
TAPS = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]


def layout(S: int) -> dict:
    """(offset, shape) of every block of the flat parameter vector."""
    blocks = [("w1", (27, C16)), ("b1", (C16,)), ("w2", (27, C16, C16)), ("b2", (C16,)),
              ("w3", (27, C16, C16)), ("b3", (C16,)), ("w4", (27, C16, C16)), ("b4", (C16,)),
              ("wh", (S, C16)), ("bh", (S,))]
    out, o = {}, 0
    for name, shape in blocks:
        out[name] = (o, shape)
        o += int(np.prod(shape))
    out["total"] = o
    return out


def tiles8(shape_zyx):
    return tuple((int(s) + 7) // 8 for s in shape_zyx)


def _torch():
    import torch
    return torch


@dataclass
class Example:
    vol: "object"      # torch float32 (nz, ny, nx) on the device
    scale: "object"    # torch float32 (nz,)
    target: "object"   # torch float32 (tiles, S)
    iteration: int = 0
    seed: int = 0


class ProposalNet:
    """Handle of one proposal network for S search offsets on one device."""

    def __init__(self, n_offsets: int, device: int = 0):
        L = _lib.load()
        self._h = C.c_void_p(None)
        _lib.check(L.inlm_proposal_create(int(n_offsets), int(device), C.byref(self._h)),
                   "proposal_create")
        n = C.c_int64(0)
        _lib.check(L.inlm_proposal_n_params(self._h, C.byref(n)), "proposal_n_params")
        self.S = int(n_offsets)
        self.n_params = int(n.value)
        self.device = int(device)
        assert self.n_params == layout(self.S)["total"]

    # ---- parameters ----
    def init(self, seed: int = 0, prior: Optional[np.ndarray] = None) -> np.ndarray:
        """He-normal conv weights, zero biases, small head weights; the head
        bias is log(prior) when a prior offset distribution is given."""
        rng = np.random.default_rng(seed)
        lay = layout(self.S)
        p = np.zeros(self.n_params, np.float32)
        for name, fan_in in (("w1", 27), ("w2", 27 * C16), ("w3", 27 * C16), ("w4", 27 * C16)):
            o, shape = lay[name]
            n = int(np.prod(shape))
            p[o:o + n] = rng.standard_normal(n) * np.sqrt(2.0 / fan_in)
        o, shape = lay["wh"]
        p[o:o + int(np.prod(shape))] = rng.standard_normal(int(np.prod(shape))) * 0.01
        if prior is not None:
            o, _ = lay["bh"]
            p[o:o + self.S] = np.log(np.maximum(np.asarray(prior, np.float64), 1e-12))
        self.set_params(p)
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.n_params
        _lib.check(_lib.load().inlm_proposal_set_params(self._h, p.ctypes.data, p.size),
                   "proposal_set_params")

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.n_params, np.float32)
        _lib.check(_lib.load().inlm_proposal_get_params(self._h, p.ctypes.data, p.size),
                   "proposal_get_params")
        return p

    def set_tensor_cores(self, on: bool, training: bool = False) -> None:
        """Layers 2-4 on the tensor cores (tcgen05, TF32 operands, FP32
        accumulation) or on the CUDA cores (FP32 activations, the reference of
        the tensor-core path): `on` for inference (the default), `training`
        for the forward pass and input gradients of train_step / gradients
        (off by default; weight gradients always run on the CUDA cores)."""
        mode = (1 if on else 0) | (2 if training else 0)
        _lib.check(_lib.load().inlm_proposal_set_tensor_cores(self._h, mode), "proposal_set_tensor_cores")

    def save(self, path: str, **meta) -> None:
        np.savez(path, params=self.get_params(), S=self.S, **meta)

    @classmethod
    def load(cls, path: str, device: int = 0) -> "ProposalNet":
        z = np.load(path)
        net = cls(int(z["S"]), device)
        net.set_params(z["params"])
        return net

    # ---- compute ----
    def logits(self, vol, scale):
        torch = _torch()
        nz, ny, nx = vol.shape
        out = torch.empty((int(np.prod(tiles8(vol.shape))), self.S), dtype=torch.float32,
                          device=vol.device)
        torch.cuda.synchronize(vol.device)
        _lib.check(_lib.load().inlm_proposal_logits(self._h, vol.data_ptr(), scale.data_ptr(),
                                                    (C.c_int * 3)(nx, ny, nz), out.data_ptr()),
                   "proposal_logits")
        return out

    def _examples_c(self, examples: Sequence[Example]):
        n = len(examples)
        vols = (C.c_void_p * n)(*[e.vol.data_ptr() for e in examples])
        scales = (C.c_void_p * n)(*[e.scale.data_ptr() for e in examples])
        targets = (C.c_void_p * n)(*[e.target.data_ptr() for e in examples])
        shapes = (C.c_int * (3 * n))()
        for i, e in enumerate(examples):
            nz, ny, nx = e.vol.shape
            shapes[3 * i:3 * i + 3] = [nx, ny, nz]
        return n, vols, scales, targets, shapes

    def gradients(self, examples: Sequence[Example]):
        """(loss, gradient) of the batch without an update."""
        _torch().cuda.synchronize()
        n, vols, scales, targets, shapes = self._examples_c(examples)
        g = np.zeros(self.n_params, np.float32)
        loss = C.c_double(0)
        _lib.check(_lib.load().inlm_proposal_train(self._h, n, vols, scales, targets, shapes, 0.0,
                                                   C.byref(loss), g.ctypes.data),
                   "proposal_train")
        return loss.value, g

    def train_step(self, examples: Sequence[Example], lr: float) -> float:
        _torch().cuda.synchronize()
        n, vols, scales, targets, shapes = self._examples_c(examples)
        loss = C.c_double(0)
        _lib.check(_lib.load().inlm_proposal_train(self._h, n, vols, scales, targets, shapes,
                                                   float(lr), C.byref(loss), None),
                   "proposal_train")
        return loss.value

    def select(self, vol, scale, k: int, min_mass: float, tiles_x: int = 1):
        """(keep bitmap int32 [lists, ceil(S/32)], predicted kept mass [lists],
        fallback lists); one list per 8^3 tile, or per tiles_x tiles along x."""
        torch = _torch()
        nz, ny, nx = vol.shape
        tz, ty, tx = tiles8(vol.shape)
        nt = (-(-tx // tiles_x)) * ty * tz
        nw = (self.S + 31) // 32
        bm = torch.zeros((nt, nw), dtype=torch.int32, device=vol.device)
        pm = torch.zeros(nt, dtype=torch.float32, device=vol.device)
        nfb = C.c_int(0)
        torch.cuda.synchronize(vol.device)
        _lib.check(_lib.load().inlm_proposal_select_grouped(
            self._h, vol.data_ptr(), scale.data_ptr(), (C.c_int * 3)(nx, ny, nz), int(tiles_x), int(k),
            float(min_mass), bm.data_ptr(), pm.data_ptr(), C.byref(nfb)), "proposal_select")
        return bm, pm, nfb.value

    def close(self) -> None:
        if self._h:
            _lib.load().inlm_proposal_destroy(self._h)
            self._h = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bitmap_to_keep(bm, S: int):
    """int32 bitmap [tiles, words] -> bool [tiles, S] (torch, on the device)."""
    torch = _torch()
    bits = torch.arange(32, device=bm.device, dtype=torch.int32)
    keep = ((bm.unsqueeze(-1) >> bits) & 1).bool().reshape(bm.shape[0], -1)
    return keep[:, :S]


def kept_mass(bm, target, S: int):
    """True kept weight mass per tile of a selection (target rows sum to 1)."""
    return (bitmap_to_keep(bm, S).float() * target).sum(dim=1)


# ---------------- training data ----------------

def training_volume(shape_zyx, seed: int, workload: str = "grain_pack_rings"):
    """Seeded synthetic volume at a training size, from the generator of a
    benchmark workload:
      grain_pack_rings  the 512^3 grain pack (noise 0.04 blurred 1.2, z-axis
                        rings of amplitude 0.02 and period 6);
      grain_pack        the learned-proposal workload (noise 0.05 blurred 1,
                        no rings);
      spheres           spheres on a background (noise 0.05)."""
    if workload == "grain_pack_rings":
        return synth.grain_pack_volume(shape_zyx, seed=seed)
    if workload == "grain_pack":
        return synth.grain_pack_volume(shape_zyx, noise_std=0.05, noise_blur=1.0, ring_amp=0.0,
                                       seed=seed)
    return synth.small_case(shape_zyx, seed=seed)


def make_examples(volumes: Sequence[np.ndarray], params: DenoiseParameters,
                  seeds: Optional[Sequence[int]] = None,
                  sigma_factors: Optional[Sequence[float]] = None) -> List[Example]:
    """Runs the iterNLM schedule in the FP16 form on each volume and records,
    per iteration, the network input and the full-search weight-mass target.
    sigma_factors[i] (optional) scales volume i's sigma estimates, so that the
    network also sees the weight maps of smaller or larger filter sigmas
    (manual sigma settings)."""
    torch = _torch()
    dev = torch.device("cuda", params.deviceID)
    out: List[Example] = []
    for vi, vol in enumerate(volumes):
        vol = np.ascontiguousarray(vol, np.float32)
        shape = vol.shape
        nt = int(np.prod(tiles8(shape)))
        g = IterativeNLM_GPU()
        g.configure_device(shape, params)
        S = g.n_search_offsets()
        nl = NoiseLevel(params.n_samples, params.patchsize, shape, seed=params.noise_seed,
                        device=params.deviceID)
        try:
            f = float(sigma_factors[vi]) if sigma_factors is not None else 1.0
            sigma0 = (nl.get_noiselevel(vol, params) * f).astype(np.float32)
            sigma = sigma0
            for it in range(1, params.maxiterations + 1):
                g.set_sigma(sigma)
                g.Run_GaussianNoise(it, vol if it == 1 else None)
                x = torch.empty(shape, dtype=torch.float32, device=dev)
                s = torch.empty(shape[0], dtype=torch.float32, device=dev)
                t = torch.empty((nt, S), dtype=torch.float32, device=dev)
                g.net_input(x.data_ptr(), s.data_ptr())
                g.weight_map(t.data_ptr())
                out.append(Example(x, s, t, it, int(seeds[vi]) if seeds is not None else vi))
                if it == 1 and params.maxiterations > 1:
                    sigma1 = nl.get_noiselevel(g.get_result(), params) * f
                    sigma = (params.alpha * sigma0 + (1 - params.alpha) * sigma1).astype(np.float32)
        finally:
            nl.close()
            g.free_device()
    return out


def mean_target(examples: Sequence[Example]) -> np.ndarray:
    """Average offset distribution over all training tiles (the static prior)."""
    acc, n = None, 0
    for e in examples:
        s = e.target.sum(dim=0).double()
        acc = s if acc is None else acc + s
        n += e.target.shape[0]
    p = (acc / max(n, 1)).cpu().numpy()
    return p / max(p.sum(), 1e-30)


def prior_params(S: int, prior: np.ndarray) -> np.ndarray:
    """A network that ignores its input and ranks offsets by `prior`: every
    weight zero, head bias log(prior). The proposal without learning."""
    p = np.zeros(layout(S)["total"], np.float32)
    o, _ = layout(S)["bh"]
    p[o:o + S] = np.log(np.maximum(np.asarray(prior, np.float64), 1e-12))
    return p


def train(net: ProposalNet, examples: Sequence[Example], steps: int, batch: int = 4,
          lr: float = 2e-3, seed: int = 0, log_every: int = 0) -> List[float]:
    """Adam on random batches; cosine decay of the learning rate."""
    rng = np.random.default_rng(seed)
    losses = []
    for step in range(steps):
        idx = rng.choice(len(examples), size=min(batch, len(examples)), replace=False)
        lr_t = lr * 0.5 * (1 + np.cos(np.pi * step / max(steps, 1)))
        losses.append(net.train_step([examples[i] for i in idx], max(lr_t, lr * 0.02)))
        if log_every and (step % log_every == 0 or step == steps - 1):
            print(f"step {step:5d} loss {losses[-1]:.5f}", flush=True)
    return losses


def evaluate(net: ProposalNet, examples: Sequence[Example], k: int, min_mass: float = 0.0):
    """Mean true kept mass of the net's top-k, its predicted kept mass, the
    fallback fraction, and the kept mass of the ideal top-k (the k offsets
    of largest true mass per tile: the bound of any proposal)."""
    torch = _torch()
    kept, pred, ideal, fb, n = 0.0, 0.0, 0.0, 0, 0
    for e in examples:
        bm, pm, nfb = net.select(e.vol, e.scale, k, min_mass)
        kept += float(kept_mass(bm, e.target, net.S).sum())
        pred += float(pm.sum())
        ideal += float(torch.topk(e.target, min(k, net.S), dim=1).values.sum())
        fb += nfb
        n += e.target.shape[0]
    return dict(kept=kept / n, predicted=pred / n, ideal=ideal / n, fallback=fb / n, tiles=n)


def default_weights(pr, sr) -> str:
    return os.path.join(WEIGHTS_DIR, f"proposal_p{pr[0]}{pr[1]}{pr[2]}_s{sr[0]}{sr[1]}{sr[2]}.npz")


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--pr", type=int, nargs=3, default=(2, 2, 2))
    ap.add_argument("--sr", type=int, nargs=3, default=(5, 5, 5))
    ap.add_argument("--volumes", type=int, default=64)
    ap.add_argument("--holdout", type=int, default=4)
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--workload", default="grain_pack_rings",
                    choices=["grain_pack_rings", "grain_pack", "spheres"])
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--k", type=int, default=256)
    ap.add_argument("--sigma-aug", type=float, default=0.0,
                    help="fraction of training volumes whose sigma is scaled by a factor "
                         "drawn from [0.3, 1]")
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    params = DenoiseParameters(radius_patchspace=tuple(a.pr), radius_searchspace=tuple(a.sr),
                               precision="f16", noise_mode="global", maxiterations=4)
    shape = (a.size, a.size, a.size)
    t0 = time.time()
    seeds = list(range(1, a.volumes + 1))
    hold = list(range(100001, 100001 + a.holdout))
    rng = np.random.default_rng(12345)
    factors = [float(rng.uniform(0.3, 1.0)) if rng.random() < a.sigma_aug else 1.0 for _ in seeds]
    train_ex = make_examples([training_volume(shape, s, a.workload) for s in seeds], params, seeds,
                             factors)
    test_ex = make_examples([training_volume(shape, s, a.workload) for s in hold], params, hold)
    S = train_ex[0].target.shape[1]
    print(f"{len(train_ex)} training examples, {len(test_ex)} held out, S={S}, "
          f"{time.time() - t0:.1f} s", flush=True)
    prior = mean_target(train_ex)
    net = ProposalNet(S)
    net.set_params(prior_params(S, prior))
    base = evaluate(net, test_ex, a.k)
    net.init(seed=0, prior=prior)
    t1 = time.time()
    train(net, train_ex, a.steps, a.batch, a.lr, log_every=100)
    print(f"training {time.time() - t1:.1f} s", flush=True)
    res = evaluate(net, test_ex, a.k)
    print(f"held-out kept mass at K={a.k}: prior {base['kept']:.4f}, trained {res['kept']:.4f} "
          f"(predicted {res['predicted']:.4f})", flush=True)
    out = a.out or default_weights(a.pr, a.sr)
    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    net.save(out, pr=np.array(a.pr), sr=np.array(a.sr), k=a.k, kept_prior=base["kept"],
             kept_trained=res["kept"], volumes=a.volumes, size=a.size, workload=a.workload,
             steps=a.steps)
    print(out)


if __name__ == "__main__":
    main()
