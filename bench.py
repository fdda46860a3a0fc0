"""Benchmark of the iterNLM hot path on B200 (one JSON line on stdout).

Workload (the 512^3 plain-filter configuration): a float32 512x512x512
grain-pack volume (uint16-quantised to [0,1], correlated noise sigma 0.04
blurred 1.2, concentric z-axis rings amplitude 0.02 period 6), patch radius 2,
search radius 5 (514 offsets, 33 taps), 4 iterations, alpha 0.5, z-adaptive
noise with a 100-slice window, 1e5 noise samples. Synthetic, seeded.

A step is one whole job: sigma0 on the raw volume, iteration 1, sigma1 on its
result, the alpha blend, iterations 2-4, all on the device (inlm_denoise).
``value`` = voxel-iterations/s with the input resident in HBM; ``e2e`` = the
same through the host-pointer API with the H2D of the raw volume and the D2H
of the result inside the timed region (pinned host memory). Inputs (537 MB)
exceed L2 (126 MB) between steps.

    python bench.py [--gpus N --steps K --warmup W]
    python bench.py --impl reference     # the reference CPU filter on host cores

Multi-GPU (torchrun, N ranks): one 512x512x(512N) volume split in z, each
rank owning 512 slices (weak scaling) and filtering them with 8 slices of
each neighbour (sharded.ZSlabJob): the neighbours' halo slices are swapped
over NCCL after every iteration and the noise estimates all-reduce the
per-sample patch stds, as the reference's n_gpus blocks split a stack
(Denoiser/iternlm_gpu.cu:1729-1886); time = max over ranks. ``--split`` runs
that path on one GPU (one rank).

``forms`` (rank 0, one GPU): the same whole job in the fused FP32 form
(fused multiply-adds, within 1e-4 relative of the reference except at
weights that cross the Pade cutoff), the FP16-storage form, and the
learned-proposal + FP16 form: one offset list per 32x8x8 block (the four 8^3
tiles' predictions summed, run by the full-width kernel) of LEARNED_K[i]
offsets in iteration i, with full search for every block whose predicted
kept weight mass is below LEARNED_REL[i] x the mean over the volume's blocks
(small lists while later iterations re-filter the result, a larger list and
the fallback in the last iteration, whose output carries the approximation);
beside it the schedule 128 x 3, 240; one k throughout (k = 208 with the
fallback at 0.9 in every iteration, k = 176 without), and k = 256 per 8^3
tile with the absolute 0.95 threshold, which falls back on every tile of
this volume. Each form reports its
speed-up over the plain FP32 job, the proposal's fallback and
evaluated-offset fractions, and its accuracy (see run_forms): PSNR against
the clean phantom over the whole volume beside the plain FP32 result's, and
max-abs error and PSNR against the FP64 full-search oracle on 64 seeded 16^3
sub-blocks.

``batch`` (rank 0, one GPU): 24 seeded volumes, sizes uniform from 64^3 to
384x384x256, spheres on a background with blurred noise of sigma uniform in
0.02-0.08, patch radius from {1,2,3} and search radius from {3,5,7} per volume,
4 iterations, global noise: the whole schedule as one CUDA graph with one
persistent kernel per iteration (inlm_batch_run), against the same volumes
run one after another (inlm_denoise each), in voxel-iterations/s.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "voxel-iter/s 512^3 p2 s5 (plain FP32, whole job incl. noise estimates)"
SHAPE = (512, 512, 512)
PR, SR, ITERS = (2, 2, 2), (5, 5, 5), 4
S_OFFSETS, P_TAPS = 514, 33
# algorithmic FLOP per voxel-iteration: per offset 2 per weighted tap, 2 for
# the squared difference, 18 for multiplier, Pade weight, cutoff and sums
FLOP_PER_VOXEL_ITER = S_OFFSETS * (2 * P_TAPS + 20)
BYTES_PER_VOXEL_ITER_F32 = 12                          # read raw + prev, write result
# learned + FP16 form of the headline line: one offset list per 32x8x8 block
# of LEARNED_K[i] offsets in iteration i, full search for the blocks whose
# predicted kept mass is below LEARNED_REL[i] x the mean over the volume's
# blocks (the last iteration's list and fallback set the accuracy)
LEARNED_K, LEARNED_MIN_MASS, LEARNED_REL = (112, 112, 112, 256), 0.0, (0.0, 0.0, 0.0, 0.9)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def workload_config():
    return {"workload": f"grain-pack {SHAPE[2]}x{SHAPE[1]}x{SHAPE[0]} f32, patch r2 (33 taps), search r5 (514 offsets), "
                        "4 iterations, alpha 0.5, z-adaptive noise (window 100, 1e5 samples)",
            "shape_xyz": [SHAPE[2], SHAPE[1], SHAPE[0]], "patch_radius": 2, "search_radius": 5,
            "iterations": ITERS, "offsets": S_OFFSETS, "taps": P_TAPS,
            "l2": "inputs (537 MB) larger than L2 (126 MB)"}


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


# DRAM traffic of one 512^3 launch of the headline filter kernel
# (nlm_tile_f32_ws_kernel<2,2,2,raw box>: 32x8x8 CTAs of 8 consumer and 8
# producer warps, raw box staged): dram__bytes_read.sum +
# dram__bytes_write.sum of one 512x512x128 launch captured by ncu
# (profiles/nlm_tile_f32_ws_p2s5_512.md gives the command), times 4: the traffic
# is the tiles' halo boxes and the result, so it grows with the tile count.
FILTER_TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum, one 512x512x128 launch of "
                         "nlm_tile_f32_ws_kernel, x4")
FILTER_TRAFFIC_BYTES_PER_LAUNCH = 4 * (338.045e6 + 125.709e6)


def fp32_arithmetic_peak(device: int):
    """FP32 CUDA-core peak in TFLOP/s: SMs x 128 FP32 lanes x 2 flop per FFMA
    x the maximum SM clock (nvidia-smi clocks.max.sm, else the driver-measured
    peaks file's sm_max_mhz)."""
    import torch
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    mhz = None
    try:
        out = subprocess.run(["nvidia-smi", "-i", str(device), "--query-gpu=clocks.max.sm",
                              "--format=csv,noheader,nounits"], capture_output=True, text=True,
                             timeout=20).stdout.strip()
        mhz = float(out.splitlines()[0])
    except Exception:
        mhz = measured_peaks().get("sm_max_mhz")
    if not mhz:
        return None, "no SM clock available"
    return sms * 128 * 2 * mhz * 1e6 / 1e12, f"{sms} SMs x 128 FP32 lanes x 2 flop x {mhz:.0f} MHz (clocks.max.sm)"


def make_volume(seed=0, return_clean=False):
    from microtomodenoise_b200 import synth
    t = time.time()
    v = synth.grain_pack_volume(SHAPE, seed=seed, return_clean=return_clean)
    log(f"generated {SHAPE} volume in {time.time() - t:.1f}s")
    return v


def psnr(a, b, peak=1.0):
    mse = float(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2))
    return float("inf") if mse == 0 else 10 * np.log10(peak * peak / mse)


def sub_block_corners(shape, n=64, size=16, seed=0):
    """n seeded lower corners (z, y, x) of size^3 blocks anywhere in the volume
    (faces, edges and corners included)."""
    rng = np.random.default_rng(seed)
    return [tuple(int(rng.integers(0, dim - size + 1)) for dim in shape) for _ in range(n)]


def batch_workload(seed=0, n=24, lo=(64, 64, 64), hi=(384, 384, 256)):
    from microtomodenoise_b200 import DenoiseParameters, synth
    rng = np.random.default_rng(seed)
    vols, params = [], []
    for i in range(n):
        nx = int(rng.integers(lo[0], hi[0] + 1))
        ny = int(rng.integers(lo[1], hi[1] + 1))
        nz = int(rng.integers(lo[2], hi[2] + 1))
        sigma = float(rng.uniform(0.02, 0.08))
        pr = int(rng.choice([1, 2, 3]))
        sr = int(rng.choice([3, 5, 7]))
        vols.append(synth.spheres_volume((nz, ny, nx), n_spheres=40, rmin=4.0, rmax=20.0,
                                         noise_std=sigma, noise_blur=1.0, seed=1000 + i))
        params.append(DenoiseParameters(radius_patchspace=(pr,) * 3, radius_searchspace=(sr,) * 3,
                                        maxiterations=ITERS, alpha=0.5, noise_mode="global",
                                        n_samples=100000, noise_seed=i))
    return vols, params


def run_batch(args, local, small=False):
    """Batched graph vs one-after-another single-volume jobs."""
    import torch
    from microtomodenoise_b200 import Batch, IterativeNLM_GPU
    t = time.time()
    vols, params = (batch_workload(seed=1, lo=(32, 32, 32), hi=(96, 96, 96)) if small
                    else batch_workload())
    log(f"batch workload generated in {time.time() - t:.1f}s")
    vox_iters = float(sum(v.size for v in vols)) * ITERS
    dev = [torch.from_numpy(v).cuda() for v in vols]
    outs = [torch.empty_like(v) for v in dev]
    torch.cuda.synchronize()
    t = time.time()
    b = Batch([v.shape for v in vols], params)
    setup_s = time.time() - t
    desc = b.describe()
    ptrs = [v.data_ptr() for v in dev]
    optrs = [o.data_ptr() for o in outs]
    b.run(ptrs, optrs, on_device=True)  # warm-up
    ms_graph = []
    for _ in range(args.form_steps):
        b.run(ptrs, optrs, on_device=True)
        ms_graph.append(b.last_ms)
    ms_b = float(np.mean(ms_graph))
    host_outs = [np.empty_like(v) for v in vols]
    t0 = time.time()
    b.run(vols, host_outs)
    e2e_s = time.time() - t0
    b.close()
    # the same jobs one after another
    stream = torch.cuda.Stream()
    total_ms = 0.0
    for v, p, o in zip(dev, params, outs):
        g = IterativeNLM_GPU()
        g.configure_device(tuple(v.shape), p)
        g.set_stream(stream.cuda_stream)
        g.denoise(v.data_ptr(), on_device=True, out=o.data_ptr())  # warm-up
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.denoise(v.data_ptr(), on_device=True, out=o.data_ptr())
        e1.record(stream)
        torch.cuda.synchronize()
        total_ms += e0.elapsed_time(e1)
        g.free_device()
    size = "32^3..96^3" if small else "64^3..384x384x256"
    return {"workload": f"24 volumes {size}, spheres + blurred noise sigma 0.02-0.08, "
                        "patch r in {1,2,3}, search r in {3,5,7}, 4 iterations, global noise",
            "voxel_iterations": vox_iters,
            "value": vox_iters / (ms_b / 1e3), "unit": "voxel-iter/s", "ms_per_job": ms_b,
            "steps": args.form_steps, "warmup": 1,
            "sequential_value": vox_iters / (total_ms / 1e3), "sequential_ms": total_ms,
            "speedup_vs_sequential": total_ms / ms_b,
            "e2e": {"value": vox_iters / e2e_s, "unit": "voxel-iter/s",
                    "h2d_bytes_per_step": int(sum(v.nbytes for v in vols)),
                    "d2h_bytes_per_step": int(sum(v.nbytes for v in vols))},
            "setup_s": setup_s, "describe": desc,
            "small_volumes": run_batch(args, local, small=True) if not small else None}


def run_forms(vol, clean, sig_iters, value_f32, args, local, stream):
    """Precision and learned forms: whole-job throughput and accuracy.

    Throughput: each form's whole job (its own noise estimates) timed like the
    headline. Accuracy: every form re-run with the FP32 job's sigma schedule
    held fixed, then
      * over the whole volume: PSNR against the clean phantom, and its
        difference to the plain FP32 result's (bit-exact to the reference's
        CPU filter, within ~1e-6 of FP64);
      * on 64 seeded 16^3 sub-blocks: max-abs error and PSNR against the FP64
        full-search oracle, and PSNR against the clean phantom next to the
        FP64 oracle's own on the same blocks."""
    import torch
    from microtomodenoise_b200 import DenoiseParameters, IterativeNLM_GPU
    from microtomodenoise_b200.proposal import ProposalNet, default_weights
    from oracle.oracle import FilterParams, Port

    net = ProposalNet.load(default_weights(PR, SR), device=local)
    forms = [("f32", "f32", None), ("f32_fused", "f32_fma", None), ("fp16", "f16", None),
             ("learned_fp16", "f16", (LEARNED_K, LEARNED_MIN_MASS, 4, LEARNED_REL)),
             ("learned_fp16_sched128", "f16", ((128, 128, 128, 240), 0.0, 4, (0.0, 0.0, 0.0, 0.9))),
             ("learned_fp16_k208_r09", "f16", (208, 0.0, 4, 0.9)),
             ("learned_fp16_k176", "f16", (176, 0.0, 4, 0.0)),
             ("learned_fp16_k256_mass095", "f16", (256, 0.95, 1, 0.0))]
    for item in filter(None, args.learned_extra.split(",")):
        f = item.split("@")
        k, t = f[0], f[1] if len(f) > 1 else "1"
        m = f[2] if len(f) > 2 else "0"
        prec = f[3] if len(f) > 3 else "f16"
        rel = [float(v) for v in m[1:].split("/")] if m.startswith("r") else [0.0]
        ks = [int(v) for v in k.split("/")]
        forms.append((f"learned_{prec}_k{k.replace('/', '-')}_t{t}_m{m.replace('/', '-')}", prec,
                      (ks if len(ks) > 1 else ks[0], 0.0 if m.startswith("r") else float(m), int(t),
                       rel if len(rel) > 1 else rel[0])))
    raw_dev = torch.from_numpy(vol).cuda()
    out_dev = torch.empty_like(raw_dev)
    vox = float(np.prod(vol.shape))
    corners = sub_block_corners(vol.shape)
    bs = 16
    crop = lambda a: [a[z:z + bs, y:y + bs, x:x + bs] for z, y, x in corners]
    cat = lambda xs: np.concatenate([x.ravel() for x in xs])
    clean_blocks = cat(crop(clean))
    res, blocks, whole = {}, {}, {}
    for name, prec, prop in forms:
        dp = DenoiseParameters(radius_patchspace=PR, radius_searchspace=SR, maxiterations=ITERS,
                               alpha=0.5, noise_mode="z-adaptive", zwindow=100, n_samples=100000,
                               noise_seed=0, deviceID=local, precision=prec)
        g = IterativeNLM_GPU()
        g.configure_device(vol.shape, dp)
        g.set_stream(stream.cuda_stream)
        if prop:
            g.attach_proposal(net, prop[0], prop[1], tiles_x=prop[2], rel_mass=prop[3] if len(prop) > 3 else 0.0)
        r = {"kernel": g.describe()}
        if name != "f32":
            g.denoise(raw_dev.data_ptr(), on_device=True, out=out_dev.data_ptr())
            g.filter_kernel_ms()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.form_steps):
                g.denoise(raw_dev.data_ptr(), on_device=True, out=out_dev.data_ptr())
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / args.form_steps
            kms, kn = g.filter_kernel_ms()
            r["kernel"] = g.describe()  # after the runs: the proposal selects the plan kernel
            r.update({"value": vox * ITERS / (ms / 1e3), "unit": "voxel-iter/s",
                      "ms_per_step": ms, "steps": args.form_steps, "warmup": 1,
                      "speedup_vs_f32": vox * ITERS / (ms / 1e3) / value_f32,
                      "filter_kernel_avg_ms": kms})
            if prop:
                r.update({"k": prop[0], "min_mass": prop[1], "tiles_per_plan": prop[2],
                          "rel_mass": prop[3] if len(prop) > 3 else 0.0})
        # accuracy run: the FP32 job's sigma schedule, fixed, for every form;
        # the proposal's lists per iteration
        fb, ev = [], []
        for it in range(ITERS):
            g.set_sigma(sig_iters[it])
            g.Run_GaussianNoise_device(it + 1, raw_dev.data_ptr() if it == 0 else None)
            if prop:
                st = g.proposal_stats()
                fb.append(st["fallback_tiles"] / max(st["tiles"], 1))
                ev.append(st["fraction_evaluated"])
        if prop:
            r.update({"fallback_fraction": fb[-1], "fallback_per_iteration": fb,
                      "fraction_evaluated": float(np.mean(ev)), "fraction_evaluated_per_iteration": ev,
                      "stats_how": "lists falling back and offsets evaluated per iteration of the accuracy "
                                   "run; fallback_fraction: the last iteration's"})
        g.get_result_device(out_dev.data_ptr())
        torch.cuda.synchronize()
        out = out_dev.cpu().numpy()
        whole[name] = psnr(out, clean)
        blocks[name] = cat(crop(out))
        res[name] = r
        g.free_device()
        del out
        log(f"form {name}: {r}")
    net.close()
    port = Port()
    t = time.time()
    ref = port.denoise_f64_blocks(vol, FilterParams(search_radius=SR, patch_radius=PR), sig_iters,
                                  corners, (bs, bs, bs))
    log(f"FP64 oracle on {len(ref)} sub-blocks: {time.time() - t:.1f}s")
    r64 = cat(ref)
    p64 = psnr(r64, clean_blocks)
    for name in res:
        got = blocks[name]
        res[name]["accuracy"] = {
            "psnr_vs_clean_db": whole[name],
            "delta_vs_f32_db": whole[name] - whole["f32"],
            "max_abs_vs_fp64": float(np.abs(got - r64).max()),
            "psnr_vs_fp64_db": psnr(got, r64),
            "blocks_psnr_vs_clean_db": psnr(got, clean_blocks),
            "blocks_fp64_psnr_vs_clean_db": p64,
            "blocks_delta_vs_fp64_oracle_db": psnr(got, clean_blocks) - p64,
            "how": "psnr_vs_clean / delta_vs_f32: whole volume against the clean phantom, minus the "
                   "plain FP32 result's; *_fp64 and blocks_*: 64 seeded 16^3 sub-blocks against the "
                   "FP64 full-search oracle (oracle/denoise_f64_blocks); sigma schedule of the FP32 "
                   "job held fixed"}
    return res


def cpu_reference_rate(vol, target_s=15.0, threads=None):
    """Rate of the reference CPU filter (oracle/_ref, else the port) on a
    bounded slab sample; returns (rate, info)."""
    from oracle.oracle import FilterParams, Port, Reference, reference_available
    threads = threads or os.cpu_count()
    p = FilterParams(search_radius=SR, patch_radius=PR)
    kind = "reference" if reference_available() else "port"
    if kind == "reference":
        impl = Reference()

        def run(slab, sig):
            out, secs = impl.denoise(slab, p, sig, n_threads=threads)
            return secs
    else:
        impl = Port()
        os.environ["OMP_NUM_THREADS"] = str(threads)

        def run(slab, sig):
            t = time.time()
            impl.denoise_f32(slab, p, sig)
            return time.time() - t
    ny, nx, nzv = vol.shape[1], vol.shape[2], vol.shape[0]
    # The reference parallelises over z-slices (iternlm_cpu.cpp:91): slab
    # depths are whole multiples of the thread count so no thread idles.
    calib = min(threads, nzv)
    z0 = max(0, nzv // 2 - calib // 2)
    slab = np.ascontiguousarray(vol[z0:z0 + calib])
    secs = run(slab, np.full((1, calib), 0.045, np.float32))
    rate = calib * ny * nx / max(secs, 1e-6)
    depth = int(target_s * rate / (ny * nx)) // threads * threads
    depth = int(np.clip(depth, calib, nzv))
    z0 = max(0, nzv // 2 - depth // 2)
    slab = np.ascontiguousarray(vol[z0:z0 + depth])
    secs = run(slab, np.full((1, depth), 0.045, np.float32))
    rate = depth * ny * nx / secs
    info = {"value": rate, "unit": "voxel-iter/s", "cores": threads, "kind": kind,
            "sample": f"{nx}x{ny}x{depth} slab (z {z0}..{z0 + depth - 1}) of the volume, 1 iteration of "
                      f"IterativeNLM_CPU::Run_GaussianNoise (p2 s5, sigma fixed), {secs:.1f}s, "
                      f"OpenMP {threads} threads"}
    return rate, info


PUBLISHED = {"job_s": 8.5, "hardware": "Tesla V100 (sm_70)", "iterations": 4,
             "shape_xyz": [256, 256, 256], "patch_radius": 1, "search_radius": 10, "nslices": 11,
             "source": "iterNLM_v0.3 README benchmark figure caption (4 iterations, 256^3)"}


def reference_gpu_rates(vol):
    """The reference's own GPU class (Denoiser/iternlm_gpu.cu compiled
    unmodified for sm_100a, oracle/_ref/libiternlm_gpu_ref.so) on this GPU,
    driven as the reference driver drives its whole-stack path: iteration 2's
    Run_GaussianNoise (reflective padding, the patch kernel and, as shipped,
    apply_filter_generic after it; the call synchronises) by host wall time.
    Two cases: a 512x512x128 slab (z 192..319) of the headline volume at p2
    s5, and the published configuration (256^3 grain pack, p1, s10, 11
    slices: 3102 offsets). Sigma fixed at 0.045."""
    from microtomodenoise_b200 import synth
    from oracle.oracle import ReferenceGPU, reference_gpu_available
    if not reference_gpu_available():
        return {"unavailable": "oracle/_ref/libiternlm_gpu_ref.so not built (needs the reference tree)"}
    ref = ReferenceGPU()
    out = {"kernel": "IterativeNLM_GPU::Run_GaussianNoise as shipped (iternlm_gpu.cu:1651-1728): "
                     "pad_reflective + apply_filter_patchNNN + apply_filter_generic, sm_100a build"}
    nz = vol.shape[0]
    z0 = max(0, nz // 2 - 64)
    cases = [("headline_slab", np.ascontiguousarray(vol[z0:z0 + 128]), PR[0], SR[0],
              f"512x512x128 slab (z {z0}..{z0 + 127}) of the 512^3 grain pack, p2 s5 (514 offsets)"),
             ("published_config", synth.grain_pack_volume((256, 256, 256), seed=0), 1, 10,
              "256^3 grain pack, p1 s10, 11 slices (3102 offsets)")]
    for name, sub, pr, sr, desc in cases:
        sig = np.full((2, sub.shape[0]), 0.045, np.float32)
        try:
            _, ms = ref.denoise(sub, pr, sr, sig, want_result=False)
        except Exception as e:
            out[name] = {"error": str(e)[:200]}
            continue
        out[name] = {"workload": desc, "iteration_ms": float(ms[1]), "first_iteration_ms": float(ms[0]),
                     "value": float(sub.size / (ms[1] / 1e3)), "unit": "voxel-iter/s"}
    return out


def run_published_config(local, stream):
    """The exact FP32 whole job of this library on the configuration of the
    reference's only published GPU figure: 256^3, patch r1, search r10, 11
    slices (3102 offsets), 4 iterations, z-adaptive noise (the reference
    defaults), on a seeded 256^3 grain pack; device-timed and end to end from
    pinned host buffers. The published 8.5 s is the reference program's wall
    time on a V100."""
    import torch
    import ctypes as C
    from microtomodenoise_b200 import DenoiseParameters, IterativeNLM_GPU, _lib, synth
    vol = synth.grain_pack_volume((256, 256, 256), seed=0)
    dp = DenoiseParameters(radius_patchspace=(1, 1, 1), radius_searchspace=(10, 10, 10), nslices=11,
                           maxiterations=4, alpha=0.5, noise_mode="z-adaptive", zwindow=100,
                           n_samples=100000, noise_seed=0, deviceID=local)
    g = IterativeNLM_GPU()
    g.configure_device(vol.shape, dp)
    g.set_stream(stream.cuda_stream)
    raw_dev = torch.from_numpy(vol).cuda()
    out_dev = torch.empty_like(raw_dev)
    host_raw = torch.from_numpy(vol).pin_memory()
    host_out = torch.empty(vol.shape, dtype=torch.float32).pin_memory()
    s0 = np.zeros(256, np.float32)
    s1 = np.zeros(256, np.float32)
    L = _lib.load()
    for _ in range(2):
        g.denoise(raw_dev.data_ptr(), on_device=True, out=out_dev.data_ptr())
    g.filter_kernel_ms()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(2):
        g.denoise(raw_dev.data_ptr(), on_device=True, out=out_dev.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize()
    job_ms = e0.elapsed_time(e1) / 2
    kms, _ = g.filter_kernel_ms()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(2):
        _lib.check(L.inlm_denoise(g._h, host_raw.data_ptr(), host_out.data_ptr(), 0, s0.ctypes.data,
                                  s1.ctypes.data), "denoise")
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = f0.elapsed_time(f1) / 2
    desc = g.describe()
    g.free_device()
    vox_iters = float(vol.size) * 4
    return {"workload": "256^3 grain pack, patch r1 (7 taps), search r10 with 11 slices (3102 offsets), "
                        "4 iterations, alpha 0.5, z-adaptive noise (window 100, 1e5 samples)",
            "kernel": desc, "job_ms": job_ms, "e2e_job_ms": e2e_ms, "filter_ms_per_iteration": kms,
            "value": vox_iters / (e2e_ms / 1e3), "unit": "voxel-iter/s",
            "published_reference": dict(PUBLISHED, value=vox_iters / PUBLISHED["job_s"]),
            "speedup_vs_published_e2e": PUBLISHED["job_s"] * 1e3 / e2e_ms}


def run_reference_arm(args, rank):
    if rank != 0:
        return
    vol = make_volume()
    if args.reference_gpu_only:
        print(json.dumps({"impl": "reference", "reference_gpu": reference_gpu_rates(vol)}), flush=True)
        return
    threads = os.cpu_count()
    rates = []
    for i in range(args.warmup + args.steps):
        rate, info = cpu_reference_rate(vol, target_s=8.0, threads=threads)
        if i >= args.warmup:
            rates.append(rate)
    value = float(np.mean(rates))
    info["value"] = value
    try:  # the reference's own GPU class on this GPU, beside the CPU timing
        ref_gpu = reference_gpu_rates(vol)
    except Exception as e:
        ref_gpu = {"error": str(e)[:200]}
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "voxel-iter/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded grain pack)",
            "config": workload_config(), "cpu_baseline": info,
            "e2e": {"value": value, "unit": "voxel-iter/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "reference_gpu": ref_gpu}
    print(json.dumps(line), flush=True)


def psnr_chunked(a, b, peak=1.0, chunk=32):
    """PSNR over a volume without float64 copies of the whole of it."""
    se, n = 0.0, 0
    for z in range(0, a.shape[0], chunk):
        d = a[z:z + chunk].astype(np.float64) - b[z:z + chunk]
        se += float(np.sum(d * d))
        n += d.size
    return float("inf") if se == 0 else 10 * np.log10(peak * peak / (se / n))


def parse_learned(spec):
    """k@tiles_per_plan[@min_mass] with min_mass rX: relative threshold X;
    k1/k2/... and rX1/X2/...: per-iteration schedules."""
    f = spec.split("@")
    ks = [int(v) for v in f[0].split("/")]
    t = int(f[1]) if len(f) > 1 else 1
    m = f[2] if len(f) > 2 else "0"
    rels = [float(v) for v in m[1:].split("/")] if m.startswith("r") else [0.0]
    return (ks if len(ks) > 1 else ks[0]), t, (0.0 if m.startswith("r") else float(m)), \
        (rels if len(rels) > 1 else rels[0])


def run_large_workload(args):
    """One-step measurements of the two large workloads (rank 0, one GPU):

    learned1024: float32 1024x1024x512 grain pack (noise 0.05 blurred 1, no
      rings), patch r3 search r7 (1326 offsets), 4 iterations, global noise:
      the whole job in plain FP32, FP16 full search, and learned + FP16 forms
      (--k-list k@tiles[@min_mass], default the schedule 256/256/256/1024 per
      32x8x8 block with the relative fallback in the last iteration, 896 per
      block throughout, and 256 per 8^3 tile with the absolute 0.95
      threshold), PSNR against the clean phantom over the whole volume for
      every form.
    stream2048: a 2048x2048xZ grain pack (Z = --stream-depth, 1024 for the
      17 GB configuration) with noise sigma drifting 0.02 -> 0.08 along z
      (blur 1) and rings of amplitude 0.03, z-adaptive noise, patch r3 search
      r7, 4 iterations, held in host memory and streamed through the GPU in
      z-slabs of --slab slices: the plain FP32 whole job and the learned +
      FP16 whole job (--stream-learned k@tiles[@min_mass], default the schedule
      512/512/512/1024 per block with the relative fallback in the last
      iteration), each with its own
      noise estimates, PSNR against the clean phantom over the whole volume;
      then the learned form again with the plain job's sigma schedule held
      fixed (inlm_blocks_*, one iteration at a time), and the FP64
      full-search result on 64 seeded 128^3 sub-blocks with the same
      schedule (inlm_denoise_f64_blocks): max-abs error and PSNR of both forms
      against it, and PSNR against the clean phantom on those blocks."""
    import torch
    from microtomodenoise_b200 import (Blocks, DenoiseParameters, IterativeNLM_GPU, denoise_f64_blocks,
                                       stream_denoise, synth)
    from microtomodenoise_b200.proposal import ProposalNet, default_weights
    pr, sr = (3, 3, 3), (7, 7, 7)
    net = ProposalNet.load(default_weights(pr, sr))
    res = {"workload": args.workload, "forms": {}}
    t = time.time()
    if args.workload == "learned1024":
        shape = (512, 1024, 1024)
        vol, clean = synth.grain_pack_volume(shape, noise_std=0.05, noise_blur=1.0, ring_amp=0.0,
                                             seed=0, return_clean=True)
    else:
        shape = (args.stream_depth, 2048, 2048)
        try:
            import psutil
            need = 7 * 4 * float(np.prod(shape))
            have = float(psutil.virtual_memory().total)
            if have < need:
                print(json.dumps({"workload": args.workload, "skipped":
                                  f"host memory {have / 1e9:.0f} GB < {need / 1e9:.0f} GB needed"}), flush=True)
                return
        except ImportError:
            pass
        vol, clean = synth.grain_pack_volume(shape, noise_blur=1.0, ring_amp=0.03,
                                             sigma_drift=(0.02, 0.08), seed=0, return_clean=True)
    log(f"generated {shape} in {time.time() - t:.1f}s")
    res["generate_s"] = time.time() - t
    vox = float(np.prod(shape)) * ITERS
    res["config"] = {"shape_xyz": [shape[2], shape[1], shape[0]], "patch_radius": 3,
                     "search_radius": 7, "offsets": 1326, "iterations": ITERS}
    if args.workload == "learned1024":
        forms = [("f32", "f32", None), ("fp16", "f16", None)]
        for item in (args.k_list or "256/256/256/1024@4@r0/0/0/0.9,896@4@r0.9,256@1@0.95").split(","):
            k, tx, mm, rel = parse_learned(item)
            forms.append((f"learned_fp16_{item}", "f16", (k, mm, tx, rel)))
        ref_psnr = None
        for name, prec, prop in forms:
            dp = DenoiseParameters(radius_patchspace=pr, radius_searchspace=sr, maxiterations=ITERS,
                                   alpha=0.5, noise_seed=0, precision=prec, noise_mode="global")
            g = IterativeNLM_GPU()
            g.configure_device(shape, dp)
            if prop:
                g.attach_proposal(net, prop[0], prop[1], tiles_x=prop[2], rel_mass=prop[3])
            raw = torch.from_numpy(vol).cuda()
            out = torch.empty_like(raw)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            g.denoise(raw.data_ptr(), on_device=True, out=out.data_ptr())
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            r = {"ms_per_job": ms, "value": vox / (ms / 1e3), "unit": "voxel-iter/s", "kernel": g.describe()}
            if prop:
                st = g.proposal_stats()
                r.update({"k": prop[0], "min_mass": prop[1], "tiles_per_plan": prop[2], "rel_mass": prop[3],
                          "fallback_fraction": st["fallback_tiles"] / max(st["tiles"], 1),
                          "fraction_evaluated": st["fraction_evaluated"]})
            o = out.cpu().numpy()
            g.free_device()
            del raw, out
            r["psnr_vs_clean_db"] = psnr(o, clean)
            if name == "f32":
                ref_psnr = r["psnr_vs_clean_db"]
            r["delta_vs_f32_db"] = r["psnr_vs_clean_db"] - ref_psnr
            res["forms"][name] = r
            log(f"{name}: {r}")
    else:
        k, tx, mm, rel = parse_learned(args.stream_learned)
        dp32 = DenoiseParameters(radius_patchspace=pr, radius_searchspace=sr, maxiterations=ITERS, alpha=0.5,
                                 noise_seed=0, precision="f32", noise_mode="z-adaptive")
        dp16 = DenoiseParameters(radius_patchspace=pr, radius_searchspace=sr, maxiterations=ITERS, alpha=0.5,
                                 noise_seed=0, precision="f16", noise_mode="z-adaptive")
        out32, s0, s1, st = stream_denoise(vol, dp32, slab_depth=args.slab)
        r32 = {"ms_per_job": st["ms"], "value": vox / (st["ms"] / 1e3), "unit": "voxel-iter/s",
               "h2d_bytes": st["h2d_bytes"], "d2h_bytes": st["d2h_bytes"], "slabs": st["slabs"],
               "halo": st["halo"], "psnr_vs_clean_db": psnr_chunked(out32, clean)}
        log(f"f32: {r32}")
        outl, _, _, st = stream_denoise(vol, dp16, slab_depth=args.slab, net=net, k=k, min_mass=mm,
                                        tiles_x=tx, rel_mass=rel)
        rl = {"ms_per_job": st["ms"], "value": vox / (st["ms"] / 1e3), "unit": "voxel-iter/s",
              "k": k, "tiles_per_plan": tx, "min_mass": mm, "rel_mass": rel, "slabs": st["slabs"],
              "halo": st["halo"], "psnr_vs_clean_db": psnr_chunked(outl, clean)}
        rl["delta_vs_f32_db"] = rl["psnr_vs_clean_db"] - r32["psnr_vs_clean_db"]
        rl["speedup_vs_f32"] = r32["ms_per_job"] / rl["ms_per_job"]
        log(f"learned: {rl}")
        # accuracy with the FP32 job's sigma schedule held fixed
        sched = np.stack([s0] + [(np.float32(0.5) * s0 + np.float32(0.5) * s1).astype(np.float32)] * (ITERS - 1))
        t = time.time()
        b = Blocks(shape, dp16, slab_depth=args.slab)
        b.attach_proposal(net, k, mm, tiles_x=tx, rel_mass=rel)
        other = np.empty_like(vol)
        bufs, prev = [outl, other], None
        for it in range(ITERS):
            b.set_sigma(sched[it])
            o = bufs[it % 2]
            b.run_iteration(it + 1, vol, prev, o)
            prev = o
        b.close()
        fixed = prev
        rl["fixed_schedule_s"] = time.time() - t
        t = time.time()
        bs = 128
        corners = sub_block_corners(shape, n=64, size=bs, seed=0)
        ref = denoise_f64_blocks(vol, DenoiseParameters(radius_patchspace=pr, radius_searchspace=sr), sched,
                                 corners, (bs, bs, bs))
        fp64_s = time.time() - t
        crop = lambda a: np.concatenate([a[z:z + bs, y:y + bs, x:x + bs].ravel() for z, y, x in corners])
        r64, c64 = np.concatenate([x.ravel() for x in ref]), crop(clean)
        p64 = psnr(r64, c64)
        for r, o in ((r32, out32), (rl, fixed)):
            got = crop(o)
            d = np.abs(got - r64)
            per_block = [psnr(g_, w_) for g_, w_ in zip(np.split(got, len(corners)), np.split(r64, len(corners)))]
            r["accuracy"] = {"max_abs_vs_fp64": float(d.max()), "psnr_vs_fp64_db": psnr(got, r64),
                             "psnr_vs_fp64_db_per_block_min": float(np.min(per_block)),
                             "psnr_vs_fp64_db_per_block_median": float(np.median(per_block)),
                             "blocks_psnr_vs_clean_db": psnr(got, c64), "blocks_fp64_psnr_vs_clean_db": p64,
                             "blocks_delta_vs_fp64_oracle_db": psnr(got, c64) - p64}
        res["fp64"] = {"blocks": len(corners), "size": bs, "seconds": fp64_s,
                       "how": "inlm_denoise_f64_blocks (GPU, FP64 full search, bit-exact to the oracle's FP64 "
                              "restatement) with the plain job's sigma schedule"}
        res["forms"] = {"f32": r32, "learned_fp16": rl}
        log(f"accuracy: f32 {r32['accuracy']}, learned {rl['accuracy']}")
    f32 = res["forms"]["f32"]["ms_per_job"]
    for v in res["forms"].values():
        v["speedup_vs_f32"] = f32 / v["ms_per_job"]
    net.close()
    print(json.dumps(res), flush=True)


def run_rgb_workload(args):
    """The colour path (--color) on a 4096x3072 RGB image (seeded gradients,
    disks and shot noise; reference defaults: search radius 10, patch radius 1,
    4 iterations, alpha 0.5, one noise estimate per channel from 2048 samples,
    Anscombe transform, joint weights): the whole job through
    color.rgb_denoise (host planes in and out), and the reference's own colour
    job (oracle/_ref) on a 1024x768 crop on all host threads."""
    import torch
    from microtomodenoise_b200 import DenoiseParameters, synth
    from microtomodenoise_b200.color import ColorParameters, rgb_denoise
    ny, nx = 3072, 4096
    img = synth.rgb_photo(ny, nx, seed=0)
    dp = DenoiseParameters(radius_searchspace=(10, 10, 0), radius_patchspace=(1, 1, 0), nslices=1,
                           maxiterations=ITERS, alpha=0.5, noise_mode="global", n_samples=2048,
                           noise_seed=0)
    cp = ColorParameters()
    rgb_denoise([c[:256, :256] for c in img], dp, cp)  # warm-up
    times = []
    for _ in range(max(1, args.steps)):
        torch.cuda.synchronize()
        t = time.perf_counter()
        rgb_denoise(img, dp, cp)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t)
    secs = min(times)
    res = {"workload": "rgb 4096x3072, search r10, patch r1, 4 iterations, global noise (2048 samples), "
                       "Anscombe, joint weights",
           "ms_per_job": secs * 1e3, "value": ny * nx * ITERS / secs, "unit": "pixel-iter/s",
           "e2e": "host planes in and out, host wall clock (min of steps)"}
    from oracle.oracle import FilterParams, Reference, reference_available
    if reference_available():
        cy, cx = 768, 1024
        crop = [np.ascontiguousarray(c[1000:1000 + cy, 1500:1500 + cx]) for c in img]
        t = time.perf_counter()
        Reference().rgb_job(crop, FilterParams(search_radius=(10, 10, 0), patch_radius=(1, 1, 0),
                                               nslices=1), maxiterations=ITERS, mode="global",
                            n_samples=2048, seed=0, keep_iterations=False)
        csecs = time.perf_counter() - t
        res["cpu_reference"] = {"value": cy * cx * ITERS / csecs, "unit": "pixel-iter/s",
                                "cores": os.cpu_count(), "kind": "reference",
                                "sample": f"{cx}x{cy} crop, whole colour job, {csecs:.1f}s"}
        res["speedup_vs_cpu_reference"] = res["value"] / res["cpu_reference"]["value"]
    print(json.dumps(res), flush=True)


def run_train_workload(args):
    """Training speed of the proposal network for patch radius 3 / search
    radius 7 (1326 offsets, the shipped p3 s7 net's shape): Adam steps on
    batches of 4 examples of 128^3 (the shipped training's batch), the
    network input a seeded grain pack and the targets random per-tile
    distributions (a step's cost does not depend on their values), with
    layers 2-4 on the CUDA cores and then on the tensor cores (forward and
    input gradients; weight gradients on the CUDA cores in both)."""
    import torch
    from microtomodenoise_b200 import synth
    from microtomodenoise_b200.proposal import Example, ProposalNet, tiles8
    S = 1326
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(0)
    exs = []
    for i in range(4):
        v = synth.grain_pack_volume((128, 128, 128), noise_std=0.05, noise_blur=1.0, ring_amp=0.0, seed=100 + i)
        nt = int(np.prod(tiles8(v.shape)))
        t = rng.random((nt, S)).astype(np.float32) ** 4
        t /= t.sum(axis=1, keepdims=True)
        exs.append(Example(torch.from_numpy(v).to(dev), torch.full((128,), 7.0, device=dev),
                           torch.from_numpy(t).to(dev)))
    res = {"workload": "proposal training, S = 1326 (p3 s7), batches of 4 examples of 128^3"}
    for name, tc in (("cuda_cores", False), ("tensor_cores", True)):
        net = ProposalNet(S)
        net.init(seed=0)
        net.set_tensor_cores(True, training=tc)
        for _ in range(3):
            net.train_step(exs, 1e-3)
        torch.cuda.synchronize()
        t = time.perf_counter()
        n = max(args.steps, 10)
        for _ in range(n):
            net.train_step(exs, 1e-3)
        torch.cuda.synchronize()
        secs = time.perf_counter() - t
        res[name] = {"steps": n, "ms_per_step": secs / n * 1e3, "steps_per_s": n / secs}
        net.close()
        log(f"{name}: {res[name]}")
    res["speedup"] = res["tensor_cores"]["steps_per_s"] / res["cuda_cores"]["steps_per_s"]
    print(json.dumps(res), flush=True)


def run_profile_case(args):
    """Small cases of the filter kernels for ncu captures (one GPU, a few GB):

    f32:     two exact FP32 iterations (sigma 0.14) of a grain pack of --shape
             (default 128x512x512) at patch r2 search r5: the headline kernel.
    fast:    two iterations of a 64x512x512 grain pack, patch r2 search r5,
             FP16 form: iteration 1 with the shipped proposal (k = 112 per 8^3
             tile, one tile per CTA), iteration 2 full search (32-wide kernel).
    learned: the whole learned + FP16 job (noise estimates, 4 iterations,
             one list per 32x8x8 block) on a 128x512x512 grain pack.
    published: two exact FP32 iterations of a 256^3 grain pack at the
             reference's default geometry (patch r1, search r10, 11 slices:
             3102 offsets) with the default kernel there, the column form;
    slab:    the same with the tile kernel (raw staged as a z slab)."""
    import torch
    from microtomodenoise_b200 import DenoiseParameters, IterativeNLM_GPU, synth
    from microtomodenoise_b200.proposal import ProposalNet, default_weights
    case = args.case
    net = None
    if case in ("f32", "slab", "published"):
        shape = SHAPE if case == "f32" else (256, 256, 256)
        pr, sr = ((2, 2, 2), (5, 5, 5)) if case == "f32" else ((1, 1, 1), (10, 10, 10))
        vol = synth.grain_pack_volume(shape, seed=0)
        g = IterativeNLM_GPU()
        g.configure_device(vol.shape, DenoiseParameters(radius_patchspace=pr, radius_searchspace=sr,
                                                        nslices=11))
        if case == "slab":
            g.select_tile_form("tile")
        g.set_sigma(np.full(shape[0], 0.14 if case == "f32" else 0.045, np.float32))
        raw = torch.from_numpy(vol).cuda()
        g.Run_GaussianNoise_device(1, raw.data_ptr())
        g.Run_GaussianNoise_device(2)
    elif case == "fast":
        vol = synth.grain_pack_volume((64, 512, 512), seed=0)
        raw = torch.from_numpy(vol).cuda()
        net = ProposalNet.load(default_weights((2, 2, 2), (5, 5, 5)))
        g = IterativeNLM_GPU()
        g.configure_device(vol.shape, DenoiseParameters(radius_patchspace=(2, 2, 2),
                                                        radius_searchspace=(5, 5, 5), precision="f16"))
        g.set_sigma(np.full(64, 0.14, np.float32))
        g.attach_proposal(net, 112, 0.0)
        g.Run_GaussianNoise_device(1, raw.data_ptr())
        g.attach_proposal(None)
        g.Run_GaussianNoise_device(2)
    else:
        vol = synth.grain_pack_volume((128, 512, 512), seed=0)
        raw = torch.from_numpy(vol).cuda()
        out = torch.empty_like(raw)
        net = ProposalNet.load(default_weights((2, 2, 2), (5, 5, 5)))
        g = IterativeNLM_GPU()
        g.configure_device(vol.shape, DenoiseParameters(radius_patchspace=(2, 2, 2),
                                                        radius_searchspace=(5, 5, 5), precision="f16",
                                                        noise_mode="z-adaptive", n_samples=100000))
        g.attach_proposal(net, list(LEARNED_K), LEARNED_MIN_MASS, tiles_x=4, rel_mass=list(LEARNED_REL))
        g.denoise(raw.data_ptr(), on_device=True, out=out.data_ptr())
    torch.cuda.synchronize()
    ms, n = g.filter_kernel_ms()
    log(f"profile case {case}: {g.describe()}; {ms:.2f} ms per filter launch ({n})")
    g.free_device()
    if net is not None:
        net.close()


def run_split(args, rank, world, local):
    """The z-slab split of one 512x512x(512 N) volume over N ranks (see the
    module docstring): value = device-resident job (raw and result in HBM),
    e2e = the same with the rank's raw slices from host memory and its result
    slices back to it."""
    import datetime
    import torch
    import torch.distributed as dist
    from microtomodenoise_b200 import DenoiseParameters
    from microtomodenoise_b200.sharded import ZSlabJob
    if not dist.is_initialized():
        kw = {"device_id": torch.device("cuda", local)} if args.backend == "nccl" else {}
        dist.init_process_group(args.backend, timeout=datetime.timedelta(seconds=300), **kw)
    vol = make_volume(seed=0)  # this rank's 512 slices (every rank holds one copy of the pack)
    full = (SHAPE[0] * world,) + SHAPE[1:]
    dp = DenoiseParameters(radius_patchspace=PR, radius_searchspace=SR, maxiterations=ITERS, alpha=0.5,
                           noise_mode="z-adaptive", zwindow=100, n_samples=100000, noise_seed=0,
                           deviceID=local)
    job = ZSlabJob(full, dp)
    stream = job.be.stream
    sync_dev = "cuda" if args.backend == "nccl" else "cpu"

    def barrier():
        dist.barrier()
        torch.cuda.synchronize()

    def timed(fn, n):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=sync_dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t[0])

    job.load(vol)
    for _ in range(args.warmup):
        job.run_loaded()
    with ClockSampler(local) as clk:
        ms = timed(job.run_loaded, args.steps)
    ms_e2e = timed(lambda: (job.run(vol)), args.e2e_steps)
    job.close()
    vox = float(np.prod(full))
    line = {
        "metric": METRIC, "value": vox * ITERS * args.steps / (ms / 1e3), "unit": "voxel-iter/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded grain pack, 512^3 per rank)",
        "config": dict(workload_config(), split=f"one {SHAPE[2]}x{SHAPE[1]}x{full[0]} volume split in z over "
                                                f"{world} ranks ({args.backend}), {job.halo}-slice halos swapped "
                                                "after every iteration, patch stds all-reduced",
                       parallelism=f"z-slab split x{world}"),
        "e2e": {"value": vox * ITERS * args.e2e_steps / (ms_e2e / 1e3), "unit": "voxel-iter/s",
                "h2d_bytes_per_step": int(vol.nbytes), "d2h_bytes_per_step": int(vol.nbytes),
                "ms_per_step": ms_e2e / args.e2e_steps, "per": "rank (own slices in, own slices out)"},
        "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--form-steps", type=int, default=2)
    ap.add_argument("--no-forms", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-published", action="store_true")
    ap.add_argument("--reference-gpu-only", action="store_true",
                    help="--impl reference: only the reference GPU class timings")
    ap.add_argument("--workload", default="grain512",
                    choices=["grain512", "learned1024", "stream2048", "rgb4k", "profile", "train"],
                    help="grain512: the headline bench line; learned1024, stream2048, rgb4k: "
                         "one-step measurements of the large workloads (run_large_workload, "
                         "run_rgb_workload); profile: a small case for ncu (--case)")
    ap.add_argument("--case", default="f32", choices=["f32", "fast", "learned", "slab", "published"],
                    help="--workload profile: which small case (see run_profile_case)")
    ap.add_argument("--stream-depth", type=int, default=1024)
    ap.add_argument("--slab", type=int, default=64, help="stream2048: z-slab depth")
    ap.add_argument("--stream-learned", default="512/512/512/1024@4@r0/0/0/0.9",
                    help="stream2048: the learned + FP16 form, k@tiles_per_plan[@min_mass|@rX] "
                         "(k and rX may be per-iteration schedules k1/k2/..., rX1/X2/...)")
    ap.add_argument("--learned-extra", default="",
                    help="extra learned + FP16 forms in the headline run, "
                         "k@tiles_per_plan[@min_mass[@precision]][,...]; min_mass rX: relative "
                         "threshold X x the mean predicted kept mass; precision f16 or f16_df32; "
                         "per-iteration schedules as k1/k2/... and rX1/X2/...")
    ap.add_argument("--k-list", default="",
                    help="learned1024: learned + FP16 forms, k@tiles_per_plan[@min_mass|@rX][,...]")
    ap.add_argument("--split", action="store_true",
                    help="time the z-slab split path (sharded.ZSlabJob) even on one GPU")
    ap.add_argument("--backend", default="nccl", choices=["nccl", "gloo"],
                    help="process group of the split path (gloo: exchange through host memory)")
    ap.add_argument("--shape", default="512,512,512",
                    help="nz,ny,nx of the volume (smaller shapes only for profiling runs)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    global SHAPE
    SHAPE = tuple(int(v) for v in args.shape.split(","))
    if args.impl == "reference":
        run_reference_arm(args, rank)
        return
    if args.workload != "grain512":
        if rank == 0:
            import torch
            torch.cuda.set_device(local)
            if args.workload == "rgb4k":
                run_rgb_workload(args)
            elif args.workload == "profile":
                run_profile_case(args)
            elif args.workload == "train":
                run_train_workload(args)
            else:
                run_large_workload(args)
        return

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1 or args.split:
        if world == 1 and not dist.is_initialized():
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            os.environ.setdefault("MASTER_PORT", "29533")
            os.environ.setdefault("RANK", "0")
            os.environ.setdefault("WORLD_SIZE", "1")
        run_split(args, rank, world, local)
        return

    from microtomodenoise_b200 import DenoiseParameters, IterativeNLM_GPU, _lib
    import ctypes as C

    L = _lib.load()
    fp32_peak, peak_source = fp32_arithmetic_peak(local)

    vol, clean = make_volume(seed=0, return_clean=True)
    dp = DenoiseParameters(radius_patchspace=PR, radius_searchspace=SR, maxiterations=ITERS,
                           alpha=0.5, noise_mode="z-adaptive", zwindow=100, n_samples=100000,
                           noise_seed=0, deviceID=local)
    g = IterativeNLM_GPU()
    assert g.configure_device(vol.shape, dp) > 0
    stream = torch.cuda.Stream()
    g.set_stream(stream.cuda_stream)
    raw_dev = torch.from_numpy(vol).cuda()
    out_dev = torch.empty_like(raw_dev)
    torch.cuda.synchronize()

    def step():
        g.denoise(raw_dev.data_ptr(), on_device=True, out=out_dev.data_ptr())

    for _ in range(args.warmup):
        step()
    g.filter_kernel_ms()  # drop warm-up launches
    cnt = C.c_uint64(0)
    L.inlm_kernel_launches(g._h, C.byref(cnt))
    launches0 = cnt.value

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    L.inlm_kernel_launches(g._h, C.byref(cnt))
    gpu_launches = int(cnt.value - launches0)
    filt_ms, filt_n = g.filter_kernel_ms()

    # end-to-end through the host-pointer API (pinned host buffers)
    host_raw = torch.from_numpy(vol).pin_memory()
    host_out = torch.empty(vol.shape, dtype=torch.float32).pin_memory()
    nz = vol.shape[0]
    s0 = np.zeros(nz, np.float32)
    s1 = np.zeros(nz, np.float32)

    def step_e2e():
        rc = L.inlm_denoise(g._h, host_raw.data_ptr(), host_out.data_ptr(), 0, s0.ctypes.data,
                            s1.ctypes.data)
        _lib.check(rc, "denoise")

    step_e2e()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.e2e_steps):
        step_e2e()
    f1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = f0.elapsed_time(f1)

    # max over ranks
    t = torch.tensor([ms, ms_e2e], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms, ms_e2e = float(t[0]), float(t[1])

    vox = float(np.prod(SHAPE))
    value = world * vox * ITERS * args.steps / (ms / 1e3)
    value_e2e = world * vox * ITERS * args.e2e_steps / (ms_e2e / 1e3)
    achieved = FLOP_PER_VOXEL_ITER * vox / (filt_ms * 1e-3) / 1e12
    traffic = FILTER_TRAFFIC_BYTES_PER_LAUNCH * vox / (512.0 ** 3)
    line = {
        "metric": METRIC, "value": value, "unit": "voxel-iter/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded grain pack, 512^3)", "config": workload_config(),
        "e2e": {"value": value_e2e, "unit": "voxel-iter/s",
                "h2d_bytes_per_step": int(vol.nbytes), "d2h_bytes_per_step": int(vol.nbytes),
                "ms_per_step": ms_e2e / args.e2e_steps},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                     "frac": achieved / fp32_peak if fp32_peak else None,
                     "traffic": traffic, "traffic_source": FILTER_TRAFFIC_SOURCE,
                     "kernel": g.describe(), "kernel_avg_ms": filt_ms, "kernel_launches": filt_n,
                     "flop_per_voxel_iter": FLOP_PER_VOXEL_ITER,
                     "peak_source": "FP32 arithmetic peak: " + peak_source,
                     "hbm": {"achieved_gbs": BYTES_PER_VOXEL_ITER_F32 * vox / (filt_ms * 1e-3) / 1e9,
                             "peak_gbs": measured_peaks().get("hbm_gbs"),
                             "bytes_per_voxel_iter": BYTES_PER_VOXEL_ITER_F32}},
        "gpu_launches": gpu_launches,
        "clocks": clk.summary(),
    }
    g.free_device()
    if rank == 0 and world == 1 and not args.no_forms:
        sig_iters = np.stack([s0] + [(0.5 * s0 + 0.5 * s1).astype(np.float32)] * (ITERS - 1))
        try:
            line["forms"] = run_forms(vol, clean, sig_iters, value, args, local, stream)
        except Exception as e:
            line["forms"] = {"error": str(e)[:300]}
    if rank == 0 and world == 1 and not args.no_published:
        try:
            line["published_config"] = run_published_config(local, stream)
        except Exception as e:
            line["published_config"] = {"error": str(e)[:300]}
    if rank == 0 and world == 1 and not args.no_batch:
        try:
            line["batch"] = run_batch(args, local)
        except Exception as e:
            line["batch"] = {"error": str(e)[:300]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            _, info = cpu_reference_rate(vol)
            line["cpu_baseline"] = info
        except Exception as e:  # the GPU number stands without it
            line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
