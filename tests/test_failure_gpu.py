"""Failure paths on the GPU, provoked without a GPU fault.

The reference detects a failed CUDA call by comparing
cudaGetErrorString(cudaGetLastError()) with "no error", prints it and
returns (Denoiser/iternlm_gpu.cu:1608-1618). Here every C-ABI call returns a
status; these tests make the two failures a device run can meet happen on
purpose and check the status and what the handle does afterwards:

* a bounded device wait that runs out: a one-CTA kernel whose mbarrier wait
  (the wait of every TMA-staged filter kernel) is never satisfied, with a
  short budget; the call returns INLM_ERR_TIMEOUT and the handle goes on;
* device allocations that fail: every allocation point of a denoiser's
  creation and of a whole job, one after another, fails once as cudaMalloc
  fails when memory runs out; the call returns INLM_ERR_NOMEM, nothing
  allocated stays behind, and the same handle finishes the job afterwards.
"""
import ctypes as C

import numpy as np
import pytest

from microtomodenoise_b200 import DenoiseParameters, IterativeNLM_GPU, _lib, synth
from oracle.oracle import FilterParams

pytestmark = pytest.mark.gpu

ERR_NOMEM, ERR_TIMEOUT = -4, -6


def _live(L):
    n = C.c_int64(-1)
    _lib.check(L.inlm_debug_live_allocations(C.byref(n)), "live allocations")
    return n.value


def test_bounded_wait_expiry_reports_timeout_and_the_handle_recovers(gpu, port):
    L = _lib.load()
    vol = synth.small_case((12, 40, 48), seed=3)
    g = IterativeNLM_GPU()
    g.configure_device(vol.shape, DenoiseParameters(radius_patchspace=(2, 2, 2), radius_searchspace=(3, 3, 3)))
    s = np.full(12, 0.05, np.float32)
    g.set_sigma(s)
    for _ in range(2):  # twice: the error word is cleared after each report
        rc = L.inlm_debug_wait_expiry(g._h, 200000)  # ~0.1 ms of spinning
        assert rc == ERR_TIMEOUT, (rc, L.inlm_last_error())
        assert b"wait gave up" in L.inlm_last_error()
    g.Run_GaussianNoise(1, vol)
    got = g.get_result()
    g.free_device()
    want = port.denoise_f32(vol, FilterParams(search_radius=(3, 3, 3), patch_radius=(2, 2, 2)), s[None])
    assert np.array_equal(got, want)


def test_allocation_failures_at_creation_return_nomem_without_leaks(gpu):
    L = _lib.load()
    p = DenoiseParameters(radius_patchspace=(2, 2, 2), radius_searchspace=(3, 3, 3)).to_c()
    shape = (C.c_int * 3)(48, 40, 12)
    live0 = _live(L)
    failed = 0
    for k in range(64):
        L.inlm_debug_fail_allocation(k)
        h = C.c_void_p(None)
        rc = L.inlm_denoiser_create(shape, C.byref(p), C.byref(h))
        L.inlm_debug_fail_allocation(-1)
        if rc == 0:
            L.inlm_denoiser_destroy(h)
            break
        assert rc == ERR_NOMEM, (k, rc, L.inlm_last_error())
        assert not h.value
        assert _live(L) == live0, f"allocation {k} failed: {_live(L) - live0} allocations left behind"
        failed += 1
    assert rc == 0 and failed >= 4, (failed, rc)
    assert _live(L) == live0


def test_allocation_failures_during_a_job_leave_the_handle_usable(gpu):
    """The allocations a whole job makes on first use (noise estimator,
    staging, EM scratch) fail one after another; each time inlm_denoise
    returns INLM_ERR_NOMEM, and the same handle then completes the job with
    the result of an undisturbed run."""
    L = _lib.load()
    vol = synth.small_case((12, 40, 48), seed=8)
    dp = DenoiseParameters(radius_patchspace=(1, 1, 1), radius_searchspace=(3, 3, 3), maxiterations=2,
                           noise_mode="global", n_samples=4000, noise_seed=2)
    ref = IterativeNLM_GPU()
    ref.configure_device(vol.shape, dp)
    want, _, _ = ref.denoise(vol)
    ref.free_device()
    live0 = _live(L)
    g = IterativeNLM_GPU()
    g.configure_device(vol.shape, dp)
    live_handle = _live(L)
    failures = 0
    for k in range(64):
        L.inlm_debug_fail_allocation(k)
        try:
            got, _, _ = g.denoise(vol)
            L.inlm_debug_fail_allocation(-1)
            break
        except _lib.InlmError as e:
            L.inlm_debug_fail_allocation(-1)
            assert e.code == ERR_NOMEM, e
            failures += 1
    assert failures >= 1
    assert np.array_equal(got, want)
    assert _live(L) >= live_handle  # buffers kept by the handle for the next job
    g.free_device()
    assert _live(L) == live0
