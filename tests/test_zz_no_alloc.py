"""The allocation-free Bessel sum (kr_bessel_sum_noalloc) against the workspace entry point.

Some callers cannot allocate device memory (a host that owns the GPU's memory pool, an FFI
caller holding only device pointers, a loop that must avoid cudaMalloc's implicit device
synchronisation); kr_bessel_sum_noalloc serves them from a fixed 16 MiB static device
array.  This file is named to be collected last.  Both entry points are called through the
C ABI on the same inputs, twice in a row with different inputs and sizes (the shared array
keeps the previous call's contents), and must agree to the path's 1e-10 relative bar.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _call(fn_name, R, p, pw, dp, om, r, U, ws=None):
    from seismicinversion_b200 import _lib

    h = _lib.lib()
    st = torch.cuda.current_stream().cuda_stream
    if fn_name == "kr_bessel_sum":
        return h.kr_bessel_sum(R.data_ptr(), p.data_ptr(), pw.data_ptr(), p.numel(), dp,
                               om.data_ptr(), om.numel(), r.data_ptr(), r.numel(), U.data_ptr(),
                               ws.data_ptr(), ws.numel(), st)
    return h.kr_bessel_sum_noalloc(R.data_ptr(), p.data_ptr(), pw.data_ptr(), p.numel(), dp,
                                   om.data_ptr(), om.numel(), r.data_ptr(), r.numel(),
                                   U.data_ptr(), st)


def _inputs(seed, n_p, n_w, n_r):
    rng = np.random.default_rng(seed)
    dev = "cuda"
    R = torch.as_tensor(rng.standard_normal((n_p, n_w)) + 1j * rng.standard_normal((n_p, n_w)),
                        device=dev)
    p = torch.as_tensor(np.sort(rng.uniform(1e-3, 1.2, n_p)), device=dev)
    pw = p * torch.as_tensor(rng.uniform(0, 1, n_p), device=dev)
    om = torch.as_tensor(np.arange(1, n_w + 1) * (2 * np.pi / 64), device=dev)
    r = torch.as_tensor(rng.uniform(0.0, 50.0, n_r), device=dev)
    return R, p, pw, om, r


def test_noalloc_matches_workspace_entry_two_calls():
    from seismicinversion_b200 import _lib

    h = _lib.lib()
    for call, (n_p, n_w, n_r) in enumerate([(1500, 300, 9), (4096, 513, 100)]):
        R, p, pw, om, r = _inputs(call, n_p, n_w, n_r)
        dp = 1.2 / n_p
        ws = torch.empty(h.kr_bessel_sum_workspace_bytes(n_p, n_w, n_r), dtype=torch.uint8,
                         device="cuda")
        U_ref = torch.empty((n_r, n_w), dtype=torch.complex128, device="cuda")
        U = torch.full((n_r, n_w), float("nan"), dtype=torch.complex128, device="cuda")
        assert _call("kr_bessel_sum", R, p, pw, dp, om, r, U_ref, ws) == 0
        assert _call("kr_bessel_sum_noalloc", R, p, pw, dp, om, r, U) == 0
        torch.cuda.synchronize()
        a, b = U.cpu().numpy(), U_ref.cpu().numpy()
        err = np.max(np.abs(a - b)) / np.max(np.abs(b))
        assert err < TOL, (call, err)


def test_noalloc_rejects_sizes_beyond_scratch():
    from seismicinversion_b200 import _lib

    h = _lib.lib()
    cap = h.kr_bessel_sum_noalloc_scratch_bytes() // 16
    n_p, n_w, n_r = 1, 1024, cap // 1024 + 1  # one slice needs more than the array holds
    # buffers sized for the claimed shapes, so nothing could be read out of bounds
    R, p, pw, om, r = _inputs(7, n_p, n_w, n_r)
    U = torch.empty((n_r, n_w), dtype=torch.complex128, device="cuda")
    st = _call("kr_bessel_sum_noalloc", R, p, pw, 1e-3, om, r, U)
    assert st == 6  # KR_ERR_TOO_LARGE
    assert b"static scratch" in h.kr_last_error()
