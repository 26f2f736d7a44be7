"""The allocation-free operator entry point against the regular one.

tcu_cluster_apply_noalloc serves callers that cannot allocate device memory: it takes
device pointers only and keeps its scratch in a fixed 8 MiB static device array. Two calls
in a row (different clusters, so the second overwrites the first one's scratch) must give
the same y = (I - T C) x as tcu_cluster_apply within 1e-13 relative, and oversized
clusters must be rejected. This file runs last so that a failure here leaves every other
test already run; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(torch, a, dtype):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _noalloc_apply(torch, w, x):
    import treams_b200 as t
    from treams_b200 import _lib

    r = _dev(torch, w.radii, torch.float64)
    e = torch.view_as_real(_dev(torch, w.eps, torch.complex128)).contiguous()
    pos = _dev(torch, w.positions, torch.float64)
    xd = _dev(torch, np.asfortranarray(x).ravel(order="F"), torch.complex128)
    yd = torch.zeros_like(xd)
    stream = torch.cuda.current_stream().cuda_stream
    st = _lib.lib().tcu_cluster_apply_noalloc(ctypes.c_void_p(stream), w.lmax, w.k0, w.radii.size, r.data_ptr(),
                                              e.data_ptr(), pos.data_ptr(), x.shape[1], xd.data_ptr(), yd.data_ptr())
    _lib._check(st)
    torch.cuda.synchronize()
    return yd.cpu().numpy().reshape(x.shape, order="F")


def test_noalloc_apply_matches_the_allocating_entry_point_twice():
    import torch
    import treams_b200 as t
    from treams_b200 import workloads

    rng = np.random.default_rng(11)
    for w in (workloads.precision_cluster(count=24), workloads.small_cluster()):
        x = rng.standard_normal((w.n, 3)) + 1j * rng.standard_normal((w.n, 3))
        y = _noalloc_apply(torch, w, x)
        ref = t.cluster_apply(w.lmax, w.k0, w.radii, w.eps, w.positions, x)
        assert np.linalg.norm(y - ref) <= 1e-13 * np.linalg.norm(ref)


def test_noalloc_rejects_clusters_beyond_its_scratch():
    import torch
    from treams_b200 import _lib, workloads

    w = workloads.small_cluster()
    n_big = 50000  # 50000 spheres * lmax 3 * 64 bytes > 8 MiB
    r = torch.full((n_big,), 0.1, dtype=torch.float64, device="cuda")
    e = torch.zeros((n_big, 2), dtype=torch.float64, device="cuda")
    pos = torch.zeros((n_big, 3), dtype=torch.float64, device="cuda")
    x = torch.zeros((n_big * 30,), dtype=torch.complex128, device="cuda")
    st = _lib.lib().tcu_cluster_apply_noalloc(None, 3, w.k0, n_big, r.data_ptr(), e.data_ptr(), pos.data_ptr(), 1,
                                              x.data_ptr(), x.data_ptr())
    assert st == 1
    assert "8 MiB" in _lib.lib().tcu_last_error_message().decode()
