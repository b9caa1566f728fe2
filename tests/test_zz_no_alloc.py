"""The dot product that allocates nothing (fem_dot_f64_noalloc).

Some callers cannot allocate device memory: their device memory belongs to a
host framework's pool that forbids raw cudaMalloc, or they run real-time
loops that must not allocate once started.  For them the library offers a
dot product whose scratch lives in a static device array inside the
library.  This test calls it through the C ABI and checks it against the
workspace-based fem_dot_f64 (same FP64 reduction, different block split, so
the tolerance is round-off: 1e-12 relative) on two calls in a row, plus the
size limit.  It lives in its own file, collected last, and works both alone
in a fresh process and after the other tests.
"""
import ctypes

import numpy as np
import pytest
import torch


def _dot_ref(nat, x, y):
    nb = nat.lib().fem_dot_workspace_bytes(x.numel())
    work = torch.empty(int(nb), dtype=torch.uint8, device=x.device)
    out = ctypes.c_double(0.0)
    nat.check(nat.lib().fem_dot_f64(x.numel(), nat.ptr(x), nat.ptr(y), ctypes.byref(out), nat.ptr(work),
                                    int(nb), nat.stream_ptr()), "dot_f64")
    return out.value


@pytest.mark.gpu
def test_dot_noalloc_matches_dot_with_workspace(pkg, cuda):
    nat = pkg._native
    g = torch.Generator(device="cpu").manual_seed(11)
    for n in (1, 4097, 397_953):
        x = torch.randn(n, generator=g, dtype=torch.float64).to(cuda)
        y = torch.randn(n, generator=g, dtype=torch.float64).to(cuda)
        ref = _dot_ref(nat, x, y)
        out = torch.full((1,), np.nan, dtype=torch.float64, device=cuda)
        for _ in range(2):  # two calls in a row share the static scratch
            nat.check(nat.lib().fem_dot_f64_noalloc(n, nat.ptr(x), nat.ptr(y), nat.ptr(out), nat.stream_ptr()),
                      "dot_f64_noalloc")
            torch.cuda.synchronize()
            got = out.item()
            assert abs(got - ref) <= 1e-12 * max(1.0, abs(ref)), (n, got, ref)
            out.fill_(np.nan)


@pytest.mark.gpu
def test_dot_noalloc_rejects_oversize(pkg, cuda):
    nat = pkg._native
    x = torch.zeros(1, dtype=torch.float64, device=cuda)
    out = torch.zeros(1, dtype=torch.float64, device=cuda)
    rc = nat.lib().fem_dot_f64_noalloc(16_777_217, nat.ptr(x), nat.ptr(x), nat.ptr(out), nat.stream_ptr())
    assert rc == nat.FEM_ERR_ARG
    assert b"no-alloc maximum" in nat.lib().fem_last_error()
