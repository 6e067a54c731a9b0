"""The allocation-free statistics entry point against the context one.

paddi_compute_statistics_noalloc is meant for callers that may not let the
library allocate device memory (hosts that own all device memory through
their own allocator, loops that cannot afford an allocation's device
synchronisation).  It must give the same statistics as
paddi_compute_statistics, call after call, while reusing its one fixed
scratch array.  This file is collected last on purpose.
"""
import numpy as np
import pytest

import paddi_b200 as P
from oracle import oracle as O
from paddi_b200 import datagen

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-6, 1e-7  # the statistics tolerance of tests/test_gpu_parity.py


def _stats_ctx(ctx, dT, n, m):
    import torch
    N = n - m + 1
    mean = torch.empty(N, dtype=torch.float32, device="cuda")
    std = torch.empty(N, dtype=torch.float32, device="cuda")
    ctx.compute_statistics(dT.data_ptr(), mean.data_ptr(), std.data_ptr(), n, m)
    torch.cuda.synchronize()
    return mean.cpu().numpy(), std.cpu().numpy()


def _stats_noalloc(dT, n, m):
    import torch
    N = n - m + 1
    mean = torch.full((N,), np.nan, dtype=torch.float32, device="cuda")
    std = torch.full((N,), np.nan, dtype=torch.float32, device="cuda")
    P.compute_statistics_noalloc(dT.data_ptr(), mean.data_ptr(), std.data_ptr(), n, m)
    torch.cuda.synchronize()
    return mean.cpu().numpy(), std.cpu().numpy()


def test_noalloc_statistics_match_the_context_entry_point_twice():
    import torch
    x, _ = datagen.palmad_series(n=P.NOALLOC_MAX_WINDOWS + 127, seed=4, n_anom=6,
                                 min_len=32, max_len=200)  # includes flat runs
    with P.Context(device=0) as ctx:
        # two calls in a row with different sizes share the same scratch
        for n, m in ((len(x), 128), (50_000, 37)):
            dT = torch.from_numpy(np.ascontiguousarray(x[:n])).cuda()
            want_mean, want_std = _stats_ctx(ctx, dT, n, m)
            got_mean, got_std = _stats_noalloc(dT, n, m)
            np.testing.assert_allclose(got_mean, want_mean, rtol=RTOL, atol=ATOL)
            np.testing.assert_allclose(got_std, want_std, rtol=RTOL, atol=ATOL)
            # and independently of the CUDA kernels: the FP64 oracle's statistics
            mu, sd, _ = O.window_stats(x[:n], m)
            np.testing.assert_allclose(got_mean, mu, rtol=RTOL, atol=ATOL)
            np.testing.assert_allclose(got_std, sd, rtol=2e-6, atol=ATOL)


def test_noalloc_statistics_refuse_inputs_beyond_the_limit():
    import torch
    m = 64
    n = P.NOALLOC_MAX_WINDOWS + m  # one window too many
    dT = torch.zeros(n, dtype=torch.float32, device="cuda")
    out = torch.zeros(n, dtype=torch.float32, device="cuda")
    with pytest.raises(P.PaddiError) as e:
        P.compute_statistics_noalloc(dT.data_ptr(), out.data_ptr(), out.data_ptr(), n, m)
    assert e.value.status == P.PADDI_ERR_INVALID_ARG
    assert "limit" in str(e.value)
