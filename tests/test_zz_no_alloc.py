"""si_normalize_signs_noalloc against si_normalize_signs, through the C ABI.

The no-allocation entry point serves callers that cannot let the library
allocate device memory (a process whose HBM is reserved by another allocator,
or a latency-bound loop on a shared device).  Its temporaries live in a static
device array shared by every call, so these tests run it twice in a row on
different shapes: what the first call leaves behind must not change the
second call's result.  Sign flips are exact, so results must be bit-identical.

This file is collected last on purpose: it must pass alone in a fresh process
and after every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _block(torch, n, k, seed):
    g = torch.Generator(device="cuda:0")
    g.manual_seed(seed)
    x = torch.randn(n, k, dtype=torch.float64, device="cuda:0", generator=g)
    # ties between +a and -a in one column: the first row of largest |x| decides
    if n > 40:
        x[7, 0] = -9.0
        x[31, 0] = 9.0
        x[5, k - 1] = -0.0
    return x


def _run_both(ctx, torch, x):
    n, k = x.shape
    ref = x.clone()
    out = x.clone()
    torch.cuda.synchronize()
    ctx.check(ctx.lib.si_normalize_signs(ctx.ptr, ref.data_ptr(), n, k))
    ctx.check(ctx.lib.si_normalize_signs_noalloc(ctx.ptr, out.data_ptr(), n, k))
    return ref, out


def test_noalloc_matches_allocating_entry_twice(gpu_ctx):
    import torch
    shapes = [(200_003, 16), (1_000, 3), (4_096, 64), (1, 1)]
    for call, (n, k) in enumerate(shapes):
        x = _block(torch, n, k, seed=11 + call)
        ref, out = _run_both(gpu_ctx, torch, x)
        assert torch.equal(ref, out), f"call {call}: n={n} k={k}"
        # the first entry of largest |x| in column 0 ends up positive
        col0 = x[:, 0].abs()
        first = int(torch.nonzero(col0 == col0.max())[0])
        assert float(out[first, 0]) > 0.0


def test_noalloc_tie_takes_first_row(gpu_ctx):
    import torch
    x = torch.zeros(1_000, 2, dtype=torch.float64, device="cuda:0")
    x[100, 0] = -3.0
    x[900, 0] = 3.0
    x[10, 1] = 2.0
    x[20, 1] = -2.0
    for _ in range(2):
        ref, out = _run_both(gpu_ctx, torch, x)
        assert torch.equal(ref, out)
        assert float(out[100, 0]) == 3.0 and float(out[900, 0]) == -3.0
        assert float(out[10, 1]) == 2.0 and float(out[20, 1]) == -2.0


def test_noalloc_rejects_columns_beyond_scratch(gpu_ctx):
    import torch
    from spectral_init_b200.api import InvalidArgument
    x = torch.ones(10, 65, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    st = gpu_ctx.lib.si_normalize_signs_noalloc(gpu_ctx.ptr, x.data_ptr(), 10, 65)
    assert st != 0
    msg = gpu_ctx.lib.si_last_error(gpu_ctx.ptr).decode()
    assert "64" in msg and "65" in msg
    with pytest.raises(InvalidArgument):
        gpu_ctx.check(st)
    # empty input is a no-op, as for the allocating entry point
    gpu_ctx.check(gpu_ctx.lib.si_normalize_signs_noalloc(gpu_ctx.ptr, None, 0, 4))
    # a valid call still works after the rejection
    y = _block(torch, 5_000, 8, seed=5)
    ref, out = _run_both(gpu_ctx, torch, y)
    assert torch.equal(ref, out)
    assert np.all(np.isfinite(out.cpu().numpy()))
