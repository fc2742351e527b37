"""si_normalize_signs_noalloc against si_normalize_signs, through the C ABI.

The no-allocation entry point serves callers that cannot let the library
allocate device memory (a process whose HBM is reserved by another allocator,
or a latency-bound loop on a shared device).  Its temporaries live in a static
device array shared by every call, so these tests run it twice in a row on
different shapes: what the first call leaves behind must not change the
second call's result.  Sign flips are exact, so results must be bit-identical,
with each other and with the CPU oracle's restatement of the crate's rule
(|x| ranked by f64::total_cmp, so a NaN maximum leaves its column unflipped).

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


def _oracle(x_host):
    from oracle import spectral_oracle as O
    y = np.array(x_host, dtype=np.float64, copy=True)
    O.normalize_signs(y)
    return y


def _bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return bool(np.all((a.view(np.uint64) == b.view(np.uint64)) | (np.isnan(a) & np.isnan(b))))


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
        assert _bits_equal(out.cpu().numpy(), _oracle(x.cpu().numpy())), f"call {call}: oracle"
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


def test_noalloc_nan_column_follows_total_cmp(gpu_ctx):
    """A NaN outranks every finite |x| in the crate's reduce, and signum(NaN)
    is not negative: the column keeps its signs although its largest finite
    entry is negative.  Both entry points, twice in a row, against the oracle."""
    import torch
    x = _block(torch, 3_000, 4, seed=21)
    x[50, 1] = -1.0e6        # largest finite entry of column 1, negative
    x[2_000, 1] = float("nan")
    x[10, 2] = -float("inf")  # -inf is column 2's maximum: flipped
    host = x.cpu().numpy()
    expect = _oracle(host)
    assert expect[50, 1] == -1.0e6 and expect[10, 2] == float("inf")
    for _ in range(2):
        ref, out = _run_both(gpu_ctx, torch, x)
        assert _bits_equal(ref.cpu().numpy(), expect)
        assert _bits_equal(out.cpu().numpy(), expect)


def test_noalloc_second_context_same_device(gpu_ctx):
    """A second library context on the same device shares the device's static
    array (same CUDA context); its calls agree with the first context's."""
    import torch
    from spectral_init_b200 import Context
    other = Context(0)
    x = _block(torch, 70_001, 5, seed=33)
    a = x.clone()
    b = x.clone()
    torch.cuda.synchronize()
    gpu_ctx.check(gpu_ctx.lib.si_normalize_signs_noalloc(gpu_ctx.ptr, a.data_ptr(), 70_001, 5))
    other.check(other.lib.si_normalize_signs_noalloc(other.ptr, b.data_ptr(), 70_001, 5))
    assert torch.equal(a, b)
    assert _bits_equal(a.cpu().numpy(), _oracle(x.cpu().numpy()))
