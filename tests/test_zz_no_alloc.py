"""gs_dot_noalloc: the dot product for callers that cannot allocate device
memory when they need it (a code that gives all GPU memory to its own pool
at start-up, or a loop that cannot take cudaMalloc's implicit device
synchronisation). Its scratch lives in a fixed array inside the library.

Checked through the C ABI against gs_dot, the entry point that keeps its
scratch in memory the library allocates, on two calls in a row (the second
call finds the array holding the first call's contents); that a run of calls
leaves the device's free memory unchanged; and the empty vector. This file is
collected last on purpose; it passes alone in a fresh process and after the
other tests.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_N = 8_388_608


@pytest.mark.parametrize("dtype_name", ["float64", "float32"])
def test_dot_noalloc_matches_dot_twice(gs, device, dtype_name):
    import torch
    kind = gs.F64 if dtype_name == "float64" else gs.F32
    tol = 1e-12 if kind == gs.F64 else 1e-5  # the dot tolerances of the other tests
    dt = getattr(torch, dtype_name)
    rng = np.random.default_rng(7)
    for n in (1_000_003, MAX_N):  # two calls in a row, different sizes
        x = torch.tensor(rng.uniform(-1, 1, n), dtype=dt, device="cuda")
        y = torch.tensor(rng.uniform(-1, 1, n), dtype=dt, device="cuda")
        ref = torch.zeros(1, dtype=dt, device="cuda")
        got = torch.full((1,), float("nan"), dtype=dt, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        gs.dot(n, x.data_ptr(), y.data_ptr(), ref.data_ptr(), kind, stream)
        gs.dot_noalloc(n, x.data_ptr(), y.data_ptr(), got.data_ptr(), kind, stream)
        torch.cuda.synchronize()
        r, g = ref.item(), got.item()
        assert abs(g - r) <= tol * max(1.0, abs(r)), (n, g, r)


def test_dot_noalloc_leaves_free_memory_unchanged(gs, device):
    """After one warm-up call (which loads the library's device image on this
    device), a run of calls with no other library call in between changes
    the device's free memory by nothing, and every result is right."""
    import torch
    rng = np.random.default_rng(11)
    sizes = (3, 2049, 777_777, MAX_N)
    xs = [torch.tensor(rng.uniform(-1, 1, n), dtype=torch.float64, device="cuda") for n in sizes]
    ys = [torch.tensor(rng.uniform(-1, 1, n), dtype=torch.float64, device="cuda") for n in sizes]
    want = [float(np.dot(x.cpu().numpy(), y.cpu().numpy())) for x, y in zip(xs, ys)]
    out = torch.full((len(sizes),), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    gs.dot_noalloc(sizes[0], xs[0].data_ptr(), ys[0].data_ptr(), out.data_ptr(), gs.F64, stream)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        for i, n in enumerate(sizes):
            gs.dot_noalloc(n, xs[i].data_ptr(), ys[i].data_ptr(), out.data_ptr() + 8 * i, gs.F64, stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    got = out.cpu().numpy()
    for g, w in zip(got, want):
        assert abs(g - w) <= 1e-12 * max(1.0, abs(w)), (g, w)


def test_dot_noalloc_empty_vector_is_zero(gs, device):
    import torch
    x = torch.ones(4, dtype=torch.float64, device="cuda")
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    gs.dot_noalloc(0, x.data_ptr(), x.data_ptr(), out.data_ptr(), gs.F64)
    torch.cuda.synchronize()
    assert out.item() == 0.0


def test_dot_noalloc_rejects_oversize(gs, device):
    import torch
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    # the host check refuses before any launch, nothing is read
    with pytest.raises(gs.SolverError, match="exceeds the maximum"):
        gs.dot_noalloc(MAX_N + 1, x.data_ptr(), x.data_ptr(), out.data_ptr(), gs.F64)
