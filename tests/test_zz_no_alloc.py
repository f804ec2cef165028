"""wap_multislice_fwd_noalloc: the forward for callers that cannot allocate
device memory while they run (graph capture under a framework that forbids
allocation, fixed-pool hosts, plugin hosts that only hand over buffers).

Collected last on purpose.  Calls the entry point through the C ABI twice in
a row (the second call reuses the library's fixed scratch array and takes no
device memory) and records it into a CUDA graph, checking every result against
wap_multislice_fwd (the regular entry point) within the parity tolerance of
the other GPU tests.  Runs alone in a fresh process or after the rest of the
suite.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-5


def rel(a, b):
    a = a.to(torch.complex128) if a.is_complex() else a.double()
    b = b.to(torch.complex128) if b.is_complex() else b.double()
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


@pytest.mark.parametrize("ny,nx,B", [(256, 256, 3), (128, 512, 2)])
def test_noalloc_matches_regular_entry_point(ny, nx, B):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wideanglepropagation_b200 import _lib
    from wideanglepropagation_b200.propagation import get_plan, split_transfer
    L = _lib.lib()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(ny + nx)
    N, dz, E = 5, 2.0, 300e3
    V = torch.as_tensor(rng.uniform(0, 40, (N, ny, nx)).astype(np.float32), device=dev)
    probe = torch.as_tensor((rng.normal(size=(ny, nx)) + 1j * rng.normal(size=(ny, nx))).astype(np.complex64),
                            device=dev)
    pos = torch.as_tensor(np.stack([rng.integers(0, ny, B), rng.integers(0, nx, B)], 1).astype(np.int32), device=dev)
    H128 = torch.exp(1j * torch.as_tensor(rng.uniform(-3, 3, (ny, nx)), device=dev))
    H, H_lo = split_transfer(H128, dev)
    p = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    # regular entry point (plan-based)
    plan = get_plan(ny, nx, B, _lib.WAP_OP_FRESNEL_AS)
    ref_exit = torch.empty((B, ny, nx), dtype=torch.complex64, device=dev)
    ref_dp = torch.empty((B, ny, nx), dtype=torch.float32, device=dev)
    ref_stack = torch.empty((B, N, ny, nx), dtype=torch.complex64, device=dev)
    _lib.check(L.wap_multislice_fwd(plan.handle, p(V), N, 1, None, p(probe), B, 0, p(pos), p(H), p(H_lo), dz, E,
                                    p(ref_exit), p(ref_dp), p(ref_stack), stream))

    for call in range(2):
        ex = torch.full((B, ny, nx), float("nan"), dtype=torch.complex64, device=dev)
        dp = torch.full((B, ny, nx), float("nan"), dtype=torch.float32, device=dev)
        st = torch.full((B, N, ny, nx), float("nan"), dtype=torch.complex64, device=dev)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info(dev)[0]
        _lib.check(L.wap_multislice_fwd_noalloc(p(V), N, ny, nx, p(probe), B, 0, p(pos), p(H), p(H_lo), dz, E,
                                                p(ex), p(dp), p(st), stream))
        torch.cuda.synchronize()
        if call == 1:
            # the second call takes no device memory at all (the first may load
            # the kernels' code, which the driver does on first use)
            assert torch.cuda.mem_get_info(dev)[0] == free0
        assert rel(ex, ref_exit) < TOL, call
        assert rel(dp, ref_dp) < TOL, call
        assert rel(st, ref_stack) < TOL, call


def test_noalloc_captures_in_cuda_graph():
    """The documented use: the call recorded into a CUDA graph in global
    capture mode (which fails any allocation or synchronising call made while
    capturing), then replayed twice with new inputs copied into the captured
    buffers; each replay matches the regular entry point."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wideanglepropagation_b200 import _lib
    from wideanglepropagation_b200.propagation import get_plan, split_transfer
    L = _lib.lib()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    ny = nx = 256
    B, N, dz, E = 2, 4, 2.0, 200e3
    rng = np.random.default_rng(7)
    p = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None
    H128 = torch.exp(1j * torch.as_tensor(rng.uniform(-3, 3, (ny, nx)), device=dev))
    H, H_lo = split_transfer(H128, dev)
    pos = torch.as_tensor(np.array([[5, 200], [128, 17]], np.int32), device=dev)
    V = torch.empty((N, ny, nx), dtype=torch.float32, device=dev)
    probe = torch.empty((ny, nx), dtype=torch.complex64, device=dev)
    ex = torch.empty((B, ny, nx), dtype=torch.complex64, device=dev)
    dp = torch.empty((B, ny, nx), dtype=torch.float32, device=dev)

    def inputs(seed):
        r = np.random.default_rng(seed)
        V.copy_(torch.as_tensor(r.uniform(0, 40, (N, ny, nx)).astype(np.float32)))
        probe.copy_(torch.as_tensor((r.normal(size=(ny, nx)) + 1j * r.normal(size=(ny, nx))).astype(np.complex64)))

    def reference():
        plan = get_plan(ny, nx, B, _lib.WAP_OP_FRESNEL_AS)
        rex = torch.empty_like(ex)
        rdp = torch.empty_like(dp)
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        _lib.check(L.wap_multislice_fwd(plan.handle, p(V), N, 1, None, p(probe), B, 0, p(pos), p(H), p(H_lo), dz, E,
                                        p(rex), p(dp), None, st))
        torch.cuda.synchronize()
        return rex, dp.clone()

    side = torch.cuda.Stream()
    inputs(1)
    with torch.cuda.stream(side):   # warm-up outside the capture (first use loads the kernels)
        _lib.check(L.wap_multislice_fwd_noalloc(p(V), N, ny, nx, p(probe), B, 0, p(pos), p(H), p(H_lo), dz, E,
                                                p(ex), p(dp), None, ctypes.c_void_p(side.cuda_stream)))
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=side, capture_error_mode="global"):
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        _lib.check(L.wap_multislice_fwd_noalloc(p(V), N, ny, nx, p(probe), B, 0, p(pos), p(H), p(H_lo), dz, E,
                                                p(ex), p(dp), None, st))
    for seed in (2, 3):
        inputs(seed)
        rex, rdp = reference()
        ex.fill_(float("nan"))
        dp.fill_(float("nan"))
        g.replay()
        torch.cuda.synchronize()
        assert rel(ex, rex) < TOL, seed
        assert rel(dp, rdp) < TOL, seed
    del g


def test_noalloc_rejects_bad_sizes():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from wideanglepropagation_b200 import _lib
    L = _lib.lib()
    d = torch.zeros(4, device="cuda")
    ptr = ctypes.c_void_p(d.data_ptr())
    rc = L.wap_multislice_fwd_noalloc(ptr, 1, 100, 128, ptr, 1, 0, None, ptr, None, 1.0, 2e5, ptr, None, None, None)
    assert rc == _lib.WAP_ERR_UNSUPPORTED
    assert b"unsupported grid" in L.wap_last_error()
