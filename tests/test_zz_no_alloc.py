"""The no-allocation training step (jq_mlp_train_step_noalloc) against the
regular one (jq_mlp_train_step), called through the C ABI.

The no-allocation entry point is for hosts that cannot allocate device memory
once running -- an embedding host with one device pool sized at start-up, or
one whose latency limits rule out an allocation that may synchronize the
device -- so its gradient workspace is a built-in device array instead of a
caller buffer.  Kept in its own file, collected last."""
import ctypes
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NP = 128 * 24 + 128 + 128 * 128 + 128 + 128 + 1
vp = ctypes.c_void_p


class StepArgs(ctypes.Structure):
    _fields_ = [("theta", vp), ("theta16", vp), ("adam_m", vp), ("adam_v", vp), ("X", vp),
                ("T", vp), ("batch_index", vp), ("batch", ctypes.c_uint32),
                ("step", ctypes.c_uint32), ("lr", ctypes.c_float), ("apply", ctypes.c_int32),
                ("grad_out", vp), ("loss_out", vp), ("scratch", vp),
                ("scratch_ctas", ctypes.c_uint32), ("stream", vp)]


def lib():
    L = ctypes.CDLL(os.path.join(REPO, "jacquard_b200", "libjacquard_b200.so"))
    for f in ("jq_mlp_train_step", "jq_mlp_train_step_noalloc"):
        getattr(L, f).restype = ctypes.c_int
        getattr(L, f).argtypes = [ctypes.POINTER(StepArgs)]
    L.jq_mlp_sync_bf16.restype = ctypes.c_int
    L.jq_mlp_sync_bf16.argtypes = [vp, vp, vp]
    L.jq_mlp_scratch_floats.restype = ctypes.c_size_t
    L.jq_mlp_scratch_floats.argtypes = [ctypes.c_uint32]
    return L


def close(a, b):
    a, b = a.cpu().numpy(), b.cpu().numpy()
    scale = max(1e-12, float(np.abs(b).max()))
    return float(np.abs(a - b).max()) <= 2e-3 * scale


def test_noalloc_step_matches_regular_step_twice():
    L = lib()
    dev = torch.device("cuda")
    rng = np.random.default_rng(7)
    n, batch, ctas = 900, 512, 12
    X = torch.from_numpy(rng.normal(size=(n, 24)).astype(np.float32)).to(torch.bfloat16).view(torch.int16).to(dev)
    T = torch.from_numpy(rng.normal(size=n).astype(np.float32)).to(dev)
    theta0 = torch.from_numpy((rng.uniform(-1, 1, NP) * 0.2).astype(np.float32)).to(dev)
    st = torch.cuda.current_stream().cuda_stream

    def state():
        th = theta0.clone()
        th16 = torch.empty(NP, dtype=torch.int16, device=dev)
        assert L.jq_mlp_sync_bf16(th.data_ptr(), th16.data_ptr(), st) == 0
        return th, th16, torch.zeros(NP, device=dev), torch.zeros(NP, device=dev)

    regular, noalloc = state(), state()
    scratch = torch.empty(L.jq_mlp_scratch_floats(ctas), dtype=torch.float32, device=dev)
    for step in (1, 2):  # two calls in a row on each entry point
        idx = torch.from_numpy(rng.integers(0, n, size=batch).astype(np.int32)).to(dev)
        outs = []
        for (th, th16, m, v), fn, scr in ((regular, L.jq_mlp_train_step, scratch),
                                          (noalloc, L.jq_mlp_train_step_noalloc, None)):
            g = torch.empty(NP, device=dev)
            loss = torch.empty(1, device=dev)
            a = StepArgs(th.data_ptr(), th16.data_ptr(), m.data_ptr(), v.data_ptr(), X.data_ptr(),
                         T.data_ptr(), idx.data_ptr(), batch, step, 1e-3, 1, g.data_ptr(),
                         loss.data_ptr(), scr.data_ptr() if scr is not None else None, ctas, st)
            assert fn(ctypes.byref(a)) == 0
            outs.append((g, loss))
        torch.cuda.synchronize()
        (g_r, l_r), (g_n, l_n) = outs
        assert close(g_n, g_r)
        assert abs(float(l_n) - float(l_r)) <= 1e-4 * max(1.0, abs(float(l_r)))
        assert close(noalloc[0], regular[0])  # updated parameters
        assert close(noalloc[2], regular[2]) and close(noalloc[3], regular[3])


def test_noalloc_limit_and_no_device_allocation():
    """16 CTAs (the built-in array's capacity) run and match the regular step
    with free device memory unchanged across the call; 17 are refused with
    JQ_ERR_NOALLOC_LIMIT and a NULL argument block with JQ_ERR_INVALID_ARG."""
    L = lib()
    dev = torch.device("cuda")
    rng = np.random.default_rng(11)
    n, batch, ctas = 700, 384, 16
    X = torch.from_numpy(rng.normal(size=(n, 24)).astype(np.float32)).to(torch.bfloat16).view(torch.int16).to(dev)
    T = torch.from_numpy(rng.normal(size=n).astype(np.float32)).to(dev)
    theta = torch.from_numpy((rng.uniform(-1, 1, NP) * 0.2).astype(np.float32)).to(dev)
    th16 = torch.empty(NP, dtype=torch.int16, device=dev)
    st = torch.cuda.current_stream().cuda_stream
    assert L.jq_mlp_sync_bf16(theta.data_ptr(), th16.data_ptr(), st) == 0
    idx = torch.from_numpy(rng.integers(0, n, size=batch).astype(np.int32)).to(dev)
    scratch = torch.empty(L.jq_mlp_scratch_floats(ctas), dtype=torch.float32, device=dev)
    g_r, g_n = torch.empty(NP, device=dev), torch.empty(NP, device=dev)
    l_r, l_n = torch.empty(1, device=dev), torch.empty(1, device=dev)

    def args(g, loss, scr, k):  # gradient only: theta stays as it is
        return StepArgs(theta.data_ptr(), th16.data_ptr(), None, None, X.data_ptr(), T.data_ptr(),
                        idx.data_ptr(), batch, 1, 1e-3, 0, g.data_ptr(), loss.data_ptr(),
                        scr.data_ptr() if scr is not None else None, k, st)

    assert L.jq_mlp_train_step(ctypes.byref(args(g_r, l_r, scratch, ctas))) == 0
    assert L.jq_mlp_train_step_noalloc(ctypes.byref(args(g_n, l_n, None, ctas))) == 0  # loads, resolves
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    alloc0 = torch.cuda.memory_allocated()
    g_n.zero_()
    torch.cuda.synchronize()
    assert L.jq_mlp_train_step_noalloc(ctypes.byref(args(g_n, l_n, None, ctas))) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert torch.cuda.memory_allocated() == alloc0
    assert close(g_n, g_r)
    assert abs(float(l_n) - float(l_r)) <= 1e-4 * max(1.0, abs(float(l_r)))
    assert L.jq_mlp_train_step_noalloc(ctypes.byref(args(g_n, l_n, None, 17))) == -6
    assert L.jq_mlp_train_step_noalloc(None) == -1
