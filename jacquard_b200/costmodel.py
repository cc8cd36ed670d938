"""Learned partition cost model.

A 24 -> 128 -> 128 -> 1 ReLU MLP predicting log(kernel SM cycles) of a
partition work item from its features (jacquard_b200/csrc/frontend/costmodel.cpp
`partition_features`).  Training data are timings the batched interpreter
measures itself (per-partition clock spans, `part_cycles`); training and
inference run on the GPU through the hand-written BF16/FP32 kernels of
csrc/costmodel.cu (jq_mlp_* in the C ABI).  The trained model is handed to the
front end, whose partitioner then accepts a merge of two partitions when the
predicted time of the merged one is below the sum of the two.
"""
import ctypes
import math

import numpy as np
import torch

from ._native import load
from .frontend import COST_MODEL_FLOATS, NFEAT

H = 128
NP = H * NFEAT + H + H * H + H + H + 1
OW1, OB1 = 0, H * NFEAT
OW2 = OB1 + H
OB2 = OW2 + H * H
OW3 = OB2 + H
OB3 = OW3 + H
vp = ctypes.c_void_p


class StepArgs(ctypes.Structure):
    _fields_ = [("theta", vp), ("theta16", vp), ("adam_m", vp), ("adam_v", vp), ("X", vp),
                ("T", vp), ("batch_index", vp), ("batch", ctypes.c_uint32),
                ("step", ctypes.c_uint32), ("lr", ctypes.c_float), ("apply", ctypes.c_int32),
                ("grad_out", vp), ("loss_out", vp), ("scratch", vp),
                ("scratch_ctas", ctypes.c_uint32), ("stream", vp)]


def lib():
    L = load("libjacquard_b200.so")
    if not getattr(L, "_jq_mlp_typed", False):
        L.jq_mlp_sync_bf16.restype = ctypes.c_int
        L.jq_mlp_sync_bf16.argtypes = [vp, vp, vp]
        L.jq_mlp_forward.restype = ctypes.c_int
        L.jq_mlp_forward.argtypes = [vp, vp, vp, ctypes.c_size_t, vp, vp]
        L.jq_mlp_scratch_floats.restype = ctypes.c_size_t
        L.jq_mlp_scratch_floats.argtypes = [ctypes.c_uint32]
        L.jq_mlp_train_step.restype = ctypes.c_int
        L.jq_mlp_train_step.argtypes = [ctypes.POINTER(StepArgs)]
        L._jq_mlp_typed = True
    return L


def _check(rc, what):
    if rc:
        raise RuntimeError(f"{what} failed ({rc})")


def init_theta(seed=5):
    """He-uniform weights, zero biases (fp32)."""
    rng = np.random.default_rng(seed)
    th = np.zeros(NP, np.float32)
    th[OW1:OB1] = rng.uniform(-1, 1, H * NFEAT) * math.sqrt(6.0 / NFEAT)
    th[OW2:OB2] = rng.uniform(-1, 1, H * H) * math.sqrt(6.0 / H)
    th[OW3:OB3] = rng.uniform(-1, 1, H) * math.sqrt(6.0 / H)
    return th


def bf16_bits(a):
    """float32 array -> bf16 bit patterns (round to nearest even), as int16."""
    t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(torch.bfloat16)
    return t.view(torch.int16)


class CostModel:
    def __init__(self, device="cuda", seed=5, scratch_ctas=32):
        self.device = torch.device(device)
        self.theta = torch.from_numpy(init_theta(seed)).to(self.device)
        self.theta16 = torch.empty(NP, dtype=torch.int16, device=self.device)
        self.m = torch.zeros(NP, dtype=torch.float32, device=self.device)
        self.v = torch.zeros_like(self.m)
        self.ctas = scratch_ctas
        self.scratch = torch.empty(lib().jq_mlp_scratch_floats(scratch_ctas), dtype=torch.float32,
                                   device=self.device)
        self.mean = np.zeros(NFEAT, np.float32)
        self.inv_std = np.ones(NFEAT, np.float32)
        self.step_count = 0
        self._sync()

    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def _sync(self):
        _check(lib().jq_mlp_sync_bf16(self.theta.data_ptr(), self.theta16.data_ptr(), self._stream()),
               "jq_mlp_sync_bf16")

    def set_theta(self, theta):
        self.theta.copy_(torch.from_numpy(np.ascontiguousarray(theta, np.float32)))
        self._sync()

    def normalise(self, feats):
        return (np.asarray(feats, np.float32) - self.mean) * self.inv_std

    def features_to_device(self, feats):
        return bf16_bits(self.normalise(feats)).to(self.device)

    def grad(self, Xd, Td, idx):
        """Summed gradient and loss of one batch (no update)."""
        g = torch.empty(NP, dtype=torch.float32, device=self.device)
        loss = torch.empty(1, dtype=torch.float32, device=self.device)
        a = StepArgs(self.theta.data_ptr(), self.theta16.data_ptr(), None, None, Xd.data_ptr(),
                     Td.data_ptr(), idx.data_ptr(), idx.numel(), 0, 0.0, 0, g.data_ptr(),
                     loss.data_ptr(), self.scratch.data_ptr(), self.ctas, self._stream())
        _check(lib().jq_mlp_train_step(ctypes.byref(a)), "jq_mlp_train_step")
        return g, loss

    def fit(self, feats, targets, steps=2000, batch=512, lr=1e-3, seed=0):
        """Adam on mean squared error of log-time.  Returns the loss history."""
        f = np.asarray(feats, np.float32)
        self.mean = f.mean(axis=0)
        sd = f.std(axis=0)
        self.inv_std = np.where(sd > 1e-6, 1.0 / np.maximum(sd, 1e-6), 0.0).astype(np.float32)
        Xd = self.features_to_device(f)
        Td = torch.from_numpy(np.asarray(targets, np.float32)).to(self.device)
        rng = np.random.default_rng(seed)
        loss = torch.empty(1, dtype=torch.float32, device=self.device)
        hist = []
        n = f.shape[0]
        for it in range(steps):
            idx = torch.from_numpy(rng.integers(0, n, size=batch).astype(np.int32)).to(self.device)
            self.step_count += 1
            a = StepArgs(self.theta.data_ptr(), self.theta16.data_ptr(), self.m.data_ptr(),
                         self.v.data_ptr(), Xd.data_ptr(), Td.data_ptr(), idx.data_ptr(), batch,
                         self.step_count, lr, 1, None, loss.data_ptr(), self.scratch.data_ptr(),
                         self.ctas, self._stream())
            _check(lib().jq_mlp_train_step(ctypes.byref(a)), "jq_mlp_train_step")
            if it % 100 == 0 or it == steps - 1:
                hist.append((it, float(loss.item())))
        return hist

    def predict(self, feats):
        Xd = self.features_to_device(feats)
        y = torch.empty(Xd.shape[0], dtype=torch.float32, device=self.device)
        _check(lib().jq_mlp_forward(self.theta.data_ptr(), self.theta16.data_ptr(), Xd.data_ptr(),
                                    Xd.shape[0], y.data_ptr(), self._stream()), "jq_mlp_forward")
        return y.cpu().numpy()

    def pack(self):
        """Flat model for the front end: weights, then feature mean and 1/std."""
        th = self.theta.cpu().numpy()
        out = np.concatenate([th, self.mean, self.inv_std]).astype(np.float32)
        assert out.size == COST_MODEL_FLOATS
        return out

    def save(self, path):
        np.savez(path, theta=self.theta.cpu().numpy(), mean=self.mean, inv_std=self.inv_std)

    @classmethod
    def load(cls, path, device="cuda"):
        z = np.load(path)
        m = cls(device)
        m.set_theta(z["theta"])
        m.mean, m.inv_std = z["mean"], z["inv_std"]
        return m


def packed_from_file(path):
    """Flat front-end model from a saved .npz (no GPU needed)."""
    z = np.load(path)
    return np.concatenate([z["theta"], z["mean"], z["inv_std"]]).astype(np.float32)
