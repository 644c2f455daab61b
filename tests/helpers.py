"""Shared helpers for the tests (numpy <-> torch, error measures)."""
import numpy as np


def to_dev(a, device='cuda'):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(device)


def to_np(t):
    return t.detach().cpu().numpy()


def max_rel(a, b):
    """max |a - b| / max |b| (0 when both are zero)."""
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.abs(b).max() if b.size else 0.0
    num = np.abs(a - b).max() if b.size else 0.0
    return 0.0 if num == 0.0 else num / (den or 1.0)


# Parity bar for FP64 stencil and transformer outputs against the oracle:
# 1e-12 relative (max-norm).  The kernels keep the reference's operation
# order and avoid FMA contraction, so in practice the difference is 0.
RTOL_FP64 = 1e-12
