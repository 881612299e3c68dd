"""Helpers shared by the GPU tests (device buffers come from torch)."""
import numpy as np


def have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / scale
