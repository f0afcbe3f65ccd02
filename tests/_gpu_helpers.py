import numpy as np
import torch


def T(x, dev, dtype=torch.float64, grad=False):
    t = torch.tensor(np.asarray(x), dtype=dtype, device=dev)
    if grad:
        t.requires_grad_(True)
    return t


def rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    b = b.detach().cpu().numpy() if isinstance(b, torch.Tensor) else np.asarray(b)
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
