"""Helpers of the GPU tests: column-major torch CUDA tensors from numpy."""
import numpy as np


def dev(a: np.ndarray, ld: int | None = None):
    """Column-major CUDA copy of a 2-D array (optionally padded to `ld` rows)."""
    import torch
    a = np.asarray(a, dtype=np.float64)
    rows, cols = a.shape
    ld = ld or max(rows, 1)
    t = torch.zeros((cols, ld), dtype=torch.float64, device="cuda").T  # (ld, cols), stride (1, ld)
    t[:rows] = torch.from_numpy(np.ascontiguousarray(a))
    return t[:rows]


def host(t) -> np.ndarray:
    return np.asfortranarray(t.detach().cpu().numpy())


def ivec(n: int):
    import torch
    return torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")


def relerr(x, ref) -> float:
    x = np.asarray(x)
    ref = np.asarray(ref)
    return float(np.linalg.norm(x - ref) / max(np.linalg.norm(ref), 1e-300))
