"""Helpers shared by the tests: layout conversion and error norms."""
from __future__ import annotations

import numpy as np


def rel_l2(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    d = np.linalg.norm((a - b).ravel())
    n = np.linalg.norm(b.ravel())
    return float(d / n) if n > 0 else float(d)


def rel_max(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    m = np.abs(b).max()
    return float(np.abs(a - b).max() / m) if m > 0 else float(np.abs(a - b).max())


def to_dev(torch, a: np.ndarray, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def to_host(t) -> np.ndarray:
    return t.detach().cpu().numpy()


def phys_to_buffer(u: np.ndarray, dtype=np.complex128) -> np.ndarray:
    """Physical real field [nx, ny, nz] -> padded buffer viewed as complex [ny, nx, nz2] storage."""
    nx, ny, nz = u.shape
    nz2 = nz // 2 + 1
    rdt = np.float64 if dtype == np.complex128 else np.float32
    buf = np.zeros((ny, nx, nz2), dtype=dtype)
    buf.view(rdt).reshape(nx, ny, 2 * nz2)[:, :, :nz] = u
    return buf


def buffer_to_phys(buf: np.ndarray, shape) -> np.ndarray:
    nx, ny, nz = shape
    nz2 = nz // 2 + 1
    rdt = np.float64 if buf.dtype == np.complex128 else np.float32
    return buf.view(rdt).reshape(nx, ny, 2 * nz2)[:, :, :nz].copy()
