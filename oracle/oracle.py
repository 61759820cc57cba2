"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU
baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import
this module; the product path never does.

Array conventions match the reference's buffers:
  physical  padded  float64[nx, ny, 2*nz2]   (cudafuncs.cu:14-17)
  spectral  complex128[ny, nx, nz2]          (transposed; solver.cu:25)
Both views share one buffer of nx*ny*nz2 complex values.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "_build" / "liboracle.so"


class OrcCfg(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("re", ctypes.c_double), ("sc", ctypes.c_double), ("sc_c", ctypes.c_double),
        ("alpha", ctypes.c_double), ("dt", ctypes.c_double),
        ("alias_filter", ctypes.c_double), ("nu_stats", ctypes.c_double),
        ("nthreads", ctypes.c_int),
    ]


def build() -> Path:
    """Compile the oracle library (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(_LIB_PATH))
        P = ctypes.POINTER(ctypes.c_double)
        PP = ctypes.POINTER(P)
        C = ctypes.POINTER(OrcCfg)
        for name, args in [
            ("orc_forward", [C, P]), ("orc_inverse", [C, P]), ("orc_dealias", [C, P]),
            ("orc_vorticity", [C, P, P, P, P, P, P]), ("orc_gradient", [C, P, P, P, P]),
            ("orc_make_rhs", [C, P, P, P, P, P]),
            ("orc_step_cnab2", [C, PP, PP, ctypes.c_int]),
            ("orc_step_rk3if", [C, PP, PP, ctypes.c_int]),
            ("orc_stats", [C, PP, P]),
            ("orc_turb_stats", [C, PP, P, P]),
            ("orc_fft_c2c", [ctypes.c_int, ctypes.c_int, P, ctypes.c_int]),
        ]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        _lib = L
    return _lib


def cfg(n=None, nx=None, ny=None, nz=None, lx=2 * np.pi, ly=2 * np.pi, lz=2 * np.pi, re=1000.0, sc=0.7,
        sc_c=0.7, alpha=0.0, dt=1e-3, alias_filter=2.0 / 3.0, nu_stats=None, nthreads=0) -> OrcCfg:
    nx = nx or n
    ny = ny or n
    nz = nz or n
    if nu_stats is None:
        nu_stats = 1.0 / re        # H/Re with H = 1
    return OrcCfg(nx, ny, nz, lx, ly, lz, re, sc, sc_c, alpha, dt, alias_filter, nu_stats, nthreads)


def _p(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _check(rc, what):
    if rc != 0:
        raise ValueError(f"oracle {what} failed with status {rc}")


def field_buffer(c: OrcCfg) -> np.ndarray:
    """A zeroed buffer able to hold one field (complex128[ny, nx, nz2])."""
    return np.zeros((c.ny, c.nx, c.nz // 2 + 1), dtype=np.complex128)


def phys_view(buf: np.ndarray, c: OrcCfg) -> np.ndarray:
    """Real padded view float64[nx, ny, 2*nz2] of a field buffer."""
    return buf.view(np.float64).reshape(c.nx, c.ny, 2 * (c.nz // 2 + 1))


def forward(c: OrcCfg, buf: np.ndarray) -> None:
    _check(lib().orc_forward(ctypes.byref(c), _p(buf.view(np.float64))), "forward")


def inverse(c: OrcCfg, buf: np.ndarray) -> None:
    _check(lib().orc_inverse(ctypes.byref(c), _p(buf.view(np.float64))), "inverse")


def dealias(c: OrcCfg, buf: np.ndarray) -> None:
    _check(lib().orc_dealias(ctypes.byref(c), _p(buf.view(np.float64))), "dealias")


def vorticity(c: OrcCfg, u, v, w):
    o = [field_buffer(c) for _ in range(3)]
    _check(lib().orc_vorticity(ctypes.byref(c), *[_p(a.view(np.float64)) for a in (u, v, w, *o)]), "vorticity")
    return o


def gradient(c: OrcCfg, f):
    o = [field_buffer(c) for _ in range(3)]
    _check(lib().orc_gradient(ctypes.byref(c), *[_p(a.view(np.float64)) for a in (f, *o)]), "gradient")
    return o


def _pp(arrs):
    P = ctypes.POINTER(ctypes.c_double)
    ptrs = (P * len(arrs))(*[(_p(a.view(np.float64)) if a is not None else P()) for a in arrs])
    return ptrs


def step_cnab2(c: OrcCfg, fields, rhs_old, euler: bool) -> None:
    """One reference step on fields[5] (uh, vh, wh, sh, ch), in place."""
    assert len(fields) == 5 and len(rhs_old) == 5
    _check(lib().orc_step_cnab2(ctypes.byref(c), _pp(fields), _pp(rhs_old), int(euler)), "step_cnab2")


def step_rk3if(c: OrcCfg, fields, n_scalars: int) -> None:
    hist = [field_buffer(c) for _ in fields]
    _check(lib().orc_step_rk3if(ctypes.byref(c), _pp(fields), _pp(hist), n_scalars), "step_rk3if")


STAT_NAMES = ("ke", "vrms2", "eps", "chi_s", "chi_c", "var_s", "var_c")


def stats(c: OrcCfg, fields) -> dict:
    f = list(fields) + [None] * (5 - len(fields))
    out = np.zeros(7)
    _check(lib().orc_stats(ctypes.byref(c), _pp(f), _p(out)), "stats")
    return dict(zip(STAT_NAMES, out.tolist()))


def fft_c2c(x: np.ndarray, sign: int) -> np.ndarray:
    """Batched complex FFT along axis 0 of a C-contiguous complex128[n, batch]."""
    a = np.ascontiguousarray(x, dtype=np.complex128).copy()
    n = a.shape[0]
    b = int(np.prod(a.shape[1:])) if a.ndim > 1 else 1
    _check(lib().orc_fft_c2c(n, b, _p(a.view(np.float64)), sign), "fft_c2c")
    return a


def nthreads_default() -> int:
    return os.cpu_count() or 1


TURB_NAMES = ("vrms", "ke", "epsilon", "eta", "l", "lambda", "chi", "omega", "omega_x", "omega_y", "omega_z")


def turb_stats(c: OrcCfg, fields, with_profiles: bool = True):
    """calcTurbStats_mgpu restated: (dict of TURB_NAMES, profiles [5][ny] or None)."""
    arr = _pp(list(fields) + [None] * (5 - len(fields)))
    out = (ctypes.c_double * 11)()
    prof = np.zeros((5, c.ny)) if with_profiles else None
    pp = prof.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if prof is not None else None
    _check(lib().orc_turb_stats(ctypes.byref(c), arr, out, pp), "turb_stats")
    return {k: float(out[i]) for i, k in enumerate(TURB_NAMES)}, prof
