"""The C-ABI library without a GPU: it loads, exports every entry point that
include/gnss_b200.h declares, and rejects bad arguments before any device work."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "gnss_b200.h"


def _declared():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gnss_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import gnss_b200 as G
    lib = G.load_library()
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    import gnss_b200 as G
    assert set(_declared()) <= set(G._SIGS), set(_declared()) - set(G._SIGS)


@pytest.mark.parametrize("bad", [
    dict(nx=10), dict(ny=7), dict(nz=1024), dict(n_scalars=0), dict(n_scalars=3), dict(scheme=5),
    dict(precision=2), dict(re=0.0), dict(dt=-1.0), dict(lx=0.0), dict(alias_filter=0.0),
])
def test_invalid_config_rejected(bad):
    import gnss_b200 as G
    lib = G.load_library()
    base = dict(nx=16, ny=16, nz=16, lx=6.28, ly=6.28, lz=6.28, re=100.0, sc=0.7, sc_c=0.7, alpha=0.0,
                dt=1e-3, alias_filter=2 / 3, nu_stats=0.01, n_scalars=1, scheme=0, precision=0, device=0)
    base.update(bad)
    cfg = G.GnssConfig(**base)
    h = ctypes.c_void_p()
    assert lib.gnss_create(ctypes.byref(cfg), ctypes.byref(h)) == 1   # GNSS_ERR_INVALID
    assert not h.value


def test_null_context_rejected():
    import gnss_b200 as G
    lib = G.load_library()
    assert lib.gnss_forward(None, None, None) == 1
    assert lib.gnss_step(None, None, None, 0, None) == 1
    assert lib.gnss_destroy(None) == 1
    assert lib.gnss_status_string(3) == b"out of memory"


def test_no_device_reports_cuda_error():
    """On a machine without a GPU a valid configuration fails with GNSS_ERR_CUDA
    (never a silent CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import gnss_b200 as G
    with pytest.raises(G.GnssError) as e:
        G.Context(16)
    assert e.value.status == 2


def test_initial_state_is_solenoidal_and_hermitian(oracle):
    import numpy as np
    import gnss_b200 as G
    n = 24
    f = G.jet_initial_state(n, n_scalars=2, seed=5, noise_kmax=6.0, amp=0.05)
    c = oracle.cfg(n)
    gx = oracle.gradient(c, f[0])[0]
    gy = oracle.gradient(c, f[1])[1]
    gz = oracle.gradient(c, f[2])[2]
    assert np.abs(gx + gy + gz).max() < 1e-12 * np.abs(f[1]).max()
    for a in f:
        b = a.copy()
        oracle.inverse(c, b)
        oracle.forward(c, b)
        assert np.abs(b - a).max() < 1e-12 * np.abs(a).max()
    # seeded: same seed -> same state, different seed -> different noise
    g = G.jet_initial_state(n, n_scalars=2, seed=5, noise_kmax=6.0, amp=0.05)
    h = G.jet_initial_state(n, n_scalars=2, seed=6, noise_kmax=6.0, amp=0.05)
    assert np.array_equal(f[1], g[1]) and not np.array_equal(f[1], h[1])
