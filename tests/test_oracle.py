"""CPU oracle checks (no GPU): the restated transforms against numpy's
pocketfft, and known-answer cases of the restated step (solver.cu:700-765).
"""
import math

import numpy as np
import pytest

from _util import buffer_to_phys, phys_to_buffer, rel_l2, rel_max


@pytest.mark.parametrize("n", [2, 3, 4, 6, 8, 12, 16, 24, 48, 96, 128, 192, 384, 512])
def test_fft_c2c_matches_numpy(oracle, rng, n):
    x = rng.standard_normal((n, 5)) + 1j * rng.standard_normal((n, 5))
    assert rel_max(oracle.fft_c2c(x, -1), np.fft.fft(x, axis=0)) < 2e-15 * max(1, math.log2(n))
    assert rel_max(oracle.fft_c2c(x, +1), np.fft.ifft(x, axis=0) * n) < 2e-15 * max(1, math.log2(n))


@pytest.mark.parametrize("shape", [(8, 8, 8), (12, 16, 18), (32, 32, 32), (16, 48, 24), (64, 8, 96)])
def test_forward_layout_and_inverse(oracle, rng, shape):
    """forwardTransform leaves the result transposed [ky][kx][kz] (fftfuncs.cu:315);
    inverseTransform includes 1/N^3 (cudafuncs.cu:20-31)."""
    nx, ny, nz = shape
    c = oracle.cfg(nx=nx, ny=ny, nz=nz)
    u = rng.standard_normal(shape)
    buf = phys_to_buffer(u)
    oracle.forward(c, buf)
    assert rel_max(buf, np.fft.rfftn(u).transpose(1, 0, 2)) < 1e-14
    oracle.inverse(c, buf)
    assert rel_max(buffer_to_phys(buf, shape), u) < 1e-14


def test_unsupported_size_rejected(oracle):
    c = oracle.cfg(nx=10, ny=8, nz=8)
    with pytest.raises(ValueError):
        oracle.forward(c, np.zeros((8, 10, 5), dtype=np.complex128))


@pytest.mark.parametrize("n,alias", [(32, 2.0 / 3.0), (64, 2.0 / 3.0), (32, 15.0 / 16.0), (96, 2.0 / 3.0)])
def test_dealias_mask_count(oracle, n, alias):
    """Spherical truncation k^2 > (alias*nx*pi/lx)^2 (solver.cu:17-42), counted directly."""
    c = oracle.cfg(n, alias_filter=alias)
    f = np.ones((n, n, n // 2 + 1), dtype=np.complex128)
    oracle.dealias(c, f)
    k = np.fft.fftfreq(n, 1.0 / n)
    k[n // 2] = -n // 2
    kz = np.arange(n // 2 + 1).astype(float)
    kz[n // 2] = -n // 2
    kmax = alias * (n * math.pi / (2 * math.pi))
    k2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + kz[None, None, :] ** 2
    assert int((f != 0).sum()) == int((k2 <= kmax * kmax).sum())


def _tg_state(oracle, c, n):
    x = np.arange(n) * 2 * np.pi / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    out = []
    for p in (np.sin(X) * np.cos(Y), -np.cos(X) * np.sin(Y), 0 * X, np.cos(2 * Z), np.sin(3 * Z)):
        b = phys_to_buffer(p)
        oracle.forward(c, b)
        out.append(b)
    return out


def test_taylor_green_cnab2(oracle):
    """Taylor-Green is an exact Navier-Stokes solution: the nonlinear term is a
    gradient, removed by the projection; CN/AB2 then multiplies each step by
    (1 - dt k^2/(2 Re)) / (1 + dt k^2/(2 Re))."""
    n, re, dt, steps = 16, 100.0, 1e-2, 10
    c = oracle.cfg(n, re=re, dt=dt, sc=0.7, sc_c=2.0)
    f = _tg_state(oracle, c, n)
    a0, s0, c0 = f[0].copy(), f[3].copy(), f[4].copy()
    r = [np.zeros_like(f[0]) for _ in range(5)]
    for s in range(steps):
        oracle.step_cnab2(c, f, r, euler=(s == 0))
    a = dt / re
    assert rel_l2(f[0], a0 * ((1 - a) / (1 + a)) ** steps) < 1e-14
    b = dt / 2 * 4 / (re * 0.7)
    assert rel_l2(f[3], s0 * ((1 - b) / (1 + b)) ** steps) < 1e-14
    b = dt / 2 * 9 / (re * 2.0)
    assert rel_l2(f[4], c0 * ((1 - b) / (1 + b)) ** steps) < 1e-14


def test_taylor_green_rk3if(oracle):
    n, re, dt, steps = 16, 100.0, 1e-2, 10
    c = oracle.cfg(n, re=re, dt=dt, sc=0.7)
    f = _tg_state(oracle, c, n)[:4]
    a0, s0 = f[0].copy(), f[3].copy()
    for _ in range(steps):
        oracle.step_rk3if(c, f, 1)
    assert rel_l2(f[0], a0 * np.exp(-2 / re * dt * steps)) < 1e-14
    assert rel_l2(f[3], s0 * np.exp(-4 / (re * 0.7) * dt * steps)) < 1e-14


def test_projection_idempotent_and_solenoidal(oracle, rng):
    """makeRHS: (k k^T/k^2 - I) is minus a projector: applying it twice returns
    the negated first result, and the result is divergence free."""
    n = 16
    c = oracle.cfg(n)
    import ctypes
    P = ctypes.POINTER(ctypes.c_double)
    r = [rng.standard_normal((n, n, n // 2 + 1)) + 1j * rng.standard_normal((n, n, n // 2 + 1)) for _ in range(3)]
    lib = oracle.lib()

    def mk(fs):
        fs = [a.copy() for a in fs]
        lib.orc_make_rhs(ctypes.byref(c), *[a.view(np.float64).ctypes.data_as(P) for a in fs], None, None)
        return fs

    once = mk(r)
    twice = mk(once)
    for a, b in zip(once, twice):
        assert rel_max(b, -a) < 1e-14
    gx = oracle.gradient(c, once[0])[0]
    gy = oracle.gradient(c, once[1])[1]
    gz = oracle.gradient(c, once[2])[2]
    assert np.abs(gx + gy + gz).max() < 1e-12 * np.abs(once[0]).max() * n


def test_stats_definitions(oracle):
    """KE of u = sin x on the unit-amplitude mode is 1/4 (volume mean of u^2/2)."""
    n = 16
    c = oracle.cfg(n, re=100.0)
    x = np.arange(n) * 2 * np.pi / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    fs = []
    for p in (np.sin(X), 0 * X, 0 * X, np.cos(2 * Y), 0 * X):
        b = phys_to_buffer(p)
        oracle.forward(c, b)
        fs.append(b)
    st = oracle.stats(c, fs)
    assert math.isclose(st["ke"], 0.25, rel_tol=1e-13)
    assert math.isclose(st["eps"], 0.01 * 0.5, rel_tol=1e-13)        # nu <|grad u|^2> = nu/2
    assert math.isclose(st["var_s"], 0.5, rel_tol=1e-13)             # <cos^2> = 1/2
    assert math.isclose(st["chi_s"], 2 * 0.01 / 0.7 * 4 * 0.5, rel_tol=1e-13)
