"""CUDA 3D transforms (gnss_forward / gnss_inverse) against the CPU oracle.

The oracle restates fftfuncs.cu:288-359 (unnormalised forward into the
transposed spectral layout, inverse with the 1/N^3 scale); the CUDA path is
called through the C ABI.  FP64 must agree to round-off (1e-13 relative max);
FP32 within 5e-6 relative L2.
"""
import numpy as np
import pytest

from _util import buffer_to_phys, phys_to_buffer, rel_l2, rel_max, to_dev, to_host

SHAPES = [(8, 8, 8), (16, 16, 16), (12, 16, 24), (32, 32, 32), (48, 24, 96), (64, 64, 64),
          (96, 96, 96), (128, 64, 32), (192, 16, 16), (384, 12, 16), (512, 8, 16), (16, 512, 8), (8, 16, 512),
          (256, 256, 32)]


def _ctx(G, shape, precision=0):
    nx, ny, nz = shape
    return G.Context(nx=nx, ny=ny, nz=nz, precision=precision)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", SHAPES)
def test_forward_inverse_fp64(torch_cuda, oracle, rng, shape):
    import gnss_b200 as G
    torch = torch_cuda
    nx, ny, nz = shape
    u = rng.standard_normal(shape)
    buf = phys_to_buffer(u)
    ref = buf.copy()
    oc = oracle.cfg(nx=nx, ny=ny, nz=nz)
    oracle.forward(oc, ref)
    with _ctx(G, shape) as ctx:
        t = to_dev(torch, buf)
        ctx.forward_transform(t)
        torch.cuda.synchronize()
        got = to_host(t)
        assert rel_max(got, ref) < 1e-13
        assert rel_max(got, np.fft.rfftn(u).transpose(1, 0, 2)) < 1e-13
        ctx.inverse_transform(t)
        torch.cuda.synchronize()
        back = buffer_to_phys(to_host(t), shape)
        assert rel_max(back, u) < 1e-13
        # inverse alone against the oracle on a spectral field with Hermitian planes
        spec = ref.copy()
        t2 = to_dev(torch, spec)
        ctx.inverse_transform(t2)
        oracle.inverse(oc, spec)
        torch.cuda.synchronize()
        assert rel_max(buffer_to_phys(to_host(t2), shape), buffer_to_phys(spec, shape)) < 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(16, 16, 16), (64, 64, 64), (96, 48, 128), (512, 16, 16)])
def test_forward_inverse_fp32(torch_cuda, oracle, rng, shape):
    import gnss_b200 as G
    torch = torch_cuda
    nx, ny, nz = shape
    u = rng.standard_normal(shape)
    ref = phys_to_buffer(u)
    oracle.forward(oracle.cfg(nx=nx, ny=ny, nz=nz), ref)
    with _ctx(G, shape, precision=1) as ctx:
        t = to_dev(torch, phys_to_buffer(u.astype(np.float32), dtype=np.complex64))
        ctx.forward_transform(t)
        torch.cuda.synchronize()
        assert rel_l2(to_host(t).astype(np.complex128), ref) < 5e-6
        ctx.inverse_transform(t)
        torch.cuda.synchronize()
        assert rel_l2(buffer_to_phys(to_host(t), shape), u) < 5e-6


@pytest.mark.gpu
def test_single_mode_known_answer(torch_cuda):
    """cos(2x + 3y - z) has exactly two nonzero coefficients of magnitude N^3/2."""
    import gnss_b200 as G
    torch = torch_cuda
    n = 32
    x = np.arange(n) * 2 * np.pi / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    u = np.cos(2 * X + 3 * Y - Z)
    with G.Context(n) as ctx:
        t = to_dev(torch, phys_to_buffer(u))
        ctx.forward_transform(t)
        torch.cuda.synchronize()
        F = to_host(t)
    # spectral [ky][kx][kz]; cos(2x+3y-z) = (e^{i(2,3,-1)} + e^{-i(2,3,-1)})/2 ; stored half kz >= 0:
    # (kx,ky,kz) = (-2,-3,1) carries N^3/2
    expect = np.zeros_like(F)
    expect[(-3) % n, (-2) % n, 1] = n ** 3 / 2
    assert np.abs(F - expect).max() < 1e-9 * n ** 3
