"""The allocation-free forward transform (gnss_forward_noalloc).

Some callers may not allocate device memory: code running under a memory
manager that owns the whole device, or latency-critical loops where a
cudaMalloc / cudaFree would synchronise the device.  gnss_forward_noalloc
serves them with a static scratch array inside the library.  This test calls
it through the C ABI and checks it against the context-based gnss_forward on
the same inputs, for two calls in a row (the shared array keeps the previous
call's contents, which must not leak into the next result).  The file is
named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from _util import phys_to_buffer, rel_max, to_dev, to_host


@pytest.mark.gpu
@pytest.mark.parametrize("shape,precision", [((32, 48, 64), 0), ((64, 64, 64), 0), ((128, 64, 96), 1),
                                             ((512, 16, 128), 0), ((16, 512, 48), 1)])
def test_noalloc_forward_matches_forward(torch_cuda, shape, precision):
    import gnss_b200 as G
    torch = torch_cuda
    lib = G.load_library()
    nx, ny, nz = shape
    cdt = np.complex128 if precision == 0 else np.complex64
    rdt = np.float64 if precision == 0 else np.float32
    tol = 1e-13 if precision == 0 else 1e-6
    rng = np.random.default_rng(99)
    with G.Context(nx=nx, ny=ny, nz=nz, precision=precision) as ctx:
        cfg = G.GnssConfig.from_buffer_copy(ctx.cfg)
        for call in range(2):   # two calls in a row, different data
            u = rng.standard_normal(shape).astype(rdt)
            a = to_dev(torch, phys_to_buffer(u, dtype=cdt))
            b = a.clone()
            ctx.forward_transform(a)
            st = lib.gnss_forward_noalloc(ctypes.byref(cfg), b.data_ptr(), torch.cuda.current_stream().cuda_stream)
            assert st == 0, f"call {call}: status {st}"
            torch.cuda.synchronize()
            assert rel_max(to_host(b), to_host(a)) < tol, f"call {call}"


@pytest.mark.gpu
def test_noalloc_size_sequence(torch_cuda):
    """Sizes and precisions one after another, the largest first: every call
    rewrites the twiddle slots it reads (a length-512 axis fills a whole slot)
    and the scratch it uses, so what a larger earlier call left in the shared
    array never reaches a later result."""
    import gnss_b200 as G
    torch = torch_cuda
    lib = G.load_library()
    rng = np.random.default_rng(7)
    seq = [((512, 16, 128), 0), ((512, 32, 64), 1), ((24, 32, 48), 0), ((96, 12, 16), 1), ((32, 48, 64), 0),
           ((8, 8, 8), 1)]
    for shape, precision in seq:
        nx, ny, nz = shape
        cdt = np.complex128 if precision == 0 else np.complex64
        rdt = np.float64 if precision == 0 else np.float32
        tol = 1e-13 if precision == 0 else 1e-6
        with G.Context(nx=nx, ny=ny, nz=nz, precision=precision) as ctx:
            cfg = G.GnssConfig.from_buffer_copy(ctx.cfg)
            u = rng.standard_normal(shape).astype(rdt)
            a = to_dev(torch, phys_to_buffer(u, dtype=cdt))
            b = a.clone()
            ctx.forward_transform(a)
            st = lib.gnss_forward_noalloc(ctypes.byref(cfg), b.data_ptr(), torch.cuda.current_stream().cuda_stream)
            assert st == 0, f"{shape}: status {st}"
            torch.cuda.synchronize()
            assert rel_max(to_host(b), to_host(a)) < tol, f"{shape} precision {precision}"


@pytest.mark.gpu
def test_noalloc_rejects_oversize(torch_cuda):
    import gnss_b200 as G
    torch = torch_cuda
    lib = G.load_library()
    cfg = G.GnssConfig(256, 256, 256, 6.28, 6.28, 6.28, 100.0, 0.7, 0.7, 0.0, 1e-3, 2 / 3, 0.01, 1, 0, 0, 0)
    t = torch.zeros(8, dtype=torch.complex128, device="cuda")
    assert lib.gnss_forward_noalloc(ctypes.byref(cfg), t.data_ptr(), None) == 1   # GNSS_ERR_INVALID
