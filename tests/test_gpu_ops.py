"""The reference operator surface (solver.cu kernels) on the GPU against the oracle.

Each operator is called through the C ABI and compared with the oracle's
restatement on the same seeded inputs: FP64 to round-off.
"""
import numpy as np
import pytest

from _util import buffer_to_phys, phys_to_buffer, rel_max, to_dev, to_host

SHAPE = (16, 24, 32)


def _spec(rng, shape):
    nx, ny, nz = shape
    return (rng.standard_normal((ny, nx, nz // 2 + 1)) + 1j * rng.standard_normal((ny, nx, nz // 2 + 1)))


def _ocfg(oracle, shape, **kw):
    nx, ny, nz = shape
    return oracle.cfg(nx=nx, ny=ny, nz=nz, **kw)


def _ctx(G, shape, **kw):
    nx, ny, nz = shape
    return G.Context(nx=nx, ny=ny, nz=nz, **kw)


@pytest.mark.gpu
@pytest.mark.parametrize("alias", [2.0 / 3.0, 15.0 / 16.0])
def test_dealias(torch_cuda, oracle, rng, alias):
    torch = torch_cuda
    import gnss_b200 as G
    a = _spec(rng, SHAPE)
    ref = a.copy()
    oracle.dealias(_ocfg(oracle, SHAPE, alias_filter=alias), ref)
    with _ctx(G, SHAPE, alias_filter=alias) as ctx:
        t = to_dev(torch, a)
        ctx.de_alias([t])
        torch.cuda.synchronize()
        got = to_host(t)
    assert np.array_equal(got == 0, ref == 0)
    assert rel_max(got, ref) == 0.0


@pytest.mark.gpu
def test_vorticity_gradient_divergence(torch_cuda, oracle, rng):
    torch = torch_cuda
    import gnss_b200 as G
    oc = _ocfg(oracle, SHAPE)
    u, v, w = (_spec(rng, SHAPE) for _ in range(3))
    ro = oracle.vorticity(oc, u, v, w)
    rg = oracle.gradient(oc, u)
    with _ctx(G, SHAPE) as ctx:
        tu, tv, tw = (to_dev(torch, a) for a in (u, v, w))
        outs = [torch.zeros_like(tu) for _ in range(3)]
        ctx.vorticity(tu, tv, tw, *outs)
        grads = [torch.zeros_like(tu) for _ in range(3)]
        ctx.gradient(tu, *grads)
        div = torch.zeros_like(tu)
        ctx.divergence(*grads, div)
        torch.cuda.synchronize()
        for a, b in zip(outs, ro):
            assert rel_max(to_host(a), b) < 1e-15
        for a, b in zip(grads, rg):
            assert rel_max(to_host(a), b) < 1e-15
        # div grad u = -k^2 u
        nx, ny, nz = SHAPE
        kx = np.fft.fftfreq(nx, 1.0 / nx)
        ky = np.fft.fftfreq(ny, 1.0 / ny)
        kz = np.arange(nz // 2 + 1).astype(float)
        kx[nx // 2] = -nx // 2
        ky[ny // 2] = -ny // 2
        kz[nz // 2] = -nz // 2
        k2 = ky[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2
        assert rel_max(to_host(div), -k2 * u) < 1e-14


@pytest.mark.gpu
def test_make_rhs_timestep_update(torch_cuda, oracle, rng):
    torch = torch_cuda
    import gnss_b200 as G
    oc = _ocfg(oracle, SHAPE, re=500.0, sc=0.7, sc_c=2.0, dt=3e-3)
    r = [_spec(rng, SHAPE) for _ in range(5)]
    ref = [a.copy() for a in r]
    lib = oracle.lib()
    import ctypes
    P = ctypes.POINTER(ctypes.c_double)
    lib.orc_make_rhs(ctypes.byref(oc), *[a.view(np.float64).ctypes.data_as(P) for a in ref])
    with _ctx(G, SHAPE, re=500.0, sc=0.7, sc_c=2.0, dt=3e-3, n_scalars=2) as ctx:
        t = [to_dev(torch, a) for a in r]
        ctx.make_rhs(*t)
        torch.cuda.synchronize()
        for a, b in zip(t, ref):
            assert rel_max(to_host(a), b) < 1e-14
        # timestep (Euler and AB2) and update, against direct formulas of solver.cu:547-657
        f = [_spec(rng, SHAPE) for _ in range(5)]
        ro = [_spec(rng, SHAPE) for _ in range(5)]
        tf = [to_dev(torch, a) for a in f]
        tro = [to_dev(torch, a) for a in ro]
        ctx.timestep(False, tf, t, tro)
        torch.cuda.synchronize()
        nx, ny, nz = SHAPE
        kx = np.fft.fftfreq(nx, 1.0 / nx)
        ky = np.fft.fftfreq(ny, 1.0 / ny)
        kz = np.arange(nz // 2 + 1).astype(float)
        kx[nx // 2] = -nx // 2
        ky[ny // 2] = -ny // 2
        kz[nz // 2] = -nz // 2
        k2 = ky[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2
        nums = [500.0, 500.0, 500.0, 500.0 * 0.7, 500.0 * 2.0]
        for q in range(5):
            a = 1.0 - 3e-3 / 2.0 * k2 / nums[q]
            b = 1.0 + 3e-3 / 2.0 * k2 / nums[q]
            expect = (a * f[q] + 3e-3 * (1.5 * ref[q] - 0.5 * ro[q])) / b
            assert rel_max(to_host(tf[q]), expect) < 1e-14
        ctx.update(t, tro)
        torch.cuda.synchronize()
        for q in range(5):
            assert rel_max(to_host(tro[q]), ref[q]) == 0.0
            assert np.abs(to_host(t[q])).max() == 0.0


@pytest.mark.gpu
def test_physical_products(torch_cuda, rng):
    torch = torch_cuda
    import gnss_b200 as G
    nx, ny, nz = SHAPE
    fs = [rng.standard_normal(SHAPE) for _ in range(11)]
    with _ctx(G, SHAPE, alpha=0.37, n_scalars=2) as ctx:
        t = [to_dev(torch, phys_to_buffer(a)) for a in fs]
        # cross product: o <- o x u  (omega x u, solver.cu:139-164)
        ctx.cross_product(t[0], t[1], t[2], t[3], t[4], t[5])
        u, v, w, o1, o2, o3 = fs[:6]
        exp = [o2 * w - o3 * v, -o1 * w + o3 * u, o1 * v - o2 * u]
        torch.cuda.synchronize()
        for q in range(3):
            assert rel_max(buffer_to_phys(to_host(t[3 + q]), SHAPE), exp[q]) < 1e-15
        out = torch.zeros_like(t[0])
        ctx.dot_product(t[0:3], t[6:9], out)
        torch.cuda.synchronize()
        assert rel_max(buffer_to_phys(to_host(out), SHAPE), u * fs[6] + v * fs[7] + w * fs[8]) < 1e-15
        # colloid: lap <- alpha (lap c + grad c . grad s) + u . grad c
        c, cx, cy, cz = fs[9], fs[6], fs[7], fs[8]
        sx, sy, sz = fs[3], fs[4], fs[5]
        lap = rng.standard_normal(SHAPE)
        tl = to_dev(torch, phys_to_buffer(lap))
        tc = to_dev(torch, phys_to_buffer(c))
        tsx, tsy, tsz = (to_dev(torch, phys_to_buffer(a)) for a in (sx, sy, sz))
        ctx.colloid_advection(t[0:3], tc, t[6:9], (tsx, tsy, tsz), tl)
        torch.cuda.synchronize()
        exp = 0.37 * (lap * c + cx * sx + cy * sy + cz * sz) + u * cx + v * cy + w * cz
        assert rel_max(buffer_to_phys(to_host(tl), SHAPE), exp) < 1e-15
