"""The kernel variants of the step give the same step.

At N = 256 and 512 the z stage runs register-resident line transforms
(k_zreg, or k_zws with separate inverse and forward warps in FP32 with one
scalar) and the strided x / y passes register-resident column transforms
(k_passr); at N = 64, 96, 128 and 192 the same kernels run lane-shuffle
transforms when requested; the staged kernels (k_zphys, k_pass:
per-radix-stage transforms through shared memory) serve every size.  All evaluate the nonlinear term of
solver_ps (solver.cu:700-765); here one context steps the same dealiased
state with every combination of the two options (gnss_set_option) and the
fields must agree to round-off: relative L2 <= 1e-13 in FP64 and <= 2e-6 in
FP32 after two steps.  The FP64 register path is also held to the oracle at
256^3, 96^3 and 128^3 (1e-12 after one step).
"""
import numpy as np
import pytest

from _util import rel_l2, to_dev, to_host

CASES = [
    # grid, precision, n_scalars, alpha
    (256, 0, 1, 0.0),
    (256, 0, 2, 0.05),
    (256, 1, 1, 0.0),
    (256, 1, 2, 0.0),
    (512, 1, 1, 0.0),
    ((64, 64, 512), 0, 2, 0.05),   # z length 512: forward transforms split in halves, 5 products
    ((64, 64, 512), 1, 1, 0.0),
    # lane-shuffle register transforms (N = 32 E, E = 2, 3, 4, 6)
    (64, 0, 2, 0.05),
    (96, 1, 1, 0.0),
    (128, 0, 1, 0.0),
    (192, 1, 2, 0.0),
    ((96, 64, 192), 0, 1, 0.0),
    ((128, 192, 64), 1, 2, 0.05),
]


def _shape(n):
    return (n, n, n) if isinstance(n, int) else n


def _run(G, torch, ctx, init, steps, variant, pvariant=0):
    ctx.set_option(G.GNSS_OPT_ZVARIANT, variant)
    ctx.set_option(G.GNSS_OPT_PVARIANT, pvariant)
    st = [to_dev(torch, a) for a in init]
    hi = [torch.zeros_like(st[0]) for _ in st]
    ctx.de_alias(st)
    for s in range(steps):
        ctx.solver_ps(st, hi, euler=(s == 0))
    ctx.check()
    torch.cuda.synchronize()
    return [to_host(t) for t in st]


@pytest.mark.gpu
@pytest.mark.parametrize("n,precision,ns,alpha", CASES,
                         ids=[f"n{'x'.join(map(str, _shape(c[0])))}_{'fp64' if c[1] == 0 else 'fp32'}_s{c[2]}"
                              f"{'_alpha' if c[3] else ''}" for c in CASES])
def test_register_and_staged_z_agree(torch_cuda, n, precision, ns, alpha):
    import gnss_b200 as G
    torch = torch_cuda
    nx, ny, nz = _shape(n)
    cdt = np.complex128 if precision == 0 else np.complex64
    init = G.jet_initial_state(nx, ny, nz, n_scalars=ns, seed=5, noise_kmax=8.0, amp=0.05, dtype=cdt)
    tol = 1e-13 if precision == 0 else 2e-6
    A, S = G.GNSS_VARIANT_REGISTER, G.GNSS_VARIANT_STAGED
    with G.Context(nx=nx, ny=ny, nz=nz, re=3000.0, sc=0.7, sc_c=1.0, alpha=alpha, dt=5e-4, n_scalars=ns,
                   precision=precision) as ctx:
        a = _run(G, torch, ctx, init, 2, A, A)
        W = G.GNSS_VARIANT_WARPSPEC   # the register kernel where the warp-specialised one does not exist
        for zv, pv in ((S, A), (A, S), (S, S), (W, A), (W, S)):
            b = _run(G, torch, ctx, init, 2, zv, pv)
            for q in range(3 + ns):
                err = rel_l2(a[q], b[q])
                assert err < tol, f"z {zv} pass {pv} field {q}: rel L2 {err:.3e} against the register kernels"


@pytest.mark.gpu
@pytest.mark.parametrize("n", [256, 96, 128])
def test_register_z_matches_oracle(torch_cuda, oracle, n):
    """FP64 register kernels (both z and passes) against the oracle after one step: the default (AUTO)
    selection at 256, the lane-shuffle transforms requested explicitly at 96 and 128."""
    import gnss_b200 as G
    torch = torch_cuda
    ns = 2
    init = G.jet_initial_state(n, n_scalars=ns, seed=11, noise_kmax=min(16.0, n / 8), amp=0.05)
    oc = oracle.cfg(n, re=3000.0, sc=0.7, sc_c=1.0, dt=5e-4)
    f = [x.copy() for x in init]
    r = [np.zeros_like(init[0]) for _ in range(5)]
    for a in f:
        oracle.dealias(oc, a)
    oracle.step_cnab2(oc, f, r, euler=True)
    with G.Context(n, re=3000.0, sc=0.7, sc_c=1.0, dt=5e-4, n_scalars=ns) as ctx:
        assert ctx.get_option(G.GNSS_OPT_ZVARIANT) == G.GNSS_ZVARIANT_AUTO
        v = G.GNSS_VARIANT_AUTO if n == 256 else G.GNSS_VARIANT_REGISTER
        got = _run(G, torch, ctx, init, 1, v, v)
    for q in range(3 + ns):
        err = rel_l2(got[q], f[q])
        assert err < 1e-12, f"field {q}: rel L2 {err:.3e}"


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(256, 256, 32), (512, 8, 16), (16, 512, 8), (64, 96, 16), (192, 128, 8)])
def test_register_passes_in_the_3d_transforms(torch_cuda, oracle, shape):
    """gnss_forward / gnss_inverse (fftfuncs.cu:288-359) with the register pass kernel, against the oracle."""
    import gnss_b200 as G
    from _util import buffer_to_phys, phys_to_buffer, rel_max
    torch = torch_cuda
    nx, ny, nz = shape
    u = np.random.default_rng(17).standard_normal(shape)
    buf = phys_to_buffer(u)
    ref = buf.copy()
    oc = oracle.cfg(nx=nx, ny=ny, nz=nz)
    oracle.forward(oc, ref)
    with G.Context(nx=nx, ny=ny, nz=nz) as ctx:
        ctx.set_option(G.GNSS_OPT_PVARIANT, G.GNSS_VARIANT_REGISTER)
        t = to_dev(torch, buf)
        ctx.forward_transform(t)
        torch.cuda.synchronize()
        assert rel_max(to_host(t), ref) < 1e-13
        ctx.inverse_transform(t)
        torch.cuda.synchronize()
        assert rel_max(buffer_to_phys(to_host(t), shape), u) < 1e-13


@pytest.mark.gpu
def test_z_kernel_query(torch_cuda):
    """GNSS_OPT_ZKERNEL reports the z kernel the options select (read-only)."""
    import gnss_b200 as G
    W, R, S, A = G.GNSS_VARIANT_WARPSPEC, G.GNSS_VARIANT_REGISTER, G.GNSS_VARIANT_STAGED, G.GNSS_VARIANT_AUTO
    cases = [
        # config, z option -> kernel
        (dict(n=256, precision=G.GNSS_FP32), W, W),
        (dict(n=256, precision=G.GNSS_FP64), W, W),      # FP64 with one or two scalars,
        (dict(n=256, precision=G.GNSS_FP64, n_scalars=2), W, W),
        (dict(n=256, precision=G.GNSS_FP64), A, W),      # AUTO takes it in FP64,
        (dict(n=256, precision=G.GNSS_FP32), A, R),      # not in FP32
        (dict(n=256, precision=G.GNSS_FP32, n_scalars=2), W, R),   # FP32 with one
        (dict(n=128, precision=G.GNSS_FP32), W, R),      # and z length 256 or 512 only
        (dict(n=128, precision=G.GNSS_FP32), A, R),
        (dict(n=128, precision=G.GNSS_FP32), S, S),
        (dict(n=48, precision=G.GNSS_FP32), R, S),       # no register transform of length 48
    ]
    for kw, opt, want in cases:
        n = kw.pop("n")
        with G.Context(n, **kw) as ctx:
            ctx.set_option(G.GNSS_OPT_ZVARIANT, opt)
            assert ctx.get_option(G.GNSS_OPT_ZKERNEL) == want, (n, kw, opt)
            with pytest.raises(G.GnssError):
                ctx.set_option(G.GNSS_OPT_ZKERNEL, R)
