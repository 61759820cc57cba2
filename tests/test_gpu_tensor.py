"""The tensor-core passes (GNSS_VARIANT_TENSOR: split-TF32 DFT-matrix GEMMs on
tcgen05, FP32, x / y lengths 256 and 512).

Tolerances: the 3D transforms within 3e-6 (forward) and 5e-6 (round trip)
relative L2 of numpy's FP64 transforms of the same FP32 input; one fused step within 2e-6 relative L2 of the register passes; the
mixed-precision jet (the 512^3 workload's parameters on a 256 x 256 x 64 grid)
within 1e-5 relative L2 of the FP64 step after 100 steps.
"""
import numpy as np
import pytest

from _util import buffer_to_phys, phys_to_buffer, rel_l2, to_dev, to_host

SHAPES = [(256, 256, 8), (512, 256, 16), (256, 512, 12), (512, 512, 8)]


@pytest.mark.gpu
@pytest.mark.parametrize("shape", SHAPES, ids=["x".join(map(str, s)) for s in SHAPES])
def test_tensor_transforms_match_numpy(torch_cuda, shape):
    """Forward and inverse 3D transforms with the tensor-core x / y passes
    against numpy's FP64 transforms of the same FP32 input: relative L2 within
    3e-6 forward and 5e-6 for the round trip (measured 1.0e-6 - 1.4e-6 and
    2.0e-6 - 2.7e-6 with the remainder truncated by the MMA; the register FP32
    passes, measured alongside, reach 1.5e-7 and 2.5e-7).  The split products
    leave out a_lo b_lo (2^-22 relative), and the tensor core's FP32
    accumulation of the K = 8 partial sums adds its own rounding."""
    import gnss_b200 as G
    torch = torch_cuda
    nx, ny, nz = shape
    rng = np.random.default_rng(11)
    u = rng.standard_normal(shape).astype(np.float32)
    ref = np.transpose(np.fft.rfftn(u.astype(np.float64), axes=(0, 1, 2)), (1, 0, 2))   # [ky][kx][kz]
    err = {}
    for pv in (G.GNSS_VARIANT_REGISTER, G.GNSS_VARIANT_TENSOR):
        with G.Context(nx=nx, ny=ny, nz=nz, precision=G.GNSS_FP32) as ctx:
            ctx.set_option(G.GNSS_OPT_PVARIANT, pv)
            t = to_dev(torch, phys_to_buffer(u, dtype=np.complex64))
            ctx.forward_transform(t)
            ctx.check()
            fwd = rel_l2(to_host(t), ref)
            ctx.inverse_transform(t)
            ctx.check()
            back = rel_l2(buffer_to_phys(to_host(t), shape), u)
            err[pv] = (fwd, back)
    print(f"{shape}: register passes {err[G.GNSS_VARIANT_REGISTER]}, tensor-core passes {err[G.GNSS_VARIANT_TENSOR]}")
    fwd, back = err[G.GNSS_VARIANT_TENSOR]
    assert fwd < 3e-6, f"forward: {fwd:.3e}"
    assert back < 5e-6, f"round trip: {back:.3e}"


@pytest.mark.gpu
@pytest.mark.parametrize("ns,alpha", [(1, 0.0), (2, 0.05)], ids=["1s", "2s_alpha"])
def test_tensor_step_matches_register_passes(torch_cuda, ns, alpha):
    """One fused step (every pass kind: x inverse with the dealias mask and the
    i kx multiplier, y inverse with i ky, y and x forward onto the kept rows)."""
    import gnss_b200 as G
    torch = torch_cuda
    shape = (256, 256, 32)
    init = G.jet_initial_state(*shape, n_scalars=ns, seed=2, noise_kmax=8.0, amp=0.05, dtype=np.complex64)
    out = {}
    for pv in (G.GNSS_VARIANT_REGISTER, G.GNSS_VARIANT_TENSOR):
        with G.Context(nx=shape[0], ny=shape[1], nz=shape[2], re=1000.0, sc=0.7, sc_c=1.0, alpha=alpha,
                       dt=1e-3, n_scalars=ns, precision=G.GNSS_FP32) as ctx:
            ctx.set_option(G.GNSS_OPT_PVARIANT, pv)
            st = [to_dev(torch, a) for a in init]
            hi = [torch.zeros_like(st[0]) for _ in st]
            ctx.de_alias(st)
            ctx.solver_ps(st, hi, euler=True)
            ctx.solver_ps(st, hi, euler=False)
            ctx.check()
            out[pv] = [to_host(a) for a in st]
    for q in range(3 + ns):
        err = rel_l2(out[G.GNSS_VARIANT_TENSOR][q], out[G.GNSS_VARIANT_REGISTER][q])
        assert err < 2e-6, f"field {q}: {err:.3e}"


@pytest.mark.gpu
def test_tensor_mixed_precision_error_budget(torch_cuda):
    """The 512^3 jet's parameters (Re 5000, Sc 0.7, dt 2.5e-4, one scalar,
    noise |k| <= 8 rms 0.05) on 256 x 256 x 64: the tensor-core passes keep every
    field within 1e-5 relative L2 of the FP64 step after 100 steps."""
    import gnss_b200 as G
    torch = torch_cuda
    shape, steps = (256, 256, 64), 100
    init = G.jet_initial_state(*shape, n_scalars=1, seed=0, noise_kmax=8.0, amp=0.05)
    out = {}
    for prec, cdt in ((G.GNSS_FP64, np.complex128), (G.GNSS_FP32, np.complex64)):
        with G.Context(nx=shape[0], ny=shape[1], nz=shape[2], re=5000.0, sc=0.7, dt=2.5e-4, n_scalars=1,
                       precision=prec) as ctx:
            if prec == G.GNSS_FP32:
                ctx.set_option(G.GNSS_OPT_PVARIANT, G.GNSS_VARIANT_TENSOR)
            st = [to_dev(torch, a.astype(cdt)) for a in init]
            hi = [torch.zeros_like(st[0]) for _ in st]
            ctx.de_alias(st)
            for s in range(steps):
                ctx.solver_ps(st, hi, euler=(s == 0))
            ctx.check()
            out[prec] = [to_host(a) for a in st]
    for q, name in enumerate("uvws"):
        err = rel_l2(out[G.GNSS_FP32][q].astype(np.complex128), out[G.GNSS_FP64][q])
        assert err < 1e-5, f"{name}: {err:.3e}"


@pytest.mark.gpu
def test_tensor_option_elsewhere_takes_auto(torch_cuda):
    """Where no tensor-core pass exists (FP64, or lengths other than 256 / 512)
    the option runs the AUTO kernels: bit-identical results."""
    import gnss_b200 as G
    torch = torch_cuda
    for prec, cdt, shape in ((G.GNSS_FP64, np.complex128, (256, 256, 16)), (G.GNSS_FP32, np.complex64, (64, 96, 32))):
        init = G.jet_initial_state(*shape, n_scalars=1, seed=4, noise_kmax=6.0, amp=0.05, dtype=cdt)
        res = []
        for pv in (G.GNSS_VARIANT_AUTO, G.GNSS_VARIANT_TENSOR):
            with G.Context(nx=shape[0], ny=shape[1], nz=shape[2], n_scalars=1, precision=prec) as ctx:
                ctx.set_option(G.GNSS_OPT_PVARIANT, pv)
                st = [to_dev(torch, a) for a in init]
                hi = [torch.zeros_like(st[0]) for _ in st]
                ctx.de_alias(st)
                ctx.solver_ps(st, hi, euler=True)
                res.append([to_host(a) for a in st])
        for q in range(4):
            assert np.array_equal(res[0][q], res[1][q]), (prec, q)
