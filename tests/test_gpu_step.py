"""The fused CUDA time step (gnss_step) against the oracle's restatement of
solver_ps (solver.cu:700-765) and of the IF-RK3 scheme, plus statistics.

Tolerances: FP64 relative L2 per field <= 1e-12 after one step and <= 1e-11
after several (round-off growth only); statistics within 1e-10 relative;
FP32 step within 1e-5 relative L2 of the FP64 oracle after 10 steps.
"""
import math

import numpy as np
import pytest

from _util import rel_l2, to_dev, to_host

CASES = [
    # name, n, re, sc, sc_c, alpha, dt, n_scalars
    ("k16_1s", 16, 200.0, 0.7, 1.0, 0.0, 2e-3, 1),
    ("k16_2s", 16, 200.0, 0.7, 1.0, 0.0, 2e-3, 2),
    ("k16_alpha", 16, 200.0, 0.7, 1.0, 0.05, 2e-3, 2),
    ("k24_2s", 24, 300.0, 1.0, 2.0, 0.0, 1e-3, 2),
    ("c64", 64, 1000.0, 0.7, 0.7, 0.0, 1e-3, 1),
]


def _initial(G, n, n_scalars, seed=0, kmax=None):
    kmax = kmax if kmax is not None else min(8.0, n / 4)
    return G.jet_initial_state(n, n_scalars=n_scalars, seed=seed, noise_kmax=kmax, amp=0.05)


def _oracle_run(oracle, oc, init, n_scalars, nsteps):
    f = [a.copy() for a in init] + ([np.zeros_like(init[0])] if n_scalars == 1 else [])
    r = [np.zeros_like(init[0]) for _ in range(5)]
    out = []
    for s in range(nsteps):
        oracle.step_cnab2(oc, f, r, euler=(s == 0))
        out.append(([a.copy() for a in f], oracle.stats(oc, f)))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_step_cnab2_fp64(torch_cuda, oracle, case):
    import gnss_b200 as G
    torch = torch_cuda
    name, n, re, sc, scc, al, dt, ns = case
    nsteps = 3 if n >= 64 else 5
    init = _initial(G, n, ns)
    oc = oracle.cfg(n, re=re, sc=sc, sc_c=scc, alpha=al, dt=dt)
    ref = _oracle_run(oracle, oc, init, ns, nsteps)
    with G.Context(n, re=re, sc=sc, sc_c=scc, alpha=al, dt=dt, n_scalars=ns) as ctx:
        st = [to_dev(torch, a) for a in init]
        hi = [torch.zeros_like(st[0]) for _ in st]
        # the reference dealiases the state once before the loop (main.cu:156)
        ctx.de_alias(st)
        for s in range(nsteps):
            ctx.solver_ps(st, hi, euler=(s == 0))
            stats = ctx.stats(st)
            fields, rstats = ref[s]
            tol = 1e-12 if s == 0 else 1e-11
            for q in range(3 + ns):
                err = rel_l2(to_host(st[q]), fields[q])
                assert err < tol, f"step {s + 1} field {q}: rel L2 {err:.3e}"
            for k in ("ke", "eps", "chi_s", "var_s") + (("chi_c", "var_c") if ns == 2 else ()):
                assert math.isclose(stats[k], rstats[k], rel_tol=1e-10), (s, k, stats[k], rstats[k])


# Grids whose dealiasing radius (alias_filter * nx / 2, solver.cu:29-31) keeps a Nyquist row or plane: the ky
# Nyquist row (nx >= 1.5 ny), the kz = nz/2 plane (nx >= 1.5 nz), both; with the kernels of 256 x 32 x 256
# (register x pass, warp-specialised z kernel) and with the staged passes.
NYQUIST_SHAPES = [(64, 32, 64), (64, 64, 32), (64, 32, 32), (256, 32, 256)]


@pytest.mark.gpu
@pytest.mark.parametrize("shape", NYQUIST_SHAPES, ids=["x".join(map(str, s)) for s in NYQUIST_SHAPES])
@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_step_cnab2_kept_nyquist_modes(torch_cuda, oracle, shape, precision):
    """Non-cubic grids where a Nyquist wavenumber lies inside the dealiasing sphere.  The reference's round trip of
    the velocity through physical space (solver.cu:707-722, :743-750) keeps only the Hermitian part of the kz = 0
    and kz = nz/2 planes there; three CN/AB2 steps against the oracle, which makes the same round trip."""
    import gnss_b200 as G
    torch = torch_cuda
    nx, ny, nz = shape
    init = G.jet_initial_state(nx, ny, nz, n_scalars=2, seed=1, noise_kmax=6.0, amp=0.05)
    oc = oracle.cfg(nx=nx, ny=ny, nz=nz, re=800.0, sc=0.7, sc_c=1.0, dt=1e-3)
    f = [a.copy() for a in init]
    r = [np.zeros_like(init[0]) for _ in range(5)]
    ref = []
    for s in range(3):
        oracle.step_cnab2(oc, f, r, euler=(s == 0))
        ref.append([a.copy() for a in f])
    cdt = np.complex128 if precision == 0 else np.complex64
    tol = 1e-11 if precision == 0 else 1e-5
    with G.Context(nx=nx, ny=ny, nz=nz, re=800.0, sc=0.7, sc_c=1.0, dt=1e-3, n_scalars=2, precision=precision) as ctx:
        st = [torch.from_numpy(a.astype(cdt)).to("cuda:0") for a in init]
        hi = [torch.zeros_like(st[0]) for _ in st]
        ctx.de_alias(st)
        for s in range(3):
            ctx.solver_ps(st, hi, euler=(s == 0))
            for q in range(5):
                err = rel_l2(to_host(st[q]).astype(np.complex128), ref[s][q])
                assert err < tol, f"step {s + 1} field {q}: rel L2 {err:.3e}"


@pytest.mark.gpu
@pytest.mark.parametrize("ns", [1, 2])
def test_step_rk3if_fp64(torch_cuda, oracle, ns):
    import gnss_b200 as G
    torch = torch_cuda
    n, re, dt = 24, 400.0, 2e-3
    init = _initial(G, n, ns, seed=3)
    oc = oracle.cfg(n, re=re, sc=0.7, sc_c=1.3, dt=dt)
    f = [a.copy() for a in init]
    with G.Context(n, re=re, sc=0.7, sc_c=1.3, dt=dt, n_scalars=ns, scheme=G.GNSS_SCHEME_RK3IF) as ctx:
        st = [to_dev(torch, a) for a in init]
        ctx.de_alias(st)
        for s in range(4):
            oracle.step_rk3if(oc, f, ns)
            ctx.solver_ps(st, None, euler=False)
            for q in range(3 + ns):
                err = rel_l2(to_host(st[q]), f[q])
                assert err < 1e-12, f"step {s + 1} field {q}: rel L2 {err:.3e}"


@pytest.mark.gpu
def test_step_fp32_error_budget(torch_cuda, oracle):
    """FP32 storage and transforms stay within 1e-5 relative L2 of FP64 after 10 steps."""
    import gnss_b200 as G
    torch = torch_cuda
    n, re, dt, ns = 32, 1000.0, 1e-3, 1
    init = _initial(G, n, ns)
    with G.Context(n, re=re, dt=dt, n_scalars=ns) as c64, \
            G.Context(n, re=re, dt=dt, n_scalars=ns, precision=G.GNSS_FP32) as c32:
        a = [to_dev(torch, x) for x in init]
        ha = [torch.zeros_like(a[0]) for _ in a]
        b = [to_dev(torch, x.astype(np.complex64)) for x in init]
        hb = [torch.zeros_like(b[0]) for _ in b]
        c64.de_alias(a)
        c32.de_alias(b)
        for s in range(10):
            c64.solver_ps(a, ha, euler=(s == 0))
            c32.solver_ps(b, hb, euler=(s == 0))
        torch.cuda.synchronize()
        for q in range(3 + ns):
            err = rel_l2(to_host(b[q]).astype(np.complex128), to_host(a[q]))
            assert err < 1e-5, f"field {q}: {err:.3e}"


@pytest.mark.gpu
def test_taylor_green_decay(torch_cuda):
    """2D Taylor-Green vortex: an exact solution; CN gives a known amplitude factor per step."""
    import gnss_b200 as G
    torch = torch_cuda
    n, re, dt, steps = 32, 100.0, 1e-2, 20
    x = np.arange(n) * 2 * np.pi / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    with G.Context(n, re=re, dt=dt, n_scalars=1) as ctx:
        phys = [np.sin(X) * np.cos(Y), -np.cos(X) * np.sin(Y), 0 * X, np.cos(2 * Z)]
        from _util import phys_to_buffer
        st = [to_dev(torch, phys_to_buffer(p)) for p in phys]
        for t in st:
            ctx.forward_transform(t)
        a0 = to_host(st[0]).copy()
        s0 = to_host(st[3]).copy()
        hi = [torch.zeros_like(st[0]) for _ in st]
        for s in range(steps):
            ctx.solver_ps(st, hi, euler=(s == 0))
        torch.cuda.synchronize()
        a = dt / re                       # dt/2 * k^2 / Re with k^2 = 2
        assert rel_l2(to_host(st[0]), a0 * ((1 - a) / (1 + a)) ** steps) < 1e-13
        b = dt / 2 * 4 / (re * 0.7)
        assert rel_l2(to_host(st[3]), s0 * ((1 - b) / (1 + b)) ** steps) < 1e-13


RUN_HOST_CASES = [
    # shape, scheme, precision, n_scalars, alpha
    ((32, 32, 32), 0, 0, 2, 0.0),
    ((48, 32, 64), 0, 1, 1, 0.05),
    ((32, 24, 48), 1, 0, 1, 0.0),
    ((64, 64, 64), 1, 1, 2, 0.0),
]


@pytest.mark.gpu
@pytest.mark.parametrize("shape,scheme,precision,ns,alpha", RUN_HOST_CASES,
                         ids=[f"{'x'.join(map(str, c[0]))}_{'cnab2' if c[1] == 0 else 'rk3if'}_"
                              f"{'fp64' if c[2] == 0 else 'fp32'}_s{c[3]}" for c in RUN_HOST_CASES])
def test_run_host_matches_device_steps(torch_cuda, shape, scheme, precision, ns, alpha):
    """The end-to-end host-buffer call equals the same steps on device buffers.

    The input carries energy in every mode, also outside the dealiasing box:
    gnss_run_host uploads only the kept box and dealiases it, the device path
    dealiases everything (main.cu:156); the states must agree bit for bit.  The
    per-step statistics of gnss_run_host are summed inside the update kernel,
    those of gnss_stats by their own pass: equal to round-off (1e-12 relative).
    """
    import gnss_b200 as G
    torch = torch_cuda
    nx, ny, nz = shape
    steps = 4
    cdt = np.complex128 if precision == G.GNSS_FP64 else np.complex64
    init = G.jet_initial_state(nx, ny, nz, n_scalars=max(ns, 1), seed=7, noise_kmax=6.0, amp=0.05)[:3 + ns]
    rng = np.random.default_rng(3)
    init = [(a + 1e-4 * (rng.standard_normal(a.shape) + 1j * rng.standard_normal(a.shape))).astype(cdt)
            for a in init]
    with G.Context(nx=nx, ny=ny, nz=nz, n_scalars=ns, re=800.0, sc=0.7, sc_c=2.0, alpha=alpha, dt=1e-3,
                   scheme=scheme, precision=precision) as ctx:
        st = [to_dev(torch, a) for a in init]
        hi = [torch.zeros_like(st[0]) for _ in st]
        ctx.de_alias(st)
        want = []
        for s in range(steps):
            ctx.solver_ps(st, hi, euler=(s == 0))
            want.append(ctx.stats(st))
        host = torch.from_numpy(G.pack_state(init)).pin_memory()
        out = torch.empty_like(host).pin_memory()
        stats = np.zeros((steps, G.GNSS_NSTATS))
        ctx.run_host(host, out, steps, True, stats)
        got = out.numpy().reshape(len(init), *init[0].shape)
        for q in range(len(init)):
            assert np.array_equal(got[q], to_host(st[q])), f"field {q}"
        for s in range(steps):
            for j, k in enumerate(G.STAT_NAMES):
                assert math.isclose(stats[s][j], want[s][k], rel_tol=1e-12, abs_tol=1e-300), (s, k)
        h2d, d2h = ctx.run_host_bytes()
        assert d2h == host.numel() * host.element_size()
        assert 0 < h2d < d2h
        ctx.run_host(host, host, steps, True, None)   # in place, no statistics
        assert np.array_equal(host.numpy(), out.numpy())


@pytest.mark.gpu
def test_mixed_precision_config3_128(torch_cuda):
    """The mixed-precision form with the 512^3 jet's parameters (Re 5000, Sc 0.7,
    dt 2.5e-4, one scalar, noise |k| <= 8 rms 0.05) at 128^3: every field within
    1e-5 relative L2 of the FP64 step after 100 steps from the same state.

    The mean profiles (the kx = kz = 0 line, which FP32 contexts advance in
    FP64) are compared with an FP64 run from the FP32-rounded initial state:
    only the FP32 nonlinear term's contribution to them differs (measured
    1.7e-8 for u; with the line stored in FP32 the whole u and s fields of the
    512^3 run were 0.9e-6 and 1.6e-6 off after 100 steps, now 4e-8)."""
    import gnss_b200 as G
    torch = torch_cuda
    n, re, sc, dt, steps = 128, 5000.0, 0.7, 2.5e-4, 100
    init = G.jet_initial_state(n, n_scalars=1, seed=0, noise_kmax=8.0, amp=0.05)
    init32 = [a.astype(np.complex64) for a in init]
    runs = {"fp64": (G.GNSS_FP64, init), "fp64_from32": (G.GNSS_FP64, [a.astype(np.complex128) for a in init32]),
            "fp32": (G.GNSS_FP32, init32)}
    out = {}
    for key, (prec, start) in runs.items():
        with G.Context(n, re=re, sc=sc, dt=dt, n_scalars=1, precision=prec) as ctx:
            st = [to_dev(torch, a) for a in start]
            hi = [torch.zeros_like(st[0]) for _ in st]
            ctx.de_alias(st)
            for s in range(steps):
                ctx.solver_ps(st, hi, euler=(s == 0))
            ctx.check()
            out[key] = [to_host(t).astype(np.complex128) for t in st]
    for q, name in enumerate("uvws"):
        err = rel_l2(out["fp32"][q], out["fp64"][q])
        assert err < 1e-5, f"{name}: rel L2 {err:.3e} after {steps} steps"
    for q, name in ((0, "u"), (3, "s")):
        err = rel_l2(out["fp32"][q][:, 0, 0], out["fp64_from32"][q][:, 0, 0])
        print(f"mean profile {name}: rel L2 {err:.3e} (against FP64 from the same FP32 state)")
        assert err < 5e-8, f"mean profile {name}: rel L2 {err:.3e} after {steps} steps"


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_bounded_wait_timeout_is_reported(torch_cuda, oracle, precision):
    """A bounded device wait that runs out is reported, and nothing hangs.

    GNSS_OPT_TEST_WAIT caps the z kernel's mbarrier waits at 1024 polls and
    makes its first block arm the barrier of its first line pair without
    issuing the copies (nothing is in flight), so that wait runs out: the
    block sets the error word and returns, the launch completes, and
    gnss_check reports GNSS_ERR_TIMEOUT once (the word is then cleared).  The
    context stays usable, and a fresh context steps correctly afterwards.
    """
    import gnss_b200 as G
    torch = torch_cuda
    n, re, dt = 64, 1000.0, 1e-3
    cdt = np.complex128 if precision == G.GNSS_FP64 else np.complex64
    init = _initial(G, n, 1)
    with G.Context(n, re=re, dt=dt, n_scalars=1, precision=precision) as ctx:
        st = [to_dev(torch, a.astype(cdt)) for a in init]
        hi = [torch.zeros_like(st[0]) for _ in st]
        ctx.de_alias(st)
        ctx.set_option(G.GNSS_OPT_TEST_WAIT, 1024)
        assert ctx.get_option(G.GNSS_OPT_TEST_WAIT) == 1024
        ctx.solver_ps(st, hi, euler=True)
        with pytest.raises(G.GnssError) as ei:
            ctx.check()
        assert ei.value.status == G.GNSS_ERR_TIMEOUT
        ctx.check()                       # reported once, then cleared
        ctx.set_option(G.GNSS_OPT_TEST_WAIT, 0)
        ctx.solver_ps(st, hi, euler=False)
        ctx.check()
    # a fresh context: one step against the oracle
    oc = oracle.cfg(n, re=re, dt=dt)
    ref = _oracle_run(oracle, oc, init, 1, 1)
    with G.Context(n, re=re, dt=dt, n_scalars=1, precision=precision) as ctx:
        st = [to_dev(torch, a.astype(cdt)) for a in init]
        hi = [torch.zeros_like(st[0]) for _ in st]
        ctx.de_alias(st)
        ctx.solver_ps(st, hi, euler=True)
        ctx.check()
        tol = 1e-12 if precision == G.GNSS_FP64 else 1e-5
        for q in range(4):
            err = rel_l2(to_host(st[q]).astype(np.complex128), ref[0][0][q])
            assert err < tol, f"field {q}: {err:.3e}"
