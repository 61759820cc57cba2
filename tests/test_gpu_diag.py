"""Turbulence diagnostics (gnss_turb_stats) against the oracle's restatement
of calcTurbStats_mgpu (statistics.cu:2039-2156).

The oracle follows the reference literally: vorticity and the fields are
transformed to physical space, the rms of each vorticity component and the
volume average of |omega| are taken over the grid points, and the mean
profiles are averages over x and z.  The CUDA path gets the component rms by
Parseval and the profiles from the kx = kz = 0 modes, so agreement also pins
those identities.  FP64: 1e-11 relative (statistics), 1e-12 of the profile
scale; FP32 state: 2e-5 relative.
"""
import math

import numpy as np
import pytest

from _util import to_dev

NAMES = ("vrms", "ke", "epsilon", "eta", "l", "lambda", "chi", "omega", "omega_x", "omega_y", "omega_z")


@pytest.mark.gpu
@pytest.mark.parametrize("shape,ns,precision", [((32, 32, 32), 2, 0), ((48, 32, 24), 1, 0), ((64, 64, 64), 2, 1)],
                         ids=["32_s2_fp64", "48x32x24_s1_fp64", "64_s2_fp32"])
def test_turb_stats_match_oracle(torch_cuda, oracle, shape, ns, precision):
    import gnss_b200 as G
    torch = torch_cuda
    nx, ny, nz = shape
    f = G.jet_initial_state(nx, ny, nz, n_scalars=ns, seed=9, noise_kmax=6.0, amp=0.08)
    oc = oracle.cfg(nx=nx, ny=ny, nz=nz, re=1500.0, sc=0.7, sc_c=1.0)
    for a in f:
        oracle.dealias(oc, a)
    ref, rprof = oracle.turb_stats(oc, f)
    cdt = np.complex128 if precision == 0 else np.complex64
    tol = 1e-11 if precision == 0 else 2e-5
    with G.Context(nx=nx, ny=ny, nz=nz, re=1500.0, sc=0.7, sc_c=1.0, n_scalars=ns, precision=precision) as ctx:
        st = [to_dev(torch, a.astype(cdt)) for a in f]
        got, prof = ctx.turb_stats(st)
    for k in NAMES:
        assert math.isclose(got[k], ref[k], rel_tol=tol), (k, got[k], ref[k])
    scale = np.abs(rprof).max()
    assert np.abs(prof - rprof).max() <= (1e-12 if precision == 0 else 2e-6) * scale
    if ns == 1:
        assert not prof[4].any()


@pytest.mark.gpu
def test_turb_stats_of_taylor_green(torch_cuda):
    """Known answers: u = (sin x cos y, -cos x sin y, 0) has KE 1/4, vrms^2 1/6,
    omega_z = -2 sin x sin y (rms 1, mean |omega| 8/pi^2), omega_x = omega_y = 0,
    and zero mean profiles."""
    import gnss_b200 as G
    from _util import phys_to_buffer
    torch = torch_cuda
    n = 32
    x = np.arange(n) * 2 * np.pi / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    with G.Context(n, re=100.0) as ctx:
        st = [to_dev(torch, phys_to_buffer(p)) for p in (np.sin(X) * np.cos(Y), -np.cos(X) * np.sin(Y), 0 * X, 0 * X)]
        for t in st:
            ctx.forward_transform(t)
        got, prof = ctx.turb_stats(st)
    assert math.isclose(got["ke"], 1 / 4, rel_tol=1e-13)
    assert math.isclose(got["vrms"], math.sqrt(1 / 6), rel_tol=1e-13)
    assert math.isclose(got["omega_z"], 1.0, rel_tol=1e-13)
    assert got["omega_x"] < 1e-14 and got["omega_y"] < 1e-14
    # the grid average of |2 sin x sin y| over 32 points per axis
    m = np.mean(np.abs(2 * np.sin(X[:, :, 0]) * np.sin(Y[:, :, 0])))
    assert math.isclose(got["omega"], m, rel_tol=1e-12)
    assert np.abs(prof).max() < 1e-15


STEP_TURB_CASES = [
    # shape, n_scalars, precision, alpha, scheme
    ((128, 128, 128), 2, 0, 0.0, 0),   # register z kernel: vorticity sums fused into the step
    ((96, 96, 96), 1, 1, 0.0, 0),
    ((64, 64, 64), 2, 1, 0.05, 0),     # colloid term (14 physical quantities)
    ((64, 48, 64), 1, 1, 0.0, 1),      # IF-RK3: the first substep sees the state the step starts from
    ((48, 32, 24), 1, 0, 0.0, 0),      # staged z kernel: vorticity by transforms before the step
]


@pytest.mark.gpu
@pytest.mark.parametrize("shape,ns,precision,alpha,scheme", STEP_TURB_CASES,
                         ids=[f"{'x'.join(map(str, c[0]))}_s{c[1]}_{'fp64' if c[2] == 0 else 'fp32'}"
                              f"{'_alpha' if c[3] else ''}{'_rk3' if c[4] else ''}" for c in STEP_TURB_CASES])
def test_step_turb_matches_separate_calls(torch_cuda, shape, ns, precision, alpha, scheme):
    """gnss_step_turb = gnss_turb_stats of the state before the step + gnss_step.

    Spectral statistics and profiles come from the same kernels (equal); the
    vorticity statistics from the step's own physical vorticity where the
    register z kernel serves (1e-10 relative in FP64, 2e-5 in FP32); the new
    state as gnss_step's (1e-14 / 1e-6 relative L2)."""
    import gnss_b200 as G
    from _util import rel_l2, to_host
    torch = torch_cuda
    nx, ny, nz = shape
    cdt = np.complex128 if precision == 0 else np.complex64
    f = [a.astype(cdt) for a in G.jet_initial_state(nx, ny, nz, n_scalars=ns, seed=4, noise_kmax=6.0, amp=0.08)]
    tol = 1e-10 if precision == 0 else 2e-5
    stol = 1e-14 if precision == 0 else 1e-6
    with G.Context(nx=nx, ny=ny, nz=nz, re=1500.0, sc=0.7, sc_c=1.0, alpha=alpha, dt=1e-3, n_scalars=ns,
                   precision=precision, scheme=scheme) as ctx:
        runs = []
        for fused in (False, True):
            st = [to_dev(torch, a) for a in f]
            hi = [torch.zeros_like(st[0]) for _ in st]
            ctx.de_alias(st)
            for step in range(2):   # two steps in a row (Euler, then AB2)
                if fused:
                    got, prof = ctx.step_turb(st, hi, euler=(step == 0))
                else:
                    got, prof = ctx.turb_stats(st)
                    ctx.solver_ps(st, hi, euler=(step == 0))
                runs.append((got, prof))
            torch.cuda.synchronize()
            runs.append([to_host(t) for t in st])
    sep, fus = runs[:3], runs[3:]
    for step in range(2):
        (a, pa), (b, pb) = sep[step], fus[step]
        for k in ("vrms", "ke", "epsilon", "eta", "l", "lambda", "chi"):
            assert a[k] == b[k], (step, k)
        assert np.array_equal(pa, pb)
        for k in ("omega", "omega_x", "omega_y", "omega_z"):
            assert math.isclose(a[k], b[k], rel_tol=tol), (step, k, a[k], b[k])
    for q in range(3 + ns):
        assert rel_l2(fus[2][q], sep[2][q]) <= stol, q
