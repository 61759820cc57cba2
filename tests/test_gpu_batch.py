"""Ensembles (gnss_ensemble_*) and the serving loop (gnss_server_*).

Both are schedulers over the same per-jet step (solver_ps, solver.cu:700-765):
a member of an ensemble, or a request in a server, must end bit-identical to
the same jet run alone through gnss_run_host (upload, dealias as main.cu:156,
Euler first step, AB2 after), whatever else runs beside it.  Statistics agree
to round-off: gnss_run_host sums them inside the update kernel.
"""
import math

import numpy as np
import pytest


def _cfgs(G):
    return [
        G.make_config(16, re=500.0, sc=0.7, dt=2e-3),
        G.make_config(24, re=800.0, sc=1.0, sc_c=2.0, dt=1e-3, n_scalars=2),
        G.make_config(nx=32, ny=24, nz=48, re=1200.0, sc=2.0, dt=1e-3),
        G.make_config(16, re=3000.0, sc=0.7, dt=1e-3, precision=G.GNSS_FP32),
        G.make_config(32, re=900.0, sc=0.7, sc_c=1.0, alpha=0.05, dt=1e-3, n_scalars=2),
    ]


def _init(G, cfg, seed):
    cdt = np.complex128 if cfg.precision == G.GNSS_FP64 else np.complex64
    f = G.jet_initial_state(cfg.nx, cfg.ny, cfg.nz, n_scalars=cfg.n_scalars, seed=seed, noise_kmax=4.0, amp=0.05,
                            dtype=cdt)
    return G.pack_state(f)


def _alone(G, cfg, packed, steps, choice=None):
    kw = {k: getattr(cfg, k) for k, _ in G.GnssConfig._fields_ if k not in ("nx", "ny", "nz")}
    with G.Context(nx=cfg.nx, ny=cfg.ny, nz=cfg.nz, **kw) as ctx:
        if choice is not None:   # autotuner choice: z variant + 4 * pass variant
            ctx.set_option(G.GNSS_OPT_ZVARIANT, choice & 3)
            ctx.set_option(G.GNSS_OPT_PVARIANT, choice >> 2)
        out = np.empty_like(packed)
        stats = np.zeros((steps, G.GNSS_NSTATS))
        ctx.run_host(packed, out, steps, True, stats)
    return out, stats[-1]


@pytest.mark.gpu
def test_ensemble_members_match_alone(torch_cuda):
    import gnss_b200 as G
    cfgs = _cfgs(G)
    init = [_init(G, c, seed=i) for i, c in enumerate(cfgs)]
    with G.Ensemble(cfgs, n_branches=3) as ens:
        for i, a in enumerate(init):
            ens.upload(i, a)
        ens.step(1)    # first (Euler) step, launched directly
        ens.step(5)    # captured into one graph
        ens.step(5)    # the same graph replayed
        assert ens.launches_per_step() == 6 * len(cfgs)
        got = []
        for i, a in enumerate(init):
            out = np.empty_like(a)
            ens.download(i, out)
            got.append((out, ens.stats(i)))
    for i, (c, a) in enumerate(zip(cfgs, init)):
        ref, rstats = _alone(G, c, a, 11)
        assert np.array_equal(got[i][0], ref), f"member {i} differs from the jet run alone"
        assert math.isclose(got[i][1]["ke"], rstats[0], rel_tol=1e-12)   # same state, other summation order


@pytest.mark.gpu
def test_ensemble_batched_groups_match_alone(torch_cuda):
    """With batching on, members of one geometry are stepped by one batched
    launch per stage; each keeps its own Reynolds and Schmidt numbers and
    time step, and ends bit-identical to the same jet run alone.  Groups
    (register kernels, which the batched form needs): 3 x 64^3 FP64,
    4 x 64 x 96 x 64 FP32 with two scalars, 2 x 64^3 FP64 with the colloid
    drift, and one 64^3 member of another drift coefficient (a group of its
    own)."""
    import gnss_b200 as G
    cfgs = [G.make_config(64, re=re, sc=sc, dt=dt) for re, sc, dt in ((500.0, 0.7, 2e-3), (900.0, 1.0, 1e-3),
                                                                       (1500.0, 2.0, 1.5e-3))]
    cfgs += [G.make_config(nx=64, ny=96, nz=64, re=re, sc=0.7, sc_c=scc, dt=1e-3, n_scalars=2,
                           precision=G.GNSS_FP32) for re, scc in ((700.0, 1.0), (1100.0, 2.0), (1600.0, 0.5),
                                                                  (2500.0, 1.0))]
    cfgs += [G.make_config(64, re=re, sc=0.7, sc_c=1.0, alpha=0.05, dt=2e-3, n_scalars=2) for re in (300.0, 600.0)]
    cfgs += [G.make_config(64, re=400.0, sc=0.7, sc_c=1.0, alpha=0.02, dt=2e-3, n_scalars=2)]
    init = [_init(G, c, seed=20 + i) for i, c in enumerate(cfgs)]
    with G.Ensemble(cfgs, n_branches=2) as ens:
        ens.set_batching(True)
        assert all(ens.batched(i) for i in range(len(cfgs)))
        for i, a in enumerate(init):
            ens.upload(i, a)
        ens.step(1)
        ens.step(4)
        ens.step(4)
        assert ens.launches_per_step() == 6 * 4   # four groups, six launches each
        got = []
        for i, a in enumerate(init):
            out = np.empty_like(a)
            ens.download(i, out)
            got.append(out)
    for i, (c, a) in enumerate(zip(cfgs, init)):
        ref, _ = _alone(G, c, a, 9)
        assert np.array_equal(got[i], ref), f"member {i} differs from the jet run alone"


@pytest.mark.gpu
def test_ensemble_batched_kept_nyquist_row(torch_cuda):
    """Groups whose dealiasing radius keeps the ky Nyquist row (96 x 64 x 96: alias_filter * 96 / 2 = 32 = ny / 2),
    where the velocity there is projected onto its Hermitian part at the start of each step, as the reference's round
    trip through physical space leaves it: 2 FP64 and 2 FP32 members, batched, end bit-identical to the same jets
    run alone."""
    import gnss_b200 as G
    cfgs = [G.make_config(nx=96, ny=64, nz=96, re=re, sc=0.7, sc_c=1.0, dt=1e-3, n_scalars=2, precision=p)
            for p in (G.GNSS_FP64, G.GNSS_FP32) for re in (600.0, 1300.0)]
    init = [_init(G, c, seed=40 + i) for i, c in enumerate(cfgs)]
    with G.Ensemble(cfgs, n_branches=2) as ens:
        ens.set_batching(True)
        assert all(ens.batched(i) for i in range(len(cfgs)))
        for i, a in enumerate(init):
            ens.upload(i, a)
        ens.step(1)
        ens.step(4)
        ens.step(4)
        got = []
        for i, a in enumerate(init):
            out = np.empty_like(a)
            ens.download(i, out)
            got.append(out)
    for i, (c, a) in enumerate(zip(cfgs, init)):
        ref, _ = _alone(G, c, a, 9)
        assert np.array_equal(got[i], ref), f"member {i} differs from the jet run alone"


@pytest.mark.gpu
def test_ensemble_autotune_keeps_results(torch_cuda):
    import gnss_b200 as G
    cfgs = [G.make_config(256, re=2000.0, dt=5e-4, precision=G.GNSS_FP32),
            G.make_config(32, re=2000.0, dt=5e-4, precision=G.GNSS_FP32)]
    init = [_init(G, c, seed=3 + i) for i, c in enumerate(cfgs)]
    with G.Ensemble(cfgs, n_branches=2) as ens:
        choices = ens.autotune(2)
        zallowed = (G.GNSS_VARIANT_REGISTER, G.GNSS_VARIANT_STAGED, G.GNSS_VARIANT_WARPSPEC)
        pallowed = (G.GNSS_VARIANT_REGISTER, G.GNSS_VARIANT_STAGED, G.GNSS_VARIANT_TENSOR)
        assert all(ch & 3 in zallowed and ch >> 2 in pallowed for ch in choices)
        for i, a in enumerate(init):
            ens.upload(i, a)
        ens.step(4)
        outs = []
        for i, a in enumerate(init):
            out = np.empty_like(a)
            ens.download(i, out)
            outs.append(out)
    for i, (c, a) in enumerate(zip(cfgs, init)):
        ref, _ = _alone(G, c, a, 4, choice=choices[i])
        assert np.array_equal(outs[i], ref), f"member {i}"


def _submit_all(G, srv, reqs):
    return [srv.submit(c, a, n) for c, a, n in reqs]


@pytest.mark.gpu
def test_server_result_same_alone_and_in_the_mix(torch_cuda):
    import gnss_b200 as G
    cfgs = _cfgs(G)
    target = (cfgs[1], _init(G, cfgs[1], seed=21), 37)
    others = [(c, _init(G, c, seed=40 + i), 25 + 7 * i) for i, c in enumerate(cfgs)]
    ref, rstats = _alone(G, *target)
    with G.Server(budget_bytes=8 << 30, max_active=8, steps_per_launch=10) as srv:
        rid = srv.submit(*target)
        srv.wait(rid)
        alone, s_alone, _ = srv.result(rid)
    with G.Server(budget_bytes=8 << 30, max_active=8, steps_per_launch=10) as srv:
        ids = _submit_all(G, srv, others[:3])
        rid = srv.submit(*target)
        ids += _submit_all(G, srv, others[3:])
        srv.wait(rid)
        mixed, s_mixed, times = srv.result(rid)
        for i in ids:
            srv.wait(i)
            srv.result(i)
        rep = srv.report()
    assert np.array_equal(alone, ref)
    assert np.array_equal(mixed, ref)
    assert s_alone["ke"] == s_mixed["ke"]
    assert math.isclose(s_alone["ke"], rstats[0], rel_tol=1e-12)
    assert times[0] <= times[1] <= times[2]
    assert rep["completed"] == 1 + len(others) and rep["failed"] == 0
    assert rep["active_max"] >= 2     # requests overlapped on the device


@pytest.mark.gpu
def test_server_admission_respects_budget(torch_cuda):
    import gnss_b200 as G
    cfg = G.make_config(48, re=1000.0, dt=1e-3)
    a = _init(G, cfg, seed=5)
    # one request reserves state + history + scratch; the budget fits two
    with G.Context(48) as probe:
        one = 8 * probe.field_bytes() + int(probe.lib.gnss_scratch_bytes(probe._h)) + probe.workspace_bytes()
    budget = int(2.5 * one) + (4 << 20)
    with G.Server(budget_bytes=budget, max_active=16, steps_per_launch=5) as srv:
        ids = [srv.submit(cfg, a, 12) for _ in range(6)]
        outs = []
        for i in ids:
            srv.wait(i)
            outs.append(srv.result(i)[0])
        rep = srv.report()
    assert rep["completed"] == 6
    assert rep["bytes_reserved_max"] <= budget
    assert 1 <= rep["active_max"] <= 2
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])


@pytest.mark.gpu
def test_server_rejects_what_can_never_fit(torch_cuda):
    import gnss_b200 as G
    cfg = G.make_config(64, re=1000.0, dt=1e-3)
    a = _init(G, cfg, seed=1)
    with G.Server(budget_bytes=1 << 20, max_active=4, steps_per_launch=5) as srv:
        rid = srv.submit(cfg, a, 3)
        srv.wait(rid)
        with pytest.raises(G.GnssError):
            srv.result(rid)
        assert srv.report()["failed"] == 1
