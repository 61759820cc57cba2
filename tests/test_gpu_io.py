"""States in the reference's files and the exact checkpoint.

gnss_save_state writes what save3Dfields writes (iofuncs.cu:360-432): each
field transformed to physical space (held to the oracle's inverse transform,
fftfuncs.cu:322-359, to round-off) without touching the state.
gnss_load_state reads such files back through the forward transform.  A
checkpoint restores state and history bit for bit, so a run resumed from it
ends bit-identical to the run that never stopped.
"""
import numpy as np
import pytest

from _util import rel_max, to_dev, to_host


def _state(G, torch, n, ns, precision=0, seed=2):
    cdt = np.complex128 if precision == 0 else np.complex64
    f = G.jet_initial_state(n, n_scalars=ns, seed=seed, noise_kmax=6.0, amp=0.05, dtype=cdt)
    return f, [to_dev(torch, a) for a in f]


@pytest.mark.gpu
def test_save_state_writes_physical_fields(torch_cuda, oracle, tmp_path):
    import gnss_b200 as G
    torch = torch_cuda
    n, ns = 32, 2
    f, st = _state(G, torch, n, ns)
    oc = oracle.cfg(n)
    with G.Context(n, n_scalars=ns) as ctx:
        ctx.de_alias(st)
        before = [to_host(t).copy() for t in st]
        ctx.save_state(st, tmp_path, 7)
        for q in range(len(st)):
            assert np.array_equal(to_host(st[q]), before[q]), "the state must not change"
    for q, var in enumerate("uvwzc"):
        phys = G.io_read_field(n, n, n, tmp_path / f"{var}.7")
        ref = before[q].copy()
        oracle.inverse(oc, ref)
        refp = ref.view(np.float64).reshape(n, n, -1)
        assert rel_max(phys[:, :, :n], refp[:, :, :n]) < 1e-13, var


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [(0, 1e-13), (1, 2e-6)])
def test_load_state_round_trip(torch_cuda, tmp_path, precision, tol):
    import gnss_b200 as G
    torch = torch_cuda
    n = 24
    _, st = _state(G, torch, n, 1, precision)
    with G.Context(n, precision=precision) as ctx:
        ctx.de_alias(st)
        ctx.save_state(st, tmp_path, 0)
        back = [torch.zeros_like(t) for t in st]
        ctx.load_state(tmp_path, 0, back)
        for a, b in zip(st, back):
            assert rel_max(to_host(b), to_host(a)) < tol


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", [0, 1], ids=["cnab2", "rk3if"])
def test_resume_from_checkpoint_is_exact(torch_cuda, tmp_path, scheme):
    import gnss_b200 as G
    torch = torch_cuda
    n, ns = 24, 2
    _, st = _state(G, torch, n, ns, seed=4)
    with G.Context(n, n_scalars=ns, re=800.0, dt=1e-3, scheme=scheme) as ctx:
        hi = [torch.zeros_like(st[0]) for _ in st] if scheme == 0 else None
        ctx.de_alias(st)
        for s in range(3):
            ctx.solver_ps(st, hi, euler=(s == 0))
        ctx.checkpoint_save(st, hi, 3, tmp_path / "ck.bin")
        for s in range(2):
            ctx.solver_ps(st, hi, euler=False)
        straight = [to_host(t).copy() for t in st]
        st2 = [torch.zeros_like(t) for t in st]
        hi2 = [torch.zeros_like(t) for t in st] if scheme == 0 else None
        assert ctx.checkpoint_load(tmp_path / "ck.bin", st2, hi2) == 3
        for s in range(2):
            ctx.solver_ps(st2, hi2, euler=False)
        for a, b in zip(straight, st2):
            assert np.array_equal(to_host(b), a)
    with G.Context(32, n_scalars=ns, scheme=scheme) as other:
        big = [other.empty_field() for _ in range(3 + ns)]
        with pytest.raises(G.GnssError):
            other.checkpoint_load(tmp_path / "ck.bin", big, None)
