"""The CUDA path against the reference's own CUDA code.

1. Against the committed golden vectors (tests/golden, outputs of the
   unmodified reference solver_ps): full states after 1 and several steps.
2. Live, where the reference build of oracle/build_ref.sh is present
   (oracle/_ref/<cfg>/refdrv): the 256^3 two-scalar jet (Re 3000, Sc 0.7 and
   1.0, noise |k| <= 16, dt 5e-4): relative L2 of every field after one step
   <= 1e-12, and kinetic energy, dissipation, scalar dissipation and scalar
   variance within 1e-9 over 200 steps.
"""
import json
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

from _util import rel_l2, to_dev, to_host

ROOT = Path(__file__).resolve().parents[1]
GOLD = ROOT / "tests" / "golden"


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["g12", "g16", "g16a", "c64"])
def test_cuda_step_matches_reference_goldens(torch_cuda, case):
    import gnss_b200 as G
    from golden.make_golden import _low, initial_state
    torch = torch_cuda
    z = np.load(GOLD / f"{case}.npz")
    m = json.loads(str(z["cfg"]))
    n, ns = m["n"], m["n_scalars"]
    f = initial_state(n, ns, m["seed"], m["noise_kmax"])[:3 + ns]
    with G.Context(n, re=m["re"], sc=m["sc"], sc_c=m["sc_c"], alpha=m["alpha"], dt=m["dt"], n_scalars=ns) as ctx:
        st = [to_dev(torch, a) for a in f]
        hi = [torch.zeros_like(st[0]) for _ in st]
        ctx.de_alias(st)
        for s in range(1, m["steps"] + 1):
            ctx.solver_ps(st, hi, euler=(s == 1))
            stats = ctx.stats(st)
            for i, k in enumerate(G.STAT_NAMES):
                ref = z["stats"][s][i]
                assert abs(stats[k] - ref) <= 1e-11 * abs(ref) + 1e-300, (s, k, stats[k], ref)
            if s in m["dumps"]:
                got = np.stack([to_host(t) for t in st])
                tol = 1e-12 if s == 1 else 1e-11
                if f"state_{s}" in z:
                    for q in range(3 + ns):
                        assert rel_l2(got[q], z[f"state_{s}"][q]) < tol
                        assert rel_l2(to_host(hi[q]), z[f"rhsold_{s}"][q]) < tol
                else:
                    full = np.concatenate([got, np.zeros((5 - got.shape[0],) + got.shape[1:], got.dtype)])
                    lo = _low(full, n)
                    for q in range(3 + ns):
                        assert rel_l2(lo[q], z[f"low_{s}"][q]) < tol


def _refdrv(cfg):
    p = ROOT / "oracle" / "_ref" / cfg / "refdrv"
    if not p.exists():
        pytest.skip(f"reference build {p} not present (oracle/build_ref.sh)")
    return p


@pytest.mark.gpu
def test_live_reference_256_two_scalars(torch_cuda):
    """Config: 256^3, Re 3000, Sc 0.7 / 1.0, noise |k| <= 16, dt 5e-4, 200 steps."""
    import gnss_b200 as G
    from golden.make_golden import BUILD, initial_state
    torch = torch_cuda
    exe = _refdrv("c256")
    n, ns, steps = 256, 2, 200
    b = BUILD["c256"]
    f = initial_state(n, ns, 0, 16.0)
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        with open(td / "ic.bin", "wb") as fp:
            for a in f:
                fp.write(np.ascontiguousarray(a).tobytes())
        r = subprocess.run([str(exe), "run", str(td / "ic.bin"), str(steps), str(td), "1"], capture_output=True,
                           text=True, timeout=900)
        assert r.returncode == 0, r.stderr[-2000:]
        ref_stats = np.fromfile(td / "stats.bin", dtype=np.float64).reshape(steps + 1, 7)
        ref1 = np.fromfile(td / "state_1.bin", dtype=np.complex128).reshape(5, n, n, n // 2 + 1)
    with G.Context(n, re=b["re"], sc=b["sc"], sc_c=b["sc_c"], alpha=b["alpha"], dt=b["dt"], n_scalars=ns) as ctx:
        st = [to_dev(torch, a) for a in f]
        hi = [torch.zeros_like(st[0]) for _ in st]
        ctx.de_alias(st)
        worst = 0.0
        for s in range(1, steps + 1):
            ctx.solver_ps(st, hi, euler=(s == 1))
            if s == 1:
                for q in range(5):
                    e = rel_l2(to_host(st[q]), ref1[q])
                    assert e < 1e-12, (q, e)
            stats = ctx.stats(st)
            for k, i in (("ke", 0), ("eps", 2), ("chi_s", 3), ("chi_c", 4), ("var_s", 5), ("var_c", 6)):
                rel = abs(stats[k] - ref_stats[s][i]) / abs(ref_stats[s][i])
                worst = max(worst, rel)
                assert rel < 1e-9, (s, k, stats[k], ref_stats[s][i])
    print(f"worst statistic deviation over {steps} steps: {worst:.2e}")


# Reference builds of configurations beside the cubic 2/3-rule jets (oracle/build_ref.sh):
#   n64y32  64 x 32 x 64: the dealiasing radius alias_filter * NX / 2 (solver.cu:29-31) keeps the ky Nyquist row,
#           where the velocity's round trip through physical space (solver.cu:707-722, :743-750) leaves only the
#           Hermitian part of the kz = 0 plane;
#   a64     64^3 with the reference's 15/32 truncation (dnsparams.h:91; alias_filter 15/16): kept boxes of 61 of 64
#           rows and 31 of 33 kz modes;
#   l64     64^3 in a (4 pi)^3 box: wavenumbers 2 pi / L = 1/2 (initialize.cu:686-689) and the radius scaled with them;
#   r96a    96^3 (radix 3: the lane-shuffle register kernels) with the colloid term alpha = 0.05 (14 physical
#           quantities in the z kernel);
#   m48     48 x 96 x 64 (mixed radix, nx < ny);
#   f48     48^3 with alias_filter 1 (no truncation): every Nyquist row, column and plane is kept, so the Hermitian
#           projection of the velocity acts on the kx and ky Nyquist lines of the kz = 0 plane and on the kz = 24 plane.
LIVE_CONFIGS = [("n64y32", (64, 32, 64), 2.0 / 3.0, 2.0, 0.0), ("a64", (64, 64, 64), 15.0 / 16.0, 2.0, 0.0),
                ("l64", (64, 64, 64), 2.0 / 3.0, 4.0, 0.0), ("r96a", (96, 96, 96), 2.0 / 3.0, 2.0, 0.05),
                ("m48", (48, 96, 64), 2.0 / 3.0, 2.0, 0.0), ("f48", (48, 48, 48), 1.0, 2.0, 0.0)]


@pytest.mark.gpu
@pytest.mark.parametrize("cfg,shape,alias,lpi,alpha", LIVE_CONFIGS, ids=[c[0] for c in LIVE_CONFIGS])
def test_live_reference_configs(torch_cuda, oracle, cfg, shape, alias, lpi, alpha):
    """The reference program, Re 800, Sc 0.7 / 1.0, dt 1e-3, two scalars: this library and the oracle both match its
    states after each of 4 steps (1e-12 after the first, 1e-11 after the others)."""
    import gnss_b200 as G
    torch = torch_cuda
    exe = _refdrv(cfg)
    nx, ny, nz = shape
    steps = 4
    L = lpi * np.pi
    kw = dict(lx=L, ly=L, lz=L, re=800.0, sc=0.7, sc_c=1.0, dt=1e-3, alias_filter=alias, alpha=alpha)
    f = G.jet_initial_state(nx, ny, nz, lx=L, ly=L, lz=L, n_scalars=2, seed=1, noise_kmax=6.0 * 2.0 / lpi,
                            amp=0.05)
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        with open(td / "ic.bin", "wb") as fp:
            for a in f:
                fp.write(np.ascontiguousarray(a).tobytes())
        r = subprocess.run([str(exe), "run", str(td / "ic.bin"), str(steps), str(td), "1,2,3,4"],
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        ref = [np.fromfile(td / f"state_{s}.bin", dtype=np.complex128).reshape(5, ny, nx, nz // 2 + 1)
               for s in range(1, steps + 1)]
    oc = oracle.cfg(nx=nx, ny=ny, nz=nz, **kw)
    o = [a.copy() for a in f]
    ro = [np.zeros_like(f[0]) for _ in range(5)]
    with G.Context(nx=nx, ny=ny, nz=nz, n_scalars=2, **kw) as ctx:
        st = [to_dev(torch, a) for a in f]
        hi = [torch.zeros_like(st[0]) for _ in st]
        ctx.de_alias(st)
        for s in range(steps):
            ctx.solver_ps(st, hi, euler=(s == 0))
            oracle.step_cnab2(oc, o, ro, euler=(s == 0))
            tol = 1e-12 if s == 0 else 1e-11
            for q in range(5):
                e_lib = rel_l2(to_host(st[q]), ref[s][q])
                e_orc = rel_l2(o[q], ref[s][q])
                assert e_lib < tol, (s + 1, q, "library", e_lib)
                assert e_orc < tol, (s + 1, q, "oracle", e_orc)


@pytest.mark.gpu
@pytest.mark.parametrize("cfg,n,ns,steps", [("g16a", 16, 2, 4), ("c64", 64, 1, 5)])
def test_dropin_shim_matches_reference_program(torch_cuda, cfg, n, ns, steps):
    """The same driver linked two ways: the reference's solver.o + fftfuncs.o
    (refdrv) and the B200 library through the reference-ABI shim
    (refdrv_gnss, gnss-1_b200/refabi/refabi.cu).  States and statistics agree."""
    from golden.make_golden import initial_state
    ref = _refdrv(cfg)
    new = ref.parent / "refdrv_gnss"
    if not new.exists():
        pytest.skip("drop-in build not present")
    f = initial_state(n, ns, 21, min(8.0, n / 4))
    dumps = f"1,{steps}"
    out = {}
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        with open(td / "ic.bin", "wb") as fp:
            for a in f:
                fp.write(np.ascontiguousarray(a).tobytes())
        for name, exe in (("ref", ref), ("new", new)):
            d = td / name
            d.mkdir()
            r = subprocess.run([str(exe), "run", str(td / "ic.bin"), str(steps), str(d), dumps],
                               capture_output=True, text=True, timeout=600)
            assert r.returncode == 0, r.stderr[-2000:]
            out[name] = {
                "stats": np.fromfile(d / "stats.bin", dtype=np.float64).reshape(steps + 1, 7),
                "s1": np.fromfile(d / "state_1.bin", dtype=np.complex128).reshape(5, -1),
                "sN": np.fromfile(d / f"state_{steps}.bin", dtype=np.complex128).reshape(5, -1),
                "hN": np.fromfile(d / f"rhsold_{steps}.bin", dtype=np.complex128).reshape(5, -1),
            }
    for q in range(3 + ns):
        assert rel_l2(out["new"]["s1"][q], out["ref"]["s1"][q]) < 1e-12
        assert rel_l2(out["new"]["sN"][q], out["ref"]["sN"][q]) < 1e-11
        assert rel_l2(out["new"]["hN"][q], out["ref"]["hN"][q]) < 1e-11
    a, b = out["new"]["stats"], out["ref"]["stats"]
    mask = b != 0
    assert np.all(np.abs(a[mask] - b[mask]) <= 1e-10 * np.abs(b[mask]))
