"""Golden vectors from the reference's own CUDA step (test fixtures generator).

The reference has no tests or golden data of its own, so these fixtures pin
the oracle and the CUDA path to outputs of the unmodified reference code
(solver.cu, fftfuncs.cu, ... built by oracle/build_ref.sh into
oracle/_ref/<cfg>/refdrv with a generated dnsparams.h per configuration).

    python tests/golden/make_golden.py prepare <dir>   # seeded initial states -> <dir>/<case>/ic.bin
    python tests/golden/make_golden.py run <dir>       # on a GPU machine: refdrv run ... for each case
    python tests/golden/make_golden.py package <dir>   # -> tests/golden/<case>.npz

Cases (the build configuration fixes N, Re, Sc, Sc_c, alpha, dt; see
oracle/build_ref.sh): small grids with full states, and the 64^3 jet of
20 steps (statistics every step plus the low modes |m| <= 6 of the state).
"""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "gnss-1_b200"))

# case: (build cfg, n, n_scalars, seed, noise_kmax, steps, dumps, full state in fixture)
CASES = {
    "g12": ("g12", 12, 2, 11, 3.0, 3, [1, 3], True),
    "g16": ("g16", 16, 2, 12, 4.0, 4, [1, 4], True),
    "g16a": ("g16a", 16, 2, 13, 4.0, 3, [1, 3], True),
    "c64": ("c64", 64, 1, 0, 8.0, 20, [1, 20], False),
}
# parameters of each build configuration (must match oracle/build_ref.sh)
BUILD = {
    "g12": dict(re=200.0, sc=0.7, sc_c=1.0, alpha=0.0, dt=2.0e-3),
    "g16": dict(re=200.0, sc=0.7, sc_c=1.0, alpha=0.0, dt=2.0e-3),
    "g16a": dict(re=200.0, sc=0.7, sc_c=1.0, alpha=0.05, dt=2.0e-3),
    "c64": dict(re=1000.0, sc=0.7, sc_c=0.7, alpha=0.0, dt=1.0e-3),
    "c128": dict(re=1000.0, sc=0.7, sc_c=0.7, alpha=0.0, dt=1.0e-3),
    "c256": dict(re=3000.0, sc=0.7, sc_c=1.0, alpha=0.0, dt=5.0e-4),
    "c512": dict(re=5000.0, sc=0.7, sc_c=0.7, alpha=0.0, dt=2.5e-4),
}
LOW = 6


def initial_state(n: int, n_scalars: int, seed: int, kmax: float) -> list:
    import gnss_b200 as G
    f = G.jet_initial_state(n, n_scalars=n_scalars, seed=seed, noise_kmax=kmax, amp=0.05)
    if n_scalars == 1:
        f.append(np.zeros_like(f[0]))     # the reference always carries c (zero here)
    return f


def prepare(d: Path) -> None:
    for case, (cfg, n, ns, seed, km, steps, dumps, _) in CASES.items():
        cd = d / case
        cd.mkdir(parents=True, exist_ok=True)
        f = initial_state(n, ns, seed, km)
        with open(cd / "ic.bin", "wb") as fp:
            for a in f:
                fp.write(np.ascontiguousarray(a, dtype=np.complex128).tobytes())
        print("prepared", cd)


def run(d: Path) -> None:
    for case, (cfg, n, ns, seed, km, steps, dumps, _) in CASES.items():
        cd = d / case
        exe = ROOT / "oracle" / "_ref" / cfg / "refdrv"
        cmd = [str(exe), "run", str(cd / "ic.bin"), str(steps), str(cd), ",".join(map(str, dumps))]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
        (cd / "refdrv.log").write_text(r.stdout + r.stderr)
        if r.returncode != 0:
            raise SystemExit(f"{case}: refdrv failed ({r.returncode}): {r.stderr[-500:]}")
        print(case, r.stdout.strip().splitlines()[-1])
        full = CASES[case][7]
        if not full:   # keep what comes back small: only the state dumps and the statistics
            for p in [cd / "ic.bin", *cd.glob("rhsold_*.bin")]:
                p.unlink()


def _read_state(p: Path, n: int) -> np.ndarray:
    a = np.fromfile(p, dtype=np.complex128)
    return a.reshape(5, n, n, n // 2 + 1)


def _low(a: np.ndarray, n: int) -> np.ndarray:
    idx = np.r_[0:LOW + 1, n - LOW:n]
    return a[:, idx][:, :, idx][:, :, :, :LOW + 1]


def package(d: Path) -> None:
    out = Path(__file__).resolve().parent
    for case, (cfg, n, ns, seed, km, steps, dumps, full) in CASES.items():
        cd = d / case
        stats = np.fromfile(cd / "stats.bin", dtype=np.float64).reshape(steps + 1, 7)
        rec = dict(case=np.array(case), cfg=np.array(json.dumps(dict(BUILD[cfg], n=n, n_scalars=ns, seed=seed,
                                                                      noise_kmax=km, steps=steps, dumps=dumps))),
                   stats=stats)
        for s in dumps:
            st = _read_state(cd / f"state_{s}.bin", n)
            if full:
                rec[f"state_{s}"] = st
                rec[f"rhsold_{s}"] = _read_state(cd / f"rhsold_{s}.bin", n)
            else:
                rec[f"low_{s}"] = _low(st, n)
                rec[f"norm_{s}"] = np.linalg.norm(st.reshape(5, -1), axis=1)
        np.savez_compressed(out / f"{case}.npz", **rec)
        print("wrote", out / f"{case}.npz")


if __name__ == "__main__":
    if len(sys.argv) != 3 or sys.argv[1] not in ("prepare", "run", "package"):
        raise SystemExit(__doc__)
    {"prepare": prepare, "run": run, "package": package}[sys.argv[1]](Path(sys.argv[2]))
