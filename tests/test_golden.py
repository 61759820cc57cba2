"""The oracle against golden vectors produced by the reference's own CUDA code.

tests/golden/<case>.npz hold the outputs of solver_ps (solver.cu:700-765) run
by oracle/refdriver.cu on the unmodified reference sources (see
tests/golden/make_golden.py): full spectral states and AB2 histories after
given steps for small grids, and statistics every step plus low modes for the
64^3 jet of 20 steps.  The oracle must agree to 1e-12 (it does to ~1e-15).
"""
import json
from pathlib import Path

import numpy as np
import pytest

from _util import rel_l2

GOLD = Path(__file__).resolve().parent / "golden"
CASES = ["g12", "g16", "g16a", "c64"]


def _load(case):
    z = np.load(GOLD / f"{case}.npz")
    return z, json.loads(str(z["cfg"]))


def _initial(meta):
    from golden.make_golden import initial_state
    return initial_state(meta["n"], meta["n_scalars"], meta["seed"], meta["noise_kmax"])


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference_goldens(oracle, case):
    from golden.make_golden import _low
    z, m = _load(case)
    n, ns = m["n"], m["n_scalars"]
    oc = oracle.cfg(n, re=m["re"], sc=m["sc"], sc_c=m["sc_c"], alpha=m["alpha"], dt=m["dt"])
    f = _initial(m)
    for a in f:
        oracle.dealias(oc, a)                      # main.cu:156
    r = [np.zeros_like(f[0]) for _ in range(5)]
    names = oracle.STAT_NAMES
    st = oracle.stats(oc, f)
    for i, k in enumerate(names):
        assert abs(st[k] - z["stats"][0][i]) <= 1e-12 * abs(z["stats"][0][i]) + 1e-300
    for s in range(1, m["steps"] + 1):
        oracle.step_cnab2(oc, f, r, euler=(s == 1))
        st = oracle.stats(oc, f)
        for i, k in enumerate(names):
            ref = z["stats"][s][i]
            assert abs(st[k] - ref) <= 1e-12 * abs(ref) + 1e-300, (s, k, st[k], ref)
        if s in m["dumps"]:
            if f"state_{s}" in z:
                for q in range(3 + ns):
                    assert rel_l2(f[q], z[f"state_{s}"][q]) < 1e-12
                    assert rel_l2(r[q], z[f"rhsold_{s}"][q]) < 1e-12
            else:
                lo = _low(np.stack(f), n)
                for q in range(3 + ns):
                    assert rel_l2(lo[q], z[f"low_{s}"][q]) < 1e-12
                nr = np.linalg.norm(np.stack(f).reshape(5, -1), axis=1)
                assert np.allclose(nr[:3 + ns], z[f"norm_{s}"][:3 + ns], rtol=1e-12)


def test_golden_inputs_are_reproducible():
    """The fixtures' initial states come from the seeded generator: regenerate and
    check the reference's step-0 statistics."""
    z, m = _load("g16")
    import oracle as O
    f = _initial(m)
    oc = O.cfg(m["n"], re=m["re"], sc=m["sc"], sc_c=m["sc_c"], alpha=m["alpha"], dt=m["dt"])
    for a in f:
        O.dealias(oc, a)
    st = O.stats(oc, f)
    assert abs(st["ke"] - z["stats"][0][0]) < 1e-14 * z["stats"][0][0]
