"""The reference's initial temporal jet (gnss_initial_jet) against the
reference's own generator.

tests/golden/ic_<cfg>.npz hold the spectral state that the reference program
builds before its time loop (initializeJet with generateNoise's rand() stream,
forward transforms, deAlias: main.cu:139-156), dumped by oracle/refdriver.cu
from the unmodified sources (tests/golden/make_ic_golden.py).  The library
draws the same random numbers in the same order and must reproduce the state
to the transforms' round-off: 1e-12 relative L2 per field.
"""
import math
from pathlib import Path

import numpy as np
import pytest

from _util import rel_l2, to_host

GOLD = Path(__file__).resolve().parent / "golden"


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", ["i16", "i32"])
def test_initial_jet_matches_reference(torch_cuda, cfg):
    import gnss_b200 as G
    torch = torch_cuda
    z = np.load(GOLD / f"ic_{cfg}.npz")
    n = int(z["n"])
    ref = z["fields"]
    with G.Context(n, n_scalars=2) as ctx:
        st = [ctx.empty_field() for _ in range(5)]
        ctx.initial_jet(st, h=float(z["h"]), theta=float(z["theta"]), theta_c=float(z["theta_c"]),
                        pert_amp=float(z["pert_amp"]))
        got = [to_host(t) for t in st]
        stats = ctx.stats(st)
    for q in range(5):
        err = rel_l2(got[q], ref[q])
        assert err < 1e-12, f"field {q}: rel L2 {err:.3e}"
    assert stats["ke"] > 0 and math.isfinite(stats["ke"])


@pytest.mark.gpu
def test_initial_jet_fp32_and_one_scalar(torch_cuda):
    import gnss_b200 as G
    torch = torch_cuda
    z = np.load(GOLD / "ic_i32.npz")
    ref = z["fields"]
    with G.Context(32, n_scalars=1, precision=G.GNSS_FP32) as ctx:
        st = [ctx.empty_field() for _ in range(4)]
        ctx.initial_jet(st, h=1.0, theta=0.05, theta_c=0.05, pert_amp=0.05)
        for q in range(4):
            assert rel_l2(to_host(st[q]).astype(np.complex128), ref[q]) < 2e-6
