"""Reference file formats (iofuncs.cu) written and read by the library, byte
for byte against files the reference's own writers produced
(tests/golden/io_g12/, made by tests/golden/make_io_golden.py from
write3Dfields_mgpu, writexyfields, writexzfields, writeyzfields, writeStats
and writeYprofs on a synthetic 12^3 field).  Host code only: no GPU needed.
"""
from pathlib import Path

import numpy as np
import pytest

GOLD = Path(__file__).resolve().parent / "golden" / "io_g12"
N = 12


@pytest.fixture(scope="module")
def G():
    import gnss_b200
    gnss_b200.load_library()
    return gnss_b200


@pytest.fixture(scope="module")
def field():
    return np.fromfile(GOLD / "input.bin", dtype=np.float64).reshape(N, N, 2 * (N // 2 + 1))


def _same(a: Path, b: Path):
    assert a.read_bytes() == b.read_bytes(), f"{a.name} differs from the reference's {b}"


def test_3d_field_matches_reference_writer(G, field, tmp_path):
    G.io_write_field(field, N, tmp_path / "u.3")
    _same(tmp_path / "u.3", GOLD / "u.3")


@pytest.mark.parametrize("plane,index,name", [(0, 2, "u_xy.3"), (1, 1, "u_xz.3"), (2, 4, "u_yz.3")])
def test_slices_match_reference_writers(G, field, tmp_path, plane, index, name):
    G.io_write_slice(field, N, plane, index, tmp_path / name)
    _same(tmp_path / name, GOLD / "vis" / name)


def test_stats_records_and_profile_match(G, tmp_path):
    for i, v in enumerate((1.5, 2.5, -0.125)):
        G.io_write_stat(tmp_path / "KE", v, append=i > 0)
    _same(tmp_path / "KE", GOLD / "stats" / "KE")
    prof = np.fromfile(GOLD / "prof.bin", dtype=np.float64)
    G.io_write_profile(prof, tmp_path / "u_mean.3")
    _same(tmp_path / "u_mean.3", GOLD / "Yprofs" / "u_mean.3")


def test_read_field_of_reference_file(G, field):
    got = G.io_read_field(N, N, N, GOLD / "u.3")
    assert np.array_equal(got[:, :, :N], field[:, :, :N])
    assert not got[:, :, N:].any()      # padding untouched (zero here)


def test_read_field_rejects_wrong_size(G):
    with pytest.raises(G.GnssError):
        G.io_read_field(N, N, 2 * N, GOLD / "u.3")
    with pytest.raises(G.GnssError):
        G.io_read_field(N, N, N, GOLD / "missing.3")


def test_bad_slice_arguments_are_rejected(G, field, tmp_path):
    with pytest.raises(G.GnssError):
        G.io_write_slice(field, N, 0, N, tmp_path / "x")      # z index out of range
    with pytest.raises(G.GnssError):
        G.io_write_slice(field, N, 3, 0, tmp_path / "x")      # no such plane
