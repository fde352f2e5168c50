"""Ranged and big-endian configuration transfers (ymflow_upload_sites /
ymflow_download_sites) against whole-field transfers."""
import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

N4 = (4, 4, 6, 4)


def field():
    rng = np.random.default_rng(5)
    return rng.standard_normal((N4[3], N4[2], N4[1], N4[0], 4, 18))


@pytest.mark.parametrize("precision", ["fp64", "fp32_18", "fp32_12"])
def test_ragged_ranges_equal_whole_upload(precision):
    from latticeyangmills_b200 import GluonField

    U = field()
    flat = U.reshape(-1, 72)
    V = flat.shape[0]
    with GluonField(N4, precision) as f:
        f.upload(U)
        whole = f.download()
        for a, b in [(0, 100), (100, 101), (101, V)]:
            f.upload_sites(flat[a:b], a)
        ranged = f.download()
        parts = np.concatenate([f.download_sites(a, b - a).reshape(-1) for a, b in [(0, 7), (7, 300), (300, V)]])
    assert np.array_equal(ranged, whole)
    assert np.array_equal(parts, whole.reshape(-1))
    if precision == "fp64":
        assert np.array_equal(whole, U)


def test_big_endian_reversal_on_device():
    from latticeyangmills_b200 import GluonField

    U = field()
    flat = U.reshape(-1, 72)
    V = flat.shape[0]
    with GluonField(N4, "fp64") as f:
        f.upload_sites(flat[:50].astype(">f8"), 0)
        f.upload_sites(flat[50:].astype(">f8"), 50)
        assert np.array_equal(f.download(), U)
        be = f.download_sites(0, V, big_endian=True)
    assert be.dtype == np.dtype(">f8")
    assert be.tobytes() == U.astype(">f8").tobytes()


def test_load_conf_streams_big_endian_file(tmp_path):
    from latticeyangmills_b200 import GluonField, read_conf, write_conf

    n = (4, 4, 4, 4)
    U = read_conf(GOLDEN / "g4_expiah.bin", n)
    write_conf(tmp_path / "be.bin", U, big_endian=True)
    with GluonField(n, "fp64") as f:
        f.load_conf(tmp_path / "be.bin", big_endian=True, chunk_sites=37)
        got = f.download()
        o = f.observables()
    assert np.array_equal(got, U)
    assert np.isfinite(o.plaq)


def test_ranges_are_checked():
    from latticeyangmills_b200 import GluonField, YmflowError, load

    U = field().reshape(-1, 72)
    V = U.shape[0]
    with GluonField(N4, "fp64") as f:
        with pytest.raises(YmflowError):
            f.download_sites(0, 1)  # nothing loaded yet
        with pytest.raises(YmflowError):
            f.upload_sites(U[:10], V - 5)
        with pytest.raises(YmflowError):
            f.upload_sites(U[:10], -1)
        assert load().ymflow_upload_sites(f.ctx, U.ctypes.data, 0, 1, 2) != 0
        f.upload_sites(U[:0], 0)  # empty range: no-op


def test_load_file_slabs_and_errors(tmp_path):
    """ymflow_load_file: each slab reads only its part of the file; a file of
    the wrong size is refused."""
    from latticeyangmills_b200 import GluonField, YmflowError, write_conf

    n = (8, 4, 4, 6)
    U = field6 = np.random.default_rng(3).standard_normal((n[3], n[2], n[1], n[0], 4, 18))
    write_conf(tmp_path / "c.bin", U)
    with GluonField(n, "fp64") as f:
        f.load_conf(tmp_path / "c.bin", chunk_sites=50)
        assert np.array_equal(f.download(), U)
    parts = []
    for t0, nt in ((0, 2), (2, 3), (5, 1)):
        with GluonField.slab(n, t0, nt, "fp64") as s:
            s.load_conf(tmp_path / "c.bin", chunk_sites=40)
            parts.append(s.download())
    assert np.array_equal(np.concatenate(parts), field6)
    (tmp_path / "short.bin").write_bytes((tmp_path / "c.bin").read_bytes()[:-8])
    with GluonField(n, "fp64") as f:
        with pytest.raises(YmflowError):
            f.load_conf(tmp_path / "short.bin")
        with pytest.raises(YmflowError):
            f.load_conf(tmp_path / "missing.bin")
