"""Graph and factor files: IJV text as src/IO.jl reads and writes it, and the
binary LDLinv file of the C ABI (host only, no device needed)."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

import acgpu
from acgpu import generators as G
from acgpu import io as aio
from acgpu._lib import AcgError


def _dense(a):
    return np.asarray(sp.csc_matrix(a).todense())


def test_read_graph_examples(tmp_path):
    # the two examples of read_graph's documentation (src/IO.jl:1-27)
    f1 = tmp_path / "k3.txt"
    f1.write_text("1 2\n1 3\n2 3\n")
    assert np.array_equal(_dense(aio.read_graph(f1)), np.ones((3, 3)) - np.eye(3))
    f2 = tmp_path / "path.txt"
    f2.write_text("1, 2, 1.5\n2, 3, 2.5\n")
    want = np.array([[0, 1.5, 0], [1.5, 0, 2.5], [0, 2.5, 0]])
    assert np.array_equal(_dense(aio.read_graph(f2)), want)


def test_read_graph_sums_repeated_edges(tmp_path):
    f = tmp_path / "dup.txt"
    f.write_text("1\t2\t1.0\n2 1 0.5\n1 2 2.0\n3 4 1.0\n")
    a = _dense(aio.read_graph(f))
    assert a[0, 1] == a[1, 0] == 3.5 and a[2, 3] == 1.0 and a.shape == (4, 4)


@pytest.mark.parametrize("text", ["1 2 3 4\n", "1 2\n1 2 1.0\n", "0 1\n", "1.5 2\n", ""])
def test_read_graph_rejects_malformed(tmp_path, text):
    f = tmp_path / "bad.txt"
    f.write_text(text)
    with pytest.raises(ValueError):
        aio.read_graph(f)


def test_ijv_round_trip_is_exact(tmp_path):
    a = G.grid2(7, weights="loguniform", seed=3)
    a = sp.csc_matrix(a)
    a.data *= np.pi * 1e-7  # values that need all 17 significant digits
    f = tmp_path / "g.txt"
    aio.writeIJV(f, a)
    lines = f.read_text().splitlines()
    assert len(lines) == sp.triu(a).nnz
    i, j, _ = lines[0].split(",")
    assert int(i) <= int(j)
    b = aio.read_graph(f)
    assert (b != a).nnz == 0


def test_write_formats_like_julia(tmp_path):
    a = sp.csc_matrix(np.array([[0, 1.0, 2e-7], [1.0, 0, 0.5], [2e-7, 0.5, 0]]))
    f = tmp_path / "g.txt"
    aio.write_ijv(f, a)
    assert f.read_text().splitlines() == ["1,2,1.0", "1,3,2.0e-7", "2,3,0.5"]


def test_ldlinv_file_round_trip(tmp_path):
    a = G.grid3(9, weights="loguniform", seed=11)
    acgpu.seed(5)
    f = acgpu.approx_chol(a)
    fn = tmp_path / "f.ldli"
    aio.save_ldlinv(fn, f)
    assert fn.stat().st_size == 32 + 8 * (3 * f.n - 1 + 2 * f.nnz)
    g = aio.load_ldlinv(fn)
    for k in ("col", "colptr", "rowval", "fval", "d"):
        assert np.array_equal(getattr(f, k), getattr(g, k)), k
        assert getattr(g, k).dtype == getattr(f, k).dtype


def _corrupt(src, dst, offset, data):
    b = bytearray(src.read_bytes())
    if offset is None:
        b = b[:-8]
    else:
        b[offset:offset + len(data)] = data
    dst.write_bytes(bytes(b))


def test_ldlinv_file_rejects_damage(tmp_path):
    a = G.grid2(6, seed=2)
    acgpu.seed(1)
    f = acgpu.approx_chol(a)
    good = tmp_path / "good.ldli"
    aio.save_ldlinv(good, f)
    n, F = f.n, f.nnz
    colptr_at = 32 + 8 * (n - 1)
    rowval_at = colptr_at + 8 * n
    cases = {
        "magic": (0, b"XCGLDLI1"),
        "truncated": (None, b""),
        "index base": (24, np.int64(0).tobytes()),
        "colptr start": (colptr_at, np.int64(2).tobytes()),
        "colptr order": (colptr_at + 8, np.int64(F + 5).tobytes()),
        "row id": (rowval_at, np.int64(n + 1).tobytes()),
    }
    for name, (off, data) in cases.items():
        bad = tmp_path / f"{name}.ldli"
        _corrupt(good, bad, off, data)
        with pytest.raises(AcgError) as e:
            aio.load_ldlinv(bad)
        assert e.value.code == -1, name
    with pytest.raises(AcgError):
        aio.load_ldlinv(tmp_path / "missing.ldli")
