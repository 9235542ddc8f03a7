"""Connectome loading and layouts against the reference's own objects, on CPU.

The upstream-table loader (lab/flybrain/data.py:221-259): small tables in the
upstream column layout, with repeated (pre, post) pairs and a pair that sums
to zero, loaded by ``from_parquet`` and compared with the reference's object
for the same table -- a coalesced torch sparse COO ``W[post, pre]`` -- through
``from_weights``, and with a dense sum.  The CSR by postsynaptic neuron of the
graded-spike mode, compared with torch's CSR of ``W`` (the reference's csrmv).
"""

import numpy as np
import pyarrow as pa
import pyarrow.parquet as pq
import pytest
import torch

import fis.connectome as C


def write_table(path, pre, post, val):
    pq.write_table(pa.table({
        C.UPSTREAM_PRE: pa.array(pre, pa.int64()),
        C.UPSTREAM_POST: pa.array(post, pa.int64()),
        C.UPSTREAM_VALUE: pa.array(val, pa.float32()),
    }), str(path))


def sample(seed, n=500, e=6000):
    rng = np.random.default_rng(seed)
    pre = rng.integers(0, n, e)
    post = rng.integers(0, n, e)
    val = rng.integers(-40, 41, e).astype(np.float32)  # zeros and repeats included
    pre = np.append(pre, [7, 7])  # one pair that sums to zero
    post = np.append(post, [9, 9])
    val = np.append(val, [5.0, -5.0]).astype(np.float32)
    return n, pre, post, val


def same(a, b):
    return (a.n == b.n and np.array_equal(a.row_ptr, b.row_ptr)
            and np.array_equal(a.col, b.col) and np.array_equal(a.cnt, b.cnt))


@pytest.fixture(autouse=True)
def cache_dir(tmp_path, monkeypatch):
    monkeypatch.setenv("FIS_CACHE", str(tmp_path / "cache"))
    return tmp_path / "cache"


def test_parquet_equals_the_reference_coo(tmp_path, cache_dir):
    n, pre, post, val = sample(0)
    f = tmp_path / "conn.parquet"
    write_table(f, pre, post, val)
    got = C.from_parquet(f, n=n)
    w = torch.sparse_coo_tensor(torch.from_numpy(np.vstack([post, pre])),
                                torch.from_numpy(val), (n, n)).coalesce()
    assert same(got, C.from_weights(w))
    dense = np.zeros((n, n), np.int64)
    np.add.at(dense, (pre, post), val.astype(np.int64))
    rows = np.repeat(np.arange(n), np.diff(got.row_ptr))
    assert np.array_equal(dense[rows, got.col], got.cnt)
    assert got.col.size == np.count_nonzero(dense) and (got.cnt != 0).all()
    assert int(((rows == 7) & (got.col == 9)).sum()) == (1 if dense[7, 9] else 0)
    # the second load comes from the packed-CSR cache and is the same
    assert len(list(cache_dir.glob("upstream_*.npz"))) == 1
    assert same(C.from_parquet(f, n=n), got)


def test_cache_follows_the_file(tmp_path, cache_dir):
    n, pre, post, val = sample(1)
    f = tmp_path / "conn.parquet"
    write_table(f, pre, post, val)
    a = C.from_parquet(f, n=n)
    write_table(f, pre[:-500], post[:-500], val[:-500])  # a new table, same path
    b = C.from_parquet(f, n=n)
    assert not same(a, b)
    assert same(b, C.from_parquet(f, n=n, cache=False))


def test_upstream_folder_takes_n_from_the_completeness_csv(tmp_path):
    n, pre, post, val = sample(2, n=321, e=2000)
    write_table(tmp_path / C.UPSTREAM_CONN_FILE, pre, post, val)
    with open(tmp_path / C.UPSTREAM_COMP_FILE, "w") as fh:
        fh.write(",root_id,Completed\n")
        for i in range(n):
            fh.write('%d,"72%012d",True\n' % (i, i))
    c = C.from_upstream(tmp_path)
    assert c.n == n
    assert same(c, C.from_parquet(tmp_path / C.UPSTREAM_CONN_FILE, n=n, cache=False))


def test_refusals(tmp_path):
    n, pre, post, val = sample(3, n=100, e=500)
    f = tmp_path / "frac.parquet"
    v = val.copy()
    v[3] = 2.5
    write_table(f, pre, post, v)
    with pytest.raises(C.ConnectomeError, match="integral"):
        C.from_parquet(f, n=n, cache=False)
    g = tmp_path / "range.parquet"
    p2 = pre.copy()
    p2[0] = n
    write_table(g, p2, post, val)
    with pytest.raises(C.ConnectomeError, match="outside"):
        C.from_parquet(g, n=n, cache=False)
    with pytest.raises(C.ConnectomeError, match="n="):
        C.from_parquet(g, cache=False)


def test_by_post_is_torchs_csr_of_w():
    """The graded mode's pull layout is torch's CSR of W[post, pre], the one the
    reference's csrmv reads (sim.py:357): same row pointers, column order and
    values."""
    c = C.synthetic(n=700, e=700 * 40, seed=4, cache=False)
    t_ptr, t_pre, t_val = c.by_post()
    w = c.to_torch_weights().to_sparse_csr()
    assert np.array_equal(t_ptr, w.crow_indices().numpy())
    assert np.array_equal(t_pre, w.col_indices().numpy())
    assert np.array_equal(t_val, w.values().numpy())


def test_empty_table_gives_neurons_without_edges(tmp_path):
    f = tmp_path / "empty.parquet"
    write_table(f, np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0, np.float32))
    c = C.from_parquet(f, n=17, cache=False)
    assert c.n == 17 and c.col.size == 0 and np.array_equal(c.row_ptr, np.zeros(18, np.int64))
