"""Reference binary graph format (graph_converter/compactify.cpp:172-195,
labelize.cpp:130-133; read by src/graph.h:136-193) and the generators."""
import numpy as np
import pytest


def test_roundtrip(T, tmp_path):
    g = T.gen_er(500, 8.0, 5).set_labels(4, 2)
    prefix = str(tmp_path / "g")
    g.write(prefix)
    meta = open(prefix + ".meta.txt").read().split()
    assert [int(x) for x in meta] == [g.n, g.nedges, 4, g.max_degree]
    assert np.fromfile(prefix + ".vertex.bin", np.int64).tolist() == g.rowptr.tolist()
    assert np.fromfile(prefix + ".edge.bin", np.int32).tolist() == g.colidx.tolist()
    assert np.fromfile(prefix + ".label.bin", np.int32).tolist() == g.labels.tolist()
    h = T.read_csr(prefix, labeled=True)
    assert (h.rowptr == g.rowptr).all() and (h.colidx == g.colidx).all() and (h.labels == g.labels).all()


def _write(prefix, rowptr, colidx, vid=4):
    rowptr = np.asarray(rowptr, np.int64)
    colidx = np.asarray(colidx, np.int32)
    with open(prefix + ".meta.txt", "w") as f:
        f.write(f"{len(rowptr) - 1}\n{len(colidx)}\n{vid}\n3\n")
    rowptr.tofile(prefix + ".vertex.bin")
    colidx.tofile(prefix + ".edge.bin")


@pytest.mark.parametrize("rowptr,colidx,vid,code", [
    ([0, 2, 3, 4], [2, 1, 0, 0], 4, 2),   # unsorted row
    ([0, 2, 3, 4], [1, 1, 0, 0], 4, 2),   # duplicate neighbour (reference asserts)
    ([0, 1, 2, 3], [1, 9, 0], 4, 2),      # neighbour id out of range
    ([0, 1, 2], [1, 0], 8, 2),            # vid_size must be 4
])
def test_format_errors(T, tmp_path, rowptr, colidx, vid, code):
    prefix = str(tmp_path / "bad")
    _write(prefix, rowptr, colidx, vid)
    with pytest.raises(T.TdfsError) as e:
        T.read_csr(prefix)
    assert e.value.code == code


def test_missing_files(T, tmp_path):
    with pytest.raises(T.TdfsError) as e:
        T.read_csr(str(tmp_path / "none"))
    assert e.value.code == 1
    _write(str(tmp_path / "nolab"), [0, 1, 2], [1, 0])
    with pytest.raises(T.TdfsError) as e:
        T.read_csr(str(tmp_path / "nolab"), labeled=True)
    assert e.value.code == 1


def _check_simple(g):
    rp, ci = g.rowptr, g.colidx
    src = np.repeat(np.arange(g.n), np.diff(rp))
    assert (ci != src).all(), "self loop"
    for v in range(0, g.n, max(1, g.n // 200)):
        row = ci[rp[v]:rp[v + 1]]
        assert (np.diff(row) > 0).all()
    fwd = set(zip(src.tolist(), ci.tolist()))
    assert all((b, a) in fwd for a, b in list(fwd)[:5000]), "not symmetric"


def test_er_generator(T):
    a, b = T.gen_er(4096, 16.0, 0), T.gen_er(4096, 16.0, 0)
    assert (a.colidx == b.colidx).all()
    assert abs(a.nedges / a.n - 16.0) < 0.5
    _check_simple(a)
    assert not (T.gen_er(4096, 16.0, 1).colidx[:100] == a.colidx[:100]).all()


def test_chung_lu_generator(T):
    g = T.gen_chung_lu(20000, 60000, 2.1, 600, 1)
    h = T.gen_chung_lu(20000, 60000, 2.1, 600, 1)
    assert (g.colidx == h.colidx).all()
    deg = np.diff(g.rowptr)
    assert g.nedges == 2 * 60000
    assert deg.max() <= 600 and g.max_degree == deg.max()
    assert (np.diff(deg) <= 0).all(), "ids must be in descending-degree order"
    _check_simple(g)


def test_rmat_generator(T):
    g = T.gen_rmat(12, 16, 0.57, 0.19, 0.19, 4)
    h = T.gen_rmat(12, 16, 0.57, 0.19, 0.19, 4)
    assert g.n == 4096 and (g.colidx == h.colidx).all()
    _check_simple(g)
    deg = np.diff(g.rowptr)
    assert deg[0] == deg.max()  # quadrant a = 0.57 concentrates on low ids


def test_labels_uniform(T):
    g = T.gen_er(20000, 4.0, 3).set_labels(4, 2)
    counts = np.bincount(g.labels, minlength=4)
    assert counts.min() > 4500 and g.labels.max() == 3


def test_pattern_generator(T):
    for seed in range(200):
        k = 3 + seed % 5
        text = T.gen_pattern(k, 0.4, 4, seed)
        p = T.PatternPreprocessor(text=text, labeled=True)  # compiles: connected order
        d = p.dump()
        assert d["k"] == k and 1 in d["backward_neighbors"][2]


def _edges(g):
    src = np.repeat(np.arange(g.n), np.diff(g.rowptr))
    return set(zip(src.tolist(), g.colidx.tolist()))


def test_relabel_any_graph(T):
    """Descending-degree relabelling (graph_converter/relabel.cpp:27-58):
    (degree, id) pairs sorted in descending order give the new ids, so the
    result is an isomorphic copy whose degrees never increase and whose
    ties keep the larger old id first; labels move with their vertices."""
    g = T.gen_rmat(10, 8, 0.57, 0.19, 0.19, 9).set_labels(5, 3)
    r = g.relabel()
    deg = np.diff(g.rowptr)
    order = sorted(range(g.n), key=lambda v: (deg[v], v), reverse=True)
    new = np.empty(g.n, np.int64)
    new[order] = np.arange(g.n)
    assert r.n == g.n and r.nedges == g.nedges and r.max_degree == g.max_degree
    assert (np.diff(np.diff(r.rowptr)) <= 0).all()
    assert _edges(r) == {(int(new[a]), int(new[b])) for a, b in _edges(g)}
    assert (r.labels[new] == g.labels).all()
    for v in range(r.n):
        assert (np.diff(r.colidx[r.rowptr[v]:r.rowptr[v + 1]]) > 0).all()
    # the Chung-Lu generator relabels with the same rule: a second pass only
    # permutes equal-degree ties, and the degree sequence is unchanged
    c = T.gen_chung_lu(5000, 15000, 2.1, 300, 1)
    assert (np.diff(c.relabel().rowptr) == np.diff(c.rowptr)).all()


def test_halve_any_graph(T):
    """Degree orientation (graph_converter/halve.cpp:17-32): every undirected
    edge survives once, towards the higher-degree end (the larger id on a
    tie); symmetrising the result gives the graph back."""
    g = T.gen_chung_lu(5000, 15000, 2.1, 300, 1).set_labels(4, 2)
    h = g.halve()
    deg = np.diff(g.rowptr)
    he = _edges(h)
    assert h.nedges * 2 == g.nedges and len(he) == h.nedges
    assert all(deg[d] > deg[s] or (deg[d] == deg[s] and d > s) for s, d in he)
    assert he | {(d, s) for s, d in he} == _edges(g)
    assert h.max_degree == np.diff(h.rowptr).max() and (h.labels == g.labels).all()


def test_csr_from_arrays_checks_rows(T):
    g = T.gen_er(300, 6.0, 1)
    c = T.csr_from_arrays(g.rowptr, g.colidx)
    assert (c.colidx == g.colidx).all() and c.max_degree == g.max_degree
    bad = g.colidx.copy()
    bad[g.rowptr[3]:g.rowptr[4]] = bad[g.rowptr[3]:g.rowptr[4]][::-1]
    with pytest.raises(T.TdfsError) as e:
        T.csr_from_arrays(g.rowptr, bad)
    assert e.value.code == 2


def test_convert_tool_writes_the_generators_graphs(T, tmp_path):
    """tdfs_convert (host-only, no CUDA runtime) writes the same files as the
    library's generators, and relabel/halve on disk match the C ABI."""
    import subprocess
    pre = str(tmp_path / "er")
    subprocess.run([T.CONVERT, "er", "4096", "16", "0", pre], check=True, capture_output=True)
    subprocess.run([T.CONVERT, "labels", pre, "4", "2"], check=True, capture_output=True)
    g = T.gen_er(4096, 16.0, 0).set_labels(4, 2)
    r = T.read_csr(pre, labeled=True)
    assert (r.rowptr == g.rowptr).all() and (r.colidx == g.colidx).all() and (r.labels == g.labels).all()
    for step, fn in (("relabel", g.relabel), ("halve", g.halve)):
        out = str(tmp_path / step)
        subprocess.run([T.CONVERT, step, pre, out], check=True, capture_output=True)
        a, b = T.read_csr(out, labeled=True), fn()
        assert (a.rowptr == b.rowptr).all() and (a.colidx == b.colidx).all() and (a.labels == b.labels).all()
    cl = str(tmp_path / "cl")
    subprocess.run([T.CONVERT, "cl", "20000", "60000", "2.1", "600", "1", cl], check=True, capture_output=True)
    assert (T.read_csr(cl).colidx == T.gen_chung_lu(20000, 60000, 2.1, 600, 1).colidx).all()
    bad = subprocess.run([T.CONVERT, "halve", str(tmp_path / "missing"), out], capture_output=True, text=True)
    assert bad.returncode == 1 and "cannot open" in bad.stderr
