"""Matrix Market parsed into a CSR on the GPU (gc_graph_load_mtx / gc_mtx_read_device) against the
host reader gc_mtx_read, which is pinned to the reference's CSR by the golden fixtures
(src/fast_io.c:33-222, 450-477): bit-identical V and E on every file, the golden ones included."""
import numpy as np
import pytest

import gnn_coloring as gcn

pytestmark = pytest.mark.gpu

HEADER = "%%MatrixMarket matrix coordinate pattern symmetric\n"


def both(ctx, path):
    host = gcn.mtx_read(str(path))
    dev = gcn.mtx_read_device(ctx, str(path))
    return host, dev


def same(host, dev):
    return host[0] == dev[0] and np.array_equal(host[1], dev[1]) and np.array_equal(host[2], dev[2])


def test_golden_files(gpu_ctx, golden_mtx, tmp_path):
    for name in sorted({k.split("/")[0] for k in golden_mtx.files}):
        path = tmp_path / f"{name}.mtx"
        path.write_bytes(golden_mtx[f"{name}/text"].tobytes())
        N, V, E = gcn.mtx_read_device(gpu_ctx, str(path))
        assert N == int(golden_mtx[f"{name}/N"]), name
        assert np.array_equal(V, golden_mtx[f"{name}/V"]), name
        assert np.array_equal(E, golden_mtx[f"{name}/E"]), name


@pytest.mark.parametrize("text", [
    HEADER + "5 5 3\n1 2\n% a comment between entries\n2 3\n4 5",           # no final newline
    HEADER + "5 5 3\r\n1 2\r\n2 3\r\n4 5\r\n",                               # CRLF
    HEADER + "4 4 0\n",                                                      # header only
    HEADER + "4 4 0",                                                        # header only, no newline
    HEADER + "7 3 2\n7 1\n2 3\n",                                            # N = rows > cols, empty rows
    HEADER + "3 3 3\n1 1\n2 2\n3 3\n",                                       # self-loops only
    HEADER + "6 6 4\n1 2 0.5\n2 1 7\n1 2\n6 6\n1 2\n",                       # entries past L are ignored
    "%%MatrixMarket matrix coordinate real general\n%\n%\n3 3 2 extra words\n\n1 3 1e5\n3 2 -2\n",
])
def test_edge_cases_match_host_reader(gpu_ctx, tmp_path, text):
    path = tmp_path / "g.mtx"
    path.write_bytes(text.encode())
    host, dev = both(gpu_ctx, path)
    assert same(host, dev), (host, dev)


def test_errors(gpu_ctx, tmp_path):
    bad = tmp_path / "bad.mtx"
    bad.write_text(HEADER + "3 3 2\n1 2\n0 3\n")
    with pytest.raises(gcn.GCError) as e:
        gcn.mtx_read_device(gpu_ctx, str(bad))
    assert e.value.name == "GC_ERR_FORMAT"
    big = tmp_path / "big.mtx"
    big.write_text(HEADER + "3 3 2\n1 2\n2 4\n")
    with pytest.raises(gcn.GCError) as e:
        gcn.mtx_read_device(gpu_ctx, str(big))
    assert e.value.name == "GC_ERR_FORMAT"
    trunc = tmp_path / "trunc.mtx"
    trunc.write_text(HEADER + "3 3 5\n1 2\n")
    with pytest.raises(gcn.GCError) as e:
        gcn.mtx_read_device(gpu_ctx, str(trunc))
    assert e.value.name == "GC_ERR_FORMAT"
    with pytest.raises(gcn.GCError) as e:
        gcn.mtx_read_device(gpu_ctx, str(tmp_path / "missing.mtx"))
    assert e.value.name == "GC_ERR_IO"
    # the context stays usable after each error
    N, V, E = gcn.gen_er(100, 300, 1)
    g = gcn.Graph(gpu_ctx, N, V, E)
    g.priority("LF")
    assert g.color() > 0


def test_shuffled_duplicated_entries(gpu_ctx, tmp_path):
    """Entries in random order and orientation, with duplicates, self-loops and comment lines; ids
    above 2^16 so the sorts run three digit passes."""
    rng = np.random.default_rng(7)
    n, m = 200_000, 600_000
    I = rng.integers(1, n + 1, m)
    J = rng.integers(1, n + 1, m)
    dup = rng.integers(0, m, m // 10)
    I = np.concatenate([I, J[dup]])
    J = np.concatenate([J, I[dup]])
    lines = [f"{a} {b}" for a, b in zip(I.tolist(), J.tolist())]
    for k in rng.integers(0, len(lines), 50).tolist():
        lines[k] = "% comment 12 34\n" + lines[k]
    path = tmp_path / "shuffled.mtx"
    path.write_text(HEADER + f"{n} {n} {len(I)}\n" + "\n".join(lines) + "\n")
    host, dev = both(gpu_ctx, path)
    assert same(host, dev)


def test_rmat_roundtrip_and_device_graph(gpu_ctx, tmp_path):
    """An R-MAT 2^18 file written by gc_mtx_write: the device CSR equals the source CSR, and the graph
    loaded on the device colors exactly like the graph uploaded from the host."""
    N, V, E = gcn.gen_rmat(1 << 18, 16, 3)
    path = str(tmp_path / "rmat18.mtx")
    gcn.mtx_write(path, N, V, E)
    N2, V2, E2 = gcn.mtx_read_device(gpu_ctx, path)
    assert N2 == N and np.array_equal(V2, V) and np.array_equal(E2, E)
    gd = gcn.Graph.load_mtx(gpu_ctx, path)
    gh = gcn.Graph(gpu_ctx, N, V, E)
    assert gd.N == N and gd.M == len(E)
    for heur in ("LF", "SL"):
        gd.priority(heur)
        gh.priority(heur)
        k = gd.color(recolor=1)
        assert k == gh.color(recolor=1)
        assert np.array_equal(gd.colors(), gh.colors())
        assert gd.validate() == k
