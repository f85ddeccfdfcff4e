"""Ingestion paths to a device graph: the text file (read_input), the binary
CSR file and the in-memory edge list give the same device CSR, the same
suffix tree and the same K costs; a handle writes back the file it loaded.
"""
import numpy as np
import pytest

import cases
import cpg_b200
import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["small_f32_s11", "single20k_int"])
def test_text_bin_and_edges_load_the_same_graph(tmp_path, name):
    c = cases.CASES[name]
    txt, binp = str(tmp_path / "g.txt"), str(tmp_path / "g.bin")
    d = cpg_b200.generate(cpg_b200.gen_params(**c["gen"]), text_path=txt, csr_bin_path=binp)
    k = 2_000
    results = []
    for how in ("text", "bin", "edges"):
        with cpg_b200.CpGen(division=cpg_b200.DIV_IEEE, root_seeding=cpg_b200.ROOTS_ALL) as g:
            if how == "text":
                g.read_input(txt)
            elif how == "bin":
                g.load_csr_bin(binp)
            else:
                g.load_edges(d.n, d.src, d.dst, d.w)
            g.report_paths(k)
            results.append((g.get_csr(), g.get_sfxt(), g.get_slacks(k)))
            if how == "bin":
                out = str(tmp_path / "back.bin")
                g.write_csr_bin(out)
                assert open(out, "rb").read() == open(binp, "rb").read()
    (csr0, sf0, s0) = results[0]
    for csr, sf, s in results[1:]:
        for a, b in zip(csr, csr0):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
        for a, b in zip(sf, sf0):
            assert np.array_equal(a, b)
        assert np.array_equal(s.view(np.uint32), s0.view(np.uint32))
    og = oracle.OracleGraph.from_text(txt)
    want = og.sequential(k)["slack"]
    assert np.array_equal(s0.view(np.uint32), want.view(np.uint32))


def test_bad_csr_bin_leaves_handle_usable(tmp_path):
    path = str(tmp_path / "bad.bin")
    with open(path, "wb") as f:
        f.write(np.array([3, 3, 1, 2, 2, 0, 1, 2, 2], np.int32).tobytes())
        f.write(np.ones(3, np.float32).tobytes())
    with cpg_b200.CpGen() as g:
        with pytest.raises(cpg_b200.CpgError):
            g.load_csr_bin(path)
        g.load_edges(3, np.array([0, 0, 1], np.int32), np.array([1, 2, 2], np.int32),
                     np.array([1.0, 2.0, 3.0], np.float32))
        g.report_paths(3)
        assert np.allclose(g.get_slacks(3), [2.0, 4.0])


def test_load_csr_builds_on_first_use_and_checks_heads():
    """cpg_load_csr returns once its copies have read the caller's buffers;
    the device graph is built by the first call that uses it.  The buffers
    may be overwritten right after the load, and a head out of range is
    reported by that first call, after which the handle loads and answers
    a good graph."""
    n, src, dst, w = cases.load_case("small_f32_s12")
    og = oracle.OracleGraph.from_edges(n, src, dst, w)
    adjp, adj, ww = og.csr()
    want = og.closure_topk(3000)[0]["slack"]
    with cpg_b200.CpGen(division=cpg_b200.DIV_IEEE) as g:
        a, b, c = adjp.copy(), adj.copy(), ww.copy()
        g.load_csr(n, a, b, c)
        a[:] = 0
        b[:] = -7
        c[:] = np.nan
        g.report_paths(3000)
        assert np.array_equal(g.get_slacks(3000).view(np.uint32), want.view(np.uint32))
        bad = adj.copy()
        bad[5] = n + 3
        g.load_csr(n, adjp, bad, ww)
        with pytest.raises(cpg_b200.CpgError) as e:
            g.report_paths(10)
        assert e.value.status == cpg_b200.CPG_ERR_INVALID
        with pytest.raises(cpg_b200.CpgError):
            g.report_paths(10)   # no graph is loaded after the failed build
        g.load_csr(n, adjp, adj, ww)
        g.report_paths(3000)
        assert np.array_equal(g.get_slacks(3000).view(np.uint32), want.view(np.uint32))
