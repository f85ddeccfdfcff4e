"""The CPU oracle against the reference's own known-answer tests and fixtures."""
import os

import numpy as np
import pytest

import cases
import oracle

INT_MAX = 2**31 - 1


def test_child_cost_known_answer():
    # unittests/tc_pfxt_candidates.cu:85-90:
    # candidate_slack(0.5f, 25000, 10000, 0.25f) == Approx(-0.75f)
    c = oracle.child_cost(0.5, 10000, 0.25, 25000)
    assert c == pytest.approx(-0.75)


def test_compact_deviation_csr_known_answer():
    # unittests/tc_pfxt_candidates.cu:384-407
    adjp = [0, 4, 6, 7, 7]
    adj = [1, 2, 2, 3, 2, 0, 1]
    w = [0.1, 0.2, 0.25, 0.4, 0.5, 0.6, 0.7]
    succ = [1, -1, 1, -1]
    dist = [1000, 2000, INT_MAX, 3000]
    off, dsts, deltas = oracle.deviation_csr(adjp, adj, w, succ, dist)
    assert off.tolist() == [0, 1, 2, 2, 2]
    assert dsts.tolist() == [3, 0]
    assert deltas[0] == pytest.approx(0.6)
    assert deltas[1] == pytest.approx(0.5)


def _graph(name):
    n, src, dst, w = cases.load_case(name)
    return oracle.OracleGraph.from_edges(n, src, dst, w)


def test_fixture_sizes():
    # the reference's fixture files: N line and edge lines
    assert _graph("simple").g.n == 17 and _graph("simple").g.m == 17
    assert _graph("dac21_paper_example").g.m == 14
    assert _graph("tv80_unit_wgts").g.n == 17038


def _all_path_costs(n, src, dst, w):
    """Brute force: every source-to-sink path's summed delay (float64)."""
    out = {}
    for u, v, x in zip(src.tolist(), dst.tolist(), w.tolist()):
        out.setdefault(u, []).append((v, x))
    indeg = np.bincount(dst, minlength=n)
    costs = []

    def walk(v, c):
        if v not in out:
            costs.append(c)
            return
        for h, x in out[v]:
            walk(h, c + x)

    for s0 in range(n):
        if indeg[s0] == 0:
            walk(s0, 0.0)
    return np.sort(np.array(costs))


@pytest.mark.parametrize("name", ["simple", "dac21_paper_example"])
def test_tiny_fixtures_against_brute_force(name):
    n, src, dst, w = cases.load_case(name)
    want = _all_path_costs(n, src, dst, w)
    want = want[want != 0.0]
    g = oracle.OracleGraph.from_edges(n, src, dst, w)
    seq = g.sequential(1000)["slack"]
    clo = g.closure_topk(1000, ref_roots=False)[0]["slack"]
    assert len(seq) == len(clo) == len(want)
    np.testing.assert_allclose(seq, want, rtol=1e-5)
    np.testing.assert_allclose(clo, want, rtol=1e-5)


@pytest.mark.parametrize("name,k", [("simple", 100), ("tv80_unit_wgts", 3000),
                                    ("small_f32_s11", 3000), ("small_int_s13", 3000)])
def test_sequential_matches_closure(name, k):
    g = _graph(name)
    seq = g.sequential(k)["slack"]
    clo = g.closure_topk(k, ref_roots=False)[0]["slack"]
    assert len(seq) == len(clo)
    np.testing.assert_allclose(seq, clo, rtol=1e-5, atol=0)


def test_closure_paths_are_consistent():
    g = _graph("small_f32_s12")
    out, split = g.closure_topk(2000)
    assert np.all(np.diff(out["slack"]) >= 0)
    assert out["slack"][-1] <= split
    d, s, _ = g.sfxt()
    adjp, adj, w = g.csr()
    for i, nd in enumerate(out):
        if nd["parent"] >= 0:
            p = out[nd["parent"]]
            assert nd["parent"] < i or p["slack"] == nd["slack"]
            assert nd["level"] == p["level"] + 1
            # the deviation edge exists and is not the successor edge
            row = adj[adjp[nd["from"]]:adjp[nd["from"] + 1]]
            assert nd["to"] in row and nd["to"] != s[nd["from"]]


def test_sfxt_invariants():
    g = _graph("single20k_f32")
    d, s, lvl = g.sfxt()
    adjp, adj, w = g.csr()
    fixed = (w * np.float32(10000)).astype(np.int32)
    for v in range(0, g.n, 97):
        row = slice(adjp[v], adjp[v + 1])
        if adjp[v] == adjp[v + 1]:
            assert d[v] == 0 and s[v] == -1 and lvl[v] == 0
            continue
        c = d[adj[row]] + fixed[row]
        assert d[v] == c.min()
        assert s[v] == adj[row][c == c.min()].max()
        assert lvl[v] == lvl[adj[row]].max() + 1


GOLD = os.path.join(os.path.dirname(__file__), "golden", "ref_goldens.npz")


@pytest.mark.skipif(not os.path.exists(GOLD), reason="reference goldens not packed")
def test_oracle_against_reference_goldens():
    """The oracle reproduces the reference's own outputs, run on a B200: the
    suffix tree bit for bit, and G-PathGen's costs within the fast-division
    tolerance (the oracle divides in IEEE, the reference's device code with
    --use_fast_math)."""
    z = np.load(GOLD)
    sfxt_checked = costs_checked = 0
    for name, c in cases.CASES.items():
        if c.get("large") or f"{name}/sfxt_dist" not in z:
            continue
        g = _graph(name)
        d, s, _ = g.sfxt()
        np.testing.assert_array_equal(d, z[f"{name}/sfxt_dist"])
        np.testing.assert_array_equal(s, z[f"{name}/sfxt_succ"])
        sfxt_checked += 1
        if f"{name}/costs" not in z:
            continue
        ref = z[f"{name}/costs"]
        k = int(z[f"{name}/k"])
        clo = g.closure_topk(k, ref_roots=True)[0]["slack"]
        assert len(clo) == len(ref)
        np.testing.assert_allclose(clo, ref, rtol=1e-5, atol=0)
        costs_checked += 1
    assert sfxt_checked >= 4 and costs_checked >= 3


@pytest.mark.parametrize("name", ["single20k_f32", "single20k_int", "small_f32_s11",
                                  "small_int_s14"])
def test_oracle_generator_equals_product_generator(name):
    """The oracle's restated generator and the product's cpg_dag_generate give
    the same edge list (host code only; no GPU)."""
    import cpg_b200
    gen = cases.CASES[name]["gen"]
    d = cpg_b200.generate(cpg_b200.gen_params(**gen))
    n, src, dst, w = oracle.generate(**gen)
    assert n == d.n
    np.testing.assert_array_equal(src, d.src)
    np.testing.assert_array_equal(dst, d.dst)
    np.testing.assert_array_equal(w.view(np.uint32), d.w.view(np.uint32))


def test_oracle_generator_density_settings():
    """The density-sweep settings (geometric degree, larger mean) agree too, on
    a smaller pin count."""
    import cpg_b200
    gen = {**cases.CASES["large1m_d50"]["gen"], "n_pins": 30_000, "n_first": 100,
           "n_last": 100, "n_levels": 40}
    d = cpg_b200.generate(cpg_b200.gen_params(**gen))
    n, src, dst, w = oracle.generate(**gen)
    assert n == d.n and np.array_equal(src, d.src) and np.array_equal(dst, d.dst)
    assert np.array_equal(w.view(np.uint32), d.w.view(np.uint32))


@pytest.mark.parametrize("name,k", [("simple", 100), ("tv80_unit_wgts", 5000),
                                    ("single20k_f32", 10000), ("single20k_int", 10000),
                                    ("small_f32_s11", 20000), ("small_int_s13", 20000)])
@pytest.mark.parametrize("ref_roots", [True, False])
def test_pruned_closure_equals_full_scan(name, k, ref_roots):
    """Skipping rows and chain tails that cannot hold a child <= the limit
    returns the same costs and the same final split as scanning every
    deviation edge of every chain."""
    g = _graph(name)
    a, sa = g.closure_topk(k, ref_roots=ref_roots, prune=False)
    b, sb = g.closure_topk(k, ref_roots=ref_roots, prune=True)
    assert sa == sb
    assert np.array_equal(a["slack"].view(np.uint32), b["slack"].view(np.uint32))


@pytest.mark.parametrize("name", ["small_f32_s12", "tv80_unit_wgts"])
def test_closure_path_vertices(name):
    """Each returned path's vertex sequence runs from a source to a sink over
    fan-out edges, and its cost rebuilt by the reference's left-to-right
    recurrence is the reported cost."""
    g = _graph(name)
    out, paths = g.closure_paths(1500)
    d, s, _ = g.sfxt()
    adjp, adj, w = g.csr()
    indeg = np.zeros(g.n, np.int64)
    np.add.at(indeg, adj, 1)
    assert len(paths) == out.size and len({tuple(p) for p in paths}) == out.size
    for nd, verts in zip(out, paths):
        assert indeg[verts[0]] == 0 and adjp[verts[-1]] == adjp[verts[-1] + 1]
        c = np.float32(np.float32(d[verts[0]]) / np.float32(10000))
        for a, b in zip(verts[:-1], verts[1:]):
            row = adj[adjp[a]:adjp[a + 1]]
            assert b in row
            if s[a] != b:
                e = adjp[a] + int(np.flatnonzero(row == b)[0])
                c = np.float32(oracle.child_cost(float(c), int(d[b]), float(w[e]), int(d[a])))
        assert c == nd["slack"]


PINS = os.path.join(os.path.dirname(__file__), "golden", "oracle_pins.npz")


def test_oracle_pins_reproduce():
    """The committed full-size pins are what the oracle computes: the
    1M-pin fp32 workload's suffix tree and its first 1e5 costs."""
    import hashlib
    z = np.load(PINS)
    name = "large1m_f32"
    g = _graph(name)
    d, s, lv = g.sfxt()
    sha = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
    assert sha(d) == str(z[f"{name}/sfxt_sha_dist"])
    assert sha(s) == str(z[f"{name}/sfxt_sha_succ"])
    assert sha(lv) == str(z[f"{name}/sfxt_sha_level"])
    costs = g.closure_topk(100_000, ref_roots=False)[0]["slack"]
    for p in (1000, 10_000, 100_000):
        assert sha(costs[:p]) == str(z[f"{name}/p{p}_sha"]), p
