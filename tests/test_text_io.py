"""Host-side text ingestion (cpg_dag_read_text): the reference's input format
(CpGen::read_input, gpucpg.cu:453-548) parsed on the host threads.

Checked against the generator's own edge list (file order, bit-exact delays),
the oracle's sequential parser, and the reference's error cases: a malformed
edge line fails with its 1-based line number, blank lines are skipped, and a
vertex id outside 0..N-1 is an error.  The medium case is large enough that
the parser splits the edge section across threads.
"""
import numpy as np
import pytest

import cases
import cpg_b200
import oracle


def _csr(n, src, dst, w):
    order = np.argsort(src, kind="stable")
    adjp = np.zeros(n + 1, np.int64)
    np.add.at(adjp, src.astype(np.int64) + 1, 1)
    return np.cumsum(adjp), dst[order], w[order]


@pytest.mark.parametrize("size", ["small", "medium"])
def test_read_text_equals_generator_and_oracle(tmp_path, size):
    if size == "small":
        p = cpg_b200.gen_params(**cases.CASES["small_f32_s11"]["gen"])
    else:
        p = cpg_b200.gen_params(seed=5, n_pins=60_000, n_levels=40, n_first=2_000,
                                n_last=2_000, deg_lo=3, deg_hi=8)
    path = str(tmp_path / "g.txt")
    d = cpg_b200.generate(p, text_path=path)
    got = cpg_b200.read_text(path)
    assert got.n == d.n
    assert np.array_equal(got.src, d.src) and np.array_equal(got.dst, d.dst)
    assert np.array_equal(got.w.view(np.uint32), d.w.view(np.uint32))
    adjp, adj, w = oracle.OracleGraph.from_text(path).csr()
    gadjp, gadj, gw = _csr(got.n, got.src, got.dst, got.w)
    assert np.array_equal(adjp, gadjp) and np.array_equal(adj, gadj)
    assert np.array_equal(w.view(np.uint32), gw.view(np.uint32))
    ones = cpg_b200.read_text(path, ignore_wgts=True)
    assert np.array_equal(ones.src, d.src) and np.all(ones.w == 1.0)


def _write(path, n, lines):
    with open(path, "w") as f:
        f.write(f"{n}\n")
        f.write("".join(f'"{i}";\n' for i in range(n)))
        f.write("".join(x + "\n" for x in lines))


def test_blank_lines_and_missing_weight(tmp_path):
    path = str(tmp_path / "g.txt")
    _write(path, 3, ['"0" -> "1", 2.5;', "", "   ", '"1" -> "2";', '"0" -> "2", 7;'])
    d = cpg_b200.read_text(path)
    assert d.n == 3
    assert d.src.tolist() == [0, 1, 0] and d.dst.tolist() == [1, 2, 2]
    assert d.w.tolist() == [2.5, 1.0, 7.0]


def test_last_line_without_newline(tmp_path):
    path = str(tmp_path / "g.txt")
    with open(path, "w") as f:
        f.write('2\n"0";\n"1";\n"0" -> "1",')
    d = cpg_b200.read_text(path)
    assert d.src.tolist() == [0] and d.w.tolist() == [0.0]


@pytest.mark.parametrize("bad", ['"0" -> 1, 2;', '"0" -> "5", 1;', 'junk', '"-1" -> "1", 1;'])
def test_malformed_line_reports_its_number(tmp_path, bad):
    path = str(tmp_path / "g.txt")
    _write(path, 3, ['"0" -> "1", 1;', "", bad, '"1" -> "2", 1;'])
    with pytest.raises(cpg_b200.CpgError) as e:
        cpg_b200.read_text(path)
    # header line 1, names on lines 2-4, edges from line 5; the bad one is line 7
    assert e.value.status == cpg_b200.CPG_ERR_IO
    assert "malformed edge line 7" in str(e.value)


def test_first_error_wins_across_threads(tmp_path):
    # a file large enough to be split across threads, with two bad lines far
    # apart: the error names the earlier one
    n = 1_000
    rng = np.random.default_rng(3)
    u = rng.integers(0, n, 400_000)
    v = rng.integers(0, n, 400_000)
    lines = [f'"{a}" -> "{b}", {x};' for a, b, x in zip(u.tolist(), v.tolist(), range(400_000))]
    lines[123_456] = '"1" -> "x", 1;'
    lines[345_678] = "oops"
    path = str(tmp_path / "g.txt")
    _write(path, n, lines)
    with pytest.raises(cpg_b200.CpgError) as e:
        cpg_b200.read_text(path)
    assert f"malformed edge line {n + 2 + 123_456}" in str(e.value)
    lines[123_456] = '"1" -> "2", 1;'
    _write(path, n, lines)
    with pytest.raises(cpg_b200.CpgError) as e:
        cpg_b200.read_text(path)
    assert f"malformed edge line {n + 2 + 345_678}" in str(e.value)
    lines[345_678] = '"3" -> "4", 5;'
    _write(path, n, lines)
    d = cpg_b200.read_text(path)
    assert d.src.size == 400_000 and d.src[123_456] == 1 and d.dst[345_678] == 4
    assert np.array_equal(d.w[:1000], np.arange(1000, dtype=np.float32))


def test_missing_file_and_bad_header(tmp_path):
    with pytest.raises(cpg_b200.CpgError) as e:
        cpg_b200.read_text(str(tmp_path / "absent.txt"))
    assert e.value.status == cpg_b200.CPG_ERR_IO and "cannot open" in str(e.value)
    path = str(tmp_path / "g.txt")
    with open(path, "w") as f:
        f.write("abc\n")
    with pytest.raises(cpg_b200.CpgError):
        cpg_b200.read_text(path)
    with open(path, "w") as f:
        f.write('4\n"0";\n')
    with pytest.raises(cpg_b200.CpgError) as e:
        cpg_b200.read_text(path)
    assert "missing vertex name lines" in str(e.value)


def _tricky_delays(rng):
    """Decimal strings that exercise every branch of the delay conversion."""
    out = []
    bits = rng.integers(0x00800000, 0x7F000000, 60_000, dtype=np.uint32)
    f = bits.view(np.float32)
    out += [f"{x:.9g}" for x in f.tolist()]                        # round-trip floats
    out += [f"{-x:.6g}" for x in f[:20_000].tolist()]              # short mantissas
    d = rng.uniform(-7, 7, 60_000)
    out += [repr(float(x)) for x in (10.0 ** d).tolist()]          # 17-digit doubles
    # exact float midpoints as shortest doubles (fast path defers to strtof),
    # and the doubles one ulp either side of them (fast path must be right)
    g = f[:40_000].astype(np.float64)
    nxt = np.nextafter(f[:40_000], np.float32(np.inf)).astype(np.float64)
    mid = (g + nxt) / 2
    out += [repr(float(x)) for x in mid.tolist()]
    out += [repr(float(x)) for x in np.nextafter(mid, np.inf).tolist()]
    out += [repr(float(x)) for x in np.nextafter(mid, -np.inf).tolist()]
    # random decimals: 1..21 digits, exponents -40..40
    for _ in range(60_000):
        nd = int(rng.integers(1, 22))
        digs = "".join(rng.choice(list("0123456789"), nd).tolist())
        cut = int(rng.integers(0, nd + 1))
        s = digs[:cut] + "." + digs[cut:] if cut < nd else digs
        if rng.random() < 0.5:
            s += f"e{int(rng.integers(-40, 41))}"
        out.append(("-" if rng.random() < 0.3 else "") + s)
    out += ["0.1", ".5", "5.", "-0", "+3", "0", "000123.4500", "1e30", "1e-30", "1.5e+10",
            "12345678901234567890", "9007199254740993", "16777217", "3.4028235e38",
            "3.5e38", "1e-46", "0x1p-3", "inf", "-Infinity", "1e", "1e+", "  7.25", "2.5f"]
    return out


def test_delay_conversion_matches_strtof(tmp_path):
    rng = np.random.default_rng(17)
    ws = _tricky_delays(rng)
    path = str(tmp_path / "w.txt")
    _write(path, 2, [f'"0" -> "1", {x};' for x in ws])
    got = cpg_b200.read_text(path)
    _, _, want = oracle.OracleGraph.from_text(path).csr()  # strtof, one edge row
    assert got.w.size == len(ws) == want.size
    bad = np.nonzero(got.w.view(np.uint32) != want.view(np.uint32))[0]
    assert bad.size == 0, [ws[i] for i in bad[:10]]


# ------------------------------------------------------------ binary CSR file
def test_csr_bin_layout_and_round_trip(tmp_path):
    p = cpg_b200.gen_params(**cases.CASES["small_f32_s11"]["gen"])
    lib_path = str(tmp_path / "lib.bin")
    py_path = str(tmp_path / "py.bin")
    d = cpg_b200.generate(p, csr_bin_path=lib_path)
    cpg_b200.write_csr_bin(d, py_path)
    assert open(lib_path, "rb").read() == open(py_path, "rb").read()
    # the layout: int32 N, int32 M, adjp[N+1], adjncy[M], float w[M]
    raw = np.fromfile(lib_path, np.int32)
    n, m = int(raw[0]), int(raw[1])
    assert (n, m) == (d.n, d.m) and raw.size == 2 + n + 1 + 2 * m
    adjp, adj, w = _csr(d.n, d.src, d.dst, d.w)
    assert np.array_equal(raw[2:n + 3], adjp)
    assert np.array_equal(raw[n + 3:n + 3 + m], adj)
    assert np.array_equal(raw[n + 3 + m:].view(np.float32).view(np.uint32), w.view(np.uint32))
    back = cpg_b200.read_csr_bin(lib_path)
    order = np.argsort(d.src, kind="stable")
    assert back.n == d.n
    assert np.array_equal(back.src, d.src[order]) and np.array_equal(back.dst, d.dst[order])
    assert np.array_equal(back.w.view(np.uint32), d.w[order].view(np.uint32))


def test_csr_bin_parallel_read(tmp_path):
    # large enough (over 4 MB) that the sections are read on several threads
    p = cpg_b200.gen_params(seed=9, n_pins=200_000, n_levels=50, n_first=5_000,
                            n_last=5_000, deg_lo=2, deg_hi=6)
    path = str(tmp_path / "g.bin")
    d = cpg_b200.generate(p, csr_bin_path=path)
    back = cpg_b200.read_csr_bin(path)
    order = np.argsort(d.src, kind="stable")
    assert np.array_equal(back.dst, d.dst[order])
    assert np.array_equal(back.w.view(np.uint32), d.w[order].view(np.uint32))


def _bin(path, n, adjp, adj, w):
    with open(path, "wb") as f:
        f.write(np.array([n, len(adj)], np.int32).tobytes())
        f.write(np.asarray(adjp, np.int32).tobytes())
        f.write(np.asarray(adj, np.int32).tobytes())
        f.write(np.asarray(w, np.float32).tobytes())


@pytest.mark.parametrize("case,msg", [
    ("short", "size does not match"),
    ("start", "start at 0"),
    ("end", "end at M"),
    ("falls", "offsets fall at row 1"),
    ("head", "head out of range at edge 2"),
    ("adjncy_as_offsets", "offsets"),
])
def test_csr_bin_rejects_bad_files(tmp_path, case, msg):
    path = str(tmp_path / "g.bin")
    adjp, adj, w = [0, 2, 3, 3], [1, 2, 2], [1.0, 2.0, 3.0]
    if case == "short":
        _bin(path, 3, adjp, adj, w)
        with open(path, "r+b") as f:
            f.truncate(20)
    elif case == "start":
        _bin(path, 3, [1, 2, 3, 3], adj, w)
    elif case == "end":
        _bin(path, 3, [0, 2, 3, 2], adj, w)
    elif case == "falls":
        _bin(path, 3, [0, 2, 1, 3], adj, w)
    elif case == "head":
        _bin(path, 3, adjp, [1, 2, 7], w)
    else:
        # what the reference's write_to_csr_bin produces: the first N+1
        # adjacency entries where the offsets belong
        _bin(path, 3, [1, 2, 2, 0], adj, w)
    with pytest.raises(cpg_b200.CpgError) as e:
        cpg_b200.read_csr_bin(path)
    assert e.value.status == cpg_b200.CPG_ERR_IO and msg in str(e.value)


def test_csr_bin_empty_graph(tmp_path):
    path = str(tmp_path / "g.bin")
    _bin(path, 0, [0], [], [])
    d = cpg_b200.read_csr_bin(path)
    assert d.n == 0 and d.m == 0


@pytest.mark.parametrize("m", [5_000, 400_000])
def test_csr_of_unordered_edge_list_keeps_list_order(tmp_path, m):
    # edges in random order (and repeated pairs): every row keeps the list's
    # order; the larger list is built on several threads
    rng = np.random.default_rng(m)
    n = 3_000
    src = rng.integers(0, n, m).astype(np.int32)
    dst = rng.integers(0, n, m).astype(np.int32)
    w = np.arange(m, dtype=np.float32)  # the delay records the list position
    path, binp, want = str(tmp_path / "g.txt"), str(tmp_path / "g.bin"), str(tmp_path / "w.bin")
    d = cpg_b200.Dag(n, src, dst, w)
    cpg_b200.write_text(d, path)
    cpg_b200.read_text(path, csr_bin_path=binp)
    cpg_b200.write_csr_bin(d, want)
    assert open(binp, "rb").read() == open(want, "rb").read()
