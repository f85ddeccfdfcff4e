"""The C ABI library without a GPU: it loads, exports every declared symbol,
refuses to run without a device, and its host-only generator and text I/O
agree with the oracle's restatement of the reference's parser."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

import cases
import cpg_b200
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_header_symbol():
    names = cpg_b200.header_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(cpg_b200.lib, n)]
    assert not missing, missing
    assert cpg_b200.lib.cpg_abi_version() == 3


def test_status_strings():
    assert cpg_b200.lib.cpg_status_string(0) == b"ok"
    assert cpg_b200.lib.cpg_status_string(8) == b"no cuda device"


def test_create_without_device_fails_loudly():
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a device is present")
    with pytest.raises(cpg_b200.CpgError) as e:
        cpg_b200.CpGen()
    assert e.value.status == 8


def test_null_arguments_are_rejected():
    L = cpg_b200.lib
    assert L.cpg_create(None, None) == 1
    assert L.cpg_destroy(None) == 1
    assert L.cpg_report_paths(None, 10) == 1
    assert L.cpg_levelize(None) == 1


def test_generator_is_seeded_and_levelised():
    p = cpg_b200.gen_params(**cases.CASES["single20k_f32"]["gen"])
    a = cpg_b200.generate(p)
    b = cpg_b200.generate(p)
    assert np.array_equal(a.src, b.src) and np.array_equal(a.w, b.w)
    assert a.n == 20002
    S, T = 20000, 20001
    assert np.sum(a.src == S) == 64 and np.sum(a.dst == T) == 64
    real = (a.src < S) & (a.dst < S)
    w = a.w[real]
    assert w.min() >= 0.1 and w.max() <= 10.0
    g = oracle.OracleGraph.from_edges(a.n, a.src, a.dst, a.w)
    d, s, lvl = g.sfxt()
    assert (lvl >= 0).all()                       # acyclic: every pin levelled
    indeg = np.bincount(a.dst, minlength=a.n)
    outdeg = np.bincount(a.src, minlength=a.n)
    assert np.flatnonzero(indeg == 0).tolist() == [S]
    assert np.flatnonzero(outdeg == 0).tolist() == [T]
    deg = outdeg[:S][np.isin(np.arange(S), a.dst[a.src == S], invert=True)]
    assert deg.max() <= 4 + 8                      # U{1..4} plus repair edges
    c = cpg_b200.generate(cpg_b200.gen_params(**{**cases.CASES["single20k_f32"]["gen"], "seed": 7}))
    assert not np.array_equal(a.dst, c.dst)


def test_integer_delays_are_integers():
    a = cpg_b200.generate(cpg_b200.gen_params(**cases.CASES["small_int_s13"]["gen"]))
    real = a.w[a.w > 0]
    assert np.all(real == np.round(real)) and real.min() >= 1 and real.max() <= 100


def test_text_round_trip_matches_oracle_parser(tmp_path):
    p = cpg_b200.gen_params(**cases.CASES["small_f32_s11"]["gen"])
    path = str(tmp_path / "g.txt")
    d = cpg_b200.generate(p, text_path=path)
    g = oracle.OracleGraph.from_text(path)
    adjp, adj, w = g.csr()
    ref = oracle.OracleGraph.from_edges(d.n, d.src, d.dst, d.w)
    radjp, radj, rw = ref.csr()
    assert np.array_equal(adjp, radjp) and np.array_equal(adj, radj)
    assert np.array_equal(w.view(np.uint32), rw.view(np.uint32))  # %.9g round-trips
    # python writer agrees with the library writer byte for byte
    path2 = str(tmp_path / "g2.txt")
    cpg_b200.write_text(d, path2)
    assert open(path).read() == open(path2).read()


def test_cpp_shim_compiles():
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    src = os.path.join(ROOT, "tests", "cpp", "shim_example.cpp")
    r = subprocess.run([gxx, "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), src],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
