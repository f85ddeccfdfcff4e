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


def test_cpp_shim_links_and_fails_loudly_without_device(tmp_path):
    """The reference-style C++ caller links against the library (every
    symbol the shim uses resolves) and, with no device, stops with the
    library's error instead of falling back to anything."""
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a device is present")
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    libdir = os.path.dirname(cpg_b200.LIB_PATH)
    exe = str(tmp_path / "shim_example")
    r = subprocess.run([gxx, "-std=c++17", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "cpp", "shim_example.cpp"),
                        "-L", libdir, "-lcpg_b200", f"-Wl,-rpath,{libdir}", "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([exe, str(tmp_path / "no_graph.txt"), "10"], capture_output=True, text=True)
    assert run.returncode == 1
    assert "no cuda device" in run.stderr
    assert run.stdout == ""


# ctypes mirror in cpg_b200.py -> the C typedef it must match byte for byte
_STRUCTS = {
    "Options": "cpg_options", "PathNode": "cpg_path_node", "Stats": "cpg_stats",
    "BatchStats": "cpg_batch_stats", "ServerOptions": "cpg_server_options",
    "ServerStats": "cpg_server_stats", "BvssInfo": "cpg_bvss_info",
    "BvssOpts": "cpg_bvss_opts", "BvssRunStats": "cpg_bvss_run_stats",
    "GenParams": "cpg_gen_params",
}


def test_ctypes_structs_match_header_layout(tmp_path):
    """Every struct the Python binding passes through the C ABI has the
    header's size and field offsets (a field added on one side only would
    silently shift the ones after it)."""
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no gcc")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "cpg.h"', "int main(void) {"]
    expect = []
    for py, c in _STRUCTS.items():
        cls = getattr(cpg_b200, py)
        lines.append(f'  printf("{py} size %zu\\n", sizeof({c}));')
        expect.append(f"{py} size {C.sizeof(cls)}")
        for f in cls._fields_:
            name = f[0]
            cname = name[:-1] if name.endswith("_") else name  # from_ -> from
            lines.append(f'  printf("{py}.{name} %zu\\n", offsetof({c}, {cname}));')
            expect.append(f"{py}.{name} {getattr(cls, name).offset}")
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    r = subprocess.run([gcc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = [g for g in got if g]
    diff = [(e, g) for e, g in zip(expect, got) if e != g]
    assert len(got) == len(expect) and not diff, diff


def test_options_init_defaults():
    """cpg_options_init gives the defaults the header documents."""
    o = cpg_b200.Options()
    cpg_b200.lib.cpg_options_init(C.byref(o))
    assert o.device == 0 and not o.stream
    assert o.division == cpg_b200.DIV_REFERENCE and o.frontier == cpg_b200.FRONTIER_AUTO
    assert o.hbm_budget_bytes == 0 and o.spin_limit == 0  # no cap; default poll limit
    assert o.host_stepped == 0 and o.bvss_min_bits == 0 and o.bvss_min_slices == 0
    assert o.sfxt_level_sync == 0 and o.sfxt_heap_warps == 0 and o.sfxt_late_push == 0
    assert o.sfxt_heap_mode == 0 and o.sfxt_claim_sets == 0 and o.engine_ctas == 0
