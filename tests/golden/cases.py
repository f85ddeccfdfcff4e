"""Golden cases: graphs (seeded generator settings or extracted reference
fixtures) and the K at which the reference's G-PathGen was run on them.

The synthetic settings follow the workload shapes: the 20,000-pin / 60-level
single query (out-degree U{1..4}, level span 3, 64 sources / 64 sinks), the
1,000,000-pin / 200-level query (geometric out-degree of mean 20 capped at 256,
level span 4, 2,000 sources / 2,000 sinks) in fp32 and integer delays, the
same generator at mean degree 10/30/40/50, and small random DAGs for breadth.
"""
import os

HERE = os.path.dirname(os.path.abspath(__file__))

SINGLE_20K = dict(n_pins=20000, n_levels=60, n_first=64, n_last=64, level_span=3,
                  degree_kind=0, deg_lo=1, deg_hi=4)
LARGE_1M = dict(n_pins=1_000_000, n_levels=200, n_first=2000, n_last=2000, level_span=4,
                degree_kind=1, deg_mean=20.0, deg_cap=256)
SMALL = dict(n_pins=3000, n_levels=24, n_first=16, n_last=16, level_span=3,
             degree_kind=0, deg_lo=1, deg_hi=6)

FLOAT_W = dict(weight_kind=0, w_lo=0.1, w_hi=10.0)
INT_W = dict(weight_kind=1, iw_lo=1, iw_hi=100)

CASES = {
    "simple": dict(kind="npz", ks=[1000]),
    "dac21_paper_example": dict(kind="npz", ks=[1000]),
    "tv80_unit_wgts": dict(kind="npz", ks=[10000]),
    "single20k_f32": dict(kind="gen", gen=dict(seed=1, **SINGLE_20K, **FLOAT_W), ks=[10000]),
    "single20k_int": dict(kind="gen", gen=dict(seed=1, **SINGLE_20K, **INT_W), ks=[10000]),
    "small_f32_s11": dict(kind="gen", gen=dict(seed=11, **SMALL, **FLOAT_W), ks=[20000]),
    "small_f32_s12": dict(kind="gen", gen=dict(seed=12, **SMALL, **FLOAT_W), ks=[20000]),
    "small_int_s13": dict(kind="gen", gen=dict(seed=13, **SMALL, **INT_W), ks=[20000]),
    "small_int_s14": dict(kind="gen", gen=dict(seed=14, **SMALL, **INT_W), ks=[20000]),
    "large1m_f32": dict(kind="gen", gen=dict(seed=2, **LARGE_1M, **FLOAT_W), ks=[1_000_000],
                        large=True),
    "large1m_int": dict(kind="gen", gen=dict(seed=2, **LARGE_1M, **INT_W), ks=[1_000_000],
                        large=True),
}

# density sweep on the 1M-pin generator (run separately: large text files)
SWEEP = {
    "large1m_d10": (10.0, 1_000_000),
    "large1m_d30": (30.0, 200_000),
    "large1m_d40": (40.0, 200_000),
    "large1m_d50": (50.0, 100_000),
}
for _name, (_deg, _k) in SWEEP.items():
    CASES[_name] = dict(kind="gen", gen=dict(seed=3, **{**LARGE_1M, "deg_mean": _deg}, **FLOAT_W),
                        ks=[_k], large=True, sweep=True)


def load_case(name):
    """(n, src, dst, w) numpy arrays of a case's graph.  Synthetic cases come
    from the oracle's generator, which gives the same edge lists as the
    product's cpg_dag_generate (tests/test_oracle.py checks that), so test
    inputs never depend on the library under test."""
    import numpy as np
    c = CASES[name]
    if c["kind"] == "npz":
        z = np.load(os.path.join(HERE, "inputs", name + ".npz"))
        return int(z["n"]), z["src"], z["dst"], z["w"]
    import oracle
    return oracle.generate(**c["gen"])
