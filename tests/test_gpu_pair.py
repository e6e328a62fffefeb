"""The two-step kernel (kernels_pair.cu): two outer steps per launch, step
A's surface and fluxes kept on chip.  Every candidate (warps x pipeline
stages x tile-height rule) against the FP32 oracle bit for bit on ragged grid
shapes, including widths at the tile boundaries (120-column strides, first
and last tiles without a halo) and grids fewer rows high than the tile's
halo; runs of odd length, so the last step goes through the one-step kernel;
members joining and leaving mid-run with graphs; and the same large grid
through the one-step and the two-step kernels."""
import numpy as np
import pytest

from comcot_b200 import _lib, synth
from comcot_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _case(nx, ny, seed, nsteps, ngauges=3):
    thin = min(nx, ny) <= 12
    case = synth.single_layer_case("p", nx, ny, 2.0, 2.0, nsteps, seed=seed, n_seamounts=3,
                                   shelf_cols=max(2, nx // 10), land_cols=max(1, nx // 30), source="dipole",
                                   ngauges=0 if thin else ngauges)
    if thin:  # too few rows for the random wet-gauge placement: one gauge by hand
        case.gauges = [(1, max(1, nx // 3), max(1, ny // 2), 0.25, 0.75)]
    return case


def _oracle(case, oracle_mod):
    o = oracle_mod.OracleRun(case)
    ts = o.run(case.nsteps)
    return o.layer(0), ts


def _candidates():
    lib = _lib.load()
    n1 = 2 * lib.gc_engine_num_variants()      # one-step variants x 2 tile-height rules
    return n1, list(range(n1, lib.gc_engine_num_candidates()))


def _same(got, ref, ts, what):
    for k in ("z", "m", "n", "zmax"):
        assert np.array_equal(got[k].view(np.uint32), ref[k].view(np.uint32)), (what, k)
    assert np.array_equal(got["arrival"], ref["arrival"]), what
    assert np.array_equal(got["ts"].view(np.uint32), ts.view(np.uint32)), what


SHAPES = [(97, 81), (130, 70), (33, 17), (300, 140), (128, 9), (129, 5), (248, 40), (249, 41), (367, 6),
          (12, 200)]


def test_every_pair_candidate_matches_oracle(oracle_mod):
    n1, pair = _candidates()
    assert len(pair) >= 4
    cases = [_case(nx, ny, 100 + k, 31) for k, (nx, ny) in enumerate(SHAPES)]
    refs = [_oracle(c, oracle_mod) for c in cases]
    for v in pair:
        with Engine(budget=2 << 30) as eng:
            eng.config(variant=v, use_graphs=v % 2, chunk=8)
            ids = [eng.add(c) for c in cases]
            eng.step(33)
            eng.sync()
            assert eng.variant() == v
            for c, mid, (ref, ts) in zip(cases, ids, refs):
                assert eng.done(mid)
                _same(eng.read(mid), ref, ts, (v, c.root.nx, c.root.ny))


def test_single_grid_pair_launches_match_oracle(oracle_mod):
    """one member: the single-grid form of the kernel (descriptor by value)"""
    n1, pair = _candidates()
    for (nx, ny), v in zip([(97, 81), (249, 41), (1201, 1001)], pair):
        case = _case(nx, ny, 7, 24, ngauges=6)
        ref, ts = _oracle(case, oracle_mod)
        with Engine(budget=2 << 30) as eng:
            eng.config(variant=v, use_graphs=1, chunk=8)
            mid = eng.add(case)
            eng.step(26)
            eng.sync()
            _same(eng.read(mid), ref, ts, (v, nx, ny))


def test_pair_members_joining_mid_run(oracle_mod):
    """members of different sizes, start steps (odd and even) and lengths,
    captured in graphs and stepped eagerly: pairs, single steps and gauge
    samples interleave"""
    n1, pair = _candidates()
    cases = [_case(257, 129, 91, 75), _case(97, 81, 92, 40), _case(500, 60, 93, 61), _case(61, 45, 94, 12)]
    with Engine(budget=2 << 30) as eng:
        eng.config(variant=pair[0], use_graphs=1, chunk=10)
        a = eng.add(cases[0])
        eng.step(13)
        b = eng.add(cases[1])
        eng.step(9)
        c = eng.add(cases[2])
        d = eng.add(cases[3])
        eng.step(90)
        eng.sync()
        got = [eng.read(i) for i in (a, b, c, d)]
    for g, cs in zip(got, cases):
        ref, ts = _oracle(cs, oracle_mod)
        _same(g, ref, ts, cs.root.nx)


def test_one_step_and_two_step_kernels_agree_on_a_shared_grid(oracle_mod):
    """four members on one 1201 x 1001 grid with shared bathymetry (the C4
    grid), 40 steps: the one-step kernel and the two-step kernel give the
    oracle's bits"""
    n1, pair = _candidates()
    L = synth.config_c4_grid()
    srcs = synth.ensemble_sources(L.x, L.y, 4, seed=40)
    cases = [synth.Case("C4", [synth.LayerSpec(**{**L.__dict__, "Z0": np.ascontiguousarray(z, np.float32)})], 40)
             for z in srcs]
    refs = []
    for c in cases:
        o = oracle_mod.OracleRun(c)
        o.run(40, threads=8)
        refs.append(o.layer(0))
    for v in (16, pair[0], pair[-1]):
        with Engine(budget=4 << 30) as eng:
            eng.config(variant=v, use_graphs=1, chunk=8)
            cls = eng.add_class(L)
            ids = [eng.add(c, cls=cls, gauges=[], arrival_thr=0.05) for c in cases]
            eng.step(41)
            eng.sync()
            for mid, ref in zip(ids, refs):
                got = eng.read(mid, fields=("z", "m", "n", "zmax", "arrival"))
                for k in ("z", "m", "n", "zmax"):
                    assert np.array_equal(got[k].view(np.uint32), ref[k].view(np.uint32)), (v, k)
                assert np.array_equal(got["arrival"], ref["arrival"]), v


def test_class_launch_members_of_one_grid(oracle_mod):
    """members sharing one grid class go out as a class launch (member table in
    the parameter bank): different initial surfaces, gauges, start steps and
    lengths, in graphs and eagerly, against the oracle bit for bit"""
    n1, pair = _candidates()
    base = _case(300, 140, 71, 60, ngauges=4)
    L = base.root
    rng = np.random.default_rng(72)
    z0s = [np.ascontiguousarray(L.Z0 * float(rng.uniform(0.5, 1.5)), dtype=np.float32) for _ in range(5)]
    lens = [60, 31, 44, 60, 17]
    cases = [synth.Case("k", [synth.LayerSpec(**{**L.__dict__, "Z0": z})], n, gauges=base.gauges)
             for z, n in zip(z0s, lens)]
    refs = [_oracle(c, oracle_mod) for c in cases]
    for v in (pair[0], pair[-1], pair[-2]):
        for graphs in (0, 1):
            with Engine(budget=2 << 30) as eng:
                eng.config(variant=v, use_graphs=graphs, chunk=8)
                cls = eng.add_class(L)
                ids = [eng.add(cases[0], cls=cls), eng.add(cases[1], cls=cls)]
                eng.step(7)
                ids += [eng.add(c, cls=cls) for c in cases[2:]]
                eng.step(70)
                eng.sync()
                for c, mid, (ref, ts) in zip(cases, ids, refs):
                    assert eng.done(mid)
                    _same(eng.read(mid), ref, ts, (v, graphs, c.nsteps))
