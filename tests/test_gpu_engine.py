"""Batched engine (ensemble / serving members in one launch per step) against
the FP32 oracle run of each member alone."""
import numpy as np
import pytest

from comcot_b200 import synth
from comcot_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _case(nx, ny, seed, nsteps, ngauges=3):
    return synth.single_layer_case("m", nx, ny, 2.0, 2.0, nsteps, seed=seed, n_seamounts=3,
                                   shelf_cols=max(2, nx // 10), land_cols=max(1, nx // 30), source="dipole",
                                   ngauges=ngauges)


def _oracle(case, oracle_mod):
    o = oracle_mod.OracleRun(case)
    ts = o.run(case.nsteps)
    return o.layer(0), ts


@pytest.mark.parametrize("graphs", [0, 1])
def test_engine_mixed_sizes_match_oracle(oracle_mod, graphs):
    cases = [_case(97, 81, 21, 70), _case(61, 45, 22, 40), _case(130, 70, 23, 70)]
    with Engine(budget=2 << 30) as eng:
        eng.config(variant=-1, use_graphs=graphs, chunk=16)
        ids = [eng.add(c) for c in cases]
        eng.step(80)
        eng.sync()
        for c, mid in zip(cases, ids):
            assert eng.done(mid)
            got = eng.read(mid)
            ref, ts = _oracle(c, oracle_mod)
            for k in ("z", "m", "n", "zmax"):
                assert np.array_equal(got[k].view(np.uint32), ref[k].view(np.uint32)), k
            assert np.array_equal(got["arrival"], ref["arrival"])
            assert np.array_equal(got["ts"].view(np.uint32), ts.view(np.uint32))


def test_engine_member_same_alone_and_in_mix(oracle_mod):
    a = _case(97, 81, 31, 50)
    b = _case(120, 90, 32, 60)
    with Engine(budget=2 << 30) as e1:
        ia = e1.add(a)
        e1.step(60)
        alone = e1.read(ia)
    with Engine(budget=2 << 30) as e2:
        ib = e2.add(b)
        e2.step(7)                   # b already running when a arrives
        ia = e2.add(a)
        e2.step(60)
        mixed = e2.read(ia)
    for k in ("z", "m", "n", "zmax", "ts"):
        assert np.array_equal(alone[k].view(np.uint32), mixed[k].view(np.uint32)), k


def test_engine_budget_refuses():
    c = _case(97, 81, 41, 10)
    with Engine(budget=200 << 10) as eng:      # room for the class, not the member
        cls = eng.add_class(c.root)
        assert eng.member_bytes(cls) > (200 << 10) - eng.bytes_in_use()
        with pytest.raises(MemoryError):
            eng.add(c, cls=cls)


def _nested(seed, rel_time, nsteps, child_gauges=3):
    case = synth.nested_case("n", 97, 81, 2.0, 2.0, [60, 79, 30, 49], 3, nsteps, seed=seed, rel_time=rel_time,
                             ngauges=3)
    Cl = case.layers[1]
    rng = np.random.default_rng(seed + 100)
    got = 0
    while got < child_gauges:
        i = int(rng.integers(3, Cl.nx - 3))
        j = int(rng.integers(3, Cl.ny - 3))
        if Cl.H[j, i] <= 5.0:
            continue
        x0 = float(Cl.x[i] + 0.4 * (Cl.x[i + 1] - Cl.x[i]))
        y0 = float(Cl.y[j] + 0.7 * (Cl.y[j + 1] - Cl.y[j]))
        ki, kj, cx, cy = synth.pc.locate_gauge(Cl.x, Cl.y, x0, y0, first=2)
        case.gauges.append((Cl.id, ki, kj, float(cx), float(cy)))
        got += 1
    return case


def _check_nested(got, case, oracle_mod):
    o = oracle_mod.OracleRun(case)
    ts = o.run(case.nsteps)
    ref, rc = o.layer(0), o.layer(1)
    for k in ("z", "m", "n", "zmax"):
        assert np.array_equal(got[k].view(np.uint32), ref[k].view(np.uint32)), k
    assert np.array_equal(got["arrival"], ref["arrival"])
    for k in ("z", "m", "n"):
        assert np.array_equal(got["child_" + k].view(np.uint32), rc[k].view(np.uint32)), "child " + k
    H = case.layers[1].H
    assert np.array_equal(got["child_z"] + H > 1e-5, rc["z"] + H > 1e-5)
    assert np.array_equal(got["ts"].view(np.uint32), ts.view(np.uint32))


@pytest.mark.parametrize("rel_time,graphs", [(None, 1), (2, 0), (3, 1)])
def test_engine_nested_member_matches_oracle(oracle_mod, rel_time, graphs):
    case = _nested(51, rel_time, 40)
    with Engine(budget=2 << 30) as eng:
        eng.config(variant=-1, use_graphs=graphs, chunk=8)
        mid = eng.add(case)
        eng.step(45)
        eng.sync()
        assert eng.done(mid)
        _check_nested(eng.read(mid), case, oracle_mod)


@pytest.mark.parametrize("graphs", [0, 1])
def test_engine_feedback_gauges_on_the_window(oracle_mod, graphs):
    """one child sub-step per outer step (JNZ, the window's momentum and the
    outputs in one launch): outer gauges whose stencils lie inside the JNZ
    window, across its edges and at its corner, beside child gauges, bit for
    bit against the oracle"""
    case = _nested(71, 1, 40)
    P, C = case.layers
    jj, ii = np.mgrid[0:C.ny, 0:C.nx]
    bump = 0.8 * np.exp(-((ii - 0.4 * C.nx) ** 2 + (jj - 0.6 * C.ny) ** 2) / (2.0 * 8.0 ** 2))
    C.Z0 = np.where(C.H > 0.0, bump, 0.0).astype(np.float32)  # the feedback carries a wave from the start
    is_, ie, js, je = 60, 79, 30, 49  # the child's window on the outer grid, 1-based
    for ki, kj in ((is_ + 5, js + 5), (is_ - 1, js + 3), (ie, je), (is_ + 2, je), (ie - 3, js - 1)):
        case.gauges.append((P.id, ki, kj, 0.3, 0.6))
    with Engine(budget=2 << 30) as eng:
        eng.config(variant=-1, use_graphs=graphs, chunk=8)
        mid = eng.add(case)
        eng.step(45)
        eng.sync()
        assert eng.done(mid)
        _check_nested(eng.read(mid), case, oracle_mod)


@pytest.mark.parametrize("laygov,rel_time", [(1, 1), (0, 2)])
def test_engine_wide_child_matches_oracle(oracle_mod, laygov, rel_time):
    """a 151 x 151 child (interior CONMOME blocks, two-cell JNQ + mass threads)"""
    case = synth.nested_case("w", 241, 161, 2.0, 2.0, [150, 199, 50, 99], 3, 30, seed=23, rel_time=rel_time,
                             child_laygov=laygov, ngauges=2)
    C = case.layers[1]
    jj, ii = np.mgrid[0:C.ny, 0:C.nx]
    bump = 0.8 * np.exp(-((ii - 0.45 * C.nx) ** 2 + (jj - 0.55 * C.ny) ** 2) / (2.0 * 18.0 ** 2))
    C.Z0 = np.where(C.H > 0.0, bump, 0.0).astype(np.float32)
    with Engine(budget=2 << 30) as eng:
        eng.config(variant=-1, use_graphs=1, chunk=8)
        mid = eng.add(case)
        eng.step(32)
        eng.sync()
        assert eng.done(mid)
        _check_nested(eng.read(mid), case, oracle_mod)


def test_engine_nested_and_single_members_in_one_mix(oracle_mod):
    nest = [_nested(61, 2, 34), _nested(62, None, 50)]
    single = [_case(97, 81, 63, 41), _case(70, 60, 64, 66)]
    with Engine(budget=2 << 30) as eng:
        eng.config(variant=-1, use_graphs=1, chunk=6)
        ids = [eng.add(single[0]), eng.add(nest[0])]
        eng.step(5)                                  # later arrivals join a running batch
        ids += [eng.add(nest[1]), eng.add(single[1])]
        eng.step(80)
        eng.sync()
        got = [eng.read(i) for i in ids]
    _check_nested(got[1], nest[0], oracle_mod)
    _check_nested(got[2], nest[1], oracle_mod)
    for g, c in ((got[0], single[0]), (got[3], single[1])):
        ref, ts = _oracle(c, oracle_mod)
        for k in ("z", "m", "n", "zmax"):
            assert np.array_equal(g[k].view(np.uint32), ref[k].view(np.uint32)), k
        assert np.array_equal(g["ts"].view(np.uint32), ts.view(np.uint32))


def test_every_tile_variant_matches_oracle(oracle_mod):
    """the tile variants (warps, stages, copy issue, staged or direct Z1/max)
    differ only in data movement: each must give the oracle's bits"""
    from comcot_b200 import _lib

    nvar = _lib.load().gc_engine_num_variants()
    assert nvar >= 8
    cases = [_case(97, 81, 81, 30), _case(130, 70, 82, 30), _case(33, 17, 83, 30), _case(300, 140, 84, 30)]
    refs = [_oracle(c, oracle_mod) for c in cases]
    # every variant with tile-height rule 0, and every second one with rule 1
    for v in list(range(nvar)) + list(range(nvar, 2 * nvar, 2)):
        with Engine(budget=1 << 30) as eng:
            eng.config(variant=v, use_graphs=v % 2, chunk=8)
            ids = [eng.add(c) for c in cases]
            eng.step(31)
            eng.sync()
            for c, mid, (ref, ts) in zip(cases, ids, refs):
                got = eng.read(mid)
                for k in ("z", "m", "n", "zmax"):
                    assert np.array_equal(got[k].view(np.uint32), ref[k].view(np.uint32)), (v, c.root.nx, k)
                assert np.array_equal(got["arrival"], ref["arrival"]), v
                assert np.array_equal(got["ts"].view(np.uint32), ts.view(np.uint32)), v


def test_members_joining_mid_run(oracle_mod):
    """members of different sizes, start steps and lengths, captured in
    graphs and stepped eagerly, with the default tile variant"""
    cases = [_case(257, 129, 91, 75), _case(97, 81, 92, 40), _case(500, 60, 93, 61)]
    with Engine(budget=1 << 30) as eng:
        eng.config(variant=15, use_graphs=1, chunk=10)
        a = eng.add(cases[0])
        eng.step(13)
        b = eng.add(cases[1])
        eng.step(9)
        c = eng.add(cases[2])
        eng.step(90)
        eng.sync()
        got = [eng.read(i) for i in (a, b, c)]
    for g, cs in zip(got, cases):
        ref, ts = _oracle(cs, oracle_mod)
        for k in ("z", "m", "n", "zmax"):
            assert np.array_equal(g[k].view(np.uint32), ref[k].view(np.uint32)), (cs.root.nx, k)
        assert np.array_equal(g["arrival"], ref["arrival"])
        assert np.array_equal(g["ts"].view(np.uint32), ts.view(np.uint32))


@pytest.mark.parametrize("kind", ["sc_option_1", "sc_option_1_rel1", "dispersion_cartesian", "nonlinear_spherical",
                                  "dispersion_spherical"])
def test_engine_nested_child_kinds_match_oracle(oracle_mod, kind):
    """nested engine members whose child is coupled by SC_OPTION = 1 (UTM
    tables, band forecast in member scratch), or runs MASS_C_D/MOMT_C_D,
    CONMASS_S/CONMOME_S or MASS_S_D/MOMT_S_D: bitwise equal to the oracle,
    with graphs, rel_time 2 (and 1 for SC_OPTION = 1, where JNZ_SC falls in
    the first sub-step and reads the child's row and column 0 before UPDATE)"""
    if kind == "sc_option_1":
        case = synth.nested_sc_case("k", 97, 81, 2.0, 2.0, [60, 79, 30, 49], 3, 40, seed=3, rel_time=2)
    elif kind == "sc_option_1_rel1":
        case = synth.nested_sc_case("k", 97, 81, 2.0, 2.0, [60, 79, 30, 49], 3, 40, seed=3, rel_time=1)
    elif kind == "dispersion_cartesian":
        case = synth.nested_case("k", 97, 81, 2.0, 2.0, [60, 79, 30, 49], 3, 40, seed=5, rel_time=2, child_laygov=2)
    elif kind == "nonlinear_spherical":
        case = synth.nested_case("k", 97, 81, 2.0, 2.0, [60, 79, 30, 49], 3, 40, seed=5, rel_time=2,
                                 child_laycord=0, child_laygov=1)
    else:
        case = synth.nested_case("k", 97, 81, 2.0, 2.0, [60, 79, 30, 49], 3, 40, seed=5, rel_time=2,
                                 child_laycord=0, child_laygov=2)
    case.gauges = case.gauges[:3]
    with Engine(budget=2 << 30) as eng:
        eng.config(variant=-1, use_graphs=1, chunk=8)
        mid = eng.add(case)
        eng.step(45)
        eng.sync()
        assert eng.done(mid)
        got = eng.read(mid)
    o = oracle_mod.OracleRun(case)
    o.run(case.nsteps)
    ref, rc = o.layer(0), o.layer(1)
    assert np.abs(rc["m"]).max() > 0
    for k in ("z", "m", "n", "zmax"):
        assert np.array_equal(got[k].view(np.uint32), ref[k].view(np.uint32)), k
    for k in ("z", "m", "n"):
        assert np.array_equal(got["child_" + k].view(np.uint32), rc[k].view(np.uint32)), "child " + k


def test_read_async_matches_read_and_outlives_release():
    """results copied behind the steps into page-locked memory equal the
    blocking read; the member is released before the copy is waited for"""
    cases = [_case(97, 81, 71, 40), _case(130, 70, 72, 33)]
    with Engine(budget=1 << 30) as eng:
        ids = [eng.add(c) for c in cases]
        eng.step(45)
        eng.sync()
        want = [eng.read(i, fields=("z", "zmax", "arrival", "ts")) for i in ids]
        pend = [eng.read_async(i, fields=("z", "zmax", "arrival", "ts")) for i in ids]
        for i in ids:
            eng.release(i)
        got = [p.take() for p in pend]
    for g, w in zip(got, want):
        for k in ("z", "zmax", "arrival", "ts"):
            assert np.array_equal(g[k], w[k]), k
