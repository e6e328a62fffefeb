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
