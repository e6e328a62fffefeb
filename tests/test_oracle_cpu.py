"""CPU checks of the oracle (test infrastructure) itself."""
import math

import numpy as np
import pytest

import numpy_restatement as nr
from comcot_b200 import synth


def _case(nx=61, ny=47, seed=5):
    return synth.single_layer_case("o", nx, ny, 2.0, 2.0, 0, seed=seed, n_seamounts=3, shelf_cols=6,
                                   land_cols=3, source="dipole", amp=2.0)


def test_oracle_matches_independent_numpy_restatement_bitwise(oracle_mod):
    case = _case()
    o = oracle_mod.OracleRun(case)
    o.run(40, arrival=False)
    z, m, n, zmax = nr.run_single(case.root, 40)
    got = o.layer(0)
    for a, b in ((got["z"], z), (got["m"], m), (got["n"], n), (got["zmax"], zmax)):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("x", [-103.0, -87.5, -20.0, -1.0, -1e-3, 0.0, 1e-7, 0.37, 1.0, 3.5, 40.0, 88.5])
def test_shared_exp_close_to_libm(oracle_mod, x):
    lib = oracle_mod.load(np.float32)
    got = lib.ocl_expf(np.float32(x))
    want = np.float32(math.exp(float(np.float32(x))))
    assert abs(int(np.float32(got).view(np.int32)) - int(want.view(np.int32))) <= 1


def test_shared_exp_random_sweep(oracle_mod):
    lib = oracle_mod.load(np.float32)
    rng = np.random.default_rng(0)
    xs = rng.uniform(-30, 30, 2000).astype(np.float32)
    bad = 0
    for x in xs:
        got = np.float32(lib.ocl_expf(x))
        want = np.float32(math.exp(float(x)))
        d = abs(int(got.view(np.int32)) - int(want.view(np.int32)))
        assert d <= 1
        bad += d
    assert bad <= 5  # correctly rounded almost everywhere


def test_shared_pow_close_to_libm(oracle_mod):
    lib = oracle_mod.load(np.float32)
    rng = np.random.default_rng(1)
    for x in np.concatenate([rng.uniform(1e-3, 300.0, 1000), [1e-3, 1.0, 2.0, 1e-30]]).astype(np.float32):
        got = np.float32(lib.ocl_powf(x, np.float32(2.3333333)))
        want = np.float32(float(x) ** float(np.float32(2.3333333)))
        assert abs(int(got.view(np.int32)) - int(want.view(np.int32))) <= 1
    assert lib.ocl_powf(np.float32(0.0), np.float32(2.3333333)) == 0.0
    assert lib.ocl_expf(np.float32(-200.0)) == 0.0
    assert math.isinf(lib.ocl_expf(np.float32(100.0)))


def test_linear_scaling_fp64_twin(oracle_mod):
    """the linear equations scale with the source amplitude (FP64 twin, far
    from the EPS clamps)"""
    case = _case(seed=9)
    o1 = oracle_mod.OracleRun(case, dtype=np.float64)
    o1.run(30, arrival=False)
    case2 = _case(seed=9)
    case2.root.Z0 = (case2.root.Z0.astype(np.float64) * 2.0).astype(np.float32)
    o2 = oracle_mod.OracleRun(case2, dtype=np.float64)
    o2.run(30, arrival=False)
    a, b = o1.layer(0)["z"], o2.layer(0)["z"]
    wet = case.root.H > 1e-5
    assert np.allclose(2.0 * a[wet], b[wet], rtol=1e-9, atol=1e-12)


def test_float_vs_fp64_error_small(oracle_mod):
    case = _case(seed=13)
    o32 = oracle_mod.OracleRun(case)
    o32.run(60, arrival=False)
    o64 = oracle_mod.OracleRun(case, dtype=np.float64)
    o64.run(60, arrival=False)
    a, b = o32.layer(0)["z"].astype(np.float64), o64.layer(0)["z"]
    assert np.abs(a - b).max() <= 1e-4 * np.abs(b).max()


def test_nested_oracle_runs_and_conserves_masks(oracle_mod):
    case = synth.nested_case("n", 97, 81, 2.0, 2.0, [60, 79, 30, 49], 3, 0, seed=3, rel_time=2)
    o = oracle_mod.OracleRun(case)
    o.run(30)
    c = o.layer(1)
    H = case.layers[1].H
    # dry cells sit at -H, wet cells have DZ = Z + H >= GX (CONMASS, mass.f90:201-218)
    dry = c["z"] + H < 1e-5
    assert np.all(c["z"][dry & (H > -50)] == -H[dry & (H > -50)])
    assert np.all(np.isfinite(c["z"]))
    assert np.all(np.abs(c["m"]) <= 20.0 * np.maximum(c["z"] + H, 0) + 1e-3)


def test_division_shortcuts_are_ieee_identities():
    """The momentum kernels skip a correctly rounded division where IEEE 754
    fixes its result: a signed zero over a positive divisor is that zero, and
    a number over exactly 1 is itself.  Checked here on the host's IEEE
    binary32 division over zeros, subnormals, normals, the largest finite
    value and infinity; a NaN or non-positive divisor never takes the
    shortcut."""
    f32 = np.float32
    tiny = np.finfo(f32).tiny
    smallest = f32(np.nextafter(f32(0), f32(1)))
    divisors = np.array([smallest, tiny, f32(1e-3), f32(1.0), f32(2.0), f32(7.25), np.finfo(f32).max, np.inf],
                        dtype=f32)
    with np.errstate(all="ignore"):
        for a in (f32(0.0), f32(-0.0)):
            q = (np.full_like(divisors, a) / divisors).astype(f32)
            assert np.array_equal(q.view(np.uint32), np.full_like(divisors, a).view(np.uint32))
        nums = np.array([f32(0.0), f32(-0.0), smallest, -smallest, tiny, f32(1e-30), f32(0.1), f32(-3.5), f32(1e30),
                         np.finfo(f32).max, np.inf, -np.inf], dtype=f32)
        q = (nums / f32(1.0)).astype(f32)
        assert np.array_equal(q.view(np.uint32), nums.view(np.uint32))
        # the cases left to the division: 0/0, 0/-x, 0/NaN are not the zero itself
        assert np.isnan(f32(0.0) / f32(0.0))
        assert (f32(0.0) / f32(-2.0)).view(np.uint32) != f32(0.0).view(np.uint32)
        assert np.isnan(f32(0.0) / f32(np.nan))


def test_arrival_definition(oracle_mod):
    """Arrival step (no counterpart in the reference; the CUDA paths share this
    definition): 0 on a wet cell whose initial surface is already above the
    threshold, else the first outer step after which its surface is above it,
    -1 where that never happens and on dry cells.  The expectation is built
    from the surfaces of a step-by-step run, then compared with one run of
    all the steps."""
    case = _case(seed=17)
    L = case.root
    thr = np.float32(case.arrival_thr)
    wet = L.H > np.float32(1e-5)            # CC_GX
    nsteps = 25
    step_by_step = oracle_mod.OracleRun(case)
    expect = np.where(wet & (L.Z0 > thr), 0, -1).astype(np.int32)
    assert np.array_equal(step_by_step.layer(0)["arrival"], expect)
    for k in range(1, nsteps + 1):
        step_by_step.run(1)
        z = step_by_step.layer(0)["z"]
        expect = np.where((expect < 0) & wet & (z > thr), k, expect).astype(np.int32)
    whole = oracle_mod.OracleRun(case)
    whole.run(nsteps)
    assert np.array_equal(whole.layer(0)["arrival"], expect)
    assert (expect == 0).sum() > 0 and (expect > 0).sum() > 0 and (expect < 0).sum() > 0


def test_split_runs_number_steps_like_one_run(oracle_mod):
    """arrival steps are the forecast's step numbers: a run continued in a
    second call gives the same state as one call (the parity checks of the
    benchmark snapshot the oracle midway)"""
    import numpy as np

    from comcot_b200 import synth

    case = synth.config_c1(nsteps=240)
    a = oracle_mod.OracleRun(case)
    a.run(240, threads=4)
    b = oracle_mod.OracleRun(case)
    b.run(100, threads=4)
    b.run(140, threads=4)
    for k in ("z", "m", "n", "zmax", "arrival"):
        assert np.array_equal(a.layer(0)[k], b.layer(0)[k]), k
    assert (a.layer(0)["arrival"] > 100).sum() > 0   # arrivals in the second call
