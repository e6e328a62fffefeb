"""GPU parity through the reference C ABI against the FP32 oracle.

The CUDA kernels evaluate the Fortran expressions in the Fortran order with
separately rounded float operations, so the expected result is bit-identical
to the oracle; the asserted bar is the stated tolerance
max|d eta| <= 1e-4 * max|eta| and max|d(M,N)| <= 1e-4 * max|M,N|, with
masks (wet/dry, arrival step) compared exactly.
"""
import numpy as np
import pytest

from comcot_b200 import synth
from comcot_b200.abi import ReferenceSession

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _cmp(a, b, what):
    scale = max(float(np.abs(b).max()), 1e-30)
    err = float(np.abs(a.astype(np.float64) - b.astype(np.float64)).max())
    assert err <= TOL * scale, f"{what}: max|diff|={err} scale={scale}"
    return err


def _run_both(case, nsteps, oracle_mod, fusion=True, arrival=True):
    s = ReferenceSession(case, fusion=fusion, arrival=arrival)
    try:
        ts = [s.step(maxamp=True) for _ in range(nsteps)]
        gpu = {"z": s.getz(1), "mn": s.getmn(1), "zmax": s.getzmax(1),
               "arrival": s.getarrival(1) if arrival else None,
               "children": [(s.getz(L.id), s.getmn(L.id)) for L in case.layers[1:]]}
    finally:
        s.close()
    o = oracle_mod.OracleRun(case)
    ots = o.run(nsteps, arrival=arrival)
    return gpu, np.array(ts, dtype=np.float32).reshape(nsteps, -1), o, ots


@pytest.mark.parametrize("fusion", [False, True])
def test_single_layer_small(oracle_mod, fusion):
    case = synth.single_layer_case("t", 97, 81, 2.0, 2.0, 0, seed=7, n_seamounts=5, shelf_cols=10,
                                   land_cols=4, ngauges=4)
    gpu, ts, o, ots = _run_both(case, 120, oracle_mod, fusion=fusion)
    ref = o.layer(0)
    _cmp(gpu["z"], ref["z"], "eta")
    _cmp(gpu["mn"][0], ref["m"], "M")
    _cmp(gpu["mn"][1], ref["n"], "N")
    _cmp(gpu["zmax"], ref["zmax"], "zmax")
    assert np.array_equal(gpu["arrival"], ref["arrival"])
    H = case.root.H
    assert np.array_equal(gpu["z"] + H > 1e-5, ref["z"] + H > 1e-5)
    if ts.size:
        _cmp(ts, ots, "gauges")
    # bit-identical is the design point
    assert np.array_equal(gpu["z"].view(np.uint32), ref["z"].view(np.uint32))
    assert np.array_equal(gpu["mn"][0].view(np.uint32), ref["m"].view(np.uint32))


@pytest.mark.parametrize("shape", [(33, 17), (130, 7), (7, 130), (257, 65)])
def test_single_layer_ragged(oracle_mod, shape):
    nx, ny = shape
    case = synth.single_layer_case("r", nx, ny, 2.0, 2.0, 0, seed=11, n_seamounts=2, shelf_cols=min(4, nx // 4),
                                   land_cols=min(2, nx // 8), ngauges=0)
    gpu, _, o, _ = _run_both(case, 40, oracle_mod)
    ref = o.layer(0)
    assert np.array_equal(gpu["z"].view(np.uint32), ref["z"].view(np.uint32))
    assert np.array_equal(gpu["mn"][0].view(np.uint32), ref["m"].view(np.uint32))
    assert np.array_equal(gpu["mn"][1].view(np.uint32), ref["n"].view(np.uint32))


@pytest.mark.parametrize("rel_time", [None, 2, 3])
def test_nested_nonlinear_child(oracle_mod, rel_time):
    case = synth.nested_case("n", 97, 81, 2.0, 2.0, [60, 79, 30, 49], 3, 0, seed=3, rel_time=rel_time)
    gpu, _, o, _ = _run_both(case, 60, oracle_mod)
    ref = o.layer(0)
    _cmp(gpu["z"], ref["z"], "parent eta")
    _cmp(gpu["mn"][0], ref["m"], "parent M")
    cz, (cm, cn) = gpu["children"][0]
    rc = o.layer(1)
    _cmp(cz, rc["z"], "child eta")
    _cmp(cm, rc["m"], "child M")
    _cmp(cn, rc["n"], "child N")
    # wet/dry mask of the child, bit-exact
    H = case.layers[1].H
    assert np.array_equal(cz + H > 1e-5, rc["z"] + H > 1e-5)
    assert np.array_equal(gpu["z"].view(np.uint32), ref["z"].view(np.uint32))
    assert np.array_equal(cz.view(np.uint32), rc["z"].view(np.uint32))


def _wide_nested(laygov, rel_time, seed):
    """a child 151 x 151 wide with a surface bump of its own: CONMOME blocks
    whose stencil window lies inside the child (fixed tile offsets) and the
    first sub-step's JNQ + mass launch with two cells per thread both run"""
    case = synth.nested_case("w", 241, 161, 2.0, 2.0, [150, 199, 50, 99], 3, 0, seed=seed, rel_time=rel_time,
                             child_laygov=laygov)
    C = case.layers[1]
    jj, ii = np.mgrid[0:C.ny, 0:C.nx]
    bump = 0.8 * np.exp(-((ii - 0.45 * C.nx) ** 2 + (jj - 0.55 * C.ny) ** 2) / (2.0 * 18.0 ** 2))
    C.Z0 = np.where(C.H > 0.0, bump, 0.0).astype(np.float32)
    return case


@pytest.mark.parametrize("laygov", [0, 1])
@pytest.mark.parametrize("rel_time", [1, 2])
def test_nested_wide_child(oracle_mod, laygov, rel_time):
    case = _wide_nested(laygov, rel_time, 21 + laygov)
    gpu, _, o, _ = _run_both(case, 30, oracle_mod)
    ref, rc = o.layer(0), o.layer(1)
    cz, (cm, cn) = gpu["children"][0]
    assert np.abs(rc["m"]).max() > 0 and np.abs(rc["n"]).max() > 0
    for a, b, what in ((gpu["z"], ref["z"], "parent eta"), (gpu["mn"][0], ref["m"], "parent M"),
                       (cz, rc["z"], "child eta"), (cm, rc["m"], "child M"), (cn, rc["n"], "child N")):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), what


@pytest.mark.parametrize("kind", ["linear_cartesian", "linear_spherical", "nonlinear_spherical"])
def test_nested_linear_child(oracle_mod, kind):
    """MASS_C/MOMT_C (LAYCORD 1, LAYGOV 0), MASS_S/MOMT_S and
    CONMASS_S/CONMOME_S (LAYCORD 0, LAYGOV 1) children"""
    kw = {"linear_cartesian": {"child_laygov": 0}, "linear_spherical": {"child_laycord": 0},
          "nonlinear_spherical": {"child_laycord": 0, "child_laygov": 1}}[kind]
    case = synth.nested_case("l", 97, 81, 2.0, 2.0, [60, 79, 30, 49], 3, 0, seed=5, rel_time=2, **kw)
    gpu, _, o, _ = _run_both(case, 50, oracle_mod)
    ref, rc = o.layer(0), o.layer(1)
    cz, (cm, cn) = gpu["children"][0]
    assert np.abs(rc["z"]).max() > 0 and np.abs(rc["m"]).max() > 0   # the child saw the wave
    for a, b, what in ((gpu["z"], ref["z"], "parent eta"), (cz, rc["z"], "child eta"), (cm, rc["m"], "child M"),
                       (cn, rc["n"], "child N")):
        _cmp(a, b, what)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), what


@pytest.mark.parametrize("shape", [(97, 81), (130, 7)])
def test_nonlinear_spherical_root(oracle_mod, shape):
    """CONMASS_S / CONMOME_S on the outermost layer, with land (wet/dry) and
    Manning friction; the fused linear kernel must not take it"""
    nx, ny = shape
    case = synth.single_layer_case("ns", nx, ny, 2.0, 2.0, 0, seed=13, n_seamounts=5, shelf_cols=min(10, nx // 4),
                                   land_cols=min(4, nx // 8), ngauges=0, laygov=1, amp=3.0)
    gpu, _, o, _ = _run_both(case, 80, oracle_mod)
    ref = o.layer(0)
    for a, b, what in ((gpu["z"], ref["z"], "eta"), (gpu["mn"][0], ref["m"], "M"), (gpu["mn"][1], ref["n"], "N"),
                       (gpu["zmax"], ref["zmax"], "zmax")):
        _cmp(a, b, what)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), what
    assert np.array_equal(gpu["arrival"], ref["arrival"])


@pytest.mark.parametrize("kind", ["sponge", "sponge_wall"])
def test_sponge_and_wall_outer_layer(oracle_mod, kind):
    """SPONGE_LAYER after the momentum step (boundaries.f90:206-247) and the
    BC_WALL bathymetry (boundaries.f90:388-428).  The coefficients are
    SPONGE_COEF's on metre axes (on degree axes they are all 0, as in the
    reference), here a band of about 7 cells along every edge."""
    from comcot_b200 import precompute as pc
    case = synth.single_layer_case("sp", 97, 81, 2.0, 2.0, 0, seed=21, n_seamounts=5, shelf_cols=10,
                                   land_cols=0, ngauges=0, amp=2.0)
    L = case.root
    if kind == "sponge_wall":
        L.H = pc.bc_wall(L.H)
        L.hp, L.hq = pc.pq_depth(L.H)
    L.sponge = pc.sponge_coef(np.arange(L.nx) * 20000.0, np.arange(L.ny) * 20000.0, L.H, 1)
    assert L.sponge[0].max() > 0
    gpu, _, o, _ = _run_both(case, 60, oracle_mod)
    ref = o.layer(0)
    assert np.isfinite(ref["m"]).all()
    band = (L.sponge[0] > 0) | (L.sponge[1] > 0)
    assert np.abs(ref["m"][band]).max() > 0   # the wave reached the band
    for a, b, what in ((gpu["z"], ref["z"], "eta"), (gpu["mn"][0], ref["m"], "M"), (gpu["mn"][1], ref["n"], "N"),
                       (gpu["zmax"], ref["zmax"], "zmax")):
        _cmp(a, b, what)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), what


@pytest.mark.parametrize("rel_time,fix_top,laygov", [(None, False, 1), (2, False, 1), (3, True, 1), (2, False, 0)])
def test_nested_sc_option_1_child(oracle_mod, rel_time, fix_top, laygov):
    """SC_OPTION = 1 (all_grids.f90:996-1425): a Cartesian child coupled to
    its spherical parent through per-node positions and bilinear weights;
    EDGE_INTERP_SC at the first sub-step, NEWQ_SC's band forecast and blend
    after it, JNZ_SC at the half step; bitwise against the oracle"""
    case = synth.nested_sc_case("sc", 97, 81, 2.0, 2.0, [60, 79, 30, 49], 3, 0, seed=3, rel_time=rel_time,
                                fix_top=fix_top, child_laygov=laygov)
    gpu, _, o, _ = _run_both(case, 50, oracle_mod)
    ref, rc = o.layer(0), o.layer(1)
    cz, (cm, cn) = gpu["children"][0]
    assert np.abs(rc["m"]).max() > 0
    for a, b, what in ((gpu["z"], ref["z"], "parent eta"), (gpu["mn"][0], ref["m"], "parent M"),
                       (cz, rc["z"], "child eta"), (cm, rc["m"], "child M"), (cn, rc["n"], "child N")):
        _cmp(a, b, what)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), what


@pytest.mark.parametrize("laygov", [2, 3])
def test_dispersion_scheme_outer_layer(oracle_mod, laygov):
    """MASS_S_D / MOMT_S_D (dispersion.f90:239-356, 544-838) as the reference
    computes them (its MASK is all zero): the modified-scheme term for
    LAYGOV 2 on the outer layer (MODSCM 0), the depth-free R2 / R4 of
    LAYGOV 3 (comcot.f90:776-795); with land"""
    case = synth.single_layer_case("d", 97, 81, 2.0, 2.0, 0, seed=13, n_seamounts=5, shelf_cols=10, land_cols=4,
                                   ngauges=0, laygov=laygov, amp=3.0)
    gpu, _, o, _ = _run_both(case, 80, oracle_mod)
    ref = o.layer(0)
    for a, b, what in ((gpu["z"], ref["z"], "eta"), (gpu["mn"][0], ref["m"], "M"), (gpu["mn"][1], ref["n"], "N"),
                       (gpu["zmax"], ref["zmax"], "zmax")):
        _cmp(a, b, what)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), what


@pytest.mark.parametrize("laygov,laycord,modscm", [(2, 1, 1), (3, 1, 0), (2, 0, 1)])
def test_dispersion_scheme_child(oracle_mod, laygov, laycord, modscm):
    """MASS_C_D / MOMT_C_D (dispersion.f90:357-543, 839-1692) and the
    spherical forms on a child: total face depth, Manning friction, dry faces
    keeping their flux; MODSCM 0 forced once to cover the modified-scheme term
    of the Cartesian form"""
    kw = {"child_laygov": laygov} if laycord == 1 else {"child_laycord": 0, "child_laygov": laygov}
    case = synth.nested_case("d", 97, 81, 2.0, 2.0, [60, 79, 30, 49], 3, 0, seed=5, rel_time=2, **kw)
    case.layers[1].modscm = modscm
    gpu, _, o, _ = _run_both(case, 50, oracle_mod)
    ref, rc = o.layer(0), o.layer(1)
    cz, (cm, cn) = gpu["children"][0]
    assert np.abs(rc["m"]).max() > 0
    for a, b, what in ((gpu["z"], ref["z"], "parent eta"), (cz, rc["z"], "child eta"), (cm, rc["m"], "child M"),
                       (cn, rc["n"], "child N")):
        _cmp(a, b, what)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), what


@pytest.mark.parametrize("modscm,rel_time", [(1, 2), (0, 2), (0, None)])
def test_nonlinear_child_update_edges(oracle_mod, modscm, rel_time):
    """UPDATE's edge copy of a nonlinear Cartesian child (all_grids.f90:323-324)
    rides in the CONMOME launch when the child has no MODSCM term (nothing
    there reads the surface on row or column 0), and is a launch of its own
    after the momentum otherwise (MODSCM 0 forced); both bitwise against the
    oracle, over sub-steps before and after JNZ"""
    case = synth.nested_case("u", 97, 81, 2.0, 2.0, [60, 79, 30, 49], 3, 0, seed=9, rel_time=rel_time)
    case.layers[1].modscm = modscm
    gpu, _, o, _ = _run_both(case, 50, oracle_mod)
    ref, rc = o.layer(0), o.layer(1)
    cz, (cm, cn) = gpu["children"][0]
    assert np.abs(rc["m"]).max() > 0
    assert np.array_equal(rc["z"][0, 1:], rc["z"][1, 1:]) and np.array_equal(rc["z"][1:, 0], rc["z"][1:, 1])
    for a, b, what in ((gpu["z"], ref["z"], "parent eta"), (cz, rc["z"], "child eta"), (cm, rc["m"], "child M"),
                       (cn, rc["n"], "child N")):
        _cmp(a, b, what)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), what
