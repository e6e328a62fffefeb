"""The Okada (1985) deformation restatement (deform.f90): float and double
twins, spherical and Cartesian layers, several faults applied in order."""
import numpy as np
import pytest

FAULT = dict(hh=10000.0, l=200000.0, w=80000.0, d=8.0, th=200.0, dl=15.0, rd=90.0, x0=144.0, y0=33.3, sw=0)


def _axes(nx=121, ny=101):
    return 140.0 + np.arange(nx) * 4 / 60.0, 30.0 + np.arange(ny) * 4 / 60.0


def test_float_and_double_agree_off_the_singular_lines(oracle_mod):
    x, y = _axes()
    z32, _ = oracle_mod.okada_apply([FAULT], 0, len(x), len(y), x, y, dtype=np.float32)
    z64, _ = oracle_mod.okada_apply([FAULT], 0, len(x), len(y), x, y, dtype=np.float64)
    scale = np.abs(z64).max()
    assert 1.0 < scale < 5.0                      # metres of uplift for 8 m of thrust
    bad = np.abs(z32.astype(np.float64) - z64) > 1e-4 * scale
    # the reference's float evaluation jumps atan branches only on the lines
    # through the fault's ends; everywhere else the twins agree
    assert bad.mean() < 0.005


def test_faults_accumulate_in_order_on_z_and_h(oracle_mod):
    x, y = _axes(60, 50)
    f2 = dict(FAULT, x0=143.0, y0=32.5, rd=60.0, sw=9)
    h0 = np.full((50, 60), 3000.0)
    z1, h1 = oracle_mod.okada_apply([FAULT], 0, 60, 50, x, y, h=h0, dtype=np.float64)
    z2, h2 = oracle_mod.okada_apply([f2], 0, 60, 50, x, y, z=z1, h=h1, dtype=np.float64)
    zb, hb = oracle_mod.okada_apply([FAULT, f2], 0, 60, 50, x, y, h=h0, dtype=np.float64)
    assert np.array_equal(zb, z2) and np.array_equal(hb, h2)
    assert np.allclose(zb + hb, 3000.0)           # Z += D, H -= D


def test_cartesian_layer_uses_origin_and_spacing(oracle_mod):
    # the reference places a Cartesian cell at X = DX*(I-1) - XL with XL the
    # origin's projected offset from the epicentre (deform.f90:150-154)
    f = dict(FAULT, xo=143.0, yo=32.0)
    z, _ = oracle_mod.okada_apply([f], 1, 80, 70, dx=4000.0, dy=4000.0, dtype=np.float64)
    assert np.isfinite(z).all() and np.abs(z).max() > 0.01
