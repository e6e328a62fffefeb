"""The C-ABI library loads without a GPU and exports every declared entry."""
import pathlib
import re

from comcot_b200 import _lib

ROOT = pathlib.Path(__file__).resolve().parents[1]


def declared():
    src = (ROOT / "include" / "gcomcot.h").read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b([a-z_][a-z0-9_]*)\s*\(", src)) - {"if", "sizeof", "defined"})


def test_library_loads_and_exports_header():
    lib = _lib.load()
    names = declared()
    assert len(names) >= 40
    for n in names:
        assert hasattr(lib, n), n


def test_reference_abi_symbols_present():
    lib = _lib.load()
    for n in ("gcomcot_init_gpu_", "gcomcot_init_layer_", "mass_launch_", "momt_launch_", "openbd_launch_",
              "all_grid_launch_", "maxamp_launch_", "cuda_update_layer_", "gcomcot_get_z_", "cuda_getz_",
              "cuda_setz_", "cuda_getz1_", "cuda_setz1_", "cuda_getmn_", "cuda_setmn_", "cuda_getmn1_",
              "cuda_setmn1_", "cuda_getzmax_", "gcomcot_show_grids_", "cuda_shutdown_", "edgeinterp_dbglaunch_",
              "jnz_dbglaunch_"):
        assert hasattr(lib, n), n


def test_signatures_table_covers_header():
    assert set(declared()) <= set(_lib.SIGNATURES)
