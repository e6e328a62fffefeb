"""The constants of the oracle (oracle/oracle_consts.h) and of the library
(gpu-comcot_b200/csrc/comcot_consts.h) against the literals of the
reference's Fortran, as tests/golden/make_ref_constants.py extracted them
(COMMON /CONS/ BLOCK DATA comcot.f90:454-470, DATA UB boundaries.f90:30,
DATA TWLVTH, the Manning exponent, the DF floor, the breaking factors and SPAN
in moment.f90, DATA CORI_W comcot.f90:709).  The two headers are written
separately; a wrong constant in either fails here, whatever the GPU/oracle
parity says.  Single-precision constants (the Fortran REALs the stencils
use) compare as float32; the metric constants PARA evaluates in double
compare as written."""
import json
import pathlib
import re

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[1]
NAMES = {"ELMAX": "CC_ELMAX", "GRAV": "CC_GRAV", "PI": "CC_PI", "R_EARTH": "CC_R_EARTH", "GX": "CC_GX",
         "EPS": "CC_EPS", "V_LIMIT": "CC_VLIMIT", "RAD_DEG": "CC_RAD_DEG", "RAD_MIN": "CC_RAD_MIN",
         "CORI_W": "CC_CORI_W", "UB": "CC_UB", "TWLVTH": "CC_TWLVTH", "MANNEXP": "CC_MANNEXP",
         "DFMIN": "CC_DFMIN", "BRK_F": "CC_BRK_F", "BRK_I": "CC_BRK_I", "SPAN": "CC_SPAN"}


def _defines(path):
    out = {}
    for m in re.finditer(r"^#define\s+(CC_[A-Z_]+)\s+\(?\s*([-+0-9.eE]+)(f?)\s*\)?\s*$", path.read_text(), re.M):
        out[m.group(1)] = (m.group(2), m.group(3) == "f")
    return out


def _fortran_value(lit):
    return float(lit.replace("D", "E").replace("d", "e"))


def test_headers_match_the_fortran_literals():
    ref = json.loads((ROOT / "tests" / "golden" / "ref_constants.json").read_text())
    assert set(ref) == set(NAMES)
    for hdr in (ROOT / "oracle" / "oracle_consts.h", ROOT / "gpu-comcot_b200" / "csrc" / "comcot_consts.h"):
        defs = _defines(hdr)
        for name, macro in NAMES.items():
            assert macro in defs, f"{hdr.name}: {macro} missing"
            text, is_float = defs[macro]
            want = _fortran_value(ref[name]["literal"])
            if is_float:
                assert np.float32(float(text)) == np.float32(want), f"{hdr.name}: {macro} vs {ref[name]}"
            else:
                assert float(text) == want, f"{hdr.name}: {macro} vs {ref[name]}"


def test_oracle_does_not_include_the_library_constants():
    src = (ROOT / "oracle" / "comcot_oracle.c").read_text()
    assert '#include "oracle_consts.h"' in src
    assert "comcot_consts.h" not in src
