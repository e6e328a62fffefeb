"""Extracts the time stepper's constants from the reference's Fortran source
text into tests/golden/ref_constants.json (run in a checkout that has the
reference; the JSON is committed so the tests need no reference tree).

Each entry is the literal as the Fortran writes it, with file:line:
COMMON /CONS/ BLOCK DATA (comcot.f90), DATA UB (boundaries.f90), DATA TWLVTH,
the Manning exponent, the DF floor, the wave-breaking factors and SPAN
(moment.f90), DATA CORI_W (comcot.f90).

usage: python tests/golden/make_ref_constants.py [reference_dir]
"""
from __future__ import annotations

import json
import pathlib
import re
import sys

HERE = pathlib.Path(__file__).resolve().parent
REF = pathlib.Path(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")

# name -> (file, regular expression whose group 1 is the literal)
PATTERNS = {
    "ELMAX": ("comcot.f90", r"DATA\s+ELMAX\s*/\s*([-+0-9.EeDd]+)\s*/"),
    "GRAV": ("comcot.f90", r"DATA\s+GRAV\s*/\s*([-+0-9.EeDd]+)\s*/"),
    "PI": ("comcot.f90", r"DATA\s+PI\s*/\s*([-+0-9.EeDd]+)\s*/"),
    "R_EARTH": ("comcot.f90", r"DATA\s+R_EARTH\s*/\s*([-+0-9.EeDd]+)\s*/"),
    "GX": ("comcot.f90", r"DATA\s+GX\s*/\s*([-+0-9.EeDd]+)\s*/"),
    "EPS": ("comcot.f90", r"DATA\s+EPS\s*/\s*([-+0-9.EeDd]+)\s*/"),
    "V_LIMIT": ("comcot.f90", r"DATA\s+V_LIMIT\s*/\s*([-+0-9.EeDd]+)\s*/"),
    "RAD_DEG": ("comcot.f90", r"DATA\s+RAD_DEG\s*/\s*([-+0-9.EeDd]+)\s*/"),
    "RAD_MIN": ("comcot.f90", r"DATA\s+RAD_MIN\s*/\s*([-+0-9.EeDd]+)\s*/"),
    "CORI_W": ("comcot.f90", r"DATA\s+CORI_W\s*/\s*([-+0-9.EeDd]+)\s*/"),
    "UB": ("boundaries.f90", r"DATA\s+UB\s*/\s*([-+0-9.EeDd]+)\s*/"),
    "TWLVTH": ("moment.f90", r"DATA\s+TWLVTH\s*/\s*([-+0-9.EeDd]+)\s*/"),
    "MANNEXP": ("moment.f90", r"DF\*\*\(?\s*([0-9.]+)\s*\)?"),
    "DFMIN": ("moment.f90", r"IF\s*\(\s*DF\s+\.LT\.\s+([-+0-9.EeDd]+)\s*\)"),
    "BRK_F": ("moment.f90", r"DZDT_F\s*=\s*([0-9.]+)\s*\*\s*C"),
    "BRK_I": ("moment.f90", r"DZDT_I\s*=\s*([0-9.]+)\s*\*\s*C"),
    "SPAN": ("moment.f90", r"^\s*SPAN\s*=\s*([0-9]+)"),
}


def main():
    out = {}
    for name, (fname, pat) in PATTERNS.items():
        lines = (REF / fname).read_text(errors="replace").splitlines()
        rx = re.compile(pat)
        for k, line in enumerate(lines, 1):
            if line.lstrip().startswith("!"):
                continue
            m = rx.search(line)
            if m:
                out[name] = {"literal": m.group(1), "source": f"{fname}:{k}"}
                break
        else:
            raise SystemExit(f"{name}: not found in {fname}")
    (HERE / "ref_constants.json").write_text(json.dumps(out, indent=1) + "\n")
    print(f"wrote {len(out)} constants")


if __name__ == "__main__":
    main()
