#!/usr/bin/env python
"""Float error of the time stepping per configuration -- TEST INFRASTRUCTURE.

Runs each configuration twice through the CPU oracle: REAL = float (the
reference's arithmetic, which the CUDA library reproduces bit for bit) and the
FP64 twin built from the same source, both from the same float coefficients
(PARA/PQ_DEPTH output), so the difference is the rounding of the stepping
alone.  Written to oracle/fp64_error.json:

    python oracle/fp64_error.py [C1 steps] [C2 steps] [C3 steps] [threads]

Per layer and field it reports the largest difference over interior cells and
over the outer ring separately.  The radiation boundary (boundaries.f90:22-202)
sets the boundary surface to +/- |flux| / c with the sign taken from one flux
component; where that component is near zero the two arithmetics can pick
opposite signs, which is a property of the scheme, so the count of such sign
flips is reported too.
"""
from __future__ import annotations

import json
import os
import pathlib
import sys
import time

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent / "gpu-comcot_b200"))
sys.path.insert(0, str(HERE))

from comcot_b200 import synth  # noqa: E402
import oracle  # noqa: E402


def _stats(a, b, interior):
    d = np.abs(a.astype(np.float64) - b.astype(np.float64))
    s = float(np.abs(b).max())
    ring = ~interior
    return {"max_abs_interior": float(d[interior].max()),
            "rel_interior": float(d[interior].max() / s) if s else 0.0,
            "max_abs_boundary": float(d[ring].max()) if ring.any() else 0.0,
            "rms_interior": float(np.sqrt((d[interior] ** 2).mean())),
            "max_abs_field": s}


def measure(case, nsteps, threads):
    o32 = oracle.OracleRun(case)
    o32.run(nsteps, threads=threads, arrival=True)
    o64 = oracle.OracleRun(case, dtype=np.float64)
    o64.run(nsteps, threads=threads, arrival=True)
    out = {}
    for k, L in enumerate(case.layers):
        a, b = o32.layer(k), o64.layer(k)
        interior = np.zeros((L.ny, L.nx), bool)
        interior[1:-1, 1:-1] = True
        e = {f: _stats(a[f], b[f], interior) for f in ("z", "m", "n")}
        if k == 0:
            e["boundary_sign_flips"] = int(((np.sign(a["z"]) != np.sign(b["z"])) & ~interior
                                            & (np.abs(b["z"]) > 1e-3)).sum())
            e["zmax"] = _stats(a["zmax"], b["zmax"], interior)
            e["arrival_cells_differing"] = int((a["arrival"] != b["arrival"]).sum())
        if L.laygov == 1:
            e["wet_mask_cells_differing"] = int(((a["z"] + L.H > 1e-5) != (b["z"] + L.H > 1e-5)).sum())
        out[f"layer{L.id}"] = e
    return out


def main():
    steps = [int(x) for x in sys.argv[1:4]] + [3600, 7200, 3600][len(sys.argv[1:4]):]
    threads = int(sys.argv[4]) if len(sys.argv) > 4 else (os.cpu_count() or 1)
    res = {}
    for (name, mk), n in zip((("C1", synth.config_c1), ("C2", lambda: synth.config_c2(ngauges=0)),
                              ("C3", synth.config_c3)), steps):
        if n <= 0:
            continue
        t = time.time()
        res[name] = {"steps": n, "layers": measure(mk(), n, threads), "seconds": round(time.time() - t, 1)}
        print(name, json.dumps(res[name]), flush=True)
    (HERE / "fp64_error.json").write_text(json.dumps(res, indent=1) + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
