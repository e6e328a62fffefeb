"""COMCOT's output files, byte for byte as the reference writes them.

- Snapshots and maxima: `z_##_######.dat`, `m_…`, `n_…` (output.f90:811-837)
  and `zmax_layer##[_####mins].dat` (output.f90:918-944). Each is one gfortran
  unformatted sequential record: a 4-byte little-endian length, NX*NY float32
  in Fortran order (I fastest), the length again.
- Maximum elevation masking (output.f90:918-931): where H + Zmax <= GX on
  land (H < 0) the value written is 0; a tide level with |tide| > GX is added
  elsewhere.
- Gauge series `ts_record####.dat` (comcot.f90:272-276,434): one `(F10.5)`
  line per step.
- Bathymetry `layer##.dat` (`(F12.4)` per cell, J outer, I inner, from I=J=1
  on layer 1 and from 2 on sub-layers), axes `layer##_x.dat` /
  `layer##_y.dat` (`(F17.6)`) (output.f90:643-736).
- Arrival times `arrival_layer##.dat` (no reference writer; the name is the
  one plot_dat.py:47 would read): `(F12.4)` minutes per cell, -1 where the
  wave never arrived.

`AsyncWriter` writes on a background thread, so a serving loop hands its
results off and continues.
"""
from __future__ import annotations

import os
import queue
import struct
import threading

import numpy as np

GX = 1.0e-5


def fortran_f(value: float, w: int, d: int) -> str:
    """Fortran Fw.d edit descriptor as gfortran prints it: right-justified in
    w columns, d decimals, leading zero kept when it fits, asterisks when the
    number does not fit."""
    v = float(value)
    if v != v:
        s = "NaN"
    elif v in (float("inf"), float("-inf")):
        s = "Infinity" if v > 0 else "-Infinity"
        if len(s) > w:
            s = "Inf" if v > 0 else "-Inf"
    else:
        s = f"{v:.{d}f}"
        if len(s) > w and s.startswith(("0.", "-0.")):
            s = s.replace("0.", ".", 1)          # the optional leading zero goes first
    if len(s) > w:
        return "*" * w
    return s.rjust(w)


def write_unformatted(path: str, field: np.ndarray):
    """one gfortran unformatted sequential record of float32 [ny, nx]"""
    a = np.ascontiguousarray(field, dtype="<f4")
    n = a.nbytes
    if n >= 2 ** 31:
        raise ValueError("records of 2 GiB or more need gfortran sub-records")
    with open(path, "wb") as f:
        f.write(struct.pack("<i", n))
        f.write(a.tobytes())
        f.write(struct.pack("<i", n))


def read_unformatted(path: str, nx: int, ny: int) -> np.ndarray:
    with open(path, "rb") as f:
        b = f.read()
    n = struct.unpack("<i", b[:4])[0]
    if n != nx * ny * 4 or struct.unpack("<i", b[4 + n:8 + n])[0] != n:
        raise ValueError(f"{path}: not one record of {nx}x{ny} floats")
    return np.frombuffer(b[4:4 + n], dtype="<f4").reshape(ny, nx)


def snapshot_name(kind: str, layer_id: int, k: int) -> str:
    """kind z, m or n (output.f90:813,823,830)"""
    return f"{kind}_{layer_id:02d}_{k:06d}.dat"


def zmax_name(layer_id: int, minutes: int | None) -> str:
    """final file when minutes is None (output.f90:932-934)"""
    return f"zmax_layer{layer_id:02d}.dat" if minutes is None else f"zmax_layer{layer_id:02d}_{minutes:04d}mins.dat"


def zmax_masked(zmax: np.ndarray, h: np.ndarray, tide_level: float = 0.0) -> np.ndarray:
    zm = zmax.astype(np.float32)
    h = h.astype(np.float32)
    out = zm.copy()
    if abs(tide_level) > GX:
        out = (zm + np.float32(tide_level)).astype(np.float32)
    dry_land = ((h + zm) <= np.float32(GX)) & (h < 0)
    out[dry_land] = 0.0
    return out


def write_text_column(path: str, values, w: int, d: int):
    with open(path, "w") as f:
        for v in values:
            f.write(fortran_f(v, w, d) + "\n")


def write_bathymetry(out_dir: str, layer_id: int, h: np.ndarray, x: np.ndarray, y: np.ndarray):
    """layer##.dat, layer##_x.dat, layer##_y.dat (output.f90:671-708)"""
    s = 0 if layer_id == 1 else 1
    write_text_column(os.path.join(out_dir, f"layer{layer_id:02d}.dat"), h[s:, s:].ravel(), 12, 4)
    write_text_column(os.path.join(out_dir, f"layer{layer_id:02d}_x.dat"), x[s:], 17, 6)
    write_text_column(os.path.join(out_dir, f"layer{layer_id:02d}_y.dat"), y[s:], 17, 6)


def write_gauges(out_dir: str, ts: np.ndarray, first: int = 1):
    """ts [nsteps, ngauges] -> ts_record####.dat, gauge g numbered first+g"""
    for g in range(ts.shape[1]):
        write_text_column(os.path.join(out_dir, f"ts_record{first + g:04d}.dat"), ts[:, g], 10, 5)


def write_arrival(out_dir: str, layer_id: int, arrival_steps: np.ndarray, dt: float):
    minutes = np.where(arrival_steps >= 0, arrival_steps.astype(np.float64) * dt / 60.0, -1.0)
    write_text_column(os.path.join(out_dir, f"arrival_layer{layer_id:02d}.dat"), minutes.ravel(), 12, 4)


def write_forecast(out_dir: str, result: dict, h: np.ndarray, dt: float, layer_id: int = 1, tide_level=0.0):
    """the products a served request returns: maximum elevation, gauge series,
    arrival times (whichever the result holds)"""
    os.makedirs(out_dir, exist_ok=True)
    if "zmax" in result:
        write_unformatted(os.path.join(out_dir, zmax_name(layer_id, None)), zmax_masked(result["zmax"], h, tide_level))
    if "ts" in result and result["ts"].size:
        write_gauges(out_dir, result["ts"])
    if "arrival" in result:
        write_arrival(out_dir, layer_id, result["arrival"], dt)


class AsyncWriter:
    """writes results on a background thread; `close()` waits for the queue"""

    def __init__(self):
        self.q: queue.Queue = queue.Queue()
        self.errors = []
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def _run(self):
        while True:
            job = self.q.get()
            if job is None:
                return
            fn, args = job
            try:
                fn(*args)
            except Exception as exc:  # reported by close()
                self.errors.append(exc)

    def submit(self, fn, *args):
        self.q.put((fn, args))

    def close(self):
        self.q.put(None)
        self.t.join()
        if self.errors:
            raise self.errors[0]
