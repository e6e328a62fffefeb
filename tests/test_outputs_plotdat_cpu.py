"""The output files read the way the reference's own reader reads them
(plot_dat.py:9-95, COMCOTdat): text files parsed with
`[float(v) for v in text.split()]` and reshaped to (len(y), len(x)); the
unformatted snapshots with `struct.unpack('f' * size, f.read(4 * size))`
from the start of the file; snapshot minutes from `int(name[5:-4])` of the
files whose name starts with 'z_%02d'.  That reader does not skip gfortran's
4-byte record marker, so it sees the marker as the first value and the field
shifted by one -- on a file written by the reference's Fortran as on ours,
since both are the same bytes.  The restated reader below mirrors those
calls (without matplotlib/basemap, which only plot)."""
import os
import struct

import numpy as np

from comcot_b200 import outputs


class PlotDatReader:
    """COMCOTdat's reading half (plot_dat.py:14-75), restated"""

    def __init__(self, base, layer=1):
        self.base = base.rstrip("/") + "/"
        self.x = self.read(self.base + "layer%02d_x.dat" % layer)
        self.y = self.read(self.base + "layer%02d_y.dat" % layer)
        self.dim = [len(self.y), len(self.x)]
        self.z = self.read(self.base + "layer%02d.dat" % layer, dim=True)
        names = sorted(i for i in os.listdir(self.base) if i[:4] == "z_%02d" % layer)
        self.eta = {int(n[5:-4]): self.read(self.base + n, dim=True, binary=True) for n in names}

    def read(self, filename, dim=False, binary=False):
        if binary:
            with open(filename, "rb") as f:
                size = self.dim[0] * self.dim[1]
                data = struct.unpack("f" * size, f.read(4 * size))
        else:
            with open(filename, "r") as f:
                data = [float(v) for v in f.read().split()]
        return np.reshape(data, self.dim) if dim else data


def _layer(nx=23, ny=17, seed=3):
    rng = np.random.default_rng(seed)
    h = rng.uniform(-200.0, 5000.0, (ny, nx)).astype(np.float32)
    x = (140.0 + np.arange(nx) / 30.0).astype(np.float64)
    y = (20.0 + np.arange(ny) / 30.0).astype(np.float64)
    return h, x, y


def test_bathymetry_and_axes_read_back_through_the_reference_reader(tmp_path):
    h, x, y = _layer()
    outputs.write_bathymetry(str(tmp_path), 1, h, x, y)
    rd = PlotDatReader(str(tmp_path))
    assert rd.dim == [h.shape[0], h.shape[1]]
    # F17.6 axes, F12.4 depths, J outer and I inner: the same grid back
    assert np.allclose(rd.x, x, atol=5e-7) and np.allclose(rd.y, y, atol=5e-7)
    assert np.allclose(rd.z, h, atol=5e-5)


def test_snapshots_read_like_a_fortran_written_file(tmp_path):
    h, x, y = _layer()
    outputs.write_bathymetry(str(tmp_path), 1, h, x, y)
    rng = np.random.default_rng(4)
    fields = {k: rng.normal(0.0, 1.0, h.shape).astype(np.float32) for k in (30, 1800)}
    for k, z in fields.items():
        outputs.write_unformatted(str(tmp_path / outputs.snapshot_name("z", 1, k)), z)
    rd = PlotDatReader(str(tmp_path))
    assert sorted(rd.eta) == sorted(fields)
    n = h.size
    for k, z in fields.items():
        raw = (tmp_path / outputs.snapshot_name("z", 1, k)).read_bytes()
        # one gfortran sequential record: length, NX*NY floats I fastest, length
        assert len(raw) == 4 * n + 8
        assert struct.unpack("<i", raw[:4])[0] == 4 * n == struct.unpack("<i", raw[-4:])[0]
        # what the reference's reader makes of those bytes: the marker, then the field less its last value
        marker = struct.unpack("<f", struct.pack("<i", 4 * n))[0]
        want = np.concatenate([[marker], z.ravel()[:-1]]).reshape(h.shape)
        assert np.array_equal(rd.eta[k].astype(np.float32), want.astype(np.float32))


def test_forecast_products_read_back(tmp_path):
    h, x, y = _layer()
    rng = np.random.default_rng(5)
    zmax = rng.uniform(0.0, 3.0, h.shape).astype(np.float32)
    arrival = rng.integers(-1, 400, h.shape).astype(np.int32)
    ts = rng.normal(0.0, 0.5, (50, 3)).astype(np.float32)
    outputs.write_forecast(str(tmp_path), {"zmax": zmax, "arrival": arrival, "ts": ts}, h, dt=2.0)
    # zmax_layer01.dat: one record, masked on dry land (output.f90:919-931)
    got = outputs.read_unformatted(str(tmp_path / "zmax_layer01.dat"), h.shape[1], h.shape[0])
    assert np.array_equal(got, outputs.zmax_masked(zmax, h))
    # gauge series: one F10.5 value per line, read back with float()
    for g in range(3):
        with open(tmp_path / ("ts_record%04d.dat" % (g + 1))) as f:
            vals = [float(v) for v in f.read().split()]
        assert np.allclose(vals, ts[:, g], atol=5e-6)
    # arrival minutes, -1 where the wave never arrived
    with open(tmp_path / "arrival_layer01.dat") as f:
        vals = np.reshape([float(v) for v in f.read().split()], h.shape)
    want = np.where(arrival >= 0, arrival * 2.0 / 60.0, -1.0)
    assert np.allclose(vals, want, atol=5e-5)
