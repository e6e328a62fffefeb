"""Output files in the reference's formats (gfortran unformatted records,
Fortran F edit descriptors), checked byte for byte against hand-built
expectations."""
import os
import struct

import numpy as np

from comcot_b200 import outputs


def test_fortran_f_descriptor():
    f = outputs.fortran_f
    assert f(0.5, 10, 5) == "   0.50000"
    assert f(-0.5, 10, 5) == "  -0.50000"
    assert f(1234.5, 10, 5) == "1234.50000"
    assert f(-1234.5, 10, 5) == "**********"           # does not fit: asterisks
    assert f(-0.123456, 8, 5) == "-0.12346"
    assert f(4000.0, 12, 4) == "   4000.0000"
    assert f(-10.0, 12, 4) == "    -10.0000"
    assert f(121.03333282470703, 17, 6) == "       121.033333"
    assert f(0.1234567, 7, 5) == "0.12346"
    assert f(-0.1234567, 7, 5) == "-.12346"              # the leading zero is dropped before asterisks


def test_unformatted_record_layout(tmp_path):
    a = np.arange(12, dtype=np.float32).reshape(3, 4)   # ny=3, nx=4, I fastest
    p = os.path.join(tmp_path, outputs.snapshot_name("z", 1, 42))
    assert p.endswith("z_01_000042.dat")
    outputs.write_unformatted(p, a)
    b = open(p, "rb").read()
    assert len(b) == 4 + 48 + 4
    assert struct.unpack("<i", b[:4])[0] == 48 and struct.unpack("<i", b[-4:])[0] == 48
    assert np.array_equal(np.frombuffer(b[4:-4], "<f4"), a.ravel())
    assert np.array_equal(outputs.read_unformatted(p, 4, 3), a)


def test_zmax_masking_and_names():
    z = np.array([[0.5, -0.2], [0.0, 2.0]], np.float32)
    h = np.array([[100.0, -1.0], [-3.0, -1.0]], np.float32)
    m = outputs.zmax_masked(z, h)
    # land cells stay dry (H + zmax <= GX, H < 0) -> 0; flooded land keeps its value
    assert m.tolist() == [[0.5, 0.0], [0.0, 2.0]]
    assert outputs.zmax_name(1, 60) == "zmax_layer01_0060mins.dat"
    assert outputs.zmax_name(2, None) == "zmax_layer02.dat"


def test_forecast_products_written_async(tmp_path):
    res = {"zmax": np.ones((3, 4), np.float32), "ts": np.array([[0.1, -0.2], [0.3, 0.4]], np.float32),
           "arrival": np.array([[-1, 3], [2, 0]], np.int32)}
    w = outputs.AsyncWriter()
    w.submit(outputs.write_forecast, str(tmp_path), res, np.ones((3, 4), np.float32), 2.0)
    w.close()
    names = sorted(os.listdir(tmp_path))
    assert names == ["arrival_layer01.dat", "ts_record0001.dat", "ts_record0002.dat", "zmax_layer01.dat"]
    assert open(os.path.join(tmp_path, "ts_record0002.dat")).read() == "  -0.20000\n   0.40000\n"
    assert open(os.path.join(tmp_path, "arrival_layer01.dat")).read().split() == ["-1.0000", "0.1000", "0.0667",
                                                                                "0.0000"]


def test_bathymetry_files_skip_the_first_row_and_column_of_sub_layers(tmp_path):
    h = np.array([[1.0, 2.0, 3.0], [4.0, 5.0, 6.0]], np.float32)
    outputs.write_bathymetry(str(tmp_path), 2, h, np.array([10.0, 11.0, 12.0]), np.array([20.0, 21.0]))
    assert open(os.path.join(tmp_path, "layer02.dat")).read() == "      5.0000\n      6.0000\n"
    assert open(os.path.join(tmp_path, "layer02_y.dat")).read() == "        21.000000\n"
