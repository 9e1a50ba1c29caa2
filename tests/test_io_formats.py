"""The caps output files written through the C ABI's host-only entry points,
checked against the Fortran edit descriptors and record layouts the
reference uses (evolution.f90:73, 582-583, 682, 707, 714-719, 746-766,
common.f90:50-70).  Expected strings are derived by hand from the
descriptors: Iw and Fw.d right-justify in w columns, Fw.d drops the
optional leading zero of |x| < 1 when it does not fit and prints w
asterisks when the value does not fit at all."""
import struct

import numpy as np
import pytest

io = pytest.importorskip("hydra_b200.io")


def _lines(p):
    return p.read_text().splitlines()


def test_synopsis_line_and_list_directed_read(tmp_path):
    p = tmp_path / "qqsynopsis.asc"
    io.append_synopsis(p, 12, 34567, 1.5, 0.25)
    io.append_synopsis(p, 3, 40, 2.0, 1.0 / 3.0)
    # (i9,1x,i10,1x,f12.5,1x,f16.12)
    assert _lines(p)[0] == "       12" + " " + "     34567" + " " + "     1.50000" + " " + "  0.250000000000"
    assert _lines(p)[1] == "        3" + " " + "        40" + " " + "     2.00000" + " " + "  0.333333333333"
    assert io.read_synopsis(p, 2) == (3, 40, 2.0, 0.333333333333)
    assert io.read_synopsis(p, 1) == (12, 34567, 1.5, 0.25)


def test_ene_norms_complexity_monitor(tmp_path):
    e = tmp_path / "ene.asc"
    io.append_ene(e, 2.5, 1.25, 0.5)
    # (f9.2,3(1x,f17.11))
    assert _lines(e) == ["     2.50" + "     1.25000000000" + "     0.50000000000" + "     1.75000000000"]
    n = tmp_path / "norms.asc"
    io.append_norms(n, 10.0, 123.456789)
    assert _lines(n) == ["    10.00" + " " + "   123.456789000"]  # (f9.2,1x,f16.9)
    c = tmp_path / "complexity.asc"
    io.append_complexity(c, 0.125, 80, 1234567)
    assert _lines(c) == [" " + "     0.12500" + " " + "       80" + " " + "   1234567"]
    m = tmp_path / "monitor.asc"
    io.append_monitor(m, 1.0, 0.5, 2.0, 3.0, 4.0, 2.5)
    # (1x,f12.5,1x,f6.4,4(1x,f12.6),1x,f5.3); third value is zzrms^2/2
    assert _lines(m) == [" " + "     1.00000" + " " + "0.5000" + " " + "    2.000000" + " " + "    2.000000"
                         + " " + "    3.000000" + " " + "    4.000000" + " " + "2.500"]


def test_fortran_f_overflow_and_leading_zero(tmp_path):
    m = tmp_path / "monitor.asc"
    # cfl = 12.5 does not fit f6.4 (needs 7) -> asterisks; twist -0.5 in f5.3
    # needs "-0.500" (6) -> the optional zero goes: "-.500"
    io.append_monitor(m, 1.0, 12.5, 0.0, 0.0, 0.0, -0.5)
    line = _lines(m)[0]
    fields = [line[1:13], line[14:20], line[-5:]]
    assert fields[1] == "******"
    assert fields[2] == "-.500"
    n = tmp_path / "norms.asc"
    io.append_norms(n, 1.0e9, 1.0)  # f9.2 of 1e9 needs 13 columns
    assert _lines(n)[0].startswith("*********")


def test_spectrum_block(tmp_path):
    p = tmp_path / "spectra.asc"
    alk = np.array([0.0, np.log10(np.sqrt(2.0)), np.log10(2 * np.sqrt(2.0))])
    qspec = np.array([0.0, 1.0e-3, 1.0e-5])
    io.append_spectrum(p, 4.0, 0.5, 0.75, 2, alk, qspec)
    lines = _lines(p)
    assert lines[0] == "     4.00" + "      0.500000000" + "      0.750000000" + "     2"
    # (2(1x,f12.8)): alk(k), log10(qspec(k))
    assert lines[1] == " " + "  0.15051500" + " " + " -3.00000000"
    assert lines[2] == " " + "  0.45154499" + " " + " -5.00000000"
    assert len(lines) == 3


def test_unformatted_records_layout_and_round_trip(tmp_path):
    npq = np.array([5, 7, 9])
    i1q = np.array([1, 6, 13])
    indq = np.array([2, 2, 3])
    pi = tmp_path / "qqindex001"
    io.write_index(pi, npq, i1q, indq)
    raw = pi.read_bytes()
    assert len(raw) == 4 + 36 + 4
    assert struct.unpack("<i", raw[:4])[0] == 36 and struct.unpack("<i", raw[-4:])[0] == 36
    assert list(struct.unpack("<9i", raw[4:40])) == [5, 7, 9, 1, 6, 13, 2, 2, 3]
    a, b, c = io.read_index(pi, 3)
    assert (a == npq).all() and (b == i1q).all() and (c == indq).all()
    x = np.linspace(-1, 1, 21)
    y = x ** 3
    pn = tmp_path / "qqnodes001"
    io.write_nodes(pn, x, y)
    raw = pn.read_bytes()
    assert len(raw) == 8 + 16 * 21 and struct.unpack("<i", raw[:4])[0] == 16 * 21
    assert np.array_equal(np.frombuffer(raw[4:4 + 168], "<f8"), x)
    xr, yr = io.read_nodes(pn, 21)
    assert np.array_equal(xr, x) and np.array_equal(yr, y)
    with pytest.raises(io.CaslError):
        io.read_nodes(pn, 20)  # record length does not match


def test_direct_access_r4(tmp_path):
    p = tmp_path / "qq.r4"
    nx, ny = 8, 4
    f2 = np.arange(nx * ny, dtype=np.float32).reshape(nx, ny)
    io.write_r4(p, 2, 2.5, f2)  # record 2 first: record 1 stays zero-filled
    io.write_r4(p, 1, 1.25, -f2)
    recl = 4 * (nx * ny + 1)
    raw = p.read_bytes()
    assert len(raw) == 2 * recl
    assert struct.unpack("<f", raw[recl:recl + 4])[0] == 2.5
    assert np.array_equal(np.frombuffer(raw[recl + 4:], "<f4").reshape(nx, ny), f2)
    t, g = io.read_r4(p, 1, nx, ny)
    assert t == 1.25 and np.array_equal(g, -f2)
