"""Host-side reference formats: config, list, Euler file, MRC, output lines."""
import os
import struct

import numpy as np
import pytest

import _helpers as H
from gisspa_b200 import formats


def test_config_parse_reference_rules(tmp_path):
    p = tmp_path / "cfg"
    p.write_text("# comment\n"
                 "input = a/b.lst\n"
                 "template=t.mrcs\n"
                 "eulerfile   ==  e.lst\n"
                 "angpix = 1.5x\n"
                 "window_size = 720\n"
                 "threshold = 7.25\n"
                 "bogus = 3\n"
                 "\n"
                 "Highres = 8\n")
    c = formats.read_config(str(p))
    assert c.inlst == "a/b.lst" and c.temp2d == "t.mrcs" and c.eulerf == "e.lst"
    assert c.apix == pytest.approx(1.5)
    assert c.padding_size == 720 and c.thres == pytest.approx(7.25)
    assert c.highres == 8.0
    assert c.unknown == ["3"]
    # reference defaults (DataReader.h:36-42)
    assert c.overlap == -1 and c.phase_flip == 0 and c.norm_type == 0 and c.first == -1
    assert set(formats.missing_required(c)) == {"phistep", "kk", "energy", "cs", "Lowres", "diameter"}


def test_lst_first_line_consumed_and_prefix(tmp_path):
    d = tmp_path / "sub"
    d.mkdir()
    p = d / "m.lst"
    p.write_text("0\tskipped.mrc\tdefocus=9\n# c\n3\tx.mrc\tdefocus=1.5\tdfdiff=0.01\tdfang=30\n"
                 "4\ty.mrc\tdefocus=2.0\n")
    e0 = formats.read_lst_entry(str(p), 0)
    assert e0.nn == 3 and e0.path == str(d) + "/x.mrc"
    assert (e0.defocus, e0.dfang) == (pytest.approx(1.5), pytest.approx(30.0))
    e1 = formats.read_lst_entry(str(p), 1)
    assert e1.nn == 4 and e1.path.endswith("/y.mrc")
    assert formats.read_lst_entry(str(p), 2) is None


def test_euler_file(tmp_path):
    p = tmp_path / "e.lst"
    p.write_text("#hdr\n 10.5\t20\t0\n\n30 40.25 0\n")
    e = formats.read_euler(str(p))
    assert e.shape == (2, 2)
    assert e.tolist() == [[10.5, 20.0], [30.0, 40.25]]


def test_mrc_roundtrip_and_sections(tmp_path):
    rng = np.random.default_rng(0)
    stack = rng.standard_normal((3, 5, 7)).astype(np.float32)
    p = str(tmp_path / "s.mrcs")
    formats.write_mrc(p, stack)
    h = formats.read_mrc_header(p)
    assert (h["nx"], h["ny"], h["nz"], h["mode"]) == (7, 5, 3, 2)
    assert np.array_equal(formats.read_mrc(p, 1), stack[1])
    assert np.array_equal(formats.read_mrc(p, 7), stack)   # out of range: whole stack


def test_mrc_big_endian_int16(tmp_path):
    a = np.arange(12, dtype=">i2").reshape(3, 4)
    hdr = bytearray(1024)
    struct.pack_into(">4i", hdr, 0, 4, 3, 1, 1)
    struct.pack_into(">i", hdr, 220, 1)
    p = tmp_path / "be.mrc"
    p.write_bytes(bytes(hdr) + a.tobytes())
    assert np.array_equal(formats.read_mrc(str(p), 0), a.astype(np.float32))


def test_mrc_rejects_invalid(tmp_path):
    p = tmp_path / "bad.mrc"
    hdr = bytearray(1024)
    struct.pack_into("<4i", hdr, 0, 4, 3, 1, 7)
    p.write_bytes(bytes(hdr) + b"\0" * 48)
    with pytest.raises(IOError):
        formats.read_mrc(str(p), 0)
    (tmp_path / "short.mrc").write_bytes(b"\0" * 10)
    with pytest.raises(IOError):
        formats.read_mrc(str(tmp_path / "short.mrc"), 0)


@pytest.mark.parametrize("name", H.SMALL_CASES)
def test_pick_line_format_roundtrip(name):
    for line in H.load_golden(name)["lines"][:50]:
        d = formats.parse_pick_line(line)
        again = formats.format_pick_line(d["nn"], d["path"], d["defocus"], d["dfdiff"], d["dfang"],
                                         d["euler"][0], d["euler"][1], d["euler"][2],
                                         d["center"][0], d["center"][1], d["score"])
        assert again.rstrip("\n") == line
