"""EMAN HDF5 input: the library's own HDF5 parser (gs_hdf_read_*).

The reference reads HDF5 through libhdf5 (EMReader/emhdf_.cpp, emhdf2_.cpp),
which is not available here.  The parser is pinned in two ways:
  - against a file written by libhdf5 itself: scipy ships a MATLAB 7.3 file
    (an HDF5 file behind a 512-byte user block) whose variable `testdouble`
    scipy also ships in MATLAB 5 format, which scipy reads; the two must agree;
  - against fixtures of the two EMAN layouts written by tests/_hdf5_writer.py
    from the file-format specification (superblocks 0 and 2, object headers 1
    and 2, symbol-table groups over several nodes and B-tree levels, compact
    links, contiguous / compact / chunked storage with shuffle + deflate,
    integer, big-endian and double data), read back value for value.
No GPU is needed.
"""
import os

import numpy as np
import pytest

import gisspa_b200 as G
import _hdf5_writer as W

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "gisspa_b200", "lib",
                   "libgisspa_b200.so")
pytestmark = pytest.mark.skipif(not os.path.exists(LIB), reason="library not built")

SCIPY_DATA = None
try:
    import scipy.io.matlab as _m

    SCIPY_DATA = os.path.join(os.path.dirname(_m.__file__), "tests", "data")
except Exception:  # pragma: no cover
    pass


@pytest.mark.skipif(SCIPY_DATA is None or not os.path.exists(
    os.path.join(SCIPY_DATA or "", "testhdf5_7.4_GLNX86.mat")), reason="scipy test data absent")
def test_parser_reads_a_file_written_by_libhdf5():
    import scipy.io
    h5 = os.path.join(SCIPY_DATA, "testhdf5_7.4_GLNX86.mat")
    v5 = os.path.join(SCIPY_DATA, "testdouble_7.4_GLNX86.mat")
    want = scipy.io.loadmat(v5)["testdouble"]
    got = G.read_hdf_dataset(h5, "/testdouble")
    # MATLAB stores column-major: the 1 x 9 row vector is a 9 x 1 HDF5 dataset
    assert got.shape == (9, 1)
    assert np.array_equal(got.ravel(), want.ravel())
    assert G.read_hdf_attribute(h5, "/testdouble", "MATLAB_class") == "double"
    assert not G.is_hdf5(h5)  # user block: the EMAN reader's signature test looks at byte 0 only
    with pytest.raises(G.GisspaError) as e:
        G.read_hdf_image(h5, 0)
    assert e.value.status == G.GS_ERR_IO


def _images(rng, n, shape, dtype=np.float32):
    return [(rng.standard_normal(shape) * 100).astype(dtype) for _ in range(n)]


@pytest.mark.parametrize("superblock", [0, 2])
def test_eman2_layout_round_trip(tmp_path, superblock):
    rng = np.random.default_rng(1)
    imgs = _images(rng, 3, (37, 53))
    p = str(tmp_path / "stack.hdf")
    W.write_eman2(p, imgs, superblock=superblock)
    assert G.is_hdf5(p)
    for n, im in enumerate(imgs):
        assert np.array_equal(G.read_hdf_image(p, n), im)
    assert np.array_equal(G.read_hdf_image(p, -4), imgs[0])  # negative index reads image 0
    assert int(G.read_hdf_attribute(p, "/MDF/images/1", "EMAN.nx")[0]) == 53
    with pytest.raises(G.GisspaError) as e:
        G.read_hdf_image(p, 3)
    assert e.value.status == G.GS_ERR_IO


@pytest.mark.parametrize("superblock", [0, 2])
def test_attributes_in_continuation_blocks(tmp_path, superblock):
    # EMAN2 puts dozens of attributes on every image group; libhdf5 then
    # spreads the group's object header over chained continuation blocks
    rng = np.random.default_rng(8)
    imgs = _images(rng, 2, (9, 14))
    extra = {"EMAN.attr%02d" % k: np.float32(k + 0.5) for k in range(40)}
    extra["EMAN.micrograph_id"] = "mic_0001"
    extra["EMAN.orientation"] = np.arange(3, dtype=np.float32)
    p = str(tmp_path / "cont.hdf")
    W.write_eman2(p, imgs, attrs={0: extra, 1: extra}, superblock=superblock, header_messages=5)
    for n, im in enumerate(imgs):
        assert np.array_equal(G.read_hdf_image(p, n), im)
    assert float(G.read_hdf_attribute(p, "/MDF/images/1", "EMAN.attr39")[0]) == 39.5
    assert G.read_hdf_attribute(p, "/MDF/images/0", "EMAN.micrograph_id") == "mic_0001"
    assert np.array_equal(G.read_hdf_attribute(p, "/MDF/images/0", "EMAN.orientation"), [0.0, 1.0, 2.0])


def test_many_images_across_symbol_nodes_and_btree_levels(tmp_path):
    # two names per symbol-table node and three children per B-tree node:
    # 23 images need 12 leaves, 4 level-1 nodes, 2 level-2 nodes and a root
    rng = np.random.default_rng(2)
    imgs = _images(rng, 23, (8, 12))
    p = str(tmp_path / "many.hdf")
    W.write_eman2(p, imgs, snod_capacity=2, btree_capacity=3)
    for n in [0, 1, 2, 9, 10, 11, 19, 20, 22]:  # names sort as strings: "10" < "2"
        assert np.array_equal(G.read_hdf_image(p, n), imgs[n]), n


def test_storage_layouts_and_types(tmp_path):
    rng = np.random.default_rng(3)
    a = (rng.standard_normal((45, 61)) * 1000)
    imgs = [a.astype(np.float32), a.astype(">f4"), a.astype(np.int16), a.astype(">i2"),
            np.abs(a).astype(np.uint8), a.astype(np.float64), a.astype(np.float32), a.astype(np.float32)]
    opts = {6: {"chunks": (16, 24), "filters": ("shuffle", "deflate")},
            7: {"chunks": (45, 61), "filters": ("deflate",)},
            1: {"compact": True}}
    p = str(tmp_path / "types.hdf")
    W.write_eman2(p, imgs, dataset_options=opts)
    for n, im in enumerate(imgs):
        got = G.read_hdf_image(p, n)
        assert got.dtype == np.float32
        assert np.array_equal(got, im.astype(np.float32)), n


def test_eman2_size_attributes_follow_emobject_int(tmp_path):
    rng = np.random.default_rng(4)
    vol = rng.standard_normal((3, 5, 7)).astype(np.float32)
    line = rng.standard_normal((1, 9)).astype(np.float32)
    img = rng.standard_normal((6, 4)).astype(np.float32)
    p = str(tmp_path / "attrs.hdf")
    # image 2: nx as a float attribute (truncated), nz missing (0 -> 2D)
    attrs = {2: {"EMAN.nx": np.float32(4.9), "EMAN.nz": np.float64(0.0)}}
    W.write_eman2(p, [vol, line, img], attrs=attrs)
    assert G.read_hdf_image(p, 0).shape == (3, 5, 7)
    assert G.read_hdf_image(p, 1).shape == (1, 9)   # ny = 1: a 1D image of nx pixels
    assert np.array_equal(G.read_hdf_image(p, 2), img)
    # a size the dataset does not have is refused (the reference would read
    # past or short of its buffer)
    p2 = str(tmp_path / "bad.hdf")
    W.write_eman2(p2, [img], attrs={0: {"EMAN.nx": np.int32(5)}})
    with pytest.raises(G.GisspaError) as e:
        G.read_hdf_image(p2, 0)
    assert e.value.status == G.GS_ERR_IO
    p3 = str(tmp_path / "nosize.hdf")
    W.write_eman2(p3, [img], attrs={0: {"EMAN.nx": "text", "EMAN.ny": np.int32(1)}})
    with pytest.raises(G.GisspaError):
        G.read_hdf_image(p3, 0)


def test_old_style_layout(tmp_path):
    rng = np.random.default_rng(5)
    imgs = _images(rng, 2, (20, 20))
    p = str(tmp_path / "old.hdf")
    W.write_eman1(p, imgs)
    for n, im in enumerate(imgs):
        got = G.read_hdf_image(p, n)
        assert np.array_equal(got, im)
    # nx = dims[0], ny = dims[1] of the dataspace (emhdf_.cpp:138-160): a
    # 20 x 30 dataset is read as nx = 20, ny = 30 over the same flat data
    rect = rng.standard_normal((20, 30)).astype(np.float32)
    p2 = str(tmp_path / "rect.hdf")
    W.write_eman1(p2, [rect])
    got = G.read_hdf_image(p2, 0)
    assert got.shape == (30, 20)
    assert np.array_equal(got.ravel(), rect.ravel())
    # anisotropic spacing: the reference refuses the image (emdata_.cpp:248-258)
    p3 = str(tmp_path / "aniso.hdf")
    W.write_eman1(p3, imgs, spacing=(1.0, 1.0, 2.0))
    with pytest.raises(G.GisspaError):
        G.read_hdf_image(p3, 0)
    # integer data: old-style images must be floating point
    p4 = str(tmp_path / "int.hdf")
    W.write_eman1(p4, [imgs[0].astype(np.int16)])
    with pytest.raises(G.GisspaError) as e:
        G.read_hdf_image(p4, 0)
    assert e.value.status == G.GS_ERR_UNSUPPORTED


def test_unsupported_and_broken_files(tmp_path):
    rng = np.random.default_rng(6)
    imgs = _images(rng, 1, (8, 8))
    p = str(tmp_path / "dense.hdf")
    W.write_eman2(p, imgs, superblock=2, dense_links=True)
    with pytest.raises(G.GisspaError) as e:
        G.read_hdf_image(p, 0)
    assert e.value.status == G.GS_ERR_UNSUPPORTED
    good = str(tmp_path / "good.hdf")
    W.write_eman2(good, imgs)
    raw = open(good, "rb").read()
    cut = str(tmp_path / "cut.hdf")
    with open(cut, "wb") as fh:
        fh.write(raw[: len(raw) // 2])
    with pytest.raises(G.GisspaError) as e:
        G.read_hdf_image(cut, 0)
    assert e.value.status == G.GS_ERR_IO
    junk = str(tmp_path / "junk.hdf")
    with open(junk, "wb") as fh:
        fh.write(W.SIG + bytes(rng.integers(0, 256, 4000, dtype=np.uint8)))
    with pytest.raises(G.GisspaError):
        G.read_hdf_image(junk, 0)
    with pytest.raises(G.GisspaError) as e:
        G.read_hdf_image(str(tmp_path / "missing.hdf"), 0)
    assert e.value.status == G.GS_ERR_IO


def test_read_image_dispatch(tmp_path):
    from gisspa_b200 import formats
    rng = np.random.default_rng(7)
    img = rng.standard_normal((16, 24)).astype(np.float32)
    h = str(tmp_path / "a.hdf")
    W.write_eman2(h, [img])
    m = str(tmp_path / "a.mrc")
    formats.write_mrc(m, img)
    assert np.array_equal(G.read_image(h, 0), G.read_image(m, 0))


def test_driver_reports_a_missing_hdf_template(tmp_path):
    # the drop-in driver reads every template before it touches the GPU
    import subprocess
    import _helpers as H
    from gisspa_b200 import build, formats
    build.build_driver()
    H.materialize("small_pf1_all", str(tmp_path))
    W.copy_case_as_hdf(str(tmp_path))
    # drop the last template image: the reference would search a 10 x 10 zero
    # image in its place (emdata_.cpp:191-196); the driver stops with the reason
    stack = formats.read_mrc(str(tmp_path / "templates.mrcs"), -1)
    W.write_eman2(str(tmp_path / "templates.hdf"), [t for t in stack[:-1]])
    r = subprocess.run([G.DRIVER_PATH, "config_hdf"], cwd=str(tmp_path), capture_output=True, text=True,
                       timeout=600)
    assert r.returncode != 0
    assert "/MDF/images/%d" % (len(stack) - 1) in r.stderr


_FUZZ = r"""
import ctypes as C, os, resource, sys
import numpy as np
sys.path.insert(0, os.path.dirname(sys.argv[1]))
import _hdf5_writer as W
resource.setrlimit(resource.RLIMIT_AS, (4 << 30, 4 << 30))
lib = C.CDLL(sys.argv[2])
rng = np.random.default_rng(11)
d = sys.argv[3]
imgs = [rng.standard_normal((12, 10)).astype(np.float32) for _ in range(5)]
files = []
p = os.path.join(d, "a.hdf"); W.write_eman2(p, imgs, snod_capacity=2, btree_capacity=3); files.append(p)
p = os.path.join(d, "b.hdf")
W.write_eman2(p, imgs, superblock=2, dataset_options={1: {"chunks": (5, 4), "filters": ("shuffle", "deflate")},
                                                     2: {"compact": True}})
files.append(p)
p = os.path.join(d, "c.hdf"); W.write_eman1(p, imgs); files.append(p)
base = [open(f, "rb").read() for f in files]
seen = set()
for it in range(900):
    b = bytearray(base[it % 3])
    for _ in range(int(rng.integers(1, 8))):
        b[int(rng.integers(8, len(b)))] = int(rng.integers(0, 256))
    q = os.path.join(d, "m.hdf")
    open(q, "wb").write(bytes(b))
    data = C.POINTER(C.c_float)(); nx, ny, nz = C.c_int(), C.c_int(), C.c_int()
    err = C.create_string_buffer(256)
    for idx in (0, 1, 3):
        r = lib.gs_hdf_read_image(q.encode(), idx, C.byref(data), C.byref(nx), C.byref(ny), C.byref(nz), err, 256)
        seen.add(r)
        if r == 0:
            lib.gs_host_free(data)
print(sorted(seen))
"""


def test_corrupt_files_fail_cleanly(tmp_path):
    # 900 files with random bytes overwritten (seeded), each read at three
    # indexes in a child process under a 4 GB address-space limit: every read
    # returns a status (no crash, no hang, no runaway allocation)
    import ast
    import subprocess
    import sys
    here = os.path.abspath(__file__)
    r = subprocess.run([sys.executable, "-c", _FUZZ, here, LIB, str(tmp_path)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    seen = ast.literal_eval(r.stdout.strip().splitlines()[-1])
    assert set(seen) <= {G.GS_OK, G.GS_ERR_IO, G.GS_ERR_UNSUPPORTED, G.GS_ERR_OOM}
    assert G.GS_OK in seen and G.GS_ERR_IO in seen


def test_huge_attribute_dataspace_is_an_io_error(tmp_path):
    # a dataspace of 2^31 x 2^31 doubles in an attribute message holding 8
    # bytes: the element count overflows any byte count; the read must return
    # GS_ERR_IO instead of sizing a buffer from it
    rng = np.random.default_rng(5)
    path = str(tmp_path / "huge_attr.hdf")
    bad = W.ClaimedShape(np.float64, (2 ** 31, 2 ** 31), b"\0" * 8)
    W.write_eman2(path, _images(rng, 1, (8, 8)), attrs={0: {"EMAN.bad": bad}})
    for call in (lambda: G.read_hdf_attribute(path, "/MDF/images/0", "EMAN.bad"),
                 lambda: G.read_hdf_image(path, 0)):
        with pytest.raises(G.GisspaError) as e:
            call()
        assert e.value.status == G.GS_ERR_IO
