"""MATLAB-style HDF5 files without an HDF5 library: the reader against a file
MATLAB wrote through libhdf5, the writer's structures against that file's
bytes, round trips of every value kind, and the reference's data files
(geometry, fields, cross sections) through the command line's loaders."""
import math
import os
import struct
import zlib

import numpy as np
import pytest

import dda_b200
from dda_b200 import cli, datafiles as F, matfile as M

# A MAT-file 7.3 written by MATLAB 7.4 (libhdf5), shipped with scipy's tests;
# it holds testdouble = 0:pi/4:2*pi (a 1x9 double, HDF5 dims [9][1]).
MATLAB_FILE = os.path.join(os.path.dirname(np.__file__), "..", "scipy", "io", "matlab", "tests", "data",
                           "testhdf5_7.4_GLNX86.mat")


def _matlab_file():
    if not os.path.exists(MATLAB_FILE):
        pytest.skip("scipy's MAT-file test data is not installed")
    return MATLAB_FILE


def test_reads_a_file_matlab_wrote():
    v = M.load(_matlab_file())
    assert list(v) == ["testdouble"]
    x = v["testdouble"]
    assert x.dtype == np.float64 and x.shape == (9, 1)
    assert np.allclose(x[:, 0], np.pi / 4 * np.arange(9), rtol=1e-15, atol=1e-15)
    assert M.reader(_matlab_file()).attrs_of("testdouble") == {"MATLAB_class": "double"}
    assert M.is_hdf5(_matlab_file())


def test_written_messages_are_those_libhdf5_writes():
    """The attribute, datatype and dataspace messages of a double [9][1] with
    MATLAB_class "double" are byte for byte those in the MATLAB file."""
    r = M.reader(_matlab_file())
    theirs = {t: bytes(b) for t, b, _ in r.messages(r.links(r.messages(r.root))["testdouble"])}
    ours_file = M.dumps({"testdouble": np.pi / 4 * np.arange(9.0).reshape(9, 1)})
    o = M._Reader(ours_file)
    ours = {t: bytes(b) for t, b, _ in o.messages(o.links(o.messages(o.root))["testdouble"])}
    for t in (0x01, 0x03, 0x0C):  # dataspace, datatype, attribute
        assert ours[t] == theirs[t], hex(t)
    # superblock version 0 after a 512-byte user block, as libhdf5 places it
    assert ours_file[512:520] == M.SIGNATURE and ours_file[124:128] == b"\x00\x02IM"
    sb = struct.unpack_from("<8BHHIQQQQ", ours_file, 520)
    assert sb[:8] == (0, 0, 0, 0, 0, 8, 8, 0) and sb[8:10] == (M.LEAF_K, M.NODE_K)
    assert sb[11] == 512 and sb[12] == M.UNDEF and sb[13] == len(ours_file) and sb[14] == M.UNDEF
    mat = open(_matlab_file(), "rb").read()
    assert struct.unpack_from("<8BHH", mat, 520) == sb[:10]  # same versions, sizes and K values
    assert struct.unpack_from("<Q", mat, 536)[0] == 512  # base address = the superblock's offset
    # the root group's local heap ends its free list with 1, as libhdf5's does
    heap = struct.unpack_from("<QQ", ours_file, 512 + 96 - 16)[1]
    assert ours_file[512 + heap:512 + heap + 4] == b"HEAP"
    assert struct.unpack_from("<Q", ours_file, 512 + heap + 16)[0] == M.HEAP_FREE_NULL


def test_round_trip_of_every_value_kind():
    rng = np.random.default_rng(1)
    vals = {"Type": "DDAField", "Empty": "", "Unicode": "héllo λ", "Flag": True,
            "S": {"a": np.array([1.5]), "b": np.arange(12, dtype=np.uint32).reshape(4, 3),
                  "c": (rng.normal(size=(5, 3)) + 1j * rng.normal(size=(5, 3))).astype(np.complex64),
                  "d": rng.normal(size=(2, 3, 4)) + 1j * rng.normal(size=(2, 3, 4)),
                  "z": np.zeros((0, 3)), "u": np.array([7], dtype=np.uint8), "i": np.array([-3], dtype=np.int32),
                  "f": np.array([0.25, -1.5], dtype=np.float32), "nested": {"x": "y", "none": None}},
            # more members than one symbol table node holds: several nodes under the B-tree
            "Many": {"m%03d" % i: np.array([float(i)]) for i in range(70)},
            "Gone": None}
    back = M.loads(M.dumps(vals))

    def check(a, b, path):
        if isinstance(a, dict):
            a = {k: v for k, v in a.items() if v is not None}
            assert set(a) == set(b), path
            for k in a:
                check(a[k], b[k], path + "/" + k)
        elif isinstance(a, str):
            assert a == b, path
        elif isinstance(a, bool):
            assert b.dtype == np.bool_ and b.tolist() == [a], path
        else:
            assert a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a, b), path

    check(vals, back, "")
    r = M._Reader(M.dumps(vals))
    assert r.attrs_of("S") == {"MATLAB_class": "struct"}
    assert r.attrs_of("S/c") == {"MATLAB_class": "single"}
    assert r.attrs_of("S/d") == {"MATLAB_class": "double"}
    assert r.attrs_of("Type") == {"MATLAB_class": "char", "MATLAB_int_decode": 2}
    assert r.attrs_of("Flag") == {"MATLAB_class": "logical", "MATLAB_int_decode": 1}


def test_chunked_deflate_and_shuffle_datasets_are_read():
    """A chunked [5][4] uint16 dataset (chunks 2 x 3, edge chunks partial)
    under a version 1 chunk B-tree, shuffled and deflated."""
    data = np.arange(20, dtype="<u2").reshape(5, 4) * 7 + 1
    buf = bytearray(64)
    entries = []
    for r0 in range(0, 5, 2):
        for c0 in range(0, 4, 3):
            chunk = np.zeros((2, 3), dtype="<u2")
            part = data[r0:r0 + 2, c0:c0 + 3]
            chunk[:part.shape[0], :part.shape[1]] = part
            raw = np.frombuffer(chunk.tobytes(), np.uint8).reshape(-1, 2).T.tobytes()  # shuffle
            raw = zlib.compress(raw)
            entries.append((len(raw), (r0, c0, 0), len(buf)))
            buf += raw
    tree = len(buf)
    node = b"TREE" + struct.pack("<BBHQQ", 1, 0, len(entries), M.UNDEF, M.UNDEF)
    for size, offs, addr in entries:
        node += struct.pack("<II3Q", size, 0, *offs) + struct.pack("<Q", addr)
    node += struct.pack("<II3Q", 0, 0, 5, 4, 0)
    buf += node
    r = M._Reader.__new__(M._Reader)
    r.d, r.base = bytes(buf), 0
    space = struct.pack("<BBBB4x", 1, 2, 0, 0) + struct.pack("<QQ", 5, 4)
    dtype = struct.pack("<BBBBIHH", 0x10, 0, 0, 0, 2, 0, 16)
    layout = struct.pack("<BBBQ3I", 3, 2, 3, tree, 2, 3, 2)
    filters = struct.pack("<BB", 2, 2) + struct.pack("<HHHI", 2, 1, 1, 2) + struct.pack("<HHHI", 1, 0, 1, 6)
    msgs = [(0x01, space, 0), (0x03, dtype, 0), (0x08, layout, 0), (0x0B, filters, 0)]
    assert np.array_equal(r.data(msgs), data)


def test_orientation_quaternion_round_trip():
    for ang in ((0, 0, 0), (30, 40, 50), (-120, 170, 10), (45, 0, 0), (10, 180, 0)):
        q = F.orientation_quaternion(ang)
        assert abs(np.linalg.norm(q) - 1) < 1e-15
        back = F.zyz_from_quaternion(q)
        assert np.allclose(F.orientation_quaternion(back) * np.sign(q @ F.orientation_quaternion(back)), q,
                           atol=1e-12)
    # Rz(90) turns x into y: q = (cos 45, 0, 0, sin 45)
    assert np.allclose(F.orientation_quaternion((90, 0, 0)), [math.sqrt(0.5), 0, 0, math.sqrt(0.5)])


def _params():
    g = dda_b200.Geometry.from_arrays(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 1], [2, 2, 1], [1, 1, 2]]),
                                      np.array([0, 1, 0, 1, 1]), "0.1um")
    return dda_b200.DDAParams(g, [1.5 + 0.1j, (1.3, 1.4 + 0.01j, 1.5)], "1um")


def test_geometry_file_loads_through_the_command_line(tmp_path):
    p = _params()
    base = str(tmp_path / "Geometry")
    F.write(base, F.geometry_file(p, orient=(20, 30, 40)), lambda path: F.geometry_txt(path, p))
    g = M.load(base + ".hdf5")
    assert g["Type"] == "Geometry" and g["Geometry"]["Size"].tolist() == [3, 3, 3]
    assert g["Geometry"]["DipolePositions"].dtype == np.uint32 and g["Geometry"]["RefractiveIndices"].shape == (2, 3)
    assert open(base + ".txt").read().splitlines()[:3] == ["#box size: 3x3x3", "Nmat=2", "0 0 0 1"]
    back = dda_b200.Geometry.load(base + ".txt", "0.1um")  # the text loader reads it (DDA/Load.cpp:37-69)
    assert np.array_equal(back.positions, p.geometry.positions) and np.array_equal(back.materials, p.geometry.materials)
    # no --grid-unit, no -m, no --orient: all three from the file (DDAMain.cpp:170-230)
    geom, refr, mie, orient = cli.build_geometry("load:file=" + str(tmp_path), None, [], 1e-6)
    assert mie is None and np.array_equal(geom.positions, p.geometry.positions)
    assert np.array_equal(geom.materials, p.geometry.materials) and geom.grid_unit == p.grid_unit
    assert refr == [1.5 + 0.1j, (1.3, 1.4 + 0.01j, 1.5)]
    assert np.allclose(orient, (20, 30, 40), atol=1e-12)
    geom, refr, _, _ = cli.build_geometry("load:file=" + base + ".hdf5", "0.1um", ["2"], 1e-6)
    assert geom.grid_unit == pytest.approx(1e-7) and refr == [2 + 0j]
    # another grid unit moves the dipoles off the stored origin's centre ...
    with pytest.raises(SystemExit, match="GridOrigin"):
        cli.build_geometry("load:file=" + base + ".hdf5", "0.2um", [], 1e-6)
    # ... and is taken where the file has no GridOrigin (the box is centred, DDAMain.cpp:217-220)
    f = F.geometry_file(p)
    del f["Geometry"]["GridOrigin"]
    M.save(str(tmp_path / "noorigin.hdf5"), f)
    geom, _, _, _ = cli.build_geometry("load:file=" + str(tmp_path / "noorigin.hdf5"), "0.2um", [], 1e-6)
    assert geom.grid_unit == pytest.approx(2e-7)


def test_geometry_file_errors(tmp_path):
    p = _params()
    f = F.geometry_file(p)
    f["Geometry"]["GridOrigin"] = f["Geometry"]["GridOrigin"] + 0.5 * p.grid_unit
    M.save(str(tmp_path / "shifted.hdf5"), f)
    with pytest.raises(SystemExit, match="GridOrigin"):
        cli.build_geometry("load:file=" + str(tmp_path / "shifted.hdf5"), None, [], 1e-6)
    f = F.geometry_file(p)
    f["Geometry"]["Periodicity"] = np.array([[1e-6, 0, 0]])
    M.save(str(tmp_path / "periodic.hdf5"), f)
    with pytest.raises(SystemExit, match="periodic"):
        cli.build_geometry("load:file=" + str(tmp_path / "periodic.hdf5"), None, [], 1e-6)
    f = F.geometry_file(p)
    del f["Geometry"]["GridSpacing"]
    M.save(str(tmp_path / "nospacing.hdf5"), f)
    with pytest.raises(SystemExit, match="GridSpacing"):
        cli.build_geometry("load:file=" + str(tmp_path / "nospacing.hdf5"), None, [], 1e-6)
    # shifted positions with the matching shifted origin are the same target (normalize)
    f = F.geometry_file(p)
    f["Geometry"]["DipolePositions"] = f["Geometry"]["DipolePositions"] + np.uint32(4)
    f["Geometry"]["GridOrigin"] = f["Geometry"]["GridOrigin"] - 4 * p.grid_unit
    M.save(str(tmp_path / "moved.hdf5"), f)
    geom, _, _, _ = cli.build_geometry("load:file=" + str(tmp_path / "moved.hdf5"), None, [], 1e-6)
    assert np.array_equal(geom.positions, p.geometry.positions)


def test_field_file_layout(tmp_path):
    p = _params()
    rng = np.random.default_rng(3)
    v = np.zeros(p.vec_size, dtype=complex)
    for c in range(3):
        v[c * p.nvs:c * p.nvs + p.nv] = rng.normal(size=p.nv) + 1j * rng.normal(size=p.nv)
    for ftype, cls, dt in (("double", "double", np.complex128), ("float", "single", np.complex64)):
        base = str(tmp_path / ("IntField-Pol2-" + ftype))
        F.write(base, F.field_file(p, F.parameters(p, "load:file=x"), F.dipole_list_geometry(p), "InternalField", 2,
                                   v, ftype))
        f = M.load(base + ".hdf5")
        assert f["Type"] == "DDAField" and f["Field"]["FieldName"] == "InternalField"
        assert f["Field"]["BeamPolarization"].dtype == np.uint32 and f["Field"]["BeamPolarization"].tolist() == [2]
        d = f["Field"]["Data"]
        assert d.dtype == dt and d.shape == (p.nv, 3)
        assert np.array_equal(d, np.asarray(v).reshape(3, p.nvs)[:, :p.nv].T.astype(dt))
        assert M.reader(base + ".hdf5").attrs_of("Field/Data") == {"MATLAB_class": cls}
        pars = f["Parameters"]
        assert pars["Method"] == "DDA" and pars["GeometryString"] == "load:file=x"
        assert pars["MethodParameters"]["Frequency"][0] == pytest.approx(F.SPEED_OF_LIGHT / 1e-6)
        assert pars["Polarizations"].shape == (0, 3)
    bad = dda_b200.DDAParams(dda_b200.Geometry.sphere("0.3um", "0.1um"), [1.5], "1um")
    with pytest.raises(ValueError):
        F.load_dip_pol(str(tmp_path / "IntField-Pol2-double"), bad)


def test_cross_section_file(tmp_path):
    base = str(tmp_path / "CrossSec-Pol1")
    F.write(base, F.cross_section_file(1, 2e-12, 0.5e-12, 1.25, 0.3125),
            lambda path: F.cross_section_txt(path, 2e-12, 0.5e-12, 1.25, 0.3125))
    f = M.load(base + ".hdf5")
    assert f["Type"] == "CrossSection" and f["BeamPolarization"].tolist() == [1]
    assert {k: v.tolist() for k, v in f["CrossSection"].items()} == {
        "Cext": [2e-12], "Cabs": [0.5e-12], "Csca": [1.5e-12], "Qext": [1.25], "Qabs": [0.3125], "Qsca": [0.9375]}
    assert open(base + ".txt").read() == ("Cext = 2e-12\nQext = 1.25\nCabs = 5e-13\nQabs = 0.3125\n"
                                          "Csca = 1.5e-12\nQsca = 0.9375\n")


def test_mie_amplitudes_identities():
    """S1, S2 of the Bohren-Huffman series: equal forward with 4/x^2 Re S(0) =
    Qext, opposite backward, |S1|^2 + |S2|^2 integrating to Qsca, and the
    Rayleigh limit S1 = -i x^3 (m^2-1)/(m^2+2), S2 = S1 cos theta."""
    from dda_b200 import postprocess as P
    x, m = 3.7, 1.5 + 0.1j
    qe, qs, _ = P.mie(x, m)
    s1, s2 = P.mie_amplitudes(x, m, np.array([0.0, math.pi]))
    assert abs(s1[0] - s2[0]) <= 1e-12 * abs(s1[0]) and abs(s1[1] + s2[1]) <= 1e-12 * abs(s1[1])
    assert 4 / x ** 2 * s1[0].real == pytest.approx(qe, rel=1e-12)
    mu, w = np.polynomial.legendre.leggauss(200)
    s1, s2 = P.mie_amplitudes(x, m, np.arccos(mu))
    assert np.sum(w * (np.abs(s1) ** 2 + np.abs(s2) ** 2)) / x ** 2 == pytest.approx(qs, rel=1e-10)
    th = np.linspace(0, math.pi, 7)
    s1, s2 = P.mie_amplitudes(0.01, m, th)
    ray = -1j * 0.01 ** 3 * (m * m - 1) / (m * m + 2)
    assert np.allclose(s1, ray, rtol=1e-3) and np.allclose(s2, ray * np.cos(th), rtol=1e-3, atol=1e-3 * abs(ray))
    j = P.mie_jones(x, m, th, 2.0)
    assert np.array_equal(j[:, 0, 1], np.zeros(7)) and np.allclose(j[:, 1, 1], -P.mie_amplitudes(x, m, th)[0] / 2)


def test_newer_attribute_and_dataspace_versions():
    """Attribute messages 2 and 3 (no padding; 3 with a character set byte)
    and version 2 dataspaces, scalar and null, as libhdf5 writes them with its
    newer format options."""
    r = M._Reader.__new__(M._Reader)
    i32 = struct.pack("<BBBBIHH", 0x10, 0x08, 0, 0, 4, 0, 32)
    s6 = struct.pack("<BBBBI", 0x13, 0, 0, 0, 6)
    scalar, null = struct.pack("<BBBB", 2, 0, 0, 0), struct.pack("<BBBB", 2, 0, 0, 2)

    def attr(ver, name, dt, space, data):
        nm = name.encode() + b"\0"
        head = struct.pack("<BBHHH", ver, 0, len(nm), len(dt), len(space)) + (b"\0" if ver == 3 else b"")
        return (0x0C, head + nm + dt + space + data, 0)

    got = r.attributes([attr(2, "MATLAB_class", s6, scalar, b"double"),
                        attr(3, "MATLAB_int_decode", i32, scalar, struct.pack("<i", 2)),
                        attr(2, "MATLAB_empty", struct.pack("<BBBBIHH", 0x10, 0, 0, 0, 1, 0, 8), null, b"")])
    assert got["MATLAB_class"] == "double" and got["MATLAB_int_decode"] == 2
    assert got["MATLAB_empty"].size == 0


def test_version_2_object_headers_and_compact_groups():
    """Superblock 2, version 2 object headers (OHDR) and a group stored as
    link messages, the structures of libhdf5's newer format: the reader walks
    them (it does not check their checksums)."""
    def ohdr(msgs):
        body = b"".join(struct.pack("<BHB", t, len(d), 0) + d for t, d in msgs)
        assert len(body) < 256
        return b"OHDR" + struct.pack("<BBB", 2, 0, len(body)) + body + b"\0" * 4

    data = np.arange(6, dtype="<f8").reshape(2, 3)
    buf = bytearray(48)  # superblock
    raw_at = len(buf)
    buf += data.tobytes()
    dt = struct.pack("<BBBBIHHBBBBI", 0x11, 0x20, 63, 0, 8, 0, 64, 52, 11, 0, 52, 1023)
    space = struct.pack("<BBBB", 2, 2, 0, 1) + struct.pack("<QQ", 2, 3)
    s6 = struct.pack("<BBBBI", 0x13, 0, 0, 0, 6)
    nm = b"MATLAB_class\0"
    attr = struct.pack("<BBHHH", 3, 0, len(nm), len(s6), 4) + b"\0" + nm + s6 + struct.pack("<BBBB", 2, 0, 0, 0) + b"double"
    ds_at = len(buf)
    buf += ohdr([(0x01, space), (0x03, dt), (0x08, struct.pack("<BBQQ", 3, 1, raw_at, data.nbytes)), (0x0C, attr)])
    link = struct.pack("<BB", 1, 0) + struct.pack("<B", 1) + b"x" + struct.pack("<Q", ds_at)
    root_at = len(buf)
    buf += ohdr([(0x06, link)])
    buf[:48] = M.SIGNATURE + struct.pack("<BBBB", 2, 8, 8, 0) + struct.pack("<QQQQ", 0, M.UNDEF, len(buf), root_at) \
        + b"\0" * 4
    v = M.loads(bytes(buf))
    assert list(v) == ["x"] and np.array_equal(v["x"], data)
    assert M._Reader(bytes(buf)).attrs_of("x") == {"MATLAB_class": "double"}


def test_version_1_header_continued_in_a_second_block():
    """A version 1 object header whose attribute sits in a continuation block
    (message 0x10), the way libhdf5 grows a header when attributes are added."""
    img = M._Image()
    data = np.arange(4, dtype="<i4")
    raw_at = img.add(data.tobytes())
    attr = M._attribute_message("MATLAB_class", "int32")
    cont_body = struct.pack("<HHB3x", 0x0C, len(M._pad8(attr)), 0) + M._pad8(attr)
    cont_at = img.add(cont_body)
    msgs = [(1, M._dataspace_message((4,)), 0), (3, M._dtype_message(data.dtype), 1),
            (8, struct.pack("<BBQQ", 3, 1, raw_at, data.nbytes), 0),
            (0x10, struct.pack("<QQ", cont_at, len(cont_body)), 0)]
    hdr = bytearray(M._object_header(msgs))
    struct.pack_into("<H", hdr, 2, len(msgs) + 1)  # the message count includes the continued one
    ds_at = img.add(bytes(hdr))
    r = M._Reader.__new__(M._Reader)
    r.d, r.base = b"".join(bytes(p) for p in img.parts), 0
    got = r.messages(ds_at)
    assert [t for t, _, _ in got] == [1, 3, 8, 0x0C]
    assert r.attributes(got) == {"MATLAB_class": "int32"} and np.array_equal(r.data(got), data)
