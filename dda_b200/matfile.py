"""MATLAB-style HDF5 files (the MAT-file 7.3 layout), written and read without
an HDF5 library.

The reference stores its results and reads geometries and polarisations
through its MATLAB serialisation (HDF5/Matlab.cpp, HDF5/Matlab.hpp):

* a 512-byte user block holding a MAT-file header (HDF5/Matlab.cpp:231-262);
* a struct is an HDF5 group with the attribute MATLAB_class = "struct"
  (HDF5/Matlab.cpp:295-304) whose members are its links; a null member is left
  out (HDF5/Matlab.hpp:766-768); the top-level struct's members are the root
  group's links (HDF5/Matlab.hpp:520-526);
* a string is a uint16 dataset of its UTF-16 code units, dims [n][1], with
  MATLAB_class "char" and MATLAB_int_decode 2 (HDF5/Matlab.cpp:323-340); a
  bool a uint8 [1] with "logical" and MATLAB_int_decode 1;
* a number is a dataset of dims [1] (HDF5/Matlab.hpp:560-572), a vector of
  numbers dims [n] (HDF5/Matlab.hpp:630-648), a vector of 3-vectors or
  diagonal matrices dims [n][3] (HDF5/MatlabVector3.hpp:46-63), a quaternion
  dims [4], a Fortran-ordered multi-array its dimensions reversed
  (HDF5/MultiArray.hpp:34-55); MATLAB_class names the element type
  ("double", "single", "uint8", "uint32", ...; HDF5/Matlab.hpp:727-739);
* a complex number is the compound {real, imag} of its real type
  (HDF5/Type.hpp:95-104);
* the attribute strings are fixed-length ASCII of the value's length with a
  scalar dataspace (HDF5/Util.cpp:26-31).

Values on the Python side: a dict is a struct, a str a char array, a bool a
logical, a numpy array a dataset of the array's shape as HDF5 dims and its
dtype (complex dtypes as the {real, imag} compound), None a missing member.

The writer uses the structures of HDF5 file format version 0, the ones
libhdf5 writes by default: superblock version 0 after the user block (base
address = the superblock's offset, other addresses relative to it, the end of
file address absolute), version 1 object headers, groups as a symbol table
(version 1 B-tree of group nodes, symbol table nodes, local heap), contiguous
datasets (layout message version 3), version 1 dataspace, datatype and
attribute messages.  The reader takes those and what libhdf5 writes with its
newer format options: superblocks 0-3, object headers 1 and 2 with
continuation blocks, symbol-table and compact (link message) groups,
contiguous, compact and chunked datasets (version 1 B-tree chunk index; the
deflate, shuffle and fletcher32 filters), attribute messages 1-3, compound
datatypes 1-3.  Anything else (dense link or attribute storage, shared
messages, variable-length, reference or array types) raises MatFileError.
"""
import struct
import zlib

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIGNATURE = b"\x89HDF\r\n\x1a\n"
USER_BLOCK = 512
LEAF_K, NODE_K = 4, 16  # group leaf node K and group internal node K (libhdf5's defaults)
ENTRY_SIZE = 40  # symbol table entry with 8-byte offsets and lengths
SNOD_SIZE = 8 + 2 * LEAF_K * ENTRY_SIZE
TREE_SIZE = 24 + 2 * NODE_K * 8 + (2 * NODE_K + 1) * 8
HEAP_FREE_NULL = 1  # end of a local heap's free list

MATLAB_CLASSES = {"f8": "double", "f4": "single", "u1": "uint8", "u2": "uint16", "u4": "uint32", "u8": "uint64",
                  "i1": "int8", "i2": "int16", "i4": "int32", "i8": "int64"}


class MatFileError(ValueError):
    pass


def _pad8(b):
    return bytes(b) + b"\0" * (-len(b) % 8)


def matlab_class(dtype):
    dt = np.dtype(dtype)
    if dt.kind == "c":
        dt = np.dtype("f%d" % (dt.itemsize // 2))
    key = "%s%d" % (dt.kind, dt.itemsize)
    if key not in MATLAB_CLASSES:
        raise MatFileError("no MATLAB class for dtype %s" % dtype)
    return MATLAB_CLASSES[key]


# --------------------------------------------------------------------------
# writer

def _dtype_message(dt):
    """Datatype message (version 1) of a little-endian numpy dtype."""
    dt = np.dtype(dt)
    if dt.kind == "c":
        part = np.dtype("<f%d" % (dt.itemsize // 2))
        member = _dtype_message(part)
        body = b""
        for i, name in enumerate((b"real", b"imag")):
            # name, byte offset, dimensionality 0, permutation, four dimension sizes
            body += _pad8(name + b"\0") + struct.pack("<IB3xI4x4I", i * part.itemsize, 0, 0, 0, 0, 0, 0) + member
        return struct.pack("<BHBI", 0x16, 2, 0, dt.itemsize) + body
    if dt.kind == "f":
        sign, ebits, mbits, bias = {8: (63, 11, 52, 1023), 4: (31, 8, 23, 127)}[dt.itemsize]
        # little-endian, implied leading mantissa bit; offset, precision,
        # exponent location and size, mantissa location and size, bias
        return struct.pack("<BBBBIHHBBBBI", 0x11, 0x20, sign, 0, dt.itemsize, 0, 8 * dt.itemsize, mbits, ebits, 0,
                           mbits, bias)
    if dt.kind in "iu":
        return struct.pack("<BBBBIHH", 0x10, 0x08 if dt.kind == "i" else 0, 0, 0, dt.itemsize, 0, 8 * dt.itemsize)
    if dt.kind == "S":  # fixed-length ASCII, null terminated
        return struct.pack("<BBBBI", 0x13, 0, 0, 0, dt.itemsize)
    raise MatFileError("cannot store dtype %s" % dt)


def _dataspace_message(shape):
    """Dataspace message (version 1); shape () is the scalar dataspace."""
    return struct.pack("<BBBB4x", 1, len(shape), 0, 0) + b"".join(struct.pack("<Q", d) for d in shape)


def _attribute_message(name, value):
    if isinstance(value, str):
        data = value.encode("ascii")
        dt = _dtype_message(np.dtype("S%d" % max(len(data), 1)))
        data = data or b"\0"
    else:
        arr = np.asarray(value)
        arr = arr.astype(arr.dtype.newbyteorder("<"))
        dt, data = _dtype_message(arr.dtype), arr.tobytes()
    space = _dataspace_message(())
    nm = name.encode("ascii") + b"\0"
    return (struct.pack("<BBHHH", 1, 0, len(nm), len(dt), len(space)) + _pad8(nm) + _pad8(dt) + _pad8(space)
            + data)


def _object_header(messages):
    """Version 1 object header of (type, data, flags) messages."""
    body = b"".join(struct.pack("<HHB3x", t, len(_pad8(d)), f) + _pad8(d) for t, d, f in messages)
    return struct.pack("<BBHII4x", 1, 0, len(messages), 1, len(body)) + body


class _Image:
    """The file after the user block, as it is laid out (relative addresses):
    a list of pieces, the datasets' raw data as views of their arrays, so
    that a large field is not copied before it is written."""

    def __init__(self):
        self.parts = [bytes(96)]  # superblock, filled in last
        self.size = 96

    def add(self, data):
        pad = -self.size % 8
        if pad:
            self.parts.append(b"\0" * pad)
            self.size += pad
        addr = self.size
        self.parts.append(data)
        self.size += len(data)
        return addr

    def next_addr(self):
        return self.size + (-self.size % 8)


def _write_dataset(img, arr, attrs):
    arr = np.ascontiguousarray(arr)
    if arr.dtype.byteorder == ">":
        arr = arr.astype(arr.dtype.newbyteorder("<"))
    raw = memoryview(arr.reshape(-1).view(np.uint8))
    addr = img.add(raw) if len(raw) else UNDEF
    msgs = [(1, _dataspace_message(arr.shape), 0), (3, _dtype_message(arr.dtype), 1),
            (8, struct.pack("<BBQQ", 3, 1, addr, len(raw)), 0)]
    msgs += [(0x0C, _attribute_message(k, v), 0) for k, v in attrs]
    return img.add(_object_header(msgs)), None


def _write_group(img, members, attrs):
    """Children first, then the local heap, symbol table nodes, B-tree and the
    group's object header.  Returns (header address, (B-tree, heap))."""
    entries = []
    for name, value in members.items():
        if value is None:
            continue
        addr, scratch = _write_value(img, value)
        entries.append((name.encode("utf-8"), addr, scratch))
    entries.sort(key=lambda e: e[0])
    if len(entries) > 2 * NODE_K * 2 * LEAF_K:
        raise MatFileError("a struct with more than %d members" % (2 * NODE_K * 2 * LEAF_K))
    heap = bytearray(8)  # the empty string at offset 0
    offsets = []
    for name, _, _ in entries:
        offsets.append(len(heap))
        heap += _pad8(name + b"\0")
    heap_addr = img.next_addr()
    img.add(b"HEAP" + bytes(4) + struct.pack("<QQQ", len(heap), HEAP_FREE_NULL, heap_addr + 32) + heap)
    children, keys = [], [0]
    for i in range(0, len(entries), 2 * LEAF_K):
        node = b"SNOD" + struct.pack("<BBH", 1, 0, len(entries[i:i + 2 * LEAF_K]))
        for (name, addr, scratch), off in zip(entries[i:i + 2 * LEAF_K], offsets[i:i + 2 * LEAF_K]):
            if scratch is None:
                node += struct.pack("<QQI4x16x", off, addr, 0)
            else:
                node += struct.pack("<QQI4xQQ", off, addr, 1, *scratch)
        children.append(img.add(node + bytes(SNOD_SIZE - len(node))))
        keys.append(offsets[min(i + 2 * LEAF_K, len(entries)) - 1])
    tree = b"TREE" + struct.pack("<BBHQQ", 0, 0, len(children), UNDEF, UNDEF) + struct.pack("<Q", keys[0])
    for child, key in zip(children, keys[1:]):
        tree += struct.pack("<QQ", child, key)
    tree_addr = img.add(tree + bytes(TREE_SIZE - len(tree)))
    msgs = [(0x11, struct.pack("<QQ", tree_addr, heap_addr), 1)]
    msgs += [(0x0C, _attribute_message(k, v), 0) for k, v in attrs]
    return img.add(_object_header(msgs)), (tree_addr, heap_addr)


def _write_value(img, value):
    if isinstance(value, dict):
        return _write_group(img, value, [("MATLAB_class", "struct")])
    if isinstance(value, str):
        units = np.frombuffer(value.encode("utf-16-le"), dtype="<u2")
        return _write_dataset(img, units.reshape(len(units), 1),
                              [("MATLAB_class", "char"), ("MATLAB_int_decode", np.int32(2))])
    if isinstance(value, (bool, np.bool_)):
        return _write_dataset(img, np.array([1 if value else 0], dtype=np.uint8),
                              [("MATLAB_class", "logical"), ("MATLAB_int_decode", np.int32(1))])
    arr = np.asarray(value)
    if arr.dtype == np.bool_:
        return _write_dataset(img, arr.astype(np.uint8),
                              [("MATLAB_class", "logical"), ("MATLAB_int_decode", np.int32(1))])
    if arr.ndim == 0:
        arr = arr.reshape(1)
    return _write_dataset(img, arr, [("MATLAB_class", matlab_class(arr.dtype))])


def user_block(text="MATLAB 7.3 MAT-file, written by dda_b200, HDF5 schema 1.00 ."):
    """The MAT-file header: text, padded with spaces to 116 bytes, an empty
    subsystem offset, version 0x0200 and the endianness indicator "IM"."""
    ub = bytearray(USER_BLOCK)
    t = text.encode("ascii")[:116]
    ub[:116] = t + b" " * (116 - len(t))
    ub[124:128] = b"\x00\x02IM"
    return bytes(ub)


def _pieces(members):
    """The file as a list of byte pieces: user block, superblock, the rest."""
    img = _Image()
    root, (tree, heap) = _write_group(img, members, [])
    sb = SIGNATURE + struct.pack("<BBBBBBBBHHI", 0, 0, 0, 0, 0, 8, 8, 0, LEAF_K, NODE_K, 0)
    sb += struct.pack("<QQQQ", USER_BLOCK, UNDEF, USER_BLOCK + img.size, UNDEF)
    sb += struct.pack("<QQI4xQQ", 0, root, 1, tree, heap)
    assert len(sb) == 96
    img.parts[0] = sb
    return [user_block()] + img.parts


def dumps(members):
    """The bytes of a file whose root group holds `members` (a dict)."""
    return b"".join(bytes(p) for p in _pieces(members))


def save(path, members):
    """Write a MATLAB-style HDF5 file (HDF5::matlabSerialize)."""
    with open(path, "wb") as f:
        for piece in _pieces(members):
            f.write(piece)


# --------------------------------------------------------------------------
# reader

def find_superblock(data):
    """Offset of the HDF5 signature: 0, 512, 1024, 2048, ... (H5Fis_hdf5)."""
    off = 0
    while off + 8 <= len(data):
        if data[off:off + 8] == SIGNATURE:
            return off
        off = 512 if off == 0 else 2 * off
    return None


def is_hdf5(path):
    try:
        with open(path, "rb") as f:
            data = f.read(1 << 20)
    except OSError:
        return False
    return find_superblock(data) is not None


class _Reader:
    def __init__(self, data):
        self.d = bytes(data)
        off = find_superblock(self.d)
        if off is None:
            raise MatFileError("not an HDF5 file")
        self.base = off  # addresses are relative to the superblock (libhdf5 adjusts a moved file the same way)
        ver = self.d[off + 8]
        if ver in (0, 1):
            so, sl = self.d[off + 13], self.d[off + 14]
            p = off + 24 + (4 if ver == 1 else 0)
            p += 32  # base, free space, end of file, driver block
            self.root = struct.unpack_from("<Q", self.d, p + 8)[0]
        elif ver in (2, 3):
            so, sl = self.d[off + 9], self.d[off + 10]
            self.root = struct.unpack_from("<Q", self.d, off + 12 + 24)[0]
        else:
            raise MatFileError("superblock version %d" % ver)
        if (so, sl) != (8, 8):
            raise MatFileError("offsets of %d and lengths of %d bytes" % (so, sl))

    def at(self, addr):
        return self.base + addr

    # object headers -------------------------------------------------------
    def messages(self, addr):
        d, a = self.d, self.at(addr)
        out = []
        if d[a:a + 4] == b"OHDR":
            flags = d[a + 5]
            p = a + 6 + (16 if flags & 0x20 else 0) + (4 if flags & 0x10 else 0)
            n = 1 << (flags & 3)
            size = int.from_bytes(d[p:p + n], "little")
            p += n
            todo = [(p, size)]
            while todo:
                p, size = todo.pop(0)
                end = p + size
                hdr = 6 if flags & 0x04 else 4
                while p + hdr <= end:
                    t, sz, mf = d[p], struct.unpack_from("<H", d, p + 1)[0], d[p + 3]
                    p += hdr
                    body = d[p:p + sz]
                    p += sz
                    if t == 0x10:
                        ca, cl = struct.unpack_from("<QQ", body)
                        c = self.at(ca)
                        if d[c:c + 4] != b"OCHK":
                            raise MatFileError("bad continuation block")
                        todo.append((c + 4, cl - 8))
                    else:
                        out.append((t, body, mf))
            return out
        if d[a] != 1:
            raise MatFileError("object header version %d" % d[a])
        nmsg, _, size = struct.unpack_from("<HII", d, a + 2)
        todo = [(a + 16, size)]
        while todo and len(out) < nmsg:
            p, size = todo.pop(0)
            end = p + size
            while p + 8 <= end:
                t, sz, mf = struct.unpack_from("<HHB", d, p)
                body = d[p + 8:p + 8 + sz]
                p += 8 + sz
                if t == 0x10:
                    ca, cl = struct.unpack_from("<QQ", body)
                    todo.append((self.at(ca), cl))
                elif t != 0:
                    out.append((t, body, mf))
        return out

    @staticmethod
    def first(msgs, t):
        for mt, body, flags in msgs:
            if mt == t:
                if flags & 0x02:
                    raise MatFileError("shared message of type %d" % t)
                return body
        return None

    # datatypes, dataspaces ----------------------------------------------
    def dtype(self, b, p=0):
        cv = b[p]
        cls, ver = cv & 0x0F, cv >> 4
        bf = b[p + 1] | (b[p + 2] << 8) | (b[p + 3] << 16)
        size = struct.unpack_from("<I", b, p + 4)[0]
        q = p + 8
        order = ">" if bf & 1 else "<"
        if cls == 0:
            return np.dtype(order + ("i" if bf & 8 else "u") + str(size)), q + 4
        if cls == 1:
            return np.dtype(order + "f" + str(size)), q + 12
        if cls == 3:
            return np.dtype("S%d" % size), q
        if cls == 6:
            fields = []
            for _ in range(bf & 0xFFFF):
                e = b.index(b"\0", q)
                name = b[q:e].decode("utf-8")
                q = q + ((e - q + 8) // 8) * 8 if ver < 3 else e + 1
                if ver == 3:
                    nb = (size.bit_length() - 1) // 8 + 1
                    off = int.from_bytes(b[q:q + nb], "little")
                    q += nb
                else:
                    off = struct.unpack_from("<I", b, q)[0]
                    q += 4
                    if ver == 1:
                        if b[q] != 0:
                            raise MatFileError("array member in a compound type")
                        q += 28
                mdt, q = self.dtype(b, q)
                fields.append((name, mdt, off))
            if ([f[0] for f in fields] == ["real", "imag"] and fields[0][1] == fields[1][1]
                    and fields[0][1].kind == "f" and fields[0][2] == 0 and fields[1][2] == fields[0][1].itemsize
                    and size == 2 * fields[0][1].itemsize):
                f = fields[0][1]
                return np.dtype(f.byteorder.replace("=", "<") + "c%d" % size), q
            return np.dtype({"names": [f[0] for f in fields], "formats": [f[1] for f in fields],
                             "offsets": [f[2] for f in fields], "itemsize": size}), q
        raise MatFileError("datatype class %d" % cls)

    @staticmethod
    def shape(b):
        ver, rank = b[0], b[1]
        if ver == 1:
            p, kind = 8, (1 if rank else 0)
        else:
            p, kind = 4, b[3]
        if kind == 2:
            return None  # null dataspace
        return tuple(struct.unpack_from("<%dQ" % rank, b, p))

    # attributes -----------------------------------------------------------
    def attributes(self, msgs):
        out = {}
        for t, b, _ in msgs:
            if t == 0x15:
                fh = struct.unpack_from("<Q", b, 2)[0]
                if fh != UNDEF:
                    raise MatFileError("dense attribute storage")
            if t != 0x0C:
                continue
            ver = b[0]
            nsize, dtsize, dssize = struct.unpack_from("<HHH", b, 2)
            p = 8
            pad = (lambda n: n + (-n % 8)) if ver == 1 else (lambda n: n)
            if ver == 3:
                p += 1
            name = b[p:p + nsize].split(b"\0")[0].decode("utf-8")
            p += pad(nsize)
            dt, _ = self.dtype(b, p)
            p += pad(dtsize)
            shp = self.shape(b[p:])
            p += pad(dssize)
            n = 0 if shp is None else int(np.prod(shp))
            val = np.frombuffer(b, dtype=dt, count=n, offset=p)
            if dt.kind == "S":
                out[name] = b"".join(val.tolist()).split(b"\0")[0].decode("latin-1")
            elif shp is None:
                out[name] = val.copy()
            elif shp == ():
                out[name] = val[0].item()
            else:
                out[name] = val.reshape(shp).copy()
        return out

    # groups ---------------------------------------------------------------
    def links(self, msgs):
        stab = self.first(msgs, 0x11)
        out = {}
        if stab is not None:
            tree, heap = struct.unpack_from("<QQ", stab)
            h = self.at(heap)
            if self.d[h:h + 4] != b"HEAP":
                raise MatFileError("bad local heap")
            dsize, _, daddr = struct.unpack_from("<QQQ", self.d, h + 8)
            names = self.d[self.at(daddr):self.at(daddr) + dsize]
            for snod in self._group_nodes(tree):
                s = self.at(snod)
                if self.d[s:s + 4] != b"SNOD":
                    raise MatFileError("bad symbol table node")
                for i in range(struct.unpack_from("<H", self.d, s + 6)[0]):
                    off, addr = struct.unpack_from("<QQ", self.d, s + 8 + ENTRY_SIZE * i)
                    out[names[off:names.index(b"\0", off)].decode("utf-8")] = addr
            return out
        for t, b, _ in msgs:
            if t == 0x02:
                fh = struct.unpack_from("<Q", b, 2 + (8 if b[1] & 1 else 0))[0]
                if fh != UNDEF:
                    raise MatFileError("dense link storage")
            if t != 0x06:
                continue
            flags, p, ltype = b[1], 2, 0
            if flags & 0x08:
                ltype, p = b[p], p + 1
            if flags & 0x04:
                p += 8
            if flags & 0x10:
                p += 1
            n = 1 << (flags & 3)
            nlen = int.from_bytes(b[p:p + n], "little")
            p += n
            name = b[p:p + nlen].decode("utf-8")
            if ltype == 0:
                out[name] = struct.unpack_from("<Q", b, p + nlen)[0]
        return out

    def _group_nodes(self, tree):
        a = self.at(tree)
        if self.d[a:a + 4] != b"TREE" or self.d[a + 4] != 0:
            raise MatFileError("bad group B-tree")
        level, n = self.d[a + 5], struct.unpack_from("<H", self.d, a + 6)[0]
        kids = [struct.unpack_from("<Q", self.d, a + 24 + 8 + 16 * i)[0] for i in range(n)]
        if level == 0:
            return kids
        return [s for k in kids for s in self._group_nodes(k)]

    # datasets -------------------------------------------------------------
    def data(self, msgs):
        shp = self.shape(self.first(msgs, 0x01))
        dt, _ = self.dtype(self.first(msgs, 0x03))
        if shp is None:
            return np.zeros(0, dtype=dt)
        n = int(np.prod(shp))
        cls, addr, raw, cdims = self.layout(self.first(msgs, 0x08))
        if cls == 2:
            return self._chunked(msgs, addr, cdims, shp, dt)
        if cls == 1:
            if addr == UNDEF:
                return np.zeros(shp, dtype=dt)
            raw = self.d[self.at(addr):self.at(addr) + n * dt.itemsize]
        if len(raw) < n * dt.itemsize:
            raise MatFileError("dataset data beyond the end of the file")
        return np.frombuffer(raw, dtype=dt, count=n).reshape(shp).copy()

    @staticmethod
    def layout(lay):
        """(class, address, compact data, chunk dims) of a layout message:
        versions 1 and 2 (dimensions with the element size last, 5 reserved
        bytes) and 3."""
        ver = lay[0]
        if ver in (1, 2):
            nd, cls = lay[1], lay[2]
            p, addr = 8, None
            if cls != 0:
                addr = struct.unpack_from("<Q", lay, p)[0]
                p += 8
            dims = struct.unpack_from("<%dI" % nd, lay, p)
            p += 4 * nd
            if cls == 0:
                size = struct.unpack_from("<I", lay, p)[0]
                return 0, None, lay[p + 4:p + 4 + size], None
            return cls, addr, None, dims[:-1]
        if ver != 3:
            raise MatFileError("layout message version %d" % ver)
        cls = lay[1]
        if cls == 0:
            size = struct.unpack_from("<H", lay, 2)[0]
            return 0, None, lay[4:4 + size], None
        if cls == 1:
            return 1, struct.unpack_from("<Q", lay, 2)[0], None, None
        if cls == 2:
            nd = lay[2]
            return 2, struct.unpack_from("<Q", lay, 3)[0], None, struct.unpack_from("<%dI" % nd, lay, 11)[:-1]
        raise MatFileError("layout class %d" % cls)

    def _filters(self, msgs):
        b = self.first(msgs, 0x0B)
        if b is None:
            return []
        ver, nf = b[0], b[1]
        p = 8 if ver == 1 else 2
        out = []
        for _ in range(nf):
            fid = struct.unpack_from("<H", b, p)[0]
            if ver == 1 or fid >= 256:
                nlen = struct.unpack_from("<H", b, p + 2)[0]
                flags, nv = struct.unpack_from("<HH", b, p + 4)
                p += 8 + (nlen + (-nlen % 8) if ver == 1 else nlen)
            else:
                flags, nv = struct.unpack_from("<HH", b, p + 2)
                p += 6
            vals = struct.unpack_from("<%dI" % nv, b, p)
            p += 4 * nv + (4 if ver == 1 and nv % 2 else 0)
            out.append((fid, vals))
        return out

    def _chunked(self, msgs, tree, cdims, shp, dt):
        nd = len(cdims) + 1
        filters = self._filters(msgs)
        out = np.zeros(shp, dtype=dt)
        if tree == UNDEF:
            return out
        csize = int(np.prod(cdims)) * dt.itemsize
        for offs, mask, size, addr in self._chunk_nodes(tree, nd):
            raw = self.d[self.at(addr):self.at(addr) + size]
            for i, (fid, vals) in reversed(list(enumerate(filters))):
                if mask & (1 << i):
                    continue
                if fid == 1:
                    raw = zlib.decompress(raw)
                elif fid == 2:
                    es = vals[0] if vals else dt.itemsize
                    raw = np.frombuffer(raw, np.uint8).reshape(es, -1).T.tobytes()
                elif fid == 3:
                    raw = raw[:-4]
                else:
                    raise MatFileError("filter %d" % fid)
            chunk = np.frombuffer(raw[:csize], dtype=dt).reshape(cdims)
            dst = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, cdims, shp))
            out[dst] = chunk[tuple(slice(0, x.stop - x.start) for x in dst)]
        return out

    def _chunk_nodes(self, tree, nd):
        a = self.at(tree)
        if self.d[a:a + 4] != b"TREE" or self.d[a + 4] != 1:
            raise MatFileError("bad chunk B-tree")
        level, n = self.d[a + 5], struct.unpack_from("<H", self.d, a + 6)[0]
        ks = 8 + 8 * nd
        p = a + 24
        for _ in range(n):
            size, mask = struct.unpack_from("<II", self.d, p)
            offs = struct.unpack_from("<%dQ" % nd, self.d, p + 8)[:-1]
            child = struct.unpack_from("<Q", self.d, p + ks)[0]
            p += ks + 8
            if level == 0:
                yield offs, mask, size, child
            else:
                yield from self._chunk_nodes(child, nd)

    # MATLAB values --------------------------------------------------------
    def value(self, addr):
        msgs = self.messages(addr)
        attrs = self.attributes(msgs)
        if self.first(msgs, 0x08) is None:
            return {k: self.value(a) for k, a in self.links(msgs).items()}
        arr = self.data(msgs)
        cls = attrs.get("MATLAB_class")
        if attrs.get("MATLAB_empty"):
            return "" if cls == "char" else np.zeros(0, dtype=arr.dtype)
        if cls == "char":
            return arr.astype("<u2").tobytes().decode("utf-16-le")
        if cls == "logical":
            return arr.astype(bool)
        if arr.dtype.byteorder == ">":
            arr = arr.astype(arr.dtype.newbyteorder("<"))
        return arr

    def attrs_of(self, path):
        """Attributes of the object at a '/'-separated path (tests, tools)."""
        addr = self.root
        for part in [p for p in path.split("/") if p]:
            addr = self.links(self.messages(addr))[part]
        return self.attributes(self.messages(addr))


def loads(data):
    r = _Reader(data)
    return r.value(r.root)


def load(path):
    """The root group's members as Python values (HDF5::matlabDeserialize)."""
    with open(path, "rb") as f:
        return loads(f.read())


def reader(path):
    with open(path, "rb") as f:
        return _Reader(f.read())
