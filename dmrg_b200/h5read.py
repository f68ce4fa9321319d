"""Read-only reader for the HDF5 files the reference writes through h5pp, in pure Python + numpy.

The image this package runs in has no HDF5 library (no libhdf5, no h5py), yet the reference's dumps of its hot-path
operands are HDF5 files:

* ``dmrg-contractions.h5`` (contraction_tblis.cpp:72-84, under ``DMRG_SAVE_CONTRACTION``): groups ``contraction_<n>``
  holding ``mps``, ``mpo``, ``envL``, ``envR``;
* ``svd-save-<seed>.h5`` (math/svd/svd_save.cpp:32-66, 112-181): groups ``svd_<n>`` / ``svd-last`` / ``svd-fail``
  holding ``A`` (or ``A_real``/``A_cplx``), ``U``, ``S``, ``VT`` and attributes ``rank_max``, ``truncation_lim`` ...;
* the SVD test matrices of tests/svd/main.cpp:69-87 (one root dataset ``svdmatrix``) and the SVD bench file of
  bench/svd/main.cpp:89-108 (groups ``svd_<n>`` with ``A``, ``U``, ``S``, ``V`` and attributes ``rank_max``,
  ``threshold``);
* the eigensolver bench's ``eigs.h5`` (bench/eig/main.cpp:45-62: groups ``eigs-<n>`` holding ``mps``, ``mpo2``,
  ``envL2``, ``envR2`` and the recorded solve as attributes) and the dense eigenproblem fixtures
  tests/testmatrices/lapacke_matrix-*.h5 (``matrix``, ``eigvals``, ``eigvecs``, ``theta``, ``overlaps``).

This module implements the part of the published HDF5 file format (HDF Group, "HDF5 File Format Specification",
versions 2.0/3.0) those files use: superblocks v0-v3; object headers v1 and v2 with continuation blocks; groups stored
as symbol tables (v1 B-tree + local heap) or as compact link messages; datasets with compact, contiguous or chunked
layout (layout message v1-v4; v1 B-tree chunk index, single-chunk and implicit indices); the deflate, shuffle and
fletcher32 filters; fixed-point, IEEE float, string (fixed and variable length, through the global heap), compound
(h5pp's ``{real, imag}`` complex pair becomes complex128) and array datatypes; attributes on groups and datasets.
Anything outside that subset raises ``H5FormatError`` naming the feature, rather than returning wrong data.

Arrays come back in the file's C (row-major) order with the file's dimensions.  h5pp converts Eigen's column-major
matrices and tensors to row-major when it writes them, so those dimensions are the Eigen dimensions (rows, cols, ...)
and ``np.asfortranarray`` of the result is the reference's in-memory layout.  The reference's eigenproblem fixtures
confirm it: their eigenvector matrices, read this way, satisfy A V = V diag(w) column by column.
"""
import mmap
import os
import zlib

import numpy as np

__all__ = ["H5File", "H5Group", "H5Dataset", "H5FormatError"]

_SIGNATURE = b"\x89HDF\r\n\x1a\n"


class H5FormatError(ValueError):
    """The file is not HDF5, is damaged, or uses a feature this reader does not implement (named in the message)."""


def _undef(addr, size):
    return addr == (1 << (8 * size)) - 1


class _Cursor:
    """Little-endian field reader over a bytes-like buffer."""

    __slots__ = ("buf", "pos", "so", "sl")

    def __init__(self, buf, pos, so=8, sl=8):
        self.buf, self.pos, self.so, self.sl = buf, pos, so, sl

    def u(self, n):
        if self.pos + n > len(self.buf):
            raise H5FormatError("read past the end of a structure")
        v = int.from_bytes(self.buf[self.pos:self.pos + n], "little")
        self.pos += n
        return v

    def off(self):
        return self.u(self.so)

    def length(self):
        return self.u(self.sl)

    def raw(self, n):
        if self.pos + n > len(self.buf):
            raise H5FormatError("read past the end of a structure")
        b = bytes(self.buf[self.pos:self.pos + n])
        self.pos += n
        return b

    def skip(self, n):
        self.pos += n

    def align(self, base, a=8):
        r = (self.pos - base) % a
        if r:
            self.pos += a - r

    def cstr(self):
        end = self.buf.find(b"\x00", self.pos)
        if end < 0:
            raise H5FormatError("unterminated name")
        s = bytes(self.buf[self.pos:end]).decode("utf-8", "replace")
        self.pos = end + 1
        return s


# ------------------------------------------------------------------------------------------------------- datatypes
class _Type:
    """A parsed datatype message: ``kind`` in {int, float, string, vlen_string, vlen_seq, compound, array, opaque,
    enum, reference}, the element ``size`` in bytes, and a numpy dtype for the raw bytes where one exists."""

    def __init__(self, kind, size, np_dtype=None, **kw):
        self.kind, self.size, self.np_dtype = kind, size, np_dtype
        self.__dict__.update(kw)


def _parse_datatype(c):
    cv = c.u(1)
    cls, version = cv & 0x0F, cv >> 4
    bits = c.u(3)
    size = c.u(4)
    if cls == 0:  # fixed-point
        c.skip(4)
        order = ">" if bits & 1 else "<"
        signed = bool(bits & 0x08)
        if size not in (1, 2, 4, 8):
            raise H5FormatError(f"fixed-point datatype of {size} bytes")
        return _Type("int", size, np.dtype(f"{order}{'i' if signed else 'u'}{size}"))
    if cls == 1:  # IEEE float
        c.skip(12)
        order = ">" if bits & 1 else "<"
        if bits & 0x40:
            raise H5FormatError("VAX-order float")
        if size not in (2, 4, 8):
            raise H5FormatError(f"float datatype of {size} bytes")
        return _Type("float", size, np.dtype(f"{order}f{size}"))
    if cls == 3:  # fixed-length string
        return _Type("string", size, np.dtype(f"S{size}"), utf8=bool((bits >> 4) & 0x0F))
    if cls == 4:  # bitfield
        c.skip(4)
        return _Type("int", size, np.dtype(f"{'>' if bits & 1 else '<'}u{size}"))
    if cls == 5:  # opaque
        taglen = bits & 0xFF
        c.skip(taglen)
        return _Type("opaque", size, np.dtype(f"V{size}"))
    if cls == 6:  # compound
        nmemb = bits & 0xFFFF
        members = []
        for _ in range(nmemb):
            start = c.pos
            name = c.cstr()
            if version < 3:
                c.align(start, 8)
                moff = c.u(4)
                if version == 1:
                    ndims = c.u(1)
                    c.skip(3 + 4 + 4 + 16)
                    if ndims:
                        raise H5FormatError("array-valued compound member (version 1)")
            else:
                nb = 1 if size < 1 << 8 else 2 if size < 1 << 16 else 3 if size < 1 << 24 else 4
                moff = c.u(nb)
            members.append((name, moff, _parse_datatype(c)))
        fields = {}
        for name, moff, t in members:
            if t.np_dtype is None:
                raise H5FormatError(f"compound member {name!r} of kind {t.kind}")
            fields[name] = (t.np_dtype, moff)
        npd = np.dtype({"names": list(fields), "formats": [f[0] for f in fields.values()],
                        "offsets": [f[1] for f in fields.values()], "itemsize": size})
        names = [m[0] for m in members]
        cplx = (len(members) == 2 and all(m[2].kind == "float" and m[2].size == members[0][2].size for m in members)
                and (names in (["real", "imag"], ["r", "i"], ["re", "im"])) and members[1][1] == members[0][2].size)
        return _Type("compound", size, npd, complex=cplx, members=members)
    if cls == 7:  # reference
        return _Type("reference", size, np.dtype(f"V{size}"))
    if cls == 8:  # enumeration
        base = _parse_datatype(c)
        n = bits & 0xFFFF
        names = []
        for _ in range(n):
            start = c.pos
            names.append(c.cstr())
            if version < 3:
                c.align(start, 8)
        values = [int.from_bytes(c.raw(base.size), "little") for _ in range(n)]
        return _Type("enum", size, base.np_dtype, names=dict(zip(values, names)))
    if cls == 9:  # variable length
        vtype = bits & 0x0F
        base = _parse_datatype(c)
        return _Type("vlen_string" if vtype == 1 else "vlen_seq", size, None, base=base)
    if cls == 10:  # array
        nd = c.u(1)
        if version < 3:
            c.skip(3)
        adims = [c.u(4) for _ in range(nd)]
        if version < 3:
            c.skip(4 * nd)
        base = _parse_datatype(c)
        if base.np_dtype is None:
            raise H5FormatError("array of a variable-length type")
        return _Type("array", size, np.dtype((base.np_dtype, tuple(adims))), base=base)
    raise H5FormatError(f"datatype class {cls}")


def _parse_dataspace(c):
    version = c.u(1)
    rank = c.u(1)
    flags = c.u(1)
    if version == 1:
        c.skip(5)
        kind = "simple" if rank else "scalar"
    elif version == 2:
        kind = {0: "scalar", 1: "simple", 2: "null"}.get(c.u(1))
        if kind is None:
            raise H5FormatError("dataspace type")
    else:
        raise H5FormatError(f"dataspace message version {version}")
    shape = tuple(c.length() for _ in range(rank))
    if kind == "null":
        return None
    return shape if kind == "simple" else ()


# ------------------------------------------------------------------------------------------------------- the file
class H5File:
    """An HDF5 file opened read-only: ``f["group/dataset"]`` gives an ``H5Group`` or ``H5Dataset``; ``f.root`` is the
    root group.  Use as a context manager or call ``close()``."""

    def __init__(self, path):
        self.path = os.fspath(path)
        self._fh = open(self.path, "rb")
        size = os.fstat(self._fh.fileno()).st_size
        if size < 64:
            self._fh.close()
            raise H5FormatError(f"{self.path}: too small for an HDF5 file")
        self._buf = mmap.mmap(self._fh.fileno(), 0, access=mmap.ACCESS_READ)
        self._headers = {}
        self._gheaps = {}
        try:
            self._parse_superblock(self._find_superblock())
        except Exception:
            self.close()
            raise

    # --- context management
    def close(self):
        if self._buf is not None:
            self._headers.clear()
            self._gheaps.clear()
            self._buf.close()
            self._fh.close()
            self._buf = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --- superblock
    def _find_superblock(self):
        pos = 0
        while pos + 8 <= len(self._buf):
            if self._buf[pos:pos + 8] == _SIGNATURE:
                return pos
            pos = 512 if pos == 0 else pos * 2
        raise H5FormatError(f"{self.path}: no HDF5 signature")

    def _parse_superblock(self, at):
        b = self._buf
        version = b[at + 8]
        if version in (0, 1):
            self.so, self.sl = b[at + 13], b[at + 14]
            c = _Cursor(b, at + 24 + (4 if version == 1 else 0), self.so, self.sl)
            self.base = c.off()
            c.off()  # free-space info
            c.off()  # end of file
            c.off()  # driver info
            c.off()  # root link name offset
            root = c.off()
        elif version in (2, 3):
            self.so, self.sl = b[at + 9], b[at + 10]
            c = _Cursor(b, at + 12, self.so, self.sl)
            self.base = c.off()
            c.off()  # superblock extension
            c.off()  # end of file
            root = c.off()
        else:
            raise H5FormatError(f"superblock version {version}")
        if self.so not in (2, 4, 8) or self.sl not in (2, 4, 8):
            raise H5FormatError("sizes of offsets/lengths")
        self.root = H5Group(self, root, "/")

    def _cursor(self, addr):
        a = self.base + addr
        if a >= len(self._buf):
            raise H5FormatError(f"address {addr:#x} beyond the end of the file")
        return _Cursor(self._buf, a, self.so, self.sl)

    # --- object headers
    def _messages(self, addr):
        """[(type, flags, data bytes)] of the object header at addr, continuation blocks followed."""
        if addr in self._headers:
            return self._headers[addr]
        b = self._buf
        a = self.base + addr
        msgs = []
        seen = set()
        if b[a:a + 4] == b"OHDR":
            c = self._cursor(addr)
            c.skip(4)
            if c.u(1) != 2:
                raise H5FormatError("object header version")
            flags = c.u(1)
            if flags & 0x20:
                c.skip(16)
            if flags & 0x10:
                c.skip(4)
            size0 = c.u(1 << (flags & 3))
            blocks = [(c.pos, size0)]
            track_order = bool(flags & 0x04)
            while blocks:
                start, size = blocks.pop(0)
                c.pos = start
                end = start + size
                while end - c.pos >= 4 + (2 if track_order else 0):
                    mtype, msize, mflags = c.u(1), c.u(2), c.u(1)
                    if track_order:
                        c.skip(2)
                    data = c.raw(msize)
                    if mtype == 0x10:
                        cc = _Cursor(data, 0, self.so, self.sl)
                        caddr, clen = cc.off(), cc.length()
                        cs = self.base + caddr
                        if b[cs:cs + 4] != b"OCHK":
                            raise H5FormatError("continuation block signature")
                        if cs in seen:
                            raise H5FormatError("object header continuation cycle")
                        seen.add(cs)
                        blocks.append((cs + 4, clen - 8))
                    else:
                        msgs.append((mtype, mflags, data))
        else:
            c = self._cursor(addr)
            if c.u(1) != 1:
                raise H5FormatError(f"object header version at {addr:#x}")
            c.skip(1)
            nmsgs = c.u(2)
            c.skip(4)
            size0 = c.u(4)
            c.skip(4)  # the header's 12 bytes are padded to 16
            blocks = [(c.pos, size0)]
            while blocks and len(msgs) < nmsgs:
                start, size = blocks.pop(0)
                c.pos = start
                end = start + size
                while c.pos + 8 <= end:
                    mtype, msize, mflags = c.u(2), c.u(2), c.u(1)
                    c.skip(3)
                    data = c.raw(msize)
                    if mtype == 0x10:
                        cc = _Cursor(data, 0, self.so, self.sl)
                        caddr, clen = cc.off(), cc.length()
                        if caddr in seen:
                            raise H5FormatError("object header continuation cycle")
                        seen.add(caddr)
                        blocks.append((self.base + caddr, clen))
                    msgs.append((mtype, mflags, data))
            msgs = [m for m in msgs if m[0] != 0x10]
        self._headers[addr] = msgs
        return msgs

    def _message_data(self, mtype, mflags, data):
        """The body of a message, following a shared-message reference to the object header that holds it."""
        if not (mflags & 0x02):
            return data
        c = _Cursor(data, 0, self.so, self.sl)
        version = c.u(1)
        stype = c.u(1)
        if version == 1:
            c.skip(6)
        if version == 3 and stype != 2:
            raise H5FormatError("shared message in the shared-message heap")
        target = c.off()
        for t, f, d in self._messages(target):
            if t == mtype:
                return self._message_data(t, f, d)
        raise H5FormatError("shared message target lacks the message")

    # --- heaps
    def _local_heap_data(self, addr):
        c = self._cursor(addr)
        if c.raw(4) != b"HEAP":
            raise H5FormatError("local heap signature")
        c.skip(4)
        size = c.length()
        c.length()
        data_addr = c.off()
        a = self.base + data_addr
        return self._buf[a:a + size]

    def _global_heap_object(self, addr, index):
        heap = self._gheaps.get(addr)
        if heap is None:
            c = self._cursor(addr)
            if c.raw(4) != b"GCOL":
                raise H5FormatError("global heap signature")
            c.skip(4)
            csize = c.length()
            end = self.base + addr + csize
            heap = {}
            while c.pos + 8 + self.sl <= end:
                idx = c.u(2)
                c.skip(6)
                osize = c.length()
                if idx == 0:
                    break
                heap[idx] = bytes(self._buf[c.pos:c.pos + osize])
                c.pos += (osize + 7) & ~7
            self._gheaps[addr] = heap
        try:
            return heap[index]
        except KeyError:
            raise H5FormatError("global heap object missing") from None

    # --- navigation
    def __getitem__(self, path):
        return self.root[path]

    def __contains__(self, path):
        try:
            self.root[path]
            return True
        except KeyError:
            return False

    def visit(self):
        """Every (path, object) in the file, depth first, in name order."""
        return self.root.visit()


class _Object:
    def __init__(self, f, addr, name):
        self.file, self.addr, self.name = f, addr, name
        self._attrs = None

    def _msgs(self, mtype):
        return [self.file._message_data(t, fl, d) for t, fl, d in self.file._messages(self.addr) if t == mtype]

    @property
    def attrs(self):
        """Attributes stored in the object header: {name: numpy scalar/array or str}."""
        if self._attrs is None:
            self._attrs = {}
            for data in self._msgs(0x0C):
                name, value = _parse_attribute(self.file, data)
                self._attrs[name] = value
            for data in self._msgs(0x15):  # attribute info: dense storage would hold the attributes in a fractal heap
                c = _Cursor(data, 0, self.file.so, self.file.sl)
                c.skip(1)
                fl = c.u(1)
                if fl & 1:
                    c.skip(2)
                if not _undef(c.off(), self.file.so):
                    raise H5FormatError("dense attribute storage (fractal heap)")
        return self._attrs


def _object(f, addr, name):
    types = {t for t, _, _ in f._messages(addr)}
    if 0x11 in types or 0x06 in types or 0x02 in types:
        return H5Group(f, addr, name)
    if 0x08 in types:
        return H5Dataset(f, addr, name)
    if 0x03 in types:
        raise H5FormatError(f"{name}: committed datatype objects are not readable as data")
    return H5Group(f, addr, name)


class H5Group(_Object):
    """A group: mapping of link names to groups and datasets."""

    def _links(self):
        if getattr(self, "_link_cache", None) is not None:
            return self._link_cache
        f = self.file
        links = {}
        for data in self._msgs(0x11):
            c = _Cursor(data, 0, f.so, f.sl)
            btree, heap = c.off(), c.off()
            names = f._local_heap_data(heap)
            self._walk_group_btree(btree, names, links)
        for data in self._msgs(0x06):
            name, addr = _parse_link(data, f.so)
            if addr is not None:
                links[name] = addr
        for data in self._msgs(0x02):
            c = _Cursor(data, 0, f.so, f.sl)
            c.skip(1)
            fl = c.u(1)
            if fl & 1:
                c.skip(8)
            if not _undef(c.off(), f.so):
                raise H5FormatError(f"{self.name}: dense link storage (fractal heap)")
        self._link_cache = dict(sorted(links.items()))
        return self._link_cache

    def _walk_group_btree(self, addr, names, links):
        f = self.file
        c = f._cursor(addr)
        if c.raw(4) != b"TREE" or c.u(1) != 0:
            raise H5FormatError("group B-tree node")
        level, used = c.u(1), c.u(2)
        c.off()
        c.off()
        children = []
        for _ in range(used):
            c.length()  # key: heap offset of the left name
            children.append(c.off())
        for ch in children:
            if level > 0:
                self._walk_group_btree(ch, names, links)
                continue
            s = f._cursor(ch)
            if s.raw(4) != b"SNOD":
                raise H5FormatError("symbol table node signature")
            s.skip(2)
            n = s.u(2)
            for _ in range(n):
                name_off = s.off()
                obj = s.off()
                s.skip(4 + 4 + 16)
                end = names.find(b"\x00", name_off)
                links[bytes(names[name_off:end]).decode("utf-8", "replace")] = obj

    def keys(self):
        return list(self._links())

    def __iter__(self):
        return iter(self._links())

    def __len__(self):
        return len(self._links())

    def __getitem__(self, path):
        parts = [p for p in path.split("/") if p]
        obj = self
        for i, p in enumerate(parts):
            if not isinstance(obj, H5Group):
                raise KeyError(path)
            links = obj._links()
            if p not in links:
                raise KeyError(path)
            prefix = obj.name.rstrip("/")
            obj = _object(self.file, links[p], f"{prefix}/{p}")
        return obj

    def __contains__(self, name):
        try:
            self[name]
            return True
        except KeyError:
            return False

    def items(self):
        return [(k, self[k]) for k in self._links()]

    def visit(self):
        out = []
        for k, v in self.items():
            out.append((v.name, v))
            if isinstance(v, H5Group):
                out.extend(v.visit())
        return out

    def __repr__(self):
        return f"<H5Group {self.name} ({len(self)} links)>"


def _parse_link(data, so):
    c = _Cursor(data, 0, so, 8)
    if c.u(1) != 1:
        raise H5FormatError("link message version")
    flags = c.u(1)
    ltype = c.u(1) if flags & 0x08 else 0
    if flags & 0x04:
        c.skip(8)
    if flags & 0x10:
        c.skip(1)
    nlen = c.u(1 << (flags & 3))
    name = c.raw(nlen).decode("utf-8", "replace")
    if ltype == 0:
        return name, c.off()
    return name, None  # soft and external links are not followed


class H5Dataset(_Object):
    """A dataset: ``shape``, ``dtype`` (numpy; complex128 for h5pp's complex pair), ``read()`` -> numpy array."""

    def _meta(self):
        if getattr(self, "_meta_cache", None) is not None:
            return self._meta_cache
        f = self.file
        space = self._msgs(0x01)
        dtype = self._msgs(0x03)
        layout = self._msgs(0x08)
        if not (space and dtype and layout):
            raise H5FormatError(f"{self.name}: dataset without dataspace/datatype/layout")
        shape = _parse_dataspace(_Cursor(space[0], 0, f.so, f.sl))
        t = _parse_datatype(_Cursor(dtype[0], 0, f.so, f.sl))
        filters = []
        for data in self._msgs(0x0B):
            filters = _parse_filters(data)
        self._meta_cache = (shape, t, _parse_layout(layout[0], f.so, f.sl), filters)
        return self._meta_cache

    @property
    def shape(self):
        return self._meta()[0]

    @property
    def dtype(self):
        t = self._meta()[1]
        if t.kind == "compound" and t.complex:
            return np.dtype(np.complex128 if t.members[0][2].size == 8 else np.complex64)
        if t.kind in ("vlen_string", "string"):
            return np.dtype(object)
        return t.np_dtype.newbyteorder("=") if t.np_dtype is not None else None

    def read(self):
        shape, t, layout, filters = self._meta()
        if shape is None:
            return None
        n = int(np.prod(shape, dtype=np.int64)) if shape else 1
        raw = _read_layout(self.file, layout, filters, shape, t.size, n)
        return _decode(self.file, raw, t, shape if shape else ())

    def __array__(self, dtype=None, copy=None):
        a = self.read()
        return a if dtype is None else a.astype(dtype)

    def __repr__(self):
        return f"<H5Dataset {self.name} shape={self.shape}>"


def _parse_filters(data):
    c = _Cursor(data, 0)
    version = c.u(1)
    n = c.u(1)
    if version == 1:
        c.skip(6)
    out = []
    for _ in range(n):
        fid = c.u(2)
        nlen = c.u(2) if (version == 1 or fid >= 256) else 0
        flags = c.u(2)
        nvals = c.u(2)
        if nlen:
            c.skip(((nlen + 7) & ~7) if version == 1 else nlen)
        vals = [c.u(4) for _ in range(nvals)]
        if version == 1 and nvals % 2:
            c.skip(4)
        out.append((fid, flags, vals))
    return out


def _parse_layout(data, so, sl):
    c = _Cursor(data, 0, so, sl)
    version = c.u(1)
    if version in (1, 2):
        nd = c.u(1)
        cls = c.u(1)
        c.skip(5)
        addr = c.off() if cls != 0 else None
        ldims = [c.u(4) for _ in range(nd)]
        if cls == 0:
            size = c.u(4)
            return {"class": "compact", "data": c.raw(size)}
        if cls == 1:
            return {"class": "contiguous", "addr": addr}
        return {"class": "chunked", "index": "btree1", "addr": addr, "chunk": ldims[:-1]}
    if version in (3, 4):
        cls = c.u(1)
        if cls == 0:
            size = c.u(2)
            return {"class": "compact", "data": c.raw(size)}
        if cls == 1:
            return {"class": "contiguous", "addr": c.off()}
        if cls == 2 and version == 3:
            nd = c.u(1)
            addr = c.off()
            ldims = [c.u(4) for _ in range(nd)]
            return {"class": "chunked", "index": "btree1", "addr": addr, "chunk": ldims[:-1]}
        if cls == 2:
            flags = c.u(1)
            nd = c.u(1)
            enc = c.u(1)
            ldims = [c.u(enc) for _ in range(nd)]
            itype = c.u(1)
            out = {"class": "chunked", "chunk": ldims[:-1] if len(ldims) > 1 else ldims}
            if itype == 1:
                if flags & 0x02:
                    out["filtered_size"] = c.length()
                    out["filter_mask"] = c.u(4)
                out["index"] = "single"
            elif itype == 2:
                out["index"] = "implicit"
            else:
                raise H5FormatError(f"chunk index type {itype} (fixed/extensible array or v2 B-tree)")
            out["addr"] = c.off()
            return out
        raise H5FormatError(f"layout class {cls}")
    raise H5FormatError(f"layout message version {version}")


def _unfilter(chunk, filters, mask):
    for i in range(len(filters) - 1, -1, -1):
        fid, _, vals = filters[i]
        if mask & (1 << i):
            continue
        if fid == 1:
            chunk = zlib.decompress(chunk)
        elif fid == 2:
            es = vals[0] if vals else 1
            if es > 1:
                a = np.frombuffer(chunk, np.uint8)
                nel = len(a) // es
                body = a[:nel * es].reshape(es, nel).T.reshape(-1)
                chunk = body.tobytes() + bytes(a[nel * es:])
        elif fid == 3:
            chunk = chunk[:-4]
        else:
            raise H5FormatError(f"filter {fid}")
    return chunk


def _read_layout(f, layout, filters, shape, esize, n):
    nbytes = n * esize
    kind = layout["class"]
    if kind == "compact":
        data = layout["data"]
        if len(data) < nbytes:
            raise H5FormatError("compact data shorter than the dataspace")
        return data[:nbytes]
    if kind == "contiguous":
        if _undef(layout["addr"], f.so):
            return bytes(nbytes)
        a = f.base + layout["addr"]
        if a + nbytes > len(f._buf):
            raise H5FormatError("contiguous data beyond the end of the file")
        return f._buf[a:a + nbytes]
    chunk = [int(x) for x in layout["chunk"]]
    rank = len(shape)
    if rank == 0:
        chunk, shape = [1], (1,)
        rank = 1
    if len(chunk) != rank:
        raise H5FormatError("chunk rank differs from the dataspace rank")
    out = np.zeros(nbytes, np.uint8).reshape(tuple(shape) + (esize,))
    cbytes = int(np.prod(chunk)) * esize

    def place(offsets, payload):
        blk = np.frombuffer(payload[:cbytes], np.uint8)
        if blk.size < cbytes:
            raise H5FormatError("chunk shorter than its dimensions")
        blk = blk.reshape(tuple(chunk) + (esize,))
        dst, src = [], []
        for o, cdim, sdim in zip(offsets, chunk, shape):
            e = min(o + cdim, sdim)
            if o >= sdim:
                return
            dst.append(slice(o, e))
            src.append(slice(0, e - o))
        out[tuple(dst)] = blk[tuple(src)]

    if _undef(layout["addr"], f.so):
        return out.reshape(-1).tobytes()
    if layout["index"] == "single":
        size = layout.get("filtered_size", cbytes)
        a = f.base + layout["addr"]
        place([0] * rank, _unfilter(bytes(f._buf[a:a + size]), filters, layout.get("filter_mask", 0)))
    elif layout["index"] == "implicit":
        grid = [-(-s // cdim) for s, cdim in zip(shape, chunk)]
        a = f.base + layout["addr"]
        for k, idx in enumerate(np.ndindex(*grid)):
            place([i * cdim for i, cdim in zip(idx, chunk)], bytes(f._buf[a + k * cbytes:a + (k + 1) * cbytes]))
    else:
        _walk_chunk_btree(f, layout["addr"], rank, filters, place)
    return out.reshape(-1).tobytes()


def _walk_chunk_btree(f, addr, rank, filters, place):
    c = f._cursor(addr)
    if c.raw(4) != b"TREE" or c.u(1) != 1:
        raise H5FormatError("chunk B-tree node")
    level, used = c.u(1), c.u(2)
    c.off()
    c.off()
    entries = []
    for _ in range(used):
        size, mask = c.u(4), c.u(4)
        offs = [c.u(8) for _ in range(rank + 1)]
        entries.append((size, mask, offs[:rank], c.off()))
    for size, mask, offs, child in entries:
        if level > 0:
            _walk_chunk_btree(f, child, rank, filters, place)
        else:
            a = f.base + child
            place(offs, _unfilter(bytes(f._buf[a:a + size]), filters, mask))


def _decode(f, raw, t, shape):
    if t.kind == "vlen_string" or (t.kind == "vlen_seq"):
        n = int(np.prod(shape, dtype=np.int64)) if shape else 1
        c = _Cursor(raw, 0, f.so, f.sl)
        vals = []
        for _ in range(n):
            length, gaddr, gidx = c.u(4), c.off(), c.u(4)
            if length == 0 or _undef(gaddr, f.so) or gaddr == 0:
                obj = b""
            else:
                obj = f._global_heap_object(gaddr, gidx)
            if t.kind == "vlen_string":
                vals.append(obj[:length].split(b"\x00", 1)[0].decode("utf-8", "replace"))
            else:
                vals.append(np.frombuffer(obj[:length * t.base.size], t.base.np_dtype).copy())
        return vals[0] if shape == () else np.array(vals, dtype=object).reshape(shape)
    a = np.frombuffer(raw, t.np_dtype, count=int(np.prod(shape, dtype=np.int64)) if shape else 1).reshape(shape)
    if t.kind == "compound" and t.complex:
        names = [m[0] for m in t.members]
        a = a[names[0]].astype(np.float64) + 1j * a[names[1]].astype(np.float64)
        return a.astype(np.complex128 if t.members[0][2].size == 8 else np.complex64)
    if t.kind == "string":
        vals = np.vectorize(lambda s: s.split(b"\x00", 1)[0].decode("utf-8", "replace"), otypes=[object])(a)
        return vals.item() if shape == () else vals
    a = a.astype(t.np_dtype.newbyteorder("="), copy=True)
    return a


def _parse_attribute(f, data):
    c = _Cursor(data, 0, f.so, f.sl)
    version = c.u(1)
    c.skip(1)
    nsize, tsize, ssize = c.u(2), c.u(2), c.u(2)
    if version == 3:
        c.skip(1)
    pad = (lambda n: (n + 7) & ~7) if version == 1 else (lambda n: n)
    start = c.pos
    name = bytes(data[start:start + nsize]).split(b"\x00", 1)[0].decode("utf-8", "replace")
    c.pos = start + pad(nsize)
    tstart = c.pos
    t = _parse_datatype(_Cursor(data, tstart, f.so, f.sl))
    c.pos = tstart + pad(tsize)
    shape = _parse_dataspace(_Cursor(data, c.pos, f.so, f.sl))
    c.pos += pad(ssize)
    if shape is None:
        return name, None
    n = int(np.prod(shape, dtype=np.int64)) if shape else 1
    raw = bytes(data[c.pos:c.pos + n * t.size])
    value = _decode(f, raw, t, shape)
    if isinstance(value, np.ndarray) and value.shape == () and value.dtype != object:
        value = value[()]
    return name, value
