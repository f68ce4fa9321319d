"""Minimal HDF5 writer for tests of dmrg_b200.h5read (the image has no HDF5 library to make test files with).

It writes the structures the reference's h5pp dumps contain, following the published HDF5 file format specification:
superblock v0; groups as symbol tables (v1 B-tree + symbol node + local heap) or, with ``links=True``, as a version-2
object header holding link messages; datasets in version-1 (or, with ``ohdr_v2=True``, version-2) object headers with
dataspace v1, float64 / int64 / h5pp complex compound / fixed and variable-length string datatypes, and compact,
contiguous or chunked (v1 B-tree index, optional shuffle + deflate + fletcher32 filters) layouts through layout
messages version 1-3, or version 4 with a single-chunk or implicit index; attribute messages version 1-3.
Checksums of version-2 headers and fletcher32 are written as zeros: the reader under test does not verify them.
"""
import struct
import zlib

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF


def _pad8(b):
    return b + bytes((-len(b)) % 8)


def _float_type(size=8):
    if size == 8:
        return bytes([0x11, 0x20, 0x3F, 0x00]) + struct.pack("<I", 8) + struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
    return bytes([0x11, 0x20, 0x1F, 0x00]) + struct.pack("<I", 4) + struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)


def _int_type(size=8, signed=True):
    return bytes([0x10, 0x08 if signed else 0x00, 0, 0]) + struct.pack("<I", size) + struct.pack("<HH", 0, 8 * size)


def _complex_type(fsize=8):
    out = bytes([0x16]) + struct.pack("<I", 2)[:3] + struct.pack("<I", 2 * fsize)
    for name, off in (("real", 0), ("imag", fsize)):
        out += _pad8(name.encode() + b"\x00") + struct.pack("<I", off) + bytes(1 + 3 + 4 + 4 + 16) + _float_type(fsize)
    return out


def _fixed_string_type(n):
    return bytes([0x13, 0x00, 0x00, 0x00]) + struct.pack("<I", n)


def _vlen_string_type():
    return bytes([0x19, 0x01, 0x00, 0x00]) + struct.pack("<I", 16) + _int_type(1, signed=False)


def _dataspace(shape):
    return bytes([1, len(shape), 0, 0]) + bytes(4) + b"".join(struct.pack("<Q", int(s)) for s in shape)


class Writer:
    def __init__(self):
        self.buf = bytearray(96)  # the superblock is written last

    def alloc(self, data, align=8):
        self.buf += bytes((-len(self.buf)) % align)
        addr = len(self.buf)
        self.buf += data
        return addr

    # --- object headers
    def ohdr_v1(self, msgs):
        body = b""
        for t, flags, data in msgs:
            data = _pad8(data)
            body += struct.pack("<HHB3x", t, len(data), flags) + data
        head = struct.pack("<BBHII", 1, 0, len(msgs), 1, len(body)) + bytes(4)
        return self.alloc(head + body)

    def ohdr_v2(self, msgs):
        body = b""
        for t, flags, data in msgs:
            body += struct.pack("<BHB", t, len(data), flags) + data
        head = b"OHDR" + bytes([2, 0x02]) + struct.pack("<I", len(body))
        return self.alloc(head + body + bytes(4))

    # --- heaps
    def global_heap(self, objects):
        body = b""
        for i, o in enumerate(objects, 1):
            body += struct.pack("<HH4xQ", i, 1, len(o)) + _pad8(o)
        body += struct.pack("<HH4xQ", 0, 0, 0)
        head = b"GCOL" + bytes([1, 0, 0, 0]) + struct.pack("<Q", 16 + len(body))
        return self.alloc(head + body)

    # --- values -> (datatype, dataspace, raw bytes)
    def encode(self, value):
        if isinstance(value, str):
            gh = self.global_heap([value.encode()])
            return _vlen_string_type(), _dataspace(()), struct.pack("<IQI", len(value.encode()), gh, 1)
        if isinstance(value, bytes):
            return _fixed_string_type(len(value)), _dataspace(()), value
        a = np.asarray(value)
        if a.dtype.kind == "c":
            a = a.astype(np.complex128)
            return _complex_type(), _dataspace(a.shape), np.ascontiguousarray(a).tobytes()
        if a.dtype.kind == "f":
            if a.dtype == np.float32:
                return _float_type(4), _dataspace(a.shape), np.ascontiguousarray(a).tobytes()
            a = a.astype(np.float64)
            return _float_type(), _dataspace(a.shape), np.ascontiguousarray(a).tobytes()
        if a.dtype.kind in "iub":
            a = a.astype(np.int64)
            return _int_type(), _dataspace(a.shape), np.ascontiguousarray(a).tobytes()
        raise TypeError(a.dtype)

    def attribute(self, name, value, version=1):
        """Attribute message: version 1 pads name, datatype and dataspace to 8 bytes; 2 does not; 3 adds the name's
        character-set byte."""
        dt, ds, raw = self.encode(value)
        nm = name.encode() + b"\x00"
        if version == 1:
            return struct.pack("<BBHHH", 1, 0, len(nm), len(dt), len(ds)) + _pad8(nm) + _pad8(dt) + _pad8(ds) + raw
        head = struct.pack("<BBHHH", version, 0, len(nm), len(dt), len(ds)) + (b"\x00" if version == 3 else b"")
        return head + nm + dt + ds + raw

    # --- datasets
    def dataset(self, value, layout="contiguous", chunk=None, filters=(), attrs=None, ohdr_v2=False, layout_version=3, index="btree",
                attr_version=1):
        """layout_version 1 or 2: the old layout message (dimensions + element size as 4-byte fields); 3: the
        default; 4 with index "single" (one chunk, optionally filtered) or "implicit" (unfiltered chunks stored in
        order), otherwise the v1 B-tree through a version-3 message."""
        dt, ds, raw = self.encode(value)
        shape = np.asarray(value).shape
        esize = len(raw) // max(1, int(np.prod(shape)))
        msgs = [(0x01, 0, ds), (0x03, 1, dt)]
        dims4 = b"".join(struct.pack("<I", d) for d in list(shape) + [esize])
        if layout in ("compact", "contiguous") and layout_version in (1, 2):
            cls = 0 if layout == "compact" else 1
            body = bytes([layout_version, len(shape) + 1, cls]) + bytes(5)
            if cls == 1:
                body += struct.pack("<Q", self.alloc(raw)) + dims4
            else:
                body += dims4 + struct.pack("<I", len(raw)) + raw
            msgs.append((0x08, 0, body))
        elif layout == "compact":
            msgs.append((0x08, 0, bytes([3, 0]) + struct.pack("<H", len(raw)) + raw))
        elif layout == "contiguous":
            addr = self.alloc(raw)
            msgs.append((0x08, 0, bytes([3, 1]) + struct.pack("<QQ", addr, len(raw))))
        elif layout_version == 4 and index in ("single", "implicit"):
            chunk = list(chunk)
            cdims = b"".join(struct.pack("<I", c) for c in chunk + [esize])
            if index == "single":
                assert list(chunk) == list(shape), "a single chunk covers the dataset"
                payload = raw
                for f in filters:
                    if f == "shuffle" and esize > 1:
                        payload = np.frombuffer(payload, np.uint8).reshape(-1, esize).T.tobytes()
                    elif f == "deflate":
                        payload = zlib.compress(payload, 6)
                if filters:
                    msgs.append((0x0B, 0, self.filter_pipeline(filters, esize)))
                addr = self.alloc(payload)
                flags = 0x02 if filters else 0
                body = bytes([4, 2, flags, len(shape) + 1, 4]) + cdims + bytes([1])
                if filters:
                    body += struct.pack("<QI", len(payload), 0)
                msgs.append((0x08, 0, body + struct.pack("<Q", addr)))
            else:
                assert not filters, "implicit indices hold unfiltered chunks"
                full = np.frombuffer(raw, np.uint8).reshape(tuple(shape) + (esize,))
                grid = [-(-d // c) for d, c in zip(shape, chunk)]
                blob = b""
                for idx in np.ndindex(*grid):
                    offs = [i * c for i, c in zip(idx, chunk)]
                    blk = np.zeros(tuple(chunk) + (esize,), np.uint8)
                    src = tuple(slice(o, min(o + c, d)) for o, c, d in zip(offs, chunk, shape))
                    blk[tuple(slice(0, sl.stop - sl.start) for sl in src)] = full[src]
                    blob += blk.tobytes()
                addr = self.alloc(blob)
                msgs.append((0x08, 0, bytes([4, 2, 0, len(shape) + 1, 4]) + cdims + bytes([2]) + struct.pack("<Q", addr)))
        else:
            if filters:
                msgs.append((0x0B, 0, self.filter_pipeline(filters, esize)))
            btree = self.chunk_btree(np.asarray(value), raw, esize, chunk, filters)
            if layout_version in (1, 2):
                body = bytes([layout_version, len(shape) + 1, 2]) + bytes(5) + struct.pack("<Q", btree)
            else:
                body = bytes([3, 2, len(shape) + 1]) + struct.pack("<Q", btree)
            msgs.append((0x08, 0, body + b"".join(struct.pack("<I", c) for c in chunk) + struct.pack("<I", esize)))
        for k, v in (attrs or {}).items():
            msgs.append((0x0C, 0, self.attribute(k, v, attr_version)))
        return self.ohdr_v2(msgs) if ohdr_v2 else self.ohdr_v1(msgs)

    def filter_pipeline(self, filters, esize):
        fl = b""
        for f in filters:
            vals = {"shuffle": [esize], "deflate": [6], "fletcher32": []}[f]
            fid = {"deflate": 1, "shuffle": 2, "fletcher32": 3}[f]
            fl += struct.pack("<HHHH", fid, 0, 0, len(vals)) + b"".join(struct.pack("<I", v) for v in vals)
            if len(vals) % 2:
                fl += bytes(4)
        return bytes([1, len(filters)]) + bytes(6) + fl

    def chunk_btree(self, a, raw, esize, chunk, filters):
        shape = a.shape
        full = np.frombuffer(raw, np.uint8).reshape(tuple(shape) + (esize,))
        grid = [-(-s // c) for s, c in zip(shape, chunk)]
        entries = []
        for idx in np.ndindex(*grid):
            offs = [i * c for i, c in zip(idx, chunk)]
            blk = np.zeros(tuple(chunk) + (esize,), np.uint8)
            src = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, chunk, shape))
            blk[tuple(slice(0, sl.stop - sl.start) for sl in src)] = full[src]
            payload = blk.tobytes()
            for f in filters:  # applied in pipeline order
                if f == "shuffle" and esize > 1:
                    payload = np.frombuffer(payload, np.uint8).reshape(-1, esize).T.tobytes()
                elif f == "deflate":
                    payload = zlib.compress(payload, 6)
                elif f == "fletcher32":
                    payload = payload + bytes(4)
            entries.append((len(payload), offs, self.alloc(payload)))
        node = b"TREE" + bytes([1, 0]) + struct.pack("<HQQ", len(entries), UNDEF, UNDEF)
        for size, offs, addr in entries:
            node += struct.pack("<II", size, 0) + b"".join(struct.pack("<Q", o) for o in offs + [0]) + struct.pack("<Q", addr)
        node += struct.pack("<II", 0, 0) + b"".join(struct.pack("<Q", s) for s in list(shape) + [0])
        return self.alloc(node)

    # --- groups
    def group_symbol_table(self, children, attrs=None):
        """children: [(name, object header address)] -> (group header address, btree, heap)."""
        names = b"\x00" * 8
        offs = []
        for name, _ in children:
            offs.append(len(names))
            names += _pad8(name.encode() + b"\x00")
        heap_data = self.alloc(names)
        heap = self.alloc(b"HEAP" + bytes(4) + struct.pack("<QQQ", len(names), UNDEF, heap_data))
        snods = []
        for i in range(0, max(len(children), 1), 8):
            part = list(zip(children[i:i + 8], offs[i:i + 8]))
            body = b"SNOD" + bytes([1, 0]) + struct.pack("<H", len(part))
            for (_, obj), off in part:
                body += struct.pack("<QQII", off, obj, 0, 0) + bytes(16)
            snods.append((self.alloc(body), part[-1][1] if part else 0))
        node = b"TREE" + bytes([0, 0]) + struct.pack("<HQQ", len(snods), UNDEF, UNDEF) + struct.pack("<Q", 0)
        for addr, key in snods:
            node += struct.pack("<QQ", addr, key)
        btree = self.alloc(node)
        msgs = [(0x11, 0, struct.pack("<QQ", btree, heap))]
        for k, v in (attrs or {}).items():
            msgs.append((0x0C, 0, self.attribute(k, v)))
        return self.ohdr_v1(msgs), btree, heap

    def group_links(self, children, attrs=None):
        msgs = [(0x02, 0, bytes([0, 0]) + struct.pack("<QQ", UNDEF, UNDEF)), (0x0A, 0, bytes([0, 0]))]
        for name, obj in children:
            nm = name.encode()
            msgs.append((0x06, 0, bytes([1, 0, len(nm)]) + nm + struct.pack("<Q", obj)))
        for k, v in (attrs or {}).items():
            msgs.append((0x0C, 0, self.attribute(k, v)))
        return self.ohdr_v2(msgs)

    def tree(self, node, links=False):
        """node: {name: ndarray | dict (subgroup) | Dataset spec dict with key '__data__'}; '__attrs__' holds attributes."""
        attrs = node.get("__attrs__")
        children = []
        for name, v in node.items():
            if name.startswith("__"):
                continue
            if isinstance(v, dict) and "__data__" in v:
                spec = dict(v)
                children.append((name, self.dataset(spec.pop("__data__"), **{k.strip("_"): x for k, x in spec.items()})))
            elif isinstance(v, dict):
                sub = self.tree(v, links=links)
                children.append((name, sub))
            else:
                children.append((name, self.dataset(v)))
        if links:
            return self.group_links(children, attrs)
        return self.group_symbol_table(children, attrs)[0]

    def finish(self, path, root):
        """Writes the file with ``root`` (a dict, see tree()) as the root group, always a symbol table."""
        attrs = root.get("__attrs__")
        children = []
        for name, v in root.items():
            if name.startswith("__"):
                continue
            if isinstance(v, dict) and "__data__" in v:
                spec = dict(v)
                children.append((name, self.dataset(spec.pop("__data__"), **{k.strip("_"): x for k, x in spec.items()})))
            elif isinstance(v, dict):
                children.append((name, self.tree(v, links=bool(v.get("__links__")))))
            else:
                children.append((name, self.dataset(v)))
        hdr, btree, heap = self.group_symbol_table(children, attrs)
        sb = (b"\x89HDF\r\n\x1a\n" + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", 4, 16, 0)
              + struct.pack("<QQQQ", 0, UNDEF, len(self.buf), UNDEF)
              + struct.pack("<QQII", 0, hdr, 1, 0) + struct.pack("<QQ", btree, heap))
        assert len(sb) == 96
        self.buf[:96] = sb
        with open(path, "wb") as fh:
            fh.write(self.buf)


def write(path, root):
    Writer().finish(path, root)
