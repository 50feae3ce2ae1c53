"""A small, dependency-free reader and writer for the subset of HDF5 that Gale's checkpoint
and dump files use (numpy only; no libhdf5).

Gale writes its fields with the HDF5 1.8 C library at default settings:
- `_FeVariable_SaveToFile` (StgFEM/Discretisation/src/FeVariable.cxx:1986-2140) writes
  dataset "/data" (one row per node: `[global node id?], dof values`) and attributes;
- `SwarmDump` (StgDomain/Swarm/src/SwarmDump.cxx:304) writes one dataset per swarm
  variable ("/Position", "/MaterialIndex", ...);
- the mesh checkpoint writes "/vertices" and element tables.

Those files are superblock version 0 with 8-byte offsets and lengths, groups stored as
symbol tables (a version-1 B-tree of symbol-table nodes plus a local heap) and version-1
object headers.  This module reads exactly that: groups, datasets with contiguous, compact
or chunked (optionally deflate-compressed) storage, fixed-point and IEEE floating-point
element types, and attributes.  It writes the same subset (superblock 0, one root group,
contiguous datasets, array attributes) with the objects, message versions and field values
that the HDF5 1.8 library wrote into the reference's checkpoint files, so that Gale reads them
back (`FeVariable_ReadFromFile`, `SwarmDump`'s reader).

The layouts follow the published HDF5 File Format Specification (version 2.0 of the
document; superblock 0, object header 1, message types 0x01, 0x03, 0x05, 0x08, 0x0B,
0x0C, 0x10, 0x11, 0x12).
"""
from __future__ import annotations

import struct
import zlib
from typing import Dict, List, Optional, Tuple

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


class H5Error(RuntimeError):
    pass


# ---------------------------------------------------------------------------- reading


class _Reader:
    def __init__(self, data: bytes):
        self.d = data
        if data[:8] != SIGNATURE:
            raise H5Error("not an HDF5 file (signature)")
        ver = data[8]
        if ver not in (0, 1):
            raise H5Error(f"superblock version {ver} is outside the supported subset (0, 1)")
        self.so, self.sl = data[13], data[14]
        if self.so != 8 or self.sl != 8:
            raise H5Error("only 8-byte offsets and lengths are supported")
        p = 24 if ver == 0 else 28
        self.base = self.u(p, 8)
        p += 32  # base, free-space, end-of-file, driver block addresses
        # root group symbol table entry
        self.root_header = self.u(p + 8, 8)

    def u(self, p: int, n: int) -> int:
        return int.from_bytes(self.d[p:p + n], "little")

    # ---- object headers
    def messages(self, addr: int) -> List[Tuple[int, int, bytes]]:
        """(type, flags, body) of every message of the version-1 object header at addr."""
        d = self.d
        if d[addr] != 1:
            raise H5Error(f"object header version {d[addr]} at {addr} is outside the subset (1)")
        nmsg = self.u(addr + 2, 2)
        size = self.u(addr + 8, 4)
        blocks = [(addr + 16, size)]  # messages start 8-byte aligned after the 12-byte prefix
        out = []
        while blocks and len(out) < nmsg:
            p, n = blocks.pop(0)
            end = p + n
            while p + 8 <= end and len(out) < nmsg:
                mtype, msize, mflags = self.u(p, 2), self.u(p + 2, 2), d[p + 4]
                body = d[p + 8:p + 8 + msize]
                if mtype == 0x10:  # continuation
                    blocks.append((self.u(p + 8, 8), self.u(p + 16, 8)))
                out.append((mtype, mflags, body))
                p += 8 + msize
        return out

    # ---- groups
    def group_links(self, header: int) -> Dict[str, int]:
        for mtype, _, body in self.messages(header):
            if mtype == 0x11:
                btree = int.from_bytes(body[0:8], "little")
                heap = int.from_bytes(body[8:16], "little")
                return self._symbols(btree, heap)
        raise H5Error("group without a symbol table message (new-style groups are outside the subset)")

    def _heap_data(self, heap: int) -> int:
        if self.d[heap:heap + 4] != b"HEAP":
            raise H5Error("bad local heap signature")
        return self.u(heap + 24, 8)

    def _symbols(self, btree: int, heap: int) -> Dict[str, int]:
        hdata = self._heap_data(heap)
        links: Dict[str, int] = {}

        def node(addr):
            d = self.d
            if d[addr:addr + 4] != b"TREE":
                raise H5Error("bad B-tree signature")
            level, used = d[addr + 5], self.u(addr + 6, 2)
            p = addr + 24 + 8  # header, then key 0
            for _ in range(used):
                child = self.u(p, 8)
                p += 16  # child, next key
                if level > 0:
                    node(child)
                else:
                    snod(child)

        def snod(addr):
            d = self.d
            if d[addr:addr + 4] != b"SNOD":
                raise H5Error("bad symbol table node signature")
            n = self.u(addr + 6, 2)
            p = addr + 8
            for _ in range(n):
                name_off, obj = self.u(p, 8), self.u(p + 8, 8)
                s = hdata + name_off
                e = d.index(b"\x00", s)
                links[d[s:e].decode()] = obj
                p += 40

        node(btree)
        return links

    # ---- datasets
    @staticmethod
    def dtype(body: bytes) -> np.dtype:
        cls, ver = body[0] & 0x0F, body[0] >> 4
        bits0 = body[1]
        size = int.from_bytes(body[4:8], "little")
        order = ">" if bits0 & 1 else "<"
        if cls == 0:
            signed = bool(bits0 & 0x08)
            return np.dtype(f"{order}{'i' if signed else 'u'}{size}")
        if cls == 1:
            return np.dtype(f"{order}f{size}")
        if cls == 3:
            return np.dtype(f"S{size}")
        raise H5Error(f"datatype class {cls} (version {ver}) is outside the subset")

    @staticmethod
    def dataspace(body: bytes) -> Tuple[int, ...]:
        ver, rank, flags = body[0], body[1], body[2]
        p = 8 if ver == 1 else 4
        if ver == 2 and body[3] == 0:  # scalar
            return ()
        return tuple(int.from_bytes(body[p + 8 * i:p + 8 * i + 8], "little") for i in range(rank))

    def read_dataset(self, header: int) -> np.ndarray:
        shape, dt, layout, filters = None, None, None, []
        for mtype, _, body in self.messages(header):
            if mtype == 0x01:
                shape = self.dataspace(body)
            elif mtype == 0x03:
                dt = self.dtype(body)
            elif mtype == 0x08:
                layout = body
            elif mtype == 0x0B:
                filters = self._filters(body)
        if shape is None or dt is None or layout is None:
            raise H5Error("dataset header without dataspace, datatype or layout")
        count = int(np.prod(shape)) if shape else 1
        raw = self._layout_bytes(layout, shape, dt, filters)
        return np.frombuffer(raw, dtype=dt, count=count).reshape(shape).copy()

    @staticmethod
    def _filters(body: bytes) -> List[int]:
        ver, n = body[0], body[1]
        p = 8 if ver == 1 else 2
        ids = []
        for _ in range(n):
            fid = int.from_bytes(body[p:p + 2], "little")
            if ver == 1 or fid >= 256:
                name_len = int.from_bytes(body[p + 2:p + 4], "little")
            else:
                name_len = 0
            nvals = int.from_bytes(body[p + 6:p + 8], "little")
            q = p + 8 + name_len
            if ver == 1:
                q += (8 - name_len % 8) % 8 if name_len else 0
            q += 4 * nvals
            if ver == 1 and nvals % 2:
                q += 4
            ids.append(fid)
            p = q
        for fid in ids:
            if fid != 1:
                raise H5Error(f"filter {fid} is outside the subset (deflate only)")
        return ids

    def _layout_bytes(self, lay: bytes, shape, dt: np.dtype, filters) -> bytes:
        ver = lay[0]
        nbytes = (int(np.prod(shape)) if shape else 1) * dt.itemsize
        if ver == 3:
            cls = lay[1]
            if cls == 0:
                n = int.from_bytes(lay[2:4], "little")
                return lay[4:4 + n]
            if cls == 1:
                addr = int.from_bytes(lay[2:10], "little")
                if addr == UNDEF:
                    return bytes(nbytes)
                return self.d[addr:addr + nbytes]
            if cls == 2:
                rank = lay[2]
                addr = int.from_bytes(lay[3:11], "little")
                cdims = [int.from_bytes(lay[11 + 4 * i:15 + 4 * i], "little") for i in range(rank)]
                return self._chunked(addr, cdims[:-1], shape, dt, filters)
            raise H5Error(f"layout class {cls} is outside the subset")
        if ver in (1, 2):
            rank, cls = lay[1], lay[2]
            p = 8
            if cls == 0:
                p_dims = p
                n = int.from_bytes(lay[p_dims + 4 * rank:p_dims + 4 * rank + 4], "little")
                return lay[p_dims + 4 * rank + 4:p_dims + 4 * rank + 4 + n]
            addr = int.from_bytes(lay[p:p + 8], "little")
            dims = [int.from_bytes(lay[p + 8 + 4 * i:p + 12 + 4 * i], "little") for i in range(rank)]
            if cls == 1:
                return self.d[addr:addr + nbytes] if addr != UNDEF else bytes(nbytes)
            if cls == 2:
                return self._chunked(addr, dims[:-1], shape, dt, filters)
        raise H5Error(f"layout message version {ver} is outside the subset")

    def _chunked(self, btree: int, cdims, shape, dt: np.dtype, filters) -> bytes:
        out = np.zeros(shape, dtype=dt)
        rank = len(shape)

        def node(addr):
            d = self.d
            if d[addr:addr + 4] != b"TREE" or d[addr + 4] != 1:
                raise H5Error("bad chunk B-tree node")
            level, used = d[addr + 5], self.u(addr + 6, 2)
            keysz = 8 + 8 * (rank + 1)
            p = addr + 24
            for _ in range(used):
                csize, mask = self.u(p, 4), self.u(p + 4, 4)
                offs = [self.u(p + 8 + 8 * i, 8) for i in range(rank)]
                child = self.u(p + keysz, 8)
                if level > 0:
                    node(child)
                else:
                    raw = self.d[child:child + csize]
                    if filters and not (mask & 1):
                        raw = zlib.decompress(raw)
                    blk = np.frombuffer(raw, dtype=dt, count=int(np.prod(cdims))).reshape(cdims)
                    sl = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, cdims, shape))
                    out[sl] = blk[tuple(slice(0, s.stop - s.start) for s in sl)]
                p += keysz + 8

        node(btree)
        return out.tobytes()

    def attributes(self, header: int) -> Dict[str, np.ndarray]:
        attrs = {}
        for mtype, _, body in self.messages(header):
            if mtype != 0x0C:
                continue
            ver = body[0]
            name_len = int.from_bytes(body[2:4], "little")
            dt_len = int.from_bytes(body[4:6], "little")
            ds_len = int.from_bytes(body[6:8], "little")
            pad = (lambda n: (n + 7) // 8 * 8) if ver == 1 else (lambda n: n)
            p = 8
            name = body[p:p + name_len].split(b"\x00")[0].decode()
            p += pad(name_len)
            dt = self.dtype(body[p:p + dt_len])
            p += pad(dt_len)
            shape = self.dataspace(body[p:p + ds_len])
            p += pad(ds_len)
            count = int(np.prod(shape)) if shape else 1
            attrs[name] = np.frombuffer(body[p:p + count * dt.itemsize], dtype=dt, count=count).reshape(shape).copy()
        return attrs


class File:
    """Read-only view of an HDF5 file of the supported subset: `f.keys()`, `f[name]` (a numpy
    array for a dataset, a `File`-like group for a group), `f.attrs(name)`."""

    def __init__(self, path_or_bytes, _reader: Optional[_Reader] = None, _header: Optional[int] = None):
        if _reader is None:
            data = path_or_bytes if isinstance(path_or_bytes, (bytes, bytearray)) else open(path_or_bytes, "rb").read()
            _reader = _Reader(bytes(data))
            _header = _reader.root_header
        self._r, self._h = _reader, _header
        self._links = self._r.group_links(self._h)

    def keys(self):
        return list(self._links)

    def __contains__(self, name):
        return self._obj(name) is not None

    def _obj(self, name: str) -> Optional[int]:
        parts = [p for p in name.split("/") if p]
        h, links = self._h, self._links
        for i, part in enumerate(parts):
            if part not in links:
                return None
            h = links[part]
            if i + 1 < len(parts):
                links = self._r.group_links(h)
        return h

    def _is_group(self, h: int) -> bool:
        return any(t == 0x11 for t, _, _ in self._r.messages(h))

    def __getitem__(self, name: str):
        h = self._obj(name)
        if h is None:
            raise KeyError(name)
        if self._is_group(h):
            return File(None, self._r, h)
        return self._r.read_dataset(h)

    def attrs(self, name: str = "/") -> Dict[str, np.ndarray]:
        h = self._h if name in ("", "/") else self._obj(name)
        if h is None:
            raise KeyError(name)
        return self._r.attributes(h)


def read(path) -> Dict[str, np.ndarray]:
    """Every dataset of the root group of `path` as {name: array}."""
    f = File(path)
    return {k: f[k] for k in f.keys() if not isinstance(f[k], File)}


# ---------------------------------------------------------------------------- writing

_GROUP_LEAF_K = 4        # symbol-table node holds 2K entries
_GROUP_INTERNAL_K = 16   # B-tree node holds 2K children
_HEAP_FREE_NULL = 1      # the library's "no free block" marker in a local heap


def _u(v: int, n: int) -> bytes:
    return int(v).to_bytes(n, "little")


def _pad8(b: bytes) -> bytes:
    return b + bytes((8 - len(b) % 8) % 8)


def _dtype_msg(dt: np.dtype) -> bytes:
    """Datatype message (version 1) of a fixed-point or IEEE floating-point numpy type."""
    big = dt.byteorder == ">" or (dt.byteorder == "=" and np.little_endian is False)
    if dt.kind == "f":
        prec = dt.itemsize * 8
        exp_loc, exp_size, man_size, bias = {4: (23, 8, 23, 127), 8: (52, 11, 52, 1023)}[dt.itemsize]
        bits = bytes([0x20 | (1 if big else 0), prec - 1, 0])  # normalisation: implied msb; sign bit
        props = _u(0, 2) + _u(prec, 2) + bytes([exp_loc, exp_size, 0, man_size]) + _u(bias, 4)
        return bytes([0x11]) + bits + _u(dt.itemsize, 4) + props
    if dt.kind in "iu":
        bits = bytes([(1 if big else 0) | (0x08 if dt.kind == "i" else 0), 0, 0])
        return bytes([0x10]) + bits + _u(dt.itemsize, 4) + _u(0, 2) + _u(dt.itemsize * 8, 2)
    raise H5Error(f"numpy type {dt} is outside the writable subset")


def _space_msg(shape) -> bytes:
    """Dataspace message version 1, no maximum dimensions."""
    return bytes([1, len(shape), 0, 0]) + bytes(4) + b"".join(_u(d, 8) for d in shape)


def _message(mtype: int, body: bytes, flags: int = 0) -> bytes:
    body = _pad8(body)
    return _u(mtype, 2) + _u(len(body), 2) + bytes([flags]) + bytes(3) + body


def _header(messages: List[bytes]) -> bytes:
    body = b"".join(messages)
    return bytes([1, 0]) + _u(len(messages), 2) + _u(1, 4) + _u(len(body), 4) + bytes(4) + body


def _attribute(name: str, value: np.ndarray) -> bytes:
    value = np.atleast_1d(np.asarray(value))
    nm = name.encode() + b"\x00"
    dtm, spm = _dtype_msg(value.dtype), _space_msg(value.shape)
    body = (bytes([1, 0]) + _u(len(nm), 2) + _u(len(dtm), 2) + _u(len(spm), 2)
            + _pad8(nm) + _pad8(dtm) + _pad8(spm) + value.tobytes())
    return _message(0x0C, body)


def write(path: str, datasets: Dict[str, np.ndarray], attrs: Optional[Dict[str, np.ndarray]] = None) -> None:
    """Write an HDF5 file (superblock 0) whose root group holds `datasets` (contiguous,
    numpy dtype and shape kept) and `attrs` as root-group attributes.  At most 8 datasets
    (one symbol-table node), which covers every checkpoint file of the reference."""
    names = sorted(datasets, key=lambda k: k.encode())
    if len(names) > 2 * _GROUP_LEAF_K:
        raise H5Error("more datasets than one symbol-table node holds")
    arrays = {k: np.ascontiguousarray(datasets[k]) for k in names}
    # local heap data: the empty name at offset 0, then each name, 8-byte padded
    heap_data = bytearray(8)
    name_off = {}
    for k in names:
        name_off[k] = len(heap_data)
        heap_data += _pad8(k.encode() + b"\x00")
    # fixed-size pieces
    SB = 96
    root_msgs_len = len(_message(0x11, bytes(16))) + sum(
        len(_attribute(a, v)) for a, v in (attrs or {}).items())
    root_hdr_len = 16 + root_msgs_len
    heap_hdr_len = 32
    btree_len = 24 + 8 * (2 * _GROUP_INTERNAL_K + 1) + 8 * (2 * _GROUP_INTERNAL_K)
    snod_len = 8 + 40 * 2 * _GROUP_LEAF_K

    def ds_header(arr, addr):
        return _header([
            _message(0x05, bytes([2, 2, 2, 1]) + _u(0, 4), flags=1),      # fill value: none
            _message(0x03, _dtype_msg(arr.dtype), flags=1),
            _message(0x01, _space_msg(arr.shape)),
            _message(0x08, bytes([3, 1]) + _u(addr, 8) + _u(arr.nbytes, 8)),  # contiguous
        ])

    a_root = SB
    a_heap = a_root + root_hdr_len
    a_heap_data = a_heap + heap_hdr_len
    a_btree = a_heap_data + len(heap_data)
    a_snod = a_btree + btree_len
    a = a_snod + snod_len
    a_hdr = {}
    for k in names:
        a_hdr[k] = a
        a += len(ds_header(arrays[k], 0))
    a_raw = {}
    for k in names:
        a = (a + 7) // 8 * 8
        a_raw[k] = a
        a += arrays[k].nbytes
    eof = a

    out = bytearray()
    # superblock 0 + root group symbol-table entry (cache type 1: B-tree and heap addresses)
    out += SIGNATURE + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + _u(_GROUP_LEAF_K, 2) + _u(_GROUP_INTERNAL_K, 2)
    out += _u(0, 4) + _u(0, 8) + _u(UNDEF, 8) + _u(eof, 8) + _u(UNDEF, 8)
    out += _u(0, 8) + _u(a_root, 8) + _u(1, 4) + _u(0, 4) + _u(a_btree, 8) + _u(a_heap, 8)
    assert len(out) == SB
    msgs = [_message(0x11, _u(a_btree, 8) + _u(a_heap, 8))]
    msgs += [_attribute(k, v) for k, v in (attrs or {}).items()]
    out += _header(msgs)
    assert len(out) == a_heap
    out += b"HEAP" + bytes([0, 0, 0, 0]) + _u(len(heap_data), 8) + _u(_HEAP_FREE_NULL, 8) + _u(a_heap_data, 8)
    out += heap_data
    assert len(out) == a_btree
    bt = bytearray(b"TREE" + bytes([0, 0]) + _u(1 if names else 0, 2) + _u(UNDEF, 8) + _u(UNDEF, 8))
    bt += _u(0, 8) + _u(a_snod, 8) + _u(name_off[names[-1]] if names else 0, 8)
    bt += bytes(btree_len - len(bt))
    out += bt
    sn = bytearray(b"SNOD" + bytes([1, 0]) + _u(len(names), 2))
    for k in names:
        sn += _u(name_off[k], 8) + _u(a_hdr[k], 8) + _u(0, 4) + _u(0, 4) + bytes(16)
    sn += bytes(snod_len - len(sn))
    out += sn
    for k in names:
        assert len(out) == a_hdr[k]
        out += ds_header(arrays[k], a_raw[k])
    for k in names:
        out += bytes(a_raw[k] - len(out))
        out += arrays[k].tobytes()
    assert len(out) == eof
    with open(path, "wb") as f:
        f.write(bytes(out))
