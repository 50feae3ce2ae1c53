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
contiguous datasets, scalar or array attributes), which the HDF5 library itself reads.

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
