"""A small HDF5 reader and writer for SeisCL's job files.

SeisCL exchanges its inputs and outputs as HDF5 files (``<base>_csts.mat``,
``_model.mat``, ``_din.mat``, ``_res.mat``, ``_dout.mat``, ``_gout.mat``,
``_rms.mat``, ``_movie.mat``): flat files whose root group holds numeric
datasets (src/read_hdf5.c:461-787, src/writehdf5.c:190-316, written and read
with h5py by SeisCL/SeisCL.py:414-770).  h5py and libhdf5 are not available
to this package, so this module implements the part of the HDF5 file format
(the HDF Group's "HDF5 File Format Specification", version 3.0) those files
use:

reading
  * superblock versions 0 and 1 (symbol-table root group) and 2 and 3
    (object-header root group), with or without a user block (the
    reference's MATLAB 7.3 style outputs carry a 512-byte one);
  * object headers version 1 and 2, with continuation blocks;
  * groups stored as a symbol table (v1 B-tree of symbol nodes + local
    heap) or as compact link messages; nested groups are entered;
  * datasets with a simple or scalar dataspace; fixed-point (8 to 64 bit,
    either byte order, signed or not), IEEE floating point (32/64 bit) and
    fixed-length string types; compact, contiguous and chunked layouts
    (v1 B-tree chunk index) with the deflate and shuffle filters.
  Dense link storage (fractal heaps), virtual and external layouts, and
  compound/variable-length types raise ``H5Error``.

writing
  superblock version 0, one root group stored as a symbol table, and one
  contiguous dataset per array (little-endian integers and IEEE floats).

Arrays are read and written in the file's own (C, last index fastest)
order; callers transpose as SeisCL.py does.
"""
from __future__ import annotations

import struct
import zlib
from typing import Dict, List, Tuple

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


class H5Error(ValueError):
    """A file this subset cannot read (or not an HDF5 file)."""


# ------------------------------------------------------------------ reading
class _Reader:
    def __init__(self, buf: bytes):
        self.b = buf
        self.base = None
        for sb in (0, 512, 1024, 2048, 4096, 8192, 16384, 32768, 65536):
            if self.b[sb:sb + 8] == SIGNATURE:
                self.sb = sb
                break
        else:
            raise H5Error("no HDF5 signature")
        self.out: Dict[str, np.ndarray] = {}
        self._seen = set()

    # primitive unpacking
    def u(self, off: int, n: int) -> int:
        return int.from_bytes(self.b[off:off + n], "little")

    def addr(self, a: int) -> int:
        """Absolute file offset of a file address."""
        return self.base + a

    def parse_superblock(self):
        p = self.sb + 8
        ver = self.b[p]
        if ver in (0, 1):
            self.so, self.sl = self.b[p + 5], self.b[p + 6]
            self.leaf_k = self.u(p + 8, 2)
            q = p + 16 + (4 if ver == 1 else 0)
            base = self.u(q, self.so)
            # every other address is relative to the base address (the
            # superblock's own offset when a user block precedes it)
            self.base = base if base != UNDEF else self.sb
            q += 4 * self.so
            ent = self.sym_entry(q)
            return ("symtab", ent)
        if ver in (2, 3):
            self.so, self.sl = self.b[p + 1], self.b[p + 2]
            q = p + 4
            base = self.u(q, self.so)
            self.base = self.sb if base == UNDEF else base
            root = self.u(q + 3 * self.so, self.so)
            return ("ohdr", root)
        raise H5Error("superblock version %d not supported" % ver)

    def sym_entry(self, q: int):
        so = self.so
        name_off = self.u(q, so)
        ohdr = self.u(q + so, so)
        cache = self.u(q + 2 * so, 4)
        scratch = (self.u(q + 2 * so + 8, so), self.u(q + 3 * so + 8, so)) if cache == 1 else None
        return name_off, ohdr, cache, scratch

    # object headers ----------------------------------------------------
    def messages(self, a: int) -> List[Tuple[int, int, int]]:
        """(type, absolute offset of data, size) of every message."""
        p = self.addr(a)
        out: List[Tuple[int, int, int]] = []
        if self.b[p:p + 4] == b"OHDR":
            ver, flags = self.b[p + 4], self.b[p + 5]
            q = p + 6
            if flags & 0x20:
                q += 16
            if flags & 0x10:
                q += 4
            nsz = 1 << (flags & 3)
            size = self.u(q, nsz)
            q += nsz
            self._msgs_v2(q, q + size, flags, out)
            return out
        if self.b[p] != 1:
            raise H5Error("object header version %d not supported" % self.b[p])
        nmsg = self.u(p + 2, 2)
        size = self.u(p + 8, 4)
        blocks = [(p + 16, p + 16 + size)]
        while blocks and len(out) < nmsg:
            lo, hi = blocks.pop(0)
            q = lo
            while q + 8 <= hi and len(out) < nmsg:
                mt, ms = self.u(q, 2), self.u(q + 2, 2)
                if mt == 0x10:
                    blocks.append((self.addr(self.u(q + 8, self.so)),
                                   self.addr(self.u(q + 8, self.so)) + self.u(q + 8 + self.so, self.sl)))
                out.append((mt, q + 8, ms))
                q += 8 + ms
        return out

    def _msgs_v2(self, lo, hi, flags, out):
        q = lo
        while hi - q >= 4:   # what is left below a message header is a gap
            mt, ms, mf = self.b[q], self.u(q + 1, 2), self.b[q + 3]
            q += 4
            if flags & 0x04:
                q += 2
            if mt == 0x10:
                a = self.addr(self.u(q, self.so))
                ln = self.u(q + self.so, self.sl)
                if self.b[a:a + 4] != b"OCHK":
                    raise H5Error("bad continuation block")
                self._msgs_v2(a + 4, a + ln - 4, flags, out)
            elif mt != 0:
                out.append((mt, q, ms))
            q += ms

    # groups ------------------------------------------------------------
    def walk_group(self, ohdr: int, path: str, scratch=None):
        if ohdr in self._seen:
            return
        self._seen.add(ohdr)
        msgs = self.messages(ohdr)
        links: List[Tuple[str, int]] = []
        symtab = [m for m in msgs if m[0] == 0x11]
        if symtab:
            q = symtab[0][1]
            links += self.symtab_links(self.u(q, self.so), self.u(q + self.so, self.so))
        elif scratch:
            links += self.symtab_links(*scratch)
        links += [self.link_msg(q) for mt, q, _ in msgs if mt == 0x06]
        linfo = [m for m in msgs if m[0] == 0x02]
        if linfo and not links:
            q = linfo[0][1]
            fheap = self.u(q + 2 + (8 if self.b[q + 1] & 1 else 0), self.so)
            if fheap != UNDEF:
                raise H5Error("dense link storage is not supported")
        for name, a in links:
            sub = self.messages(a)
            st = {x[0] for x in sub}
            if 0x08 in st:
                self.out[path + name] = self.dataset(sub)
            elif st & {0x11, 0x02, 0x06}:
                self.walk_group(a, path + name + "/")

    def symtab_links(self, btree: int, heap: int) -> List[Tuple[str, int]]:
        hp = self.addr(heap)
        if self.b[hp:hp + 4] != b"HEAP":
            raise H5Error("bad local heap")
        data = self.addr(self.u(hp + 8 + 2 * self.sl, self.so))
        out: List[Tuple[str, int]] = []

        def name_at(off):
            e = self.b.index(b"\x00", data + off)
            return self.b[data + off:e].decode("utf-8", "replace")

        def node(a):
            p = self.addr(a)
            if self.b[p:p + 4] == b"SNOD":
                n = self.u(p + 6, 2)
                q = p + 8
                for _ in range(n):
                    no, oh, _, _ = self.sym_entry(q)
                    out.append((name_at(no), oh))
                    q += 2 * self.so + 24
                return
            if self.b[p:p + 4] != b"TREE":
                raise H5Error("bad group B-tree node")
            used = self.u(p + 6, 2)
            q = p + 8 + 2 * self.so + self.sl   # past the header and key 0
            for _ in range(used):
                node(self.u(q, self.so))
                q += self.so + self.sl

        node(btree)
        return out

    def link_msg(self, q: int) -> Tuple[str, int]:
        flags = self.b[q + 1]
        p = q + 2
        ltype = 0
        if flags & 0x08:
            ltype = self.b[p]
            p += 1
        if flags & 0x04:
            p += 8
        if flags & 0x10:
            p += 1
        nl = 1 << (flags & 3)
        ln = self.u(p, nl)
        p += nl
        name = self.b[p:p + ln].decode("utf-8", "replace")
        p += ln
        if ltype != 0:
            raise H5Error("soft or external link %r is not supported" % name)
        return name, self.u(p, self.so)

    # datasets ----------------------------------------------------------
    def dataspace(self, q: int):
        ver, rank, flags = self.b[q], self.b[q + 1], self.b[q + 2]
        if ver == 1:
            p = q + 8
        elif ver == 2:
            if self.b[q + 3] == 2:
                return None
            p = q + 4
        else:
            raise H5Error("dataspace version %d" % ver)
        return tuple(self.u(p + i * self.sl, self.sl) for i in range(rank))

    def datatype(self, q: int):
        cv = self.b[q]
        cls = cv & 0x0F
        bf = self.b[q + 1:q + 4]
        size = self.u(q + 4, 4)
        order = ">" if bf[0] & 1 else "<"
        if cls == 0:
            signed = bool(bf[0] & 0x08)
            if size not in (1, 2, 4, 8):
                raise H5Error("integer size %d" % size)
            return np.dtype("%s%s%d" % (order, "i" if signed else "u", size))
        if cls == 1:
            if size not in (2, 4, 8):
                raise H5Error("float size %d" % size)
            return np.dtype("%sf%d" % (order, size))
        if cls == 3:
            return np.dtype("S%d" % size)
        raise H5Error("datatype class %d is not supported" % cls)

    def dataset(self, msgs):
        shape = dtype = None
        layout = None
        filters: List[int] = []
        for mt, q, ms in msgs:
            if mt == 0x01:
                shape = self.dataspace(q)
            elif mt == 0x03:
                dtype = self.datatype(q)
            elif mt == 0x08:
                layout = q
            elif mt == 0x0B:
                filters = self.filter_ids(q)
        if dtype is None or layout is None:
            raise H5Error("dataset without a datatype or layout")
        if shape is None:
            return np.zeros(0, dtype)
        n = int(np.prod(shape)) if shape else 1
        nbytes = n * dtype.itemsize
        ver = self.b[layout]
        if ver in (1, 2):
            rank, cls = self.b[layout + 1], self.b[layout + 2]
            p = layout + 8
            if cls == 0:
                raw = self.b[p + 4 * rank + 4:p + 4 * rank + 4 + nbytes]
            elif cls == 1:
                a = self.u(p, self.so)
                raw = self.b[self.addr(a):self.addr(a) + nbytes]
            else:
                a = self.u(p, self.so)
                cdims = [self.u(p + self.so + 4 * i, 4) for i in range(rank)]
                raw = self.chunked(a, cdims, shape, dtype, filters)
        elif ver in (3, 4):
            cls = self.b[layout + 1]
            p = layout + 2
            if cls == 0:
                sz = self.u(p, 2)
                raw = self.b[p + 2:p + 2 + sz]
            elif cls == 1:
                a = self.u(p, self.so)
                raw = b"" if a == UNDEF else self.b[self.addr(a):self.addr(a) + nbytes]
            elif cls == 2 and ver == 3:
                rank = self.b[p]
                a = self.u(p + 1, self.so)
                cdims = [self.u(p + 1 + self.so + 4 * i, 4) for i in range(rank)]
                raw = self.chunked(a, cdims, shape, dtype, filters)
            else:
                raise H5Error("layout class %d (version %d) is not supported" % (cls, ver))
        else:
            raise H5Error("layout version %d" % ver)
        if len(raw) < nbytes:   # never written: the library's default fill
            raw = bytes(raw) + b"\x00" * (nbytes - len(raw))
        arr = np.frombuffer(bytes(raw[:nbytes]), dtype=dtype).reshape(shape if shape else ())
        return arr.astype(dtype.newbyteorder("=")) if dtype.kind in "iuf" else arr.copy()

    def filter_ids(self, q: int) -> List[int]:
        ver, nf = self.b[q], self.b[q + 1]
        p = q + (8 if ver == 1 else 2)
        ids = []
        for _ in range(nf):
            fid = self.u(p, 2)
            if ver == 1 or fid >= 256:
                nl = self.u(p + 2, 2)
                ncv = self.u(p + 6, 2)
                p += 8 + ((nl + 7) // 8 * 8 if ver == 1 else nl)
            else:
                ncv = self.u(p + 4, 2)
                p += 6
            p += 4 * ncv
            if ver == 1 and ncv % 2:
                p += 4
            ids.append(fid)
        return ids

    def chunked(self, btree: int, cdims, shape, dtype, filters) -> bytes:
        rank = len(shape)
        elem = cdims[-1] if len(cdims) == rank + 1 else dtype.itemsize
        cshape = cdims[:rank]
        out = np.zeros(shape, dtype=np.dtype("V%d" % dtype.itemsize)) if shape else None
        if out is None:
            raise H5Error("chunked scalar")

        def walk(a):
            p = self.addr(a)
            if self.b[p:p + 4] != b"TREE" or self.b[p + 4] != 1:
                raise H5Error("bad chunk B-tree node")
            level, used = self.b[p + 5], self.u(p + 6, 2)
            q = p + 8 + 2 * self.so
            ksz = 8 + 8 * (rank + 1)
            for _ in range(used):
                csize, fmask = self.u(q, 4), self.u(q + 4, 4)
                offs = [self.u(q + 8 + 8 * i, 8) for i in range(rank)]
                child = self.u(q + ksz, self.so)
                if level > 0:
                    walk(child)
                else:
                    data = self.b[self.addr(child):self.addr(child) + csize]
                    for fid in reversed(filters):
                        if fmask & (1 << filters.index(fid)):
                            continue
                        if fid == 1:
                            data = zlib.decompress(data)
                        elif fid == 2:
                            a2 = np.frombuffer(data, np.uint8).reshape(elem, -1)
                            data = a2.T.tobytes()
                        else:
                            raise H5Error("filter %d is not supported" % fid)
                    blk = np.frombuffer(bytes(data), dtype=out.dtype)[:int(np.prod(cshape))].reshape(cshape)
                    sl = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, cshape, shape))
                    out[sl] = blk[tuple(slice(0, x.stop - x.start) for x in sl)]
                q += ksz + self.so

        if btree != UNDEF:
            walk(btree)
        return out.tobytes()


def read(path: str) -> Dict[str, np.ndarray]:
    """Every dataset of the file, keyed by its path below the root group
    ("N", "src_pos", "grp/x", ...).  Scalars come back as 0-d arrays."""
    with open(path, "rb") as fh:
        buf = fh.read()
    r = _Reader(buf)
    kind, root = r.parse_superblock()
    if kind == "symtab":
        _, ohdr, _, scratch = root
        r.walk_group(ohdr, "", scratch)
    else:
        r.walk_group(root, "")
    return r.out


# ------------------------------------------------------------------ writing
def _pad8(b: bytes) -> bytes:
    return b + b"\x00" * (-len(b) % 8)


def _msg(mtype: int, data: bytes, flags: int = 0) -> bytes:
    data = _pad8(data)
    return struct.pack("<HHB3x", mtype, len(data), flags) + data


def _ohdr_v1(msgs: List[bytes]) -> bytes:
    body = b"".join(msgs)
    return struct.pack("<BBHII4x", 1, 0, len(msgs), 1, len(body)) + body


def _dtype_msg(dt: np.dtype) -> bytes:
    if dt.kind == "f":
        if dt.itemsize == 4:
            props = struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
            return struct.pack("<B3BI", 0x11, 0x20, 31, 0, 4) + props
        if dt.itemsize == 8:
            props = struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
            return struct.pack("<B3BI", 0x11, 0x20, 63, 0, 8) + props
    if dt.kind in "iu" and dt.itemsize in (1, 2, 4, 8):
        bits = 0x08 if dt.kind == "i" else 0x00
        return struct.pack("<B3BI", 0x10, bits, 0, 0, dt.itemsize) + struct.pack("<HH", 0, 8 * dt.itemsize)
    raise H5Error("cannot write dtype %s" % dt)


def _space_msg(shape) -> bytes:
    return struct.pack("<BBBB4x", 1, len(shape), 0, 0) + b"".join(struct.pack("<Q", int(d)) for d in shape)


def _as_writable(v) -> np.ndarray:
    a = np.asarray(v)
    if a.dtype == np.bool_:
        a = a.astype(np.int64)
    if a.dtype.kind not in "iuf":
        raise H5Error("cannot write %r" % (a.dtype,))
    return np.array(a, dtype=a.dtype.newbyteorder("<"), order="C")   # keeps 0-d arrays 0-d


def write(path: str, data: Dict[str, object]) -> None:
    """Write a flat file: one contiguous dataset per entry of ``data`` in the
    root group (numbers become scalar datasets, arrays keep their shape and
    C order; int64/float64/float32/int32 and the other numeric types)."""
    items = sorted(((str(k), _as_writable(v)) for k, v in data.items()), key=lambda kv: kv[0].encode())
    for k, _ in items:
        if not k or "/" in k or "\x00" in k:
            raise H5Error("invalid dataset name %r" % k)
    leaf_k, int_k = 4, 16
    per_node = 2 * leaf_k
    nnodes = max(1, -(-len(items) // per_node))
    if nnodes > 2 * int_k:
        raise H5Error("at most %d datasets per file" % (2 * int_k * per_node))

    # local heap data: "" at offset 0, then every name (8-byte padded)
    heap = bytearray(b"\x00" * 8)
    name_off = {}
    for k, _ in items:
        name_off[k] = len(heap)
        heap += _pad8(k.encode() + b"\x00")
    heap_data_size = max(len(heap), 88)
    heap += b"\x00" * (heap_data_size - len(heap))

    out = bytearray()
    SB = 96
    out += b"\x00" * SB
    # root object header (symbol table message)
    root_at = len(out)
    root_len = len(_ohdr_v1([_msg(0x11, b"\x00" * 16)]))
    out += b"\x00" * root_len
    # local heap header + data
    heap_at = len(out)
    heap_hdr = 32
    out += b"\x00" * heap_hdr
    heap_data_at = len(out)
    out += heap
    # B-tree node (full capacity: 2K children)
    btree_at = len(out)
    btree_len = 24 + (2 * int_k + 1) * 8 + 2 * int_k * 8
    out += b"\x00" * btree_len
    # symbol table nodes
    snod_len = 8 + per_node * 40
    snod_at = []
    for _ in range(nnodes):
        snod_at.append(len(out))
        out += b"\x00" * snod_len
    # datasets: object header, then raw data (8-byte aligned)
    ds_at = {}
    for k, a in items:
        raw_len = a.nbytes
        hdr_probe = _ohdr_v1([_msg(0x01, _space_msg(a.shape)), _msg(0x03, _dtype_msg(a.dtype)),
                              _msg(0x05, struct.pack("<BBBB", 2, 2, 2, 0)),
                              _msg(0x08, struct.pack("<BBQQ", 3, 1, 0, raw_len))])
        oh_at = len(out)
        data_at = oh_at + len(hdr_probe)
        data_at += -data_at % 8
        hdr = _ohdr_v1([_msg(0x01, _space_msg(a.shape)), _msg(0x03, _dtype_msg(a.dtype)),
                        _msg(0x05, struct.pack("<BBBB", 2, 2, 2, 0)),
                        _msg(0x08, struct.pack("<BBQQ", 3, 1, data_at if raw_len else UNDEF, raw_len))])
        out += hdr
        out += b"\x00" * (data_at - len(out))
        out += a.tobytes()
        out += b"\x00" * (-len(out) % 8)
        ds_at[k] = oh_at

    def put(at, b):
        out[at:at + len(b)] = b

    # superblock v0
    sb = SIGNATURE + struct.pack("<BBBBBBBBHHI", 0, 0, 0, 0, 0, 8, 8, 0, leaf_k, int_k, 0)
    sb += struct.pack("<QQQQ", 0, UNDEF, len(out), UNDEF)
    sb += struct.pack("<QQII", 0, root_at, 1, 0) + struct.pack("<QQ", btree_at, heap_at)
    put(0, sb)
    put(root_at, _ohdr_v1([_msg(0x11, struct.pack("<QQ", btree_at, heap_at))]))
    put(heap_at, b"HEAP" + struct.pack("<B3xQQQ", 0, heap_data_size, UNDEF, heap_data_at))
    # symbol table nodes, names in byte order
    groups = [items[i * per_node:(i + 1) * per_node] for i in range(nnodes)]
    for g, at in zip(groups, snod_at):
        b = b"SNOD" + struct.pack("<BBH", 1, 0, len(g))
        for k, _ in g:
            b += struct.pack("<QQII", name_off[k], ds_at[k], 0, 0) + b"\x00" * 16
        put(at, b)
    # B-tree: key i bounds child i from below; key i+1 = last name in child i
    b = b"TREE" + struct.pack("<BBHQQ", 0, 0, nnodes, UNDEF, UNDEF)
    b += struct.pack("<Q", 0)
    for g, at in zip(groups, snod_at):
        last = g[-1][0] if g else ""
        b += struct.pack("<QQ", at, name_off.get(last, 0))
    put(btree_at, b)
    with open(path, "wb") as fh:
        fh.write(bytes(out))
