"""Minimal HDF5 reader for box catalogs (HDF5 File Format Specification 3.0).

The reference reads box catalogs from HDF5 with h5py (src/cosmonpc/
catalog_processor.py:16-88): every requested name that is a top-level dataset
of the file, all rows, files of a list concatenated in order.  h5py is not
available here, so this module parses the file itself.  Supported -- what
HDF5 writes for one-dimensional numeric datasets in the root group:

* superblock versions 0-3; object headers versions 1 and 2 (with
  continuation blocks); groups as symbol tables (v1 B-tree + local heap) or
  as compact link messages;
* datasets of rank 1 with fixed-point (signed/unsigned, 1-8 bytes) or IEEE
  floating-point (4 or 8 bytes) elements of either byte order;
* data layouts compact, contiguous, and chunked with a version-1 B-tree chunk
  index (layout message version 3) through the deflate, shuffle and
  Fletcher-32 filters.

Anything else (dense link storage, layout version 4 chunk indices, other
filters, compound or variable-length types) raises NotImplementedError.

``DatasetInfo`` describes where a dataset's raw elements are, so that a
contiguous dataset can be copied to the device unchanged and decoded there
(``catalog_processor.read_box_hdf5``).
"""
from __future__ import annotations

import mmap
import zlib
from dataclasses import dataclass

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


@dataclass
class DatasetInfo:
    name: str
    n: int                  # elements
    dtype: np.dtype         # element type with its byte order
    layout: str             # "contiguous", "compact" or "chunked"
    offset: int = -1        # file offset of the elements (contiguous)
    data: bytes = b""       # the elements (compact)
    chunks: list = None     # [(file offset, stored size, filter mask, first element)] (chunked)
    chunk_elems: int = 0
    filters: list = None    # [(filter id, client values)]


class _File:
    def __init__(self, path):
        self.path = path
        with open(path, "rb") as f:
            size = f.seek(0, 2)
            # mapped read-only: a contiguous dataset is then copied out without
            # reading the whole file
            self.buf = mmap.mmap(f.fileno(), 0, access=mmap.ACCESS_READ) if size else b""
        self.base = 0
        self._superblock()

    # ------------------------------------------------------------ primitives
    def u(self, off, n):
        return int.from_bytes(self.buf[off:off + n], "little")

    def addr(self, off):
        return self.u(off, self.so)

    def length(self, off):
        return self.u(off, self.sl)

    def _superblock(self):
        pos = 0
        while True:  # the superblock sits at 0, 512, 1024, ... (user block)
            if self.buf[pos:pos + 8] == SIGNATURE:
                break
            pos = 512 if pos == 0 else pos * 2
            if pos + 8 > len(self.buf):
                raise ValueError(f"{self.path}: not an HDF5 file")
        v = self.buf[pos + 8]
        if v in (0, 1):
            self.so, self.sl = self.buf[pos + 13], self.buf[pos + 14]
            p = pos + 24 + (4 if v == 1 else 0)
            self.base = self.addr(p)
            p += 4 * self.so  # base, free space, end of file, driver info
            # root group symbol table entry: name offset, object header address, cache type, scratch
            self.root_header = self.addr(p + self.so)
            cache = self.u(p + 2 * self.so, 4)
            self.root_stab = None
            if cache == 1:
                s = p + 2 * self.so + 8
                self.root_stab = (self.addr(s), self.addr(s + self.so))
        elif v in (2, 3):
            self.so, self.sl = self.buf[pos + 9], self.buf[pos + 10]
            p = pos + 12
            self.base = self.addr(p)
            self.root_header = self.addr(p + 3 * self.so)
            self.root_stab = None
        else:
            raise NotImplementedError(f"{self.path}: superblock version {v}")

    # ------------------------------------------------------- object headers
    def messages(self, addr):
        """[(type, body offset, size)] of the object header at ``addr``."""
        a = self.base + addr
        out = []
        if self.buf[a:a + 4] == b"OHDR":
            ver, flags = self.buf[a + 4], self.buf[a + 5]
            p = a + 6
            if flags & 0x20:
                p += 16
            if flags & 0x10:
                p += 4
            sz = 1 << (flags & 3)
            chunk = self.u(p, sz)
            p += sz
            self._v2_messages(p, p + chunk, flags, out)
        else:
            if self.buf[a] != 1:
                raise NotImplementedError(f"{self.path}: object header version {self.buf[a]}")
            nmsg = self.u(a + 2, 2)
            size = self.u(a + 8, 4)
            blocks = [(a + 16, size)]
            while blocks and len(out) < nmsg:
                p, left = blocks.pop(0)
                end = p + left
                while p + 8 <= end and len(out) < nmsg:
                    t, sz = self.u(p, 2), self.u(p + 2, 2)
                    body = p + 8
                    if t == 0x10:
                        blocks.append((self.base + self.addr(body), self.length(body + self.so)))
                    out.append((t, body, sz))
                    p = body + sz
        return out

    def _v2_messages(self, p, end, flags, out):
        # messages fill [p, end); a tail shorter than a message header is a gap
        while p + 4 <= end:
            t, sz, mflags = self.buf[p], self.u(p + 1, 2), self.buf[p + 3]
            body = p + 4 + (2 if flags & 0x04 else 0)
            if t == 0x10:
                c = self.base + self.addr(body)
                clen = self.length(body + self.so)
                if self.buf[c:c + 4] != b"OCHK":
                    raise ValueError(f"{self.path}: bad continuation block")
                self._v2_messages(c + 4, c + clen - 4, flags, out)  # signature .. checksum
            elif t != 0:
                out.append((t, body, sz))
            p = body + sz

    # ------------------------------------------------------------------ groups
    def root_links(self):
        """{name: object header address} of the root group."""
        links = {}
        stab = self.root_stab
        for t, body, _ in self.messages(self.root_header):
            if t == 0x11:
                stab = (self.addr(body), self.addr(body + self.so))
            elif t == 0x06:
                name, target = self._link(body)
                if target is not None:
                    links[name] = target
            elif t == 0x02:
                heap = self.addr(body + 2 + (8 if self.buf[body + 1] & 1 else 0))
                if heap != UNDEF:
                    raise NotImplementedError(f"{self.path}: dense link storage")
        if stab is not None:
            btree, heap = stab
            names = self._local_heap(heap)
            self._group_btree(btree, names, links)
        return links

    def _link(self, p):
        flags = self.buf[p + 1]
        q = p + 2
        ltype = 0
        if flags & 0x08:
            ltype = self.buf[q]
            q += 1
        if flags & 0x04:
            q += 8
        if flags & 0x10:
            q += 1
        nlen_size = 1 << (flags & 3)
        nlen = self.u(q, nlen_size)
        q += nlen_size
        name = self.buf[q:q + nlen].decode("utf-8")
        q += nlen
        return name, (self.addr(q) if ltype == 0 else None)

    def _local_heap(self, addr):
        a = self.base + addr
        if self.buf[a:a + 4] != b"HEAP":
            raise ValueError(f"{self.path}: bad local heap")
        data = self.base + self.addr(a + 8 + 2 * self.sl)
        return data

    def _cstr(self, off):
        end = self.buf.find(b"\0", off)
        return self.buf[off:end].decode("utf-8")

    def _group_btree(self, addr, heap_data, links):
        a = self.base + addr
        if self.buf[a:a + 4] != b"TREE":
            raise ValueError(f"{self.path}: bad group B-tree")
        level, used = self.buf[a + 5], self.u(a + 6, 2)
        p = a + 8 + 2 * self.so + self.sl  # past siblings and key 0
        for _ in range(used):
            child = self.addr(p)
            if level > 0:
                self._group_btree(child, heap_data, links)
            else:
                s = self.base + child
                if self.buf[s:s + 4] != b"SNOD":
                    raise ValueError(f"{self.path}: bad symbol table node")
                for e in range(self.u(s + 6, 2)):
                    ent = s + 8 + e * (2 * self.so + 24)
                    links[self._cstr(heap_data + self.length(ent))] = self.addr(ent + self.so)
            p += self.so + self.sl

    # ---------------------------------------------------------------- datasets
    def dataset(self, name, addr):
        shape = dtype = layout = None
        filters = []
        for t, body, sz in self.messages(addr):
            if t == 0x01:
                shape = self._dataspace(body)
            elif t == 0x03:
                dtype = self._datatype(body)
            elif t == 0x08:
                layout = (body, sz)
            elif t == 0x0B:
                filters = self._filters(body)
        if shape is None or dtype is None or layout is None:
            raise NotImplementedError(f"{self.path}: {name} is not a simple dataset")
        if len(shape) != 1:
            raise NotImplementedError(f"{self.path}: {name} has rank {len(shape)} (only 1-D columns)")
        n = int(shape[0])
        body, _ = layout
        ver = self.buf[body]
        if ver != 3:
            raise NotImplementedError(f"{self.path}: {name}: data layout message version {ver}")
        cls = self.buf[body + 1]
        if cls == 0:
            size = self.u(body + 2, 2)
            return DatasetInfo(name, n, dtype, "compact", data=self.buf[body + 4:body + 4 + size])
        if cls == 1:
            off = self.addr(body + 2)
            return DatasetInfo(name, n, dtype, "contiguous", offset=(self.base + off) if off != UNDEF else -1)
        if cls == 2:
            ndim = self.buf[body + 2]
            btree = self.addr(body + 3)
            dims = [self.u(body + 3 + self.so + 4 * i, 4) for i in range(ndim)]
            chunks = []
            if btree != UNDEF:
                self._chunk_btree(btree, ndim, chunks)
            return DatasetInfo(name, n, dtype, "chunked", chunks=chunks, chunk_elems=dims[0], filters=filters)
        raise NotImplementedError(f"{self.path}: {name}: layout class {cls}")

    def _dataspace(self, p):
        ver, rank, flags = self.buf[p], self.buf[p + 1], self.buf[p + 2]
        q = p + (8 if ver == 1 else 4)
        return [self.length(q + i * self.sl) for i in range(rank)]

    def _datatype(self, p):
        cls = self.buf[p] & 0x0F
        bits = self.u(p + 1, 3)
        size = self.u(p + 4, 4)
        order = ">" if bits & 1 else "<"
        if cls == 0:
            kind = "i" if bits & 0x08 else "u"
            if size not in (1, 2, 4, 8):
                raise NotImplementedError(f"{self.path}: {size}-byte integers")
            return np.dtype(f"{order}{kind}{size}")
        if cls == 1:
            if size not in (4, 8):
                raise NotImplementedError(f"{self.path}: {size}-byte floats")
            return np.dtype(f"{order}f{size}")
        raise NotImplementedError(f"{self.path}: datatype class {cls}")

    def _filters(self, p):
        ver, nf = self.buf[p], self.buf[p + 1]
        q = p + (8 if ver == 1 else 2)
        out = []
        for _ in range(nf):
            fid = self.u(q, 2)
            if ver == 1 or fid >= 256:
                nlen = self.u(q + 2, 2)
                q += 4
            else:
                nlen = 0
                q += 2
            nvals = self.u(q + 2, 2)
            q += 4
            if ver == 1:
                q += (nlen + 7) // 8 * 8
            else:
                q += nlen
            vals = [self.u(q + 4 * i, 4) for i in range(nvals)]
            q += 4 * nvals
            if ver == 1 and nvals % 2:
                q += 4
            out.append((fid, vals))
        return out

    def _chunk_btree(self, addr, ndim, chunks):
        a = self.base + addr
        if self.buf[a:a + 4] != b"TREE" or self.buf[a + 4] != 1:
            raise ValueError(f"{self.path}: bad chunk B-tree")
        level, used = self.buf[a + 5], self.u(a + 6, 2)
        p = a + 8 + 2 * self.so
        ksize = 8 + 8 * ndim
        for _ in range(used):
            size, mask = self.u(p, 4), self.u(p + 4, 4)
            first = self.u(p + 8, 8)
            child = self.addr(p + ksize)
            if level > 0:
                self._chunk_btree(child, ndim, chunks)
            else:
                chunks.append((self.base + child, size, mask, first))
            p += ksize + self.so


def _unfilter(raw, filters, mask, itemsize):
    """Undo a chunk's filter pipeline (applied in order when writing)."""
    data = raw
    for i in range(len(filters) - 1, -1, -1):
        fid, vals = filters[i]
        if mask & (1 << i):
            continue
        if fid == 1:  # deflate
            data = zlib.decompress(data)
        elif fid == 2:  # shuffle: byte planes back into elements
            es = vals[0] if vals else itemsize
            n = len(data) // es
            arr = np.frombuffer(data[:n * es], dtype=np.uint8).reshape(es, n)
            data = arr.T.tobytes() + data[n * es:]
        elif fid == 3:  # Fletcher-32: checksum appended
            data = data[:-4]
        else:
            raise NotImplementedError(f"HDF5 filter {fid}")
    return data


def open_datasets(path):
    """{name: DatasetInfo} of the root group's one-dimensional numeric datasets
    (other objects are skipped)."""
    f = _File(path)
    out = {}
    for name, addr in f.root_links().items():
        try:
            out[name] = f.dataset(name, addr)
        except NotImplementedError:
            continue
    return out, f


def read_dataset(path, name):
    """The elements of dataset ``name`` as a host array (native byte order kept)."""
    infos, f = open_datasets(path)
    return _materialise(infos[name], f)


def _materialise(d, f):
    if d.layout == "contiguous":
        if d.offset < 0:
            return np.zeros(d.n, dtype=d.dtype)
        return np.frombuffer(f.buf, dtype=d.dtype, count=d.n, offset=d.offset)
    if d.layout == "compact":
        return np.frombuffer(d.data, dtype=d.dtype, count=d.n)
    out = np.zeros(d.n, dtype=d.dtype)
    es = d.dtype.itemsize
    for off, size, mask, first in d.chunks:
        raw = _unfilter(f.buf[off:off + size], d.filters or [], mask, es)
        k = min(d.chunk_elems, d.n - first)
        if k > 0:
            out[first:first + k] = np.frombuffer(raw, dtype=d.dtype, count=k)
    return out


# ------------------------------------------------------------------ writer
def write_columns(path, columns, chunked=None):
    """Write ``{name: 1-D array}`` as HDF5 datasets in the root group
    (superblock version 0, symbol-table root group, version-1 object headers;
    contiguous layout, or for the names in ``chunked`` a chunked layout with
    the shuffle and deflate filters and a version-1 B-tree chunk index)."""
    so = 8
    chunked = dict(chunked or {})
    names = list(columns)
    arrs = [np.ascontiguousarray(columns[n]) for n in names]
    out = bytearray()

    def align(n=8):
        while len(out) % n:
            out.append(0)

    def put(b):
        off = len(out)
        out.extend(b)
        return off

    def u(v, n):
        return int(v).to_bytes(n, "little")

    # superblock v0 (root entry and addresses patched at the end)
    put(SIGNATURE + bytes([0, 0, 0, 0, 0, so, so, 0]) + u(4, 2) + u(16, 2) + u(0, 4))
    sb_addr = put(u(0, so) + u(UNDEF, so) + u(0, so) + u(UNDEF, so))  # base, free, eof, driver
    root_entry = put(b"\0" * (2 * so + 24))

    def datatype_msg(dt):
        dt = np.dtype(dt)
        order = 1 if dt.byteorder == ">" else 0
        if dt.kind == "f":
            prec = dt.itemsize * 8
            ebits, mbits, bias = (8, 23, 127) if dt.itemsize == 4 else (11, 52, 1023)
            # bit field: byte order, implied-msb mantissa (bits 4-5 = 2), sign bit position
            b = bytes([0x11, order | 0x20, 0x1F if dt.itemsize == 4 else 0x3F, 0]) + u(dt.itemsize, 4)
            b += u(0, 2) + u(prec, 2) + bytes([mbits, ebits, 0, mbits]) + u(bias, 4)
            return b
        if dt.kind in "iu":
            b = bytes([0x10, order | (0x08 if dt.kind == "i" else 0), 0, 0]) + u(dt.itemsize, 4)
            return b + u(0, 2) + u(dt.itemsize * 8, 2)
        raise ValueError(f"unsupported dtype {dt}")

    def header(msgs):
        """Version-1 object header with the given (type, body) messages."""
        align()
        body = bytearray()
        for t, m in msgs:
            m = bytes(m) + b"\0" * ((-len(m)) % 8)
            body += u(t, 2) + u(len(m), 2) + bytes([0, 0, 0, 0]) + m
        return put(bytes([1, 0]) + u(len(msgs), 2) + u(1, 4) + u(len(body), 4) + b"\0" * 4 + bytes(body))

    obj_addr = {}
    for name, a in zip(names, arrs):
        dt = a.dtype
        space = bytes([1, 1, 0, 0]) + b"\0" * 4 + u(a.size, so)
        if name in chunked:
            ce = int(chunked[name])
            chunk_recs = []
            for first in range(0, a.size, ce):
                part = np.zeros(ce, dtype=dt)
                k = min(ce, a.size - first)
                part[:k] = a[first:first + k]
                raw = part.tobytes()
                shuf = np.frombuffer(raw, dtype=np.uint8).reshape(ce, dt.itemsize).T.tobytes()
                comp = zlib.compress(shuf, 6)
                align()
                chunk_recs.append((put(comp), len(comp), first))
            align()
            node = put(b"TREE" + bytes([1, 0]) + u(len(chunk_recs), 2) + u(UNDEF, so) + u(UNDEF, so) +
                       b"".join(u(sz, 4) + u(0, 4) + u(first, 8) + u(0, 8) + u(off, so)
                                for off, sz, first in chunk_recs) +
                       u(0, 4) + u(0, 4) + u(a.size, 8) + u(0, 8))
            layout = bytes([3, 2, 2]) + u(node, so) + u(ce, 4) + u(dt.itemsize, 4)
            pipeline = bytes([1, 2]) + b"\0" * 6
            pipeline += u(2, 2) + u(0, 2) + u(0, 2) + u(1, 2) + u(dt.itemsize, 4) + u(0, 4)
            pipeline += u(1, 2) + u(0, 2) + u(0, 2) + u(1, 2) + u(6, 4) + u(0, 4)
            msgs = [(0x01, space), (0x03, datatype_msg(dt)), (0x0B, pipeline), (0x08, layout)]
        else:
            align()
            data_off = put(a.tobytes()) if a.size else UNDEF
            layout = bytes([3, 1]) + u(data_off, so) + u(a.nbytes, so)
            msgs = [(0x01, space), (0x03, datatype_msg(dt)), (0x08, layout)]
        obj_addr[name] = header(msgs)

    # local heap with the names (offset 0: the empty name)
    heap_data = bytearray(b"\0" * 8)
    name_off = {}
    for name in names:
        name_off[name] = len(heap_data)
        nb = name.encode("utf-8") + b"\0"
        heap_data += nb + b"\0" * ((-len(nb)) % 8)
    align()
    heap_data_addr = put(bytes(heap_data))
    align()
    heap_addr = put(b"HEAP" + bytes([0, 0, 0, 0]) + u(len(heap_data), so) + u(UNDEF, so) + u(heap_data_addr, so))
    # one symbol table node holding every entry, names in sorted order
    order = sorted(names)
    align()
    snod = put(b"SNOD" + bytes([1, 0]) + u(len(order), 2) +
               b"".join(u(name_off[n], so) + u(obj_addr[n], so) + u(0, 4) + u(0, 4) + b"\0" * 16 for n in order))
    align()
    btree = put(b"TREE" + bytes([0, 0]) + u(1, 2) + u(UNDEF, so) + u(UNDEF, so) + u(0, so) + u(snod, so) +
                u(name_off[order[-1]] if order else 0, so))
    root = header([(0x11, u(btree, so) + u(heap_addr, so))])
    out[root_entry:root_entry + 2 * so + 24] = (u(0, so) + u(root, so) + u(1, 4) + u(0, 4) + u(btree, so) +
                                                u(heap_addr, so))
    out[sb_addr + 2 * so:sb_addr + 3 * so] = u(len(out), so)
    with open(path, "wb") as f:
        f.write(bytes(out))
    return path
