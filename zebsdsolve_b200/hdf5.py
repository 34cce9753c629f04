"""HDF5 files, read on the host (the reference's src/io/hdf5.zig): the part of the format that EBSD
scan files use, written from the HDF5 File Format Specification (version 3.0), so that no HDF5
library is needed. Groups are followed by name, dataset headers parsed, and datasets read whole:
a contiguous dataset as a view of the memory-mapped file, a chunked one chunk by chunk into an
array.

Covered (hdf5.zig:9-16): superblock versions 0-3; object headers versions 1 and 2 (continuation
blocks included); groups stored as symbol tables (a version 1 B-tree of symbol table nodes over a
local heap, the default of every HDF5 writer) or as compact link messages; fixed-point,
floating-point, enumerated (read as its base integer), fixed-length and variable-length string
types; compact, contiguous and chunked layouts (version 1 B-tree; version 4 single-chunk and
implicit indexes); the deflate, shuffle, Fletcher-32 and LZF filters; attributes of numbers and
strings. Not covered, each refused by name (H5Unsupported): dense groups (fractal heaps), the
fixed-array, extensible-array and version 2 B-tree chunk indexes of files written with
libver="latest", external links, virtual datasets and other filters.
"""
import os
import zlib

import numpy as np

UNDEF = (1 << 64) - 1
MAX_RANK = 8


class H5Error(ValueError):
    """A file that is not HDF5, or is damaged."""


class H5Unsupported(H5Error):
    """A part of the format this reader does not cover (hdf5.zig:170-175)."""


class Dtype:
    """A stored element: kind 'u', 'i', 'f' (numbers), 'S' (fixed-length string), 'V' (variable-length
    string) or 'other'; size in bytes; byte order."""

    def __init__(self, kind, size, big=False):
        self.kind, self.size, self.big = kind, size, big

    def numpy(self):
        if self.kind in "uif":
            return np.dtype(("<>"[int(self.big)]) + self.kind + str(self.size))
        if self.kind == "S":
            return np.dtype("S%d" % self.size)
        return np.dtype("V%d" % self.size)


class Dataset:
    """A dataset's header: shape, dtype, layout ('compact', 'contiguous', 'chunked') and where its
    bytes are. Chunked: `chunk` (the chunk's shape), `index` ('btree', 'single', 'implicit'),
    `filters` [(id, client values)]."""

    def __init__(self):
        self.shape, self.dtype, self.layout = (), None, None
        self.addr, self.size, self.raw = UNDEF, 0, b""
        self.chunk, self.index, self.filters = None, None, []
        self.single_size, self.single_mask = 0, 0
        self.fill = None

    @property
    def elements(self):
        return int(np.prod(self.shape, dtype=np.int64)) if self.shape is not None else 0


def _pad8(n):
    return (n + 7) & ~7


def lzf_decompress(src, out_len):
    """LZF (Marc Lehmann's liblzf, the HDF5 filter 32000): a control byte c < 32 copies c + 1
    literal bytes; otherwise c >> 5 (7: plus the next byte) + 2 bytes are copied from
    ((c & 31) << 8 | next byte) + 1 bytes back in the output."""
    out = bytearray(out_len)
    i = o = 0
    n = len(src)
    while i < n:
        c = src[i]
        i += 1
        if c < 32:
            c += 1
            if o + c > out_len or i + c > n:
                raise H5Error("LZF: a literal run past the end")
            out[o:o + c] = src[i:i + c]
            i += c
            o += c
        else:
            ln = c >> 5
            if ln == 7:
                ln += src[i]
                i += 1
            ref = o - ((c & 31) << 8) - src[i] - 1
            i += 1
            ln += 2
            if ref < 0 or o + ln > out_len:
                raise H5Error("LZF: a back reference out of range")
            for k in range(ln):  # (may overlap its own output)
                out[o + k] = out[ref + k]
            o += ln
    if o != out_len:
        raise H5Error("LZF: the chunk decodes to the wrong size")
    return bytes(out)


class File:
    """An HDF5 file opened for reading (hdf5.zig Hdf5.open)."""

    def __init__(self, path):
        self.path = str(path)
        size = os.path.getsize(self.path)
        if size < 48:
            raise H5Error("not an HDF5 file (too short)")
        self.buf = np.memmap(self.path, np.uint8, "r")
        self.size = size
        sig = b"\x89HDF\r\n\x1a\n"
        at = 0
        while at + 8 <= size and bytes(self.buf[at:at + 8]) != sig:
            at = 512 if at == 0 else at * 2  # (after a user block: 512, 1024, 2048, ...)
        if at + 8 > size:
            raise H5Error("not an HDF5 file (no superblock signature)")
        b = self._bytes(at, min(256, size - at))
        ver = b[8]
        if ver in (0, 1):
            self.so, self.sl = b[13], b[14]
            p = 24 if ver == 0 else 28
            so = self.so
            self.base = self._int(b, p, so)
            p += 4 * so  # base, free-space info, end of file, driver info
            # the root group's symbol table entry: name offset, object header address, ...
            self.root = self._int(b, p + so, so)
        elif ver in (2, 3):
            self.so, self.sl = b[9], b[10]
            so = self.so
            self.base = self._int(b, 12, so)
            self.root = self._int(b, 12 + 3 * so, so)
        else:
            raise H5Unsupported("superblock version %d" % ver)
        if self.so not in (4, 8) or self.sl not in (4, 8):
            raise H5Unsupported("offset size")
        self._heap_cache = {}

    # ── bytes ──

    def _bytes(self, at, n):
        if at < 0 or n < 0 or at + n > self.size:
            raise H5Error("an address past the end of the file")
        return bytes(self.buf[at:at + n])

    def _abs(self, addr):
        return self.base + addr

    @staticmethod
    def _int(b, p, n):
        v = int.from_bytes(b[p:p + n], "little")
        return UNDEF if v == (1 << (8 * n)) - 1 else v

    # ── object headers ──

    def messages(self, addr):
        """Every message of the object header at `addr`: [(type, data bytes)] (hdf5.zig:191-252)."""
        at = self._abs(addr)
        head = self._bytes(at, 16)
        out = []
        if head[:4] == b"OHDR":
            if head[4] != 2:
                raise H5Unsupported("object header version")
            flags = head[5]
            p = 6 + (16 if flags & 0x20 else 0) + (4 if flags & 0x10 else 0)
            w = 1 << (flags & 3)
            b = self._bytes(at, p + w)
            size0 = self._int(b, p, w)
            blocks = [(at + p + w, size0)]
            order = 2 if flags & 0x04 else 0
            while blocks:
                start, n = blocks.pop(0)
                b = self._bytes(start, n)
                q = 0
                while q + 4 + order <= n:
                    mtype, msize, = b[q], int.from_bytes(b[q + 1:q + 3], "little")
                    q += 4 + order
                    data = b[q:q + msize]
                    q += msize
                    if mtype == 0x10:
                        c_at, c_len = self._int(data, 0, self.so), self._int(data, self.so, self.sl)
                        c = self._abs(c_at)
                        if self._bytes(c, 4) != b"OCHK":
                            raise H5Error("a continuation block without its signature")
                        blocks.append((c + 4, c_len - 8))
                    elif mtype != 0:
                        out.append((mtype, data))
            return out
        if head[0] != 1:
            raise H5Unsupported("object header version")
        nmsg = int.from_bytes(head[2:4], "little")
        hsize = int.from_bytes(head[8:12], "little")
        blocks = [(at + 16, hsize)]
        seen = 0
        while blocks and seen < nmsg:
            start, n = blocks.pop(0)
            b = self._bytes(start, n)
            q = 0
            while q + 8 <= n and seen < nmsg:
                mtype, msize = int.from_bytes(b[q:q + 2], "little"), int.from_bytes(b[q + 2:q + 4], "little")
                data = b[q + 8:q + 8 + msize]
                q += 8 + msize
                seen += 1
                if mtype == 0x10:
                    blocks.append((self._abs(self._int(data, 0, self.so)), self._int(data, self.so, self.sl)))
                elif mtype != 0:
                    out.append((mtype, data))
        return out

    # ── groups ──

    def _local_heap(self, addr):
        b = self._bytes(self._abs(addr), 8 + 2 * self.sl + self.so)
        if b[:4] != b"HEAP":
            raise H5Error("a local heap without its signature")
        size = self._int(b, 8, self.sl)
        data = self._int(b, 8 + 2 * self.sl, self.so)
        return self._bytes(self._abs(data), size)

    @staticmethod
    def _cstr(b, p):
        e = b.index(b"\0", p) if b"\0" in b[p:] else len(b)
        return b[p:e].decode("utf-8", "replace")

    def _symbol_table(self, tree, heap):
        """Names and object header addresses of a symbol-table group: the leaves of its version 1
        B-tree are symbol table nodes ("SNOD"), their entries name offsets into the local heap."""
        names = self._local_heap(heap)
        so, sl = self.so, self.sl
        out = {}
        todo = [(tree, None)]
        while todo:
            node, level = todo.pop()
            b = self._bytes(self._abs(node), 8 + 2 * so)
            if b[:4] != b"TREE" or b[4] != 0:
                raise H5Error("a group's B-tree node is damaged")
            lv, used = b[5], int.from_bytes(b[6:8], "little")
            if level is not None and lv != level:
                raise H5Error("a group's B-tree node at the wrong level")
            body = self._bytes(self._abs(node) + 8 + 2 * so, (used + 1) * sl + used * so)
            for k in range(used):
                child = self._int(body, sl + k * (sl + so), so)
                if lv > 0:
                    todo.append((child, lv - 1))
                    continue
                s = self._bytes(self._abs(child), 8)
                if s[:4] != b"SNOD":
                    raise H5Error("a symbol table node without its signature")
                count = int.from_bytes(s[6:8], "little")
                ent = 2 * so + 24
                e = self._bytes(self._abs(child) + 8, count * ent)
                for j in range(count):
                    off = self._int(e, j * ent, so)
                    out[self._cstr(names, off)] = self._int(e, j * ent + so, so)
        return out

    def members(self, group):
        """{name: object header address} of the group at `group` (hdf5.zig:254-400)."""
        out = {}
        for mtype, d in self.messages(group):
            if mtype == 0x11:  # symbol table: B-tree, local heap
                out.update(self._symbol_table(self._int(d, 0, self.so), self._int(d, self.so, self.so)))
            elif mtype == 0x02:  # link info: dense storage when the fractal heap address is defined
                p = 2 + (8 if d[1] & 1 else 0)
                if self._int(d, p, self.so) != UNDEF:
                    raise H5Unsupported('dense group (written with libver="latest")')
            elif mtype == 0x06:  # a link
                flags = d[1]
                p = 2
                kind = 0
                if flags & 0x08:
                    kind = d[p]
                    p += 1
                if flags & 0x04:
                    p += 8
                if flags & 0x10:
                    p += 1
                w = 1 << (flags & 3)
                ln = int.from_bytes(d[p:p + w], "little")
                p += w
                name = d[p:p + ln].decode("utf-8", "replace")
                p += ln
                if kind == 0:
                    out[name] = self._int(d, p, self.so)
                elif kind == 1:
                    sl_ = int.from_bytes(d[p:p + 2], "little")
                    out[name] = ("soft", d[p + 2:p + 2 + sl_].decode("utf-8", "replace"))
                else:
                    out[name] = ("external", name)
        return out

    def child(self, group, name):
        """The object named `name` in the group at `group`, or None."""
        m = self.members(group).get(name)
        if isinstance(m, tuple):
            if m[0] == "soft":
                return self.find(m[1])
            raise H5Unsupported("external link")
        return m

    def list(self, group):
        return list(self.members(group).keys())

    def find(self, path):
        """The object at a '/'-separated path from the root, or None."""
        at = self.root
        for part in [p for p in str(path).split("/") if p]:
            at = self.child(at, part)
            if at is None:
                return None
        return at

    def is_group(self, addr):
        return any(t in (0x11, 0x02, 0x06) for t, _ in self.messages(addr)) and not any(
            t == 0x08 for t, _ in self.messages(addr))

    # ── datasets ──

    def _dtype(self, d):
        cls, ver = d[0] & 0x0F, d[0] >> 4
        bits = d[1] | (d[2] << 8) | (d[3] << 16)
        size = int.from_bytes(d[4:8], "little")
        if cls == 0:
            return Dtype("i" if bits & 0x08 else "u", size, bool(bits & 1))
        if cls == 1:
            if bits & 0x40:
                raise H5Unsupported("VAX floating point")
            return Dtype("f", size, bool(bits & 1))
        if cls == 3:
            return Dtype("S", size)
        if cls == 8:  # enumerations (h5py's booleans) read as their base integer
            base = self._dtype(d[8:])
            return Dtype(base.kind, base.size, base.big)
        if cls == 9 and (bits & 0x0F) == 1:
            return Dtype("V", size)
        return Dtype("other", size)

    def _dataspace(self, d):
        ver, rank, flags = d[0], d[1], d[2]
        if ver == 1:
            p = 8
        elif ver == 2:
            if d[3] == 2:  # null dataspace: no elements
                return None
            p = 4
        else:
            raise H5Unsupported("dataspace version")
        if rank > MAX_RANK:
            raise H5Unsupported("dataset rank")
        return tuple(int.from_bytes(d[p + k * self.sl:p + (k + 1) * self.sl], "little") for k in range(rank))

    def _filters(self, d):
        ver, n = d[0], d[1]
        p = 8 if ver == 1 else 2
        out = []
        for _ in range(n):
            fid = int.from_bytes(d[p:p + 2], "little")
            if ver == 1 or fid >= 256:
                nlen = int.from_bytes(d[p + 2:p + 4], "little")
                p += 4
            else:
                nlen = 0
                p += 2
            nval = int.from_bytes(d[p + 2:p + 4], "little")
            p += 4
            p += _pad8(nlen) if ver == 1 else nlen
            vals = [int.from_bytes(d[p + 4 * k:p + 4 * k + 4], "little") for k in range(nval)]
            p += 4 * nval + (4 if ver == 1 and nval % 2 else 0)
            if fid not in (1, 2, 3, 32000):
                raise H5Unsupported("compression filter %d" % fid)
            out.append((fid, vals))
        return out

    def _layout(self, ds, d):
        ver = d[0]
        so, sl = self.so, self.sl
        if ver in (1, 2):
            nd, cls = d[1], d[2]
            p = 8
            if cls != 0:
                ds.addr = self._int(d, p, so)
                p += so
            dims = [int.from_bytes(d[p + 4 * k:p + 4 * k + 4], "little") for k in range(nd)]
            p += 4 * nd
            if cls == 0:
                ds.layout, n = "compact", int.from_bytes(d[p:p + 4], "little")
                ds.raw = d[p + 4:p + 4 + n]
            elif cls == 1:
                ds.layout = "contiguous"
            elif cls == 2:
                ds.layout, ds.index, ds.chunk = "chunked", "btree", tuple(dims[:-1])
            else:
                raise H5Unsupported("layout class")
            return
        if ver not in (3, 4):
            raise H5Unsupported("layout version")
        cls = d[1]
        if cls == 0:
            n = int.from_bytes(d[2:4], "little")
            ds.layout, ds.raw = "compact", d[4:4 + n]
        elif cls == 1:
            ds.layout, ds.addr, ds.size = "contiguous", self._int(d, 2, so), self._int(d, 2 + so, sl)
        elif cls == 2 and ver == 3:
            nd = d[2]
            if nd == 0 or nd - 1 > MAX_RANK:
                raise H5Unsupported("chunk rank")
            ds.addr = self._int(d, 3, so)
            p = 3 + so
            dims = [int.from_bytes(d[p + 4 * k:p + 4 * k + 4], "little") for k in range(nd)]
            ds.layout, ds.index, ds.chunk = "chunked", "btree", tuple(dims[:-1])
        elif cls == 2:
            flags, nd, w = d[2], d[3], d[4]
            if nd == 0 or nd - 1 > MAX_RANK:
                raise H5Unsupported("chunk rank")
            p = 5
            dims = [int.from_bytes(d[p + w * k:p + w * (k + 1)], "little") for k in range(nd)]
            p += w * nd
            kind = d[p]
            p += 1
            ds.layout, ds.chunk = "chunked", tuple(dims[:-1])
            if kind == 1:
                ds.index = "single"
                if flags & 0x02:
                    ds.single_size = self._int(d, p, sl)
                    ds.single_mask = int.from_bytes(d[p + sl:p + sl + 4], "little")
                    p += sl + 4
                ds.addr = self._int(d, p, so)
            elif kind == 2:
                ds.index, ds.addr = "implicit", self._int(d, p, so)
            elif kind == 3:
                raise H5Unsupported('fixed-array chunk index (written with libver="latest")')
            elif kind == 4:
                raise H5Unsupported('extensible-array chunk index (written with libver="latest")')
            elif kind == 5:
                raise H5Unsupported('version 2 B-tree chunk index (written with libver="latest")')
            else:
                raise H5Unsupported("chunk index")
        else:
            raise H5Unsupported("layout class")

    @staticmethod
    def _fill(d, new):
        if not new:  # the old fill value message: size, value
            n = int.from_bytes(d[0:4], "little")
            return d[4:4 + n] if n else None
        ver = d[0]
        if ver in (1, 2):
            defined = d[3]
            if ver == 2 and not defined:
                return None
            n = int.from_bytes(d[4:8], "little")
            return d[8:8 + n] if n else None
        if d[1] & 0x20:
            n = int.from_bytes(d[2:6], "little")
            return d[6:6 + n] if n else None
        return None

    def dataset(self, addr):
        """The header of the dataset at `addr` (hdf5.zig:405-552)."""
        ds = Dataset()
        have = set()
        for mtype, d in self.messages(addr):
            have.add(mtype)
            if mtype == 0x01:
                ds.shape = self._dataspace(d)
            elif mtype == 0x03:
                ds.dtype = self._dtype(d)
            elif mtype == 0x08:
                self._layout(ds, d)
            elif mtype == 0x0B:
                ds.filters = self._filters(d)
            elif mtype == 0x05:
                ds.fill = self._fill(d, True)
            elif mtype == 0x04 and ds.fill is None:
                ds.fill = self._fill(d, False)
        if 0x08 not in have or ds.dtype is None:
            raise H5Error("not a dataset")
        if ds.layout == "chunked" and ds.shape is not None and len(ds.chunk) != len(ds.shape):
            raise H5Error("a chunk of another rank than its dataset")
        return ds

    def _chunks_btree(self, ds):
        """(origin, stored size, filter mask, address) of every chunk a version 1 B-tree lists."""
        so = self.so
        rank = len(ds.shape)
        key = 8 + 8 * (rank + 1)
        out = []
        todo = [(ds.addr, None)]
        while todo:
            node, level = todo.pop()
            b = self._bytes(self._abs(node), 8 + 2 * so)
            if b[:4] != b"TREE" or b[4] != 1:
                raise H5Error("a chunk B-tree node is damaged")
            lv, used = b[5], int.from_bytes(b[6:8], "little")
            if level is not None and lv != level:
                raise H5Error("a chunk B-tree node at the wrong level")
            body = self._bytes(self._abs(node) + 8 + 2 * so, (used + 1) * key + used * so)
            for k in range(used):
                kp = k * (key + so)
                child = self._int(body, kp + key, so)
                if lv > 0:
                    todo.append((child, lv - 1))
                    continue
                size = int.from_bytes(body[kp:kp + 4], "little")
                mask = int.from_bytes(body[kp + 4:kp + 8], "little")
                origin = tuple(int.from_bytes(body[kp + 8 + 8 * j:kp + 16 + 8 * j], "little") for j in range(rank))
                out.append((origin, size, mask, child))
        return out

    def _chunks(self, ds):
        nbytes = int(np.prod(ds.chunk, dtype=np.int64)) * ds.dtype.size
        if ds.addr == UNDEF:
            return []
        if ds.index == "btree":
            return self._chunks_btree(ds)
        grid = [-(-s // c) for s, c in zip(ds.shape, ds.chunk)]
        if ds.index == "single":
            size = ds.single_size if ds.filters and ds.single_size else nbytes
            return [((0,) * len(ds.shape), size, ds.single_mask, ds.addr)]
        out = []  # implicit: unfiltered chunks back to back, row-major over the chunk grid
        for k, idx in enumerate(np.ndindex(*grid)):
            out.append((tuple(i * c for i, c in zip(idx, ds.chunk)), nbytes, 0, ds.addr + k * nbytes))
        return out

    def _decode(self, ds, raw, mask, nbytes):
        for i in range(len(ds.filters) - 1, -1, -1):
            if mask >> i & 1:
                continue  # (this filter was skipped for this chunk)
            fid, vals = ds.filters[i]
            if fid == 1:
                raw = zlib.decompress(raw)
            elif fid == 2:
                es = vals[0] if vals and vals[0] else ds.dtype.size
                n = len(raw) // es
                body = np.frombuffer(raw[:n * es], np.uint8).reshape(es, n).T.tobytes()
                raw = body + raw[n * es:]
            elif fid == 3:
                raw = raw[:-4]  # (the Fletcher-32 checksum at the end)
            elif fid == 32000:
                raw = lzf_decompress(raw, nbytes)
        if len(raw) != nbytes:
            raise H5Error("a chunk decodes to the wrong size")
        return raw

    def read(self, ds):
        """The whole dataset as an array of ds.shape in its stored type (a read-only view of the
        file where it is stored contiguously; strings as bytes)."""
        if ds.shape is None:
            return np.zeros(0, ds.dtype.numpy())
        dt = ds.dtype.numpy()
        n = ds.elements
        if ds.layout == "compact":
            return np.frombuffer(ds.raw[:n * dt.itemsize], dt, n).reshape(ds.shape)
        if ds.layout == "contiguous":
            if ds.addr == UNDEF:
                return self._filled(ds, dt)
            at = self._abs(ds.addr)
            if at + n * dt.itemsize > self.size:
                raise H5Error("a dataset past the end of the file")
            return self.buf[at:at + n * dt.itemsize].view(dt).reshape(ds.shape)
        out = self._filled(ds, dt)
        nbytes = int(np.prod(ds.chunk, dtype=np.int64)) * dt.itemsize
        for origin, size, mask, addr in self._chunks(ds):
            if addr == UNDEF:
                continue  # never written: the fill value
            if any(o >= s or o % c for o, s, c in zip(origin, ds.shape, ds.chunk)):
                raise H5Error("a chunk off its grid")
            raw = self._bytes(self._abs(addr), size)
            if ds.filters:
                raw = self._decode(ds, raw, mask, nbytes)
            elif len(raw) != nbytes:
                raise H5Error("an unfiltered chunk of the wrong size")
            arr = np.frombuffer(raw, dt).reshape(ds.chunk)
            dst = tuple(slice(o, min(o + c, s)) for o, s, c in zip(origin, ds.shape, ds.chunk))
            out[dst] = arr[tuple(slice(0, x.stop - x.start) for x in dst)]
        return out

    def _filled(self, ds, dt):
        out = np.zeros(ds.shape, dt)
        if ds.fill is not None and len(ds.fill) == dt.itemsize and any(ds.fill):
            out[...] = np.frombuffer(ds.fill, dt)[0]
        return out

    # ── values ──

    def _heap_object(self, coll, idx):
        """Object `idx` of the global heap collection at `coll` (variable-length data)."""
        key = coll
        if key not in self._heap_cache:
            head = self._bytes(self._abs(coll), 8 + self.sl)
            if head[:4] != b"GCOL":
                raise H5Error("a global heap collection without its signature")
            size = self._int(head, 8, self.sl)
            b = self._bytes(self._abs(coll), size)
            objs = {}
            p = 8 + self.sl
            while p + 8 + self.sl <= size:
                i = int.from_bytes(b[p:p + 2], "little")
                n = self._int(b, p + 8, self.sl)
                if i == 0:
                    break  # free space
                objs[i] = b[p + 8 + self.sl:p + 8 + self.sl + n]
                p += 8 + self.sl + _pad8(n)
            self._heap_cache[key] = objs
        return self._heap_cache[key].get(idx, b"")

    def _strings(self, ds, arr):
        if ds.dtype.kind == "S":
            return [bytes(x).split(b"\0", 1)[0].decode("utf-8", "replace").rstrip(" ") for x in arr.reshape(-1)]
        out = []
        for x in arr.reshape(-1):
            e = bytes(x)
            n = int.from_bytes(e[0:4], "little")
            if n == 0:
                out.append("")
                continue
            coll = self._int(e, 4, self.so)
            idx = int.from_bytes(e[4 + self.so:8 + self.so], "little")
            out.append(self._heap_object(coll, idx)[:n].decode("utf-8", "replace"))
        return out

    def numbers(self, addr):
        """A numeric dataset's values as float64, flat (hdf5.zig:1043-1055)."""
        ds = self.dataset(addr)
        if ds.dtype.kind not in "uif":
            raise H5Error("not a numeric dataset")
        return np.asarray(self.read(ds), np.float64).reshape(-1)

    def number(self, addr):
        """The first value of a numeric dataset (hdf5.zig:1057-1062)."""
        v = self.numbers(addr)
        if v.size == 0:
            raise H5Error("an empty dataset")
        return float(v[0])

    def string(self, addr):
        """The first string of a string dataset (hdf5.zig:1064-1085)."""
        ds = self.dataset(addr)
        if ds.dtype.kind not in "SV":
            raise H5Error("not a string dataset")
        s = self._strings(ds, self.read(ds))
        return s[0] if s else ""

    def attributes(self, addr):
        """{name: value} of the attributes in the object's header: numbers as arrays (a scalar as a
        float or int), strings as str."""
        out = {}
        for mtype, d in self.messages(addr):
            if mtype != 0x0C:
                continue
            ver = d[0]
            nlen, tlen, slen = (int.from_bytes(d[k:k + 2], "little") for k in (2, 4, 6))
            if ver == 1:
                p = 8
                name = d[p:p + nlen].split(b"\0", 1)[0].decode("utf-8", "replace")
                p += _pad8(nlen)
                td = d[p:p + tlen]
                p += _pad8(tlen)
                sd = d[p:p + slen]
                p += _pad8(slen)
            elif ver in (2, 3):
                p = 8 + (1 if ver == 3 else 0)
                name = d[p:p + nlen].split(b"\0", 1)[0].decode("utf-8", "replace")
                p += nlen
                td = d[p:p + tlen]
                p += tlen
                sd = d[p:p + slen]
                p += slen
            else:
                continue
            ds = Dataset()
            ds.dtype = self._dtype(td)
            ds.shape = self._dataspace(sd)
            if ds.shape is None:
                out[name] = None
                continue
            dt = ds.dtype.numpy()
            arr = np.frombuffer(d[p:p + ds.elements * dt.itemsize], dt, ds.elements).reshape(ds.shape)
            if ds.dtype.kind in "SV":
                s = self._strings(ds, arr)
                out[name] = s[0] if len(s) == 1 else s
            elif ds.dtype.kind in "uif":
                out[name] = arr.item() if arr.size == 1 else arr.copy()
        return out


def open_file(path):
    return File(path)
