"""A small HDF5 writer for the reader's tests, field by field from the HDF5 File Format
Specification (version 3.0): the layouts real writers use that the test data files do not hold —
version 2 superblocks and object headers with compact link messages, continuation blocks,
chunked datasets under multi-level version 1 B-trees, the version 4 single-chunk and implicit
chunk indexes, deflate / shuffle / Fletcher-32 / LZF filters, fill values, enumerations,
fixed and variable-length strings, and attributes.

A tree is a dict: a name maps to a dict (a group) or to a `D` (a dataset). Checksums of version 2
structures are written as zeros (the reader does not check them).
"""
import struct
import zlib

import numpy as np

UNDEF8 = b"\xff" * 8


class D:
    """A dataset to write: `data` (an array, or a list of str for variable-length strings) and how
    to store it: layout 'contiguous' | 'compact' | 'chunked' (index 'btree' | 'single' |
    'implicit'), chunk shape, filters [('deflate'|'shuffle'|'fletcher32'|'lzf', …)], the chunks left
    unwritten (grid indices), a fill value, attributes, as an enumeration, as a string type."""

    def __init__(self, data, layout="contiguous", chunk=None, index="btree", filters=(), unwritten=(),
                 fill=None, attrs=None, enum=False, big=False, vlen=False, fanout=4):
        self.data, self.layout, self.chunk, self.index = data, layout, chunk, index
        self.filters, self.unwritten, self.fill, self.attrs = list(filters), set(unwritten), fill, attrs or {}
        self.enum, self.big, self.vlen, self.fanout = enum, big, vlen, fanout


def _pad8(b):
    return b + b"\0" * (-len(b) % 8)


def lzf_literal_stream(raw):
    """LZF with literal runs only (each ≤ 32 bytes): valid input for any LZF decoder."""
    out = bytearray()
    for i in range(0, len(raw), 32):
        part = raw[i:i + 32]
        out.append(len(part) - 1)
        out += part
    return bytes(out)


class Writer:
    def __init__(self, superblock=0, header=1, user_block=0):
        self.sb, self.hv, self.ub = superblock, header, user_block
        self.buf = bytearray(b"\0" * (user_block + 256))  # (the superblock goes in at the end)

    def alloc(self, data):
        while len(self.buf) % 8:
            self.buf.append(0)
        at = len(self.buf) - self.ub
        self.buf += data
        return at

    # ── messages ──

    @staticmethod
    def dtype_msg(d):
        if d.vlen:
            base = Writer._fixed(1, False, False)
            return bytes([0x19, 0x01, 0, 0]) + struct.pack("<I", 16) + base
        a = np.asarray(d.data)
        if a.dtype.kind == "S":
            return bytes([0x13, 0x00, 0, 0]) + struct.pack("<I", a.dtype.itemsize)
        if a.dtype.kind in "ui":
            t = Writer._fixed(a.dtype.itemsize, a.dtype.kind == "i", d.big)
            if d.enum:  # an enumeration over the integer: members FALSE = 0, TRUE = 1
                names = _pad8(b"FALSE\0") + _pad8(b"TRUE\0")
                vals = np.array([0, 1], a.dtype).tobytes()
                return bytes([0x18, 2, 0, 0]) + struct.pack("<I", a.dtype.itemsize) + t + names + vals
            return t
        size = a.dtype.itemsize
        bits0 = 0x20 | (1 if d.big else 0)
        sign = 31 if size == 4 else 63
        props = (struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127) if size == 4 else
                 struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023))
        return bytes([0x11, bits0, sign, 0]) + struct.pack("<I", size) + props

    @staticmethod
    def _fixed(size, signed, big):
        return bytes([0x10, (0x08 if signed else 0) | (1 if big else 0), 0, 0]) + struct.pack("<I", size) + \
            struct.pack("<HH", 0, 8 * size)

    def space_msg(self, shape):
        if self.hv == 2:
            head = bytes([2, len(shape), 0, 1 if shape else 0])
        else:
            head = bytes([1, len(shape), 0, 0, 0, 0, 0, 0])
        return head + b"".join(struct.pack("<Q", s) for s in shape)

    def filter_msg(self, filters, elem):
        ids = {"deflate": 1, "shuffle": 2, "fletcher32": 3, "lzf": 32000}
        if self.hv == 2:
            out = bytes([2, len(filters)])
            for f in filters:
                fid = ids[f]
                vals = [elem] if f == "shuffle" else ([6] if f == "deflate" else [])
                if fid >= 256:
                    name = b"lzf\0"
                    out += struct.pack("<HHHH", fid, len(name), 0, len(vals)) + name
                else:
                    out += struct.pack("<HHH", fid, 0, len(vals))
                out += b"".join(struct.pack("<I", v) for v in vals)
            return out
        out = bytes([1, len(filters)]) + b"\0" * 6
        for f in filters:
            fid = ids[f]
            vals = [elem] if f == "shuffle" else ([6] if f == "deflate" else [])
            name = _pad8(f.encode() + b"\0")
            out += struct.pack("<HHHH", fid, len(name), 0, len(vals)) + name
            out += b"".join(struct.pack("<I", v) for v in vals) + (b"\0" * 4 if len(vals) % 2 else b"")
        return out

    def attr_msg(self, name, value):
        if isinstance(value, str):
            raw = value.encode()
            t = bytes([0x13, 0, 0, 0]) + struct.pack("<I", len(raw))
            sp = self.space_msg(())
            data = raw
        else:
            a = np.asarray(value)
            t = self.dtype_msg(D(a))
            sp = self.space_msg(a.shape)
            data = a.tobytes()
        nm = name.encode() + b"\0"
        if self.hv == 2:  # version 3: not padded, with the name's encoding
            return struct.pack("<BBHHHB", 3, 0, len(nm), len(t), len(sp), 0) + nm + t + sp + data
        return struct.pack("<BBHHH", 1, 0, len(nm), len(t), len(sp)) + _pad8(nm) + _pad8(t) + _pad8(sp) + data

    # ── data ──

    def _encode(self, raw, filters, elem):
        for f in filters:
            if f == "shuffle":
                n = len(raw) // elem
                raw = np.frombuffer(raw[:n * elem], np.uint8).reshape(n, elem).T.tobytes() + raw[n * elem:]
            elif f == "deflate":
                raw = zlib.compress(raw, 6)
            elif f == "fletcher32":
                raw = raw + b"\xde\xad\xbe\xef"
            elif f == "lzf":
                raw = lzf_literal_stream(raw)
        return raw

    def _vlen_data(self, strings):
        """A global heap collection holding the strings; the elements that point at them."""
        objs = b""
        for i, s in enumerate(strings, 1):
            b = s.encode()
            objs += struct.pack("<HHIQ", i, 1, 0, len(b)) + _pad8(b)
        size = max(4096, 16 + len(objs) + 16)
        coll = b"GCOL" + bytes([1, 0, 0, 0]) + struct.pack("<Q", size) + objs
        coll += b"\0" * (size - len(coll))
        at = self.alloc(coll)
        return b"".join(struct.pack("<IQI", len(s.encode()), at, i) for i, s in enumerate(strings, 1))

    def dataset(self, d):
        if d.vlen:
            raw = self._vlen_data(list(d.data))
            shape, elem = (len(d.data),), 16
            a = None
        else:
            a = np.asarray(d.data)
            if d.big:
                a = a.astype(a.dtype.newbyteorder(">"))
            raw, shape, elem = a.tobytes(), a.shape, a.dtype.itemsize
        msgs = [(0x01, self.space_msg(shape)), (0x03, self.dtype_msg(d))]
        if d.fill is not None:
            fv = np.asarray([d.fill], a.dtype).tobytes()
            msgs.append((0x05, bytes([2, 2, 2, 1]) + struct.pack("<I", len(fv)) + fv))
        if d.layout == "compact":
            msgs.append((0x08, bytes([3, 0]) + struct.pack("<H", len(raw)) + raw))
        elif d.layout == "contiguous":
            at = self.alloc(raw)
            msgs.append((0x08, bytes([3, 1]) + struct.pack("<QQ", at, len(raw))))
        else:
            msgs += self._chunked(d, a, elem)
        for k, v in d.attrs.items():
            msgs.append((0x0C, self.attr_msg(k, v)))
        return self.header(msgs)

    def _chunked(self, d, a, elem):
        chunk = tuple(d.chunk)
        grid = [-(-s // c) for s, c in zip(a.shape, chunk)]
        fill = np.zeros(1, a.dtype) if d.fill is None else np.asarray([d.fill], a.dtype)
        stored = []
        for idx in np.ndindex(*grid):
            box = np.full(chunk, fill[0], a.dtype)
            src = tuple(slice(i * c, min((i + 1) * c, s)) for i, c, s in zip(idx, chunk, a.shape))
            box[tuple(slice(0, x.stop - x.start) for x in src)] = a[src]
            raw = box.tobytes()
            if idx in d.unwritten:
                continue
            enc = self._encode(raw, d.filters, elem)
            stored.append((idx, enc))
        msgs = []
        if d.filters:
            msgs.append((0x0B, self.filter_msg(d.filters, elem)))
        dims = b"".join(struct.pack("<I", c) for c in chunk) + struct.pack("<I", elem)
        nd = len(chunk) + 1
        if d.index == "btree":
            root = self._btree(stored, chunk, len(chunk), d.fanout)
            msgs.append((0x08, bytes([3, 2, nd]) + struct.pack("<Q", root) + dims))
            return msgs
        dims4 = b"".join(struct.pack("<I", c) for c in chunk) + struct.pack("<I", elem)
        if d.index == "single":
            (_, enc), = stored
            at = self.alloc(enc)
            flags = 0x02 if d.filters else 0
            info = (struct.pack("<QI", len(enc), 0) if d.filters else b"") + struct.pack("<Q", at)
            msgs.append((0x08, bytes([4, 2, flags, nd, 4]) + dims4 + bytes([1]) + info))
        else:  # implicit: every chunk, unfiltered, back to back in the grid's row-major order
            at = self.alloc(b"".join(enc for _, enc in stored))
            msgs.append((0x08, bytes([4, 2, 0, nd, 4]) + dims4 + bytes([2]) + struct.pack("<Q", at)))
        return msgs

    def _btree(self, stored, chunk, rank, fanout):
        """A version 1 B-tree of chunks, `fanout` entries a node: leaves, then levels of parents."""
        def key(size, origin):
            return struct.pack("<II", size, 0) + b"".join(struct.pack("<Q", o) for o in origin) + struct.pack("<Q", 0)

        entries = []
        for idx, enc in stored:
            at = self.alloc(enc)
            entries.append((key(len(enc), [i * c for i, c in zip(idx, chunk)]), at))
        end_key = key(0, [0] * rank)
        level = 0
        while True:
            nodes = []
            for i in range(0, max(len(entries), 1), fanout):
                part = entries[i:i + fanout]
                body = b"".join(k + struct.pack("<Q", a) for k, a in part) + end_key
                node = b"TREE" + bytes([1, level]) + struct.pack("<H", len(part)) + UNDEF8 + UNDEF8 + body
                nodes.append((part[0][0] if part else end_key, self.alloc(node)))
            if len(nodes) == 1:
                return nodes[0][1]
            entries, level = nodes, level + 1

    # ── headers and groups ──

    def header(self, msgs):
        """An object header; its last message goes into a continuation block (both versions)."""
        if len(msgs) > 1:
            main, cont = msgs[:-1], msgs[-1:]
        else:
            main, cont = msgs, []
        if self.hv == 2:
            def pack(ms):
                return b"".join(struct.pack("<BHB", t, len(d), 0) + d for t, d in ms)
            c_at = None
            if cont:
                blk = b"OCHK" + pack(cont) + b"\0" * 4
                c_at = self.alloc(blk)
                main = main + [(0x10, struct.pack("<QQ", c_at, len(blk)))]
            body = pack(main)
            return self.alloc(b"OHDR" + bytes([2, 0x02]) + struct.pack("<I", len(body)) + body + b"\0" * 4)

        def pack1(ms):
            return b"".join(struct.pack("<HHB3x", t, len(_pad8(d)), 0) + _pad8(d) for t, d in ms)
        n = len(msgs)
        if cont:
            blk = pack1(cont)
            c_at = self.alloc(blk)
            main = main + [(0x10, struct.pack("<QQ", c_at, len(blk)))]
            n += 1
        body = pack1(main)
        return self.alloc(struct.pack("<BBHII", 1, 0, n, 1, len(body)) + b"\0" * 4 + body)

    def group(self, tree):
        kids = {}
        for name, v in tree.items():
            kids[name] = self.group(v) if isinstance(v, dict) else self.dataset(v)
        if self.hv == 2:  # compact link messages (and a link info message saying so)
            msgs = [(0x02, bytes([0, 0]) + UNDEF8 + UNDEF8)]
            for name, at in kids.items():
                nm = name.encode()
                msgs.append((0x06, bytes([1, 0x10 | 0x00, 0, len(nm)]) + nm + struct.pack("<Q", at)))
            return self.header(msgs)
        btree, heap = self.symbol_table(kids)
        return self.header([(0x11, struct.pack("<QQ", btree, heap))])

    def symbol_table(self, kids):
        """A local heap of the names and symbol table nodes of up to 3 entries under one B-tree node
        (several leaves: the reader must follow each)."""
        names = b"\0" * 8
        offs = {}
        for name in sorted(kids):
            offs[name] = len(names)
            names += _pad8(name.encode() + b"\0")
        data_at = self.alloc(names)
        heap = self.alloc(b"HEAP" + bytes([0, 0, 0, 0]) + struct.pack("<QQQ", len(names), (1 << 64) - 1, data_at))
        order = sorted(kids)
        leaves = []
        for i in range(0, max(len(order), 1), 3):
            part = order[i:i + 3]
            ents = b"".join(struct.pack("<QQII", offs[n], kids[n], 0, 0) + b"\0" * 16 for n in part)
            leaves.append((offs[part[-1]] if part else 0, self.alloc(b"SNOD" + bytes([1, 0]) +
                                                                       struct.pack("<H", len(part)) + ents)))
        body = struct.pack("<Q", 0) + b"".join(struct.pack("<QQ", a, k) for k, a in leaves)
        tree = self.alloc(b"TREE" + bytes([0, 0]) + struct.pack("<H", len(leaves)) + UNDEF8 + UNDEF8 + body)
        return tree, heap

    def write(self, path, tree):
        root = self.group(tree)
        eof = len(self.buf) - self.ub
        sig = b"\x89HDF\r\n\x1a\n"
        if self.sb == 0:
            if self.hv != 1:
                raise ValueError("a version 0 superblock roots a version 1 header")
            # the root's symbol table entry repeats its B-tree and heap (cache type 1)
            sb = sig + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HHI", 4, 16, 0)
            sb += struct.pack("<Q", self.ub) + UNDEF8 + struct.pack("<Q", eof) + UNDEF8
            sb += struct.pack("<QQII", 0, root, 0, 0) + b"\0" * 16
        else:
            sb = sig + bytes([2, 8, 8, 0]) + struct.pack("<Q", self.ub) + UNDEF8 + struct.pack("<QQ", eof, root)
            sb += b"\0" * 4
        self.buf[self.ub:self.ub + len(sb)] = sb
        with open(path, "wb") as fh:
            fh.write(bytes(self.buf))
