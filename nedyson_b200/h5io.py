"""Minimal HDF5 reader and writer for the simulation output and checkpoints.

The reference saves its simulations with HighFive (reference src/greens.cpp:202-239,
src/molNEsim_decomp_impl.h:107-122): groups of contiguous datasets of float64,
integers, strings and complex128 (a compound of two float64 members "r", "i").  No
HDF5 library is available here, so this module reads and writes that subset of the
file format directly:

* superblock version 0, 8-byte offsets and lengths;
* object headers version 1 (with continuation messages when reading);
* groups as symbol tables (v1 B-tree of group nodes, symbol-table nodes, local heap);
* dataspaces version 1 (scalar or simple), datatypes fixed-point, floating-point,
  fixed-length string and compound, contiguous or compact data layout (version 3).

Files written here open in the HDF5 library (the structures are the ones the library
itself writes for this subset) and files the reference wrote read here.
"""
from __future__ import annotations

import struct

import numpy as np

SIG = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


# ---------------------------------------------------------------------------- reading
class H5File:
    """Read-only view of an HDF5 file: ``f["/G/GL"]`` -> numpy array (or scalar / str)."""

    def __init__(self, path):
        with open(path, "rb") as fh:
            self.d = fh.read()
        base = self.d.find(SIG)
        if base != 0:
            raise ValueError("not an HDF5 file (no signature at offset 0)")
        if self.d[8] != 0:
            raise ValueError(f"superblock version {self.d[8]} not handled (version 0 only)")
        self.so, self.sl = self.d[13], self.d[14]
        if (self.so, self.sl) != (8, 8):
            raise ValueError("8-byte offsets and lengths only")
        p = 24 + 4 * self.so
        self.root = self._entry(p)

    def _u(self, p, n):
        return int.from_bytes(self.d[p:p + n], "little")

    def _entry(self, p):
        ent = {"name_off": self._u(p, 8), "hdr": self._u(p + 8, 8), "ctype": self._u(p + 16, 4)}
        if ent["ctype"] == 1:
            ent["btree"] = self._u(p + 24, 8)
            ent["heap"] = self._u(p + 32, 8)
        return ent

    def _messages(self, hdr):
        if self.d[hdr] != 1:
            raise ValueError("object header version 1 expected")
        nmsg = self._u(hdr + 2, 2)
        size = self._u(hdr + 8, 4)
        blocks = [(hdr + 16, size)]
        out = []
        while blocks and len(out) < nmsg:
            start, length = blocks.pop(0)
            p, end = start, start + length
            while p + 8 <= end and len(out) < nmsg:
                mtype, msize = self._u(p, 2), self._u(p + 2, 2)
                body = p + 8
                if mtype == 0x0010:  # continuation
                    blocks.append((self._u(body, 8), self._u(body + 8, 8)))
                out.append((mtype, body, msize))
                p = body + msize
        return out

    def _group_children(self, btree, heap):
        if self.d[heap:heap + 4] != b"HEAP":
            raise ValueError("local heap expected")
        hdata = self._u(heap + 24, 8)
        out = {}
        stack = [btree]
        while stack:
            node = stack.pop()
            if self.d[node:node + 4] != b"TREE":
                raise ValueError("v1 B-tree node expected")
            level, used = self.d[node + 5], self._u(node + 6, 2)
            p = node + 24
            kids = []
            for _ in range(used):
                p += 8  # key
                kids.append(self._u(p, 8))
                p += 8
            if level > 0:
                stack.extend(kids)
                continue
            for snod in kids:
                if self.d[snod:snod + 4] != b"SNOD":
                    raise ValueError("symbol table node expected")
                q = snod + 8
                for _ in range(self._u(snod + 6, 2)):
                    ent = self._entry(q)
                    e = self.d.index(b"\x00", hdata + ent["name_off"])
                    out[self.d[hdata + ent["name_off"]:e].decode()] = ent
                    q += 40
        return out

    def _group_of_header(self, hdr):
        for mtype, body, _ in self._messages(hdr):
            if mtype == 0x0011:
                return self._u(body, 8), self._u(body + 8, 8)
        return None

    def _resolve(self, path):
        ent = self.root
        btree, heap = ent["btree"], ent["heap"]
        hdr = ent["hdr"]
        for part in [x for x in path.split("/") if x]:
            if btree is None:
                raise KeyError(path)
            kids = self._group_children(btree, heap)
            if part not in kids:
                raise KeyError(path)
            ent = kids[part]
            hdr = ent["hdr"]
            g = self._group_of_header(hdr)
            btree, heap = g if g else (None, None)
        return hdr, btree is not None

    def keys(self, path="/"):
        hdr, is_group = self._resolve(path)
        if not is_group:
            raise KeyError(f"{path} is not a group")
        btree, heap = self._group_of_header(hdr) if path.strip("/") else (self.root["btree"], self.root["heap"])
        return sorted(self._group_children(btree, heap))

    def __contains__(self, path):
        try:
            self._resolve(path)
            return True
        except KeyError:
            return False

    def _dtype(self, body):
        cls, ver = self.d[body] & 0x0F, self.d[body] >> 4
        bits = self._u(body + 1, 3)
        size = self._u(body + 4, 4)
        if cls == 0:  # fixed point
            if bits & 1:
                raise ValueError("big-endian integers not handled")
            return np.dtype(("<i" if bits & 8 else "<u") + str(size)), 8 + 4
        if cls == 1:  # floating point
            if bits & 1:
                raise ValueError("big-endian floats not handled")
            return np.dtype("<f" + str(size)), 8 + 12
        if cls == 3:  # fixed-length string
            return np.dtype(f"S{size}"), 8
        if cls == 6:  # compound
            nmem = bits & 0xFFFF
            p = body + 8
            fields = []
            for _ in range(nmem):
                e = self.d.index(b"\x00", p)
                name = self.d[p:e].decode()
                nlen = e - p + 1
                p += (nlen + 7) // 8 * 8
                if ver == 1:
                    off = self._u(p, 4)
                    p += 4 + 1 + 3 + 4 + 4 + 16
                else:
                    off = self._u(p, 4)
                    p += 4
                mdt, mlen = self._dtype(p)
                p += mlen
                fields.append((name, mdt, off))
            dt = np.dtype({"names": [f[0] for f in fields], "formats": [f[1] for f in fields],
                           "offsets": [f[2] for f in fields], "itemsize": size})
            return dt, p - body
        raise ValueError(f"datatype class {cls} not handled")

    def __getitem__(self, path):
        hdr, is_group = self._resolve(path)
        if is_group:
            raise KeyError(f"{path} is a group")
        dims, dt, raw = None, None, None
        for mtype, body, msize in self._messages(hdr):
            if mtype == 0x0001:
                ver, rank = self.d[body], self.d[body + 1]
                q = body + (8 if ver == 1 else 4)
                dims = [self._u(q + 8 * i, 8) for i in range(rank)]
            elif mtype == 0x0003:
                dt, _ = self._dtype(body)
            elif mtype == 0x0008:
                if self.d[body] != 3:
                    raise ValueError("data layout version 3 expected")
                lcls = self.d[body + 1]
                if lcls == 0:
                    n = self._u(body + 2, 2)
                    raw = self.d[body + 4:body + 4 + n]
                elif lcls == 1:
                    addr, n = self._u(body + 2, 8), self._u(body + 10, 8)
                    raw = b"" if addr == UNDEF else self.d[addr:addr + n]
                else:
                    raise ValueError("chunked datasets not handled")
        count = int(np.prod(dims)) if dims else 1
        a = np.frombuffer(raw, dtype=dt, count=count) if raw else np.zeros(count, dt)
        if dt.names == ("r", "i") or (dt.names and set(dt.names) == {"r", "i"}):
            a = a["r"] + 1j * a["i"]
        if dt.kind == "S":
            return a[0].split(b"\x00")[0].decode()
        if not dims:
            return a[0].item()
        return a.reshape(dims)


# ---------------------------------------------------------------------------- writing
def _pad8(n):
    return (n + 7) // 8 * 8


def _dtype_message(a: np.ndarray | str):
    """(datatype message body, numpy dtype of the stored elements, element bytes)."""
    if isinstance(a, str):
        b = a.encode()
        size = max(1, len(b) + 1)
        body = bytes([0x13, 0x00, 0x00, 0x00]) + struct.pack("<I", size)  # version 1, string, null-term, ASCII
        return body, None, size
    dt = a.dtype
    if dt.kind == "c":
        f64 = _float_body(8)
        mem = b""
        for name, off in (("r", 0), ("i", 8)):
            nm = name.encode() + b"\x00"
            mem += nm + b"\x00" * (_pad8(len(nm)) - len(nm))
            mem += struct.pack("<I", off) + b"\x00" * 4 + b"\x00" * 4 + b"\x00" * 4 + b"\x00" * 16
            mem += f64
        body = bytes([0x16]) + struct.pack("<H", 2) + b"\x00" + struct.pack("<I", 16) + mem
        return body, np.dtype("<c16"), 16
    if dt.kind == "f":
        return _float_body(dt.itemsize), np.dtype(f"<f{dt.itemsize}"), dt.itemsize
    if dt.kind in "iu":
        bits = 0x08 if dt.kind == "i" else 0x00
        body = bytes([0x10, bits, 0, 0]) + struct.pack("<I", dt.itemsize) + struct.pack("<HH", 0, 8 * dt.itemsize)
        return body, np.dtype(f"<{dt.kind}{dt.itemsize}"), dt.itemsize
    raise TypeError(f"dtype {dt} not handled")


def _float_body(size):
    if size == 8:
        props = struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
        bits = bytes([0x20, 0x3F, 0x00])  # little-endian, mantissa normalised (msb implied), sign bit 63
    elif size == 4:
        props = struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
        bits = bytes([0x20, 0x1F, 0x00])
    else:
        raise TypeError("float32 / float64 only")
    return bytes([0x11]) + bits + struct.pack("<I", size) + props


def _message(mtype, body, flags=0):
    body = body + b"\x00" * (_pad8(len(body)) - len(body))
    return struct.pack("<HHB", mtype, len(body), flags) + b"\x00" * 3 + body


def _object_header(messages):
    data = b"".join(messages)
    return struct.pack("<BBHII", 1, 0, len(messages), 1, len(data)) + b"\x00" * 4 + data


class H5Writer:
    """Collects datasets (``w["/G/GL"] = array``) and writes them as one HDF5 file
    (``w.save(path)``).  Groups are created on the way; complex arrays are stored as the
    compound {r, i} of float64 (the reference's HighFive layout), 0-d values as scalars,
    str as fixed-length strings.  Array data are written straight from the arrays given
    (no copy into one buffer), so a file may be far larger than the free host memory."""

    LEAF_K = 4       # symbol-table node holds up to 2 K entries (the library's defaults)
    INTERNAL_K = 16  # a B-tree node holds up to 2 K children

    def __init__(self):
        self.tree = {}

    def __setitem__(self, path, value):
        parts = [x for x in path.split("/") if x]
        node = self.tree
        for p in parts[:-1]:
            node = node.setdefault(p, {})
            if not isinstance(node, dict):
                raise ValueError(f"{p} is a dataset")
        if isinstance(value, str):
            node[parts[-1]] = value
        else:
            v = np.asarray(value)
            node[parts[-1]] = v if v.flags.c_contiguous else np.ascontiguousarray(v)

    def save(self, path):
        with open(path, "w+b") as fh:
            self._write(fh)

    def _write(self, fh):
        sb_size = 8 + 8 + 4 + 4 + 4 * 8 + 40
        end = [_pad8(sb_size)]

        def alloc(n):
            a = end[0]
            end[0] += _pad8(n)
            return a

        def put(addr, data):
            fh.seek(addr)
            fh.write(data)

        def write_group(children):
            names = sorted(children, key=lambda n: n.encode())
            per = 2 * self.LEAF_K
            if len(names) > per * 2 * self.INTERNAL_K:
                raise ValueError("too many members in one group")
            # local heap: offset 0 is the empty string, then the member names, then a free block
            heap_data = bytearray(b"\x00" * 8)
            offs = {}
            for n in names:
                offs[n] = len(heap_data)
                nb = n.encode() + b"\x00"
                heap_data += nb + b"\x00" * (_pad8(len(nb)) - len(nb))
            free_off = len(heap_data)
            heap_data += struct.pack("<QQ", 1, 16)  # last free block (next = 1), 16 bytes
            data_addr = alloc(len(heap_data))
            put(data_addr, bytes(heap_data))
            heap = alloc(32)
            put(heap, b"HEAP" + bytes([0, 0, 0, 0]) + struct.pack("<QQQ", len(heap_data), free_off, data_addr))
            entries = []
            for n in names:
                v = children[n]
                if isinstance(v, dict):
                    hdr, bt, hp = write_group(v)
                    entries.append(struct.pack("<QQII", offs[n], hdr, 1, 0) + struct.pack("<QQ", bt, hp))
                else:
                    hdr = write_dataset(v)
                    entries.append(struct.pack("<QQII", offs[n], hdr, 0, 0) + b"\x00" * 16)
            # symbol-table nodes of up to 2 LEAF_K entries each, in name order; the B-tree
            # key left of child i is the largest name of child i-1 (key 0: the empty name)
            snods = []
            for i0 in range(0, len(names), per):
                chunk = entries[i0:i0 + per]
                snod = alloc(8 + per * 40)
                put(snod, b"SNOD" + bytes([1, 0]) + struct.pack("<H", len(chunk)) + b"".join(chunk))
                snods.append((snod, offs[names[min(i0 + per, len(names)) - 1]]))
            btree = alloc(24 + (2 * self.INTERNAL_K + 1) * 8 + 2 * self.INTERNAL_K * 8)
            node = b"TREE" + bytes([0, 0]) + struct.pack("<H", len(snods)) + struct.pack("<QQ", UNDEF, UNDEF)
            node += struct.pack("<Q", 0)
            for snod, last in snods:
                node += struct.pack("<QQ", snod, last)
            put(btree, node)
            hdr = alloc(16 + 24 + 8)
            put(hdr, _object_header([_message(0x0011, struct.pack("<QQ", btree, heap))]))
            return hdr, btree, heap

        def write_dataset(v):
            if isinstance(v, str):
                tbody, _, esize = _dtype_message(v)
                raw = v.encode() + b"\x00" * (esize - len(v.encode()))
                nbytes, dims = len(raw), []
            else:
                tbody, dt, esize = _dtype_message(v)
                if v.dtype != dt:
                    v = v.astype(dt)
                raw = memoryview(np.ascontiguousarray(v)).cast("B")
                nbytes, dims = v.nbytes, list(v.shape)
            # dataspace version 1 with the maximum dimensions equal to the dimensions
            dimb = b"".join(struct.pack("<Q", x) for x in dims)
            space = bytes([1, len(dims), 1 if dims else 0, 0]) + b"\x00" * 4 + dimb + (dimb if dims else b"")
            # fill value version 2: allocation late, written if set, defined with the default (size 0)
            fill = bytes([2, 2, 2, 1]) + struct.pack("<I", 0)
            daddr = alloc(nbytes) if nbytes else UNDEF
            if nbytes:
                put(daddr, raw)
            layout = bytes([3, 1]) + struct.pack("<QQ", daddr, nbytes)
            msgs = [_message(0x0001, space), _message(0x0003, tbody, flags=1), _message(0x0005, fill, flags=1),
                    _message(0x0008, layout)]
            oh = _object_header(msgs)
            hdr = alloc(len(oh))
            put(hdr, oh)
            return hdr

        root_hdr, root_bt, root_hp = write_group(self.tree)
        eof = end[0]
        fh.seek(eof - 1)
        fh.write(b"\x00")
        sb = SIG + bytes([0, 0, 0, 0, 0, 8, 8, 0]) + struct.pack("<HH", self.LEAF_K, self.INTERNAL_K)
        sb += struct.pack("<I", 0) + struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
        sb += struct.pack("<QQII", 0, root_hdr, 1, 0) + struct.pack("<QQ", root_bt, root_hp)
        assert len(sb) == sb_size
        put(0, sb)
