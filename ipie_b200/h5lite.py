"""A small HDF5 reader and writer (numpy only) for the files ipie exchanges.

ipie reads its Hamiltonians and trial wavefunctions from HDF5 through h5py
(``utils/io.py``); h5py is not part of this package's environment, so this
module implements the subset of the HDF5 file format those files use, from the
published format specification:

* superblock versions 0-3 (offsets and lengths of any size);
* groups stored as symbol tables (version-1 B-tree of type 0, local heap,
  symbol-table nodes) and compact groups of link messages;
* version-1 and version-2 object headers with continuation blocks;
* datasets with simple or scalar dataspaces, fixed-point, floating-point,
  fixed-length string, compound (complex numbers are h5py's ``{r, i}``
  compound), enum and array datatypes, and contiguous, compact or chunked
  (version-1 B-tree of type 1) layouts with the deflate, shuffle and
  fletcher32 filters.

Variable-length strings and sequences (global heap) are read.  Not supported
(``NotImplementedError``): dense link storage (fractal heaps), version-4 chunk
indexes.  The writer produces the
oldest format every HDF5 release reads: superblock 0, version-1 object
headers, symbol-table groups, contiguous datasets.

The reading API mirrors the part of h5py that ipie uses: ``File(path)`` as a
context manager, ``group["a/b"]``, ``keys()``, ``in``, ``dataset[()]``,
``dataset[:]``, ``shape``, ``dtype``.
"""
from __future__ import annotations

import struct
import zlib

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"


class _Reader:
    """Byte-level access with the file's offset and length sizes."""

    def __init__(self, data: bytes):
        self.b = data
        self.so = 8
        self.sl = 8
        self.base = 0

    def u8(self, p):
        return self.b[p]

    def u16(self, p):
        return struct.unpack_from("<H", self.b, p)[0]

    def u32(self, p):
        return struct.unpack_from("<I", self.b, p)[0]

    def uint(self, p, n):
        return int.from_bytes(self.b[p:p + n], "little")

    def off(self, p):
        return self.uint(p, self.so)

    def length(self, p):
        return self.uint(p, self.sl)

    def undef(self, v, n=None):
        return v == (1 << (8 * (n or self.so))) - 1

    def cstr(self, p):
        e = self.b.index(b"\0", p)
        return self.b[p:e].decode("utf-8")


# ---------------------------------------------------------------------------- datatypes
def _parse_dtype(r: _Reader, p: int):
    """Datatype message at p -> (numpy dtype, end position)."""
    cv = r.u8(p)
    cls, ver = cv & 0x0F, cv >> 4
    bits = r.u8(p + 1) | (r.u8(p + 2) << 8) | (r.u8(p + 3) << 16)
    size = r.u32(p + 4)
    q = p + 8
    order = ">" if bits & 1 else "<"
    if cls == 0:  # fixed point
        kind = "i" if bits & 0x08 else "u"
        return np.dtype(f"{order}{kind}{size}"), q + 4
    if cls == 1:  # floating point
        if size not in (2, 4, 8):
            raise NotImplementedError(f"floating-point size {size}")
        return np.dtype(f"{order}f{size}"), q + 12
    if cls == 3:  # fixed-length string
        return np.dtype(f"S{size}"), q
    if cls == 4:  # bitfield
        return np.dtype(f"{order}u{size}"), q + 4
    if cls == 5:  # opaque: tag, null-terminated, padded to 8
        taglen = bits & 0xFF
        return np.dtype(f"V{size}"), q + taglen
    if cls == 6:  # compound
        n = bits & 0xFFFF
        names, formats, offsets = [], [], []
        for _ in range(n):
            name = r.cstr(q)
            nl = len(name.encode()) + 1
            if ver < 3:
                q += (nl + 7) // 8 * 8
                offset = r.u32(q)
                q += 4
                if ver == 1:
                    ndim = r.u8(q)
                    q += 4 + 4 + 4 + 16  # dimensionality + reserved, permutation, reserved, dims
                    dims = [r.u32(q - 16 + 4 * i) for i in range(ndim)]
                else:
                    dims = []
            else:
                q += nl
                nb = 1 if size < 256 else 2 if size < 65536 else 3 if size < (1 << 24) else 4
                offset = r.uint(q, nb)
                q += nb
                dims = []
            mt, q = _parse_dtype(r, q)
            if dims:
                mt = np.dtype((mt, tuple(dims)))
            names.append(name)
            formats.append(mt)
            offsets.append(offset)
        dt = np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": size})
        return dt, q
    if cls == 8:  # enum: base type, then names and values
        n = bits & 0xFFFF
        base, q = _parse_dtype(r, q)
        for _ in range(n):
            name = r.cstr(q)
            nl = len(name.encode()) + 1
            q += nl if ver >= 3 else (nl + 7) // 8 * 8
        q += n * base.itemsize
        return base, q
    if cls == 9:  # variable length: element = length (4), global-heap collection address, object index (4)
        base, q = _parse_dtype(r, q)
        return _VLen(base, (bits & 0x0F) == 1, size), q
    if cls == 10:  # array
        ndim = r.u8(q)
        q += 1 if ver >= 3 else 4
        dims = [r.u32(q + 4 * i) for i in range(ndim)]
        q += 4 * ndim
        if ver < 3:
            q += 4 * ndim  # permutation
        base, q = _parse_dtype(r, q)
        return np.dtype((base, tuple(dims))), q
    raise NotImplementedError(f"HDF5 datatype class {cls}")


class _VLen:
    """A variable-length datatype (strings or sequences of ``base``); elements live in global heaps."""

    def __init__(self, base, is_string, size):
        self.base, self.is_string, self.itemsize = base, is_string, size
        self.kind = "O"
        self.names = None

    def newbyteorder(self, *_):
        return self


def _as_complex(dt):
    """h5py's complex numbers: a compound of two equal floats named r and i."""
    if dt.names is not None and len(dt.names) == 2 and set(dt.names) == {"r", "i"}:
        fr, ori = dt.fields["r"]
        fi, oi = dt.fields["i"]
        if fr == fi and fr.kind == "f" and ori == 0 and oi == fr.itemsize and dt.itemsize == 2 * fr.itemsize:
            return np.dtype(f"{fr.byteorder if fr.byteorder in '<>' else '<'}c{2 * fr.itemsize}")
    return None


# ---------------------------------------------------------------------------- objects
class _Object:
    def __init__(self, f: "File", addr: int, name: str):
        self.file = f
        self.addr = addr
        self.name = name
        self._msgs = f._messages(addr)

    def _find(self, mtype):
        return [(fl, p, n) for t, fl, p, n in self._msgs if t == mtype]


class Dataset(_Object):
    def __init__(self, f, addr, name):
        super().__init__(f, addr, name)
        r = f._r
        (_, p, _), = self._find(0x0001)
        self.shape = f._dataspace(p)
        (_, p, _), = self._find(0x0003)
        self._raw_dtype, _ = _parse_dtype(r, p)
        cdt = _as_complex(self._raw_dtype)
        self.dtype = cdt if cdt is not None else self._raw_dtype
        (_, p, _), = self._find(0x0008)
        self._layout = p
        filt = self._find(0x000B)
        self._filters = f._filters(filt[0][1]) if filt else []
        self._value = None

    @property
    def ndim(self):
        return len(self.shape)

    @property
    def size(self):
        return int(np.prod(self.shape)) if self.shape else 1

    def _read(self):
        if self._value is not None:
            return self._value
        f, r, p = self.file, self.file._r, self._layout
        dt = self._raw_dtype
        nbytes = self.size * dt.itemsize
        ver = r.u8(p)
        if ver in (1, 2):
            ndim = r.u8(p + 1)
            cls = r.u8(p + 2)
            q = p + 8
            if cls == 0:
                q += 4 * ndim
                size = r.u32(q)
                raw = r.b[q + 4:q + 4 + size]
            elif cls == 1:
                addr = r.off(q)
                raw = self._contiguous(addr, nbytes)
            else:
                addr = r.off(q)
                q += r.so
                cdims = [r.u32(q + 4 * i) for i in range(ndim)]
                raw = self._chunked(addr, cdims)
        elif ver == 3 or ver == 4:
            cls = r.u8(p + 1)
            q = p + 2
            if cls == 0:
                size = r.u16(q)
                raw = r.b[q + 2:q + 2 + size]
            elif cls == 1:
                raw = self._contiguous(r.off(q), nbytes)
            elif cls == 2 and ver == 3:
                ndim = r.u8(q)
                addr = r.off(q + 1)
                q += 1 + r.so
                cdims = [r.u32(q + 4 * i) for i in range(ndim)]
                raw = self._chunked(addr, cdims)
            else:
                raise NotImplementedError(f"HDF5 layout version {ver} class {cls}")
        else:
            raise NotImplementedError(f"HDF5 layout version {ver}")
        if isinstance(dt, _VLen):
            self._value = self._vlen(bytes(raw[:nbytes]), dt)
            return self._value
        arr = np.frombuffer(bytes(raw[:nbytes]), dtype=dt, count=self.size).reshape(self.shape)
        cdt = _as_complex(dt)
        if cdt is not None:
            out = np.empty(self.shape, dtype=cdt)
            out.real = arr["r"]
            out.imag = arr["i"]
            arr = out
        self._value = np.array(arr, dtype=arr.dtype.newbyteorder("=")) if arr.dtype.kind in "iufc" else arr.copy()
        return self._value

    def _vlen(self, raw, dt):
        """Resolve each element's global-heap object: bytes for strings, arrays for sequences."""
        r = self.file._r
        out = np.empty(self.size, dtype=object)
        for i in range(self.size):
            e = i * dt.itemsize
            n = struct.unpack_from("<I", raw, e)[0]
            coll = int.from_bytes(raw[e + 4:e + 4 + r.so], "little")
            idx = struct.unpack_from("<I", raw, e + 4 + r.so)[0]
            data = self.file._global_heap_object(coll, idx) if n else b""
            if dt.is_string:
                out[i] = data[:n]
            else:
                out[i] = np.frombuffer(data, dtype=dt.base, count=n).copy()
        return out.reshape(self.shape) if self.shape else out[0]

    def _contiguous(self, addr, nbytes):
        r = self.file._r
        if r.undef(addr):
            return bytes(nbytes)  # never written: the (zero) fill value
        a = r.base + addr
        return r.b[a:a + nbytes]

    def _chunked(self, btree, cdims):
        """Chunks indexed by a version-1 B-tree of type 1; cdims = chunk dims + element size."""
        r = self.file._r
        rank = len(self.shape)
        item = self._raw_dtype.itemsize
        out = np.zeros(self.size * item, dtype=np.uint8).reshape(tuple(self.shape) + (item,)) if rank else None
        chunk_shape = tuple(cdims[:rank])
        if r.undef(btree):
            return bytes(self.size * item)

        def visit(node):
            assert r.b[r.base + node:r.base + node + 4] == b"TREE", "bad chunk B-tree node"
            a = r.base + node
            level = r.u8(a + 5)
            used = r.u16(a + 6)
            q = a + 8 + 2 * r.so
            ksize = 8 + 8 * (rank + 1)
            for _ in range(used):
                csize = r.u32(q)
                mask = r.u32(q + 4)
                offs = [r.uint(q + 8 + 8 * i, 8) for i in range(rank)]
                child = r.off(q + ksize)
                q += ksize + r.so
                if level > 0:
                    visit(child)
                    continue
                data = r.b[r.base + child:r.base + child + csize]
                data = self._unfilter(data, mask)
                blk = np.frombuffer(data, dtype=np.uint8, count=int(np.prod(chunk_shape)) * item)
                blk = blk.reshape(chunk_shape + (item,))
                sl = tuple(slice(o, min(o + c, s)) for o, c, s in zip(offs, chunk_shape, self.shape))
                sub = tuple(slice(0, s.stop - s.start) for s in sl)
                out[sl] = blk[sub]

        visit(btree)
        return out.tobytes()

    def _unfilter(self, data, mask):
        item = self._raw_dtype.itemsize
        for i, (fid, vals) in reversed(list(enumerate(self._filters))):
            if mask & (1 << i):
                continue
            if fid == 1:
                data = zlib.decompress(data)
            elif fid == 2:
                n = len(data) // item
                a = np.frombuffer(data[: n * item], dtype=np.uint8).reshape(item, n)
                data = a.T.tobytes() + data[n * item:]
            elif fid == 3:
                data = data[:-4]
            else:
                raise NotImplementedError(f"HDF5 filter {fid}")
        return data

    def __getitem__(self, key):
        v = self._read()
        if key == () or key is Ellipsis:
            return v[()] if v.ndim == 0 else v
        return v[key]

    def __array__(self, dtype=None, copy=None):
        v = self._read()
        return v.astype(dtype) if dtype is not None else v

    def __len__(self):
        return self.shape[0]


class Group(_Object):
    def __init__(self, f, addr, name, cached_stab=None):
        super().__init__(f, addr, name)
        self._links = None
        self._cached = cached_stab

    def _entries(self):
        if self._links is not None:
            return self._links
        f = self.file
        links = {}
        stab = self._find(0x0011)
        if stab:
            p = stab[0][1]
            links.update(f._symbol_table(f._r.off(p), f._r.off(p + f._r.so)))
        elif self._cached is not None:
            links.update(f._symbol_table(*self._cached))
        for _, p, _ in self._find(0x0006):
            name, addr = f._link(p)
            if addr is not None:
                links[name] = addr
        for _, p, _ in self._find(0x0002):
            if f._link_info_dense(p):
                raise NotImplementedError("HDF5 groups in dense (fractal heap) storage")
        self._links = links
        return links

    def keys(self):
        return list(self._entries().keys())

    def __iter__(self):
        return iter(self.keys())

    def __contains__(self, key):
        try:
            self[key]
            return True
        except KeyError:
            return False

    def __getitem__(self, key):
        parts = [k for k in key.split("/") if k]
        obj = self
        for k in parts:
            if not isinstance(obj, Group):
                raise KeyError(key)
            ent = obj._entries()
            if k not in ent:
                raise KeyError(key)
            obj = obj.file._open(ent[k], obj.name.rstrip("/") + "/" + k)
        return obj


class File(Group):
    """Read-only HDF5 file (``with File(path) as f: f["x"][()]``)."""

    def __init__(self, path, mode="r"):
        if mode != "r":
            raise ValueError("h5lite.File reads only; use write_file to write")
        with open(path, "rb") as fh:
            data = fh.read()
        r = _Reader(data)
        self._r = r
        self._objs = {}
        sb = None
        for s in [0] + [512 << i for i in range(24)]:
            if s + 8 <= len(data) and data[s:s + 8] == SIGNATURE:
                sb = s
                break
            if s > len(data):
                break
        if sb is None:
            raise OSError(f"{path}: not an HDF5 file")
        ver = r.u8(sb + 8)
        cached = None
        if ver in (0, 1):
            r.so, r.sl = r.u8(sb + 13), r.u8(sb + 14)
            q = sb + 24 + (4 if ver == 1 else 0)
            r.base = r.off(q) + sb
            q += 4 * r.so
            root = r.off(q + r.so)  # symbol-table entry: name offset, object header address
            if r.u32(q + 2 * r.so) == 1:
                cached = (r.off(q + 2 * r.so + 8), r.off(q + 2 * r.so + 8 + r.so))
        elif ver in (2, 3):
            r.so, r.sl = r.u8(sb + 9), r.u8(sb + 10)
            q = sb + 12
            r.base = r.off(q) + sb
            root = r.off(q + 3 * r.so)
        else:
            raise NotImplementedError(f"HDF5 superblock version {ver}")
        Group.__init__(self, self, root, "/", cached)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def close(self):
        self._objs.clear()

    # -- object headers
    def _messages(self, addr):
        r = self._r
        a = r.base + addr
        msgs = []
        if r.b[a:a + 4] == b"OHDR":
            flags = r.u8(a + 5)
            q = a + 6
            if flags & 0x20:
                q += 16
            if flags & 0x10:
                q += 4
            nsz = 1 << (flags & 3)
            size0 = r.uint(q, nsz)
            q += nsz
            blocks = [(q, size0)]
            while blocks:
                start, ln = blocks.pop(0)
                p, end = start, start + ln
                while p + 4 <= end:
                    mtype = r.u8(p)
                    msize = r.u16(p + 1)
                    mfl = r.u8(p + 3)
                    p += 4 + (2 if flags & 0x04 else 0)
                    if mtype == 0x10:
                        blocks.append((r.base + r.off(p) + 4, r.length(p + r.so) - 8))  # skip OCHK, checksum
                    elif mtype != 0:
                        msgs.append((mtype, mfl, p, msize))
                    p += msize
            return msgs
        if r.u8(a) != 1:
            raise NotImplementedError(f"HDF5 object header version {r.u8(a)}")
        size = r.u32(a + 8)
        blocks = [(a + 16, size)]
        while blocks:
            start, ln = blocks.pop(0)
            p, end = start, start + ln
            while p + 8 <= end:
                mtype = r.u16(p)
                msize = r.u16(p + 2)
                mfl = r.u8(p + 4)
                p += 8
                if mtype == 0x10:
                    blocks.append((r.base + r.off(p), r.length(p + r.so)))
                elif mtype != 0:
                    msgs.append((mtype, mfl, p, msize))
                p += msize
        return msgs

    def _open(self, addr, name):
        obj = self._objs.get(addr)
        if obj is None:
            kinds = {t for t, _, _, _ in self._messages(addr)}
            obj = Dataset(self, addr, name) if 0x0008 in kinds else Group(self, addr, name)
            self._objs[addr] = obj
        return obj

    def _global_heap_object(self, coll, idx):
        r = self._r
        a = r.base + coll
        assert r.b[a:a + 4] == b"GCOL", "bad global heap collection"
        end = a + r.length(a + 8)
        q = a + 8 + r.sl
        while q + 8 + r.sl <= end:
            oid = r.u16(q)
            size = r.length(q + 8)
            if oid == idx:
                return r.b[q + 8 + r.sl:q + 8 + r.sl + size]
            if oid == 0:
                break
            q += 8 + r.sl + (size + 7) // 8 * 8
        raise KeyError(f"global heap object {idx} not found")

    def _dataspace(self, p):
        r = self._r
        ver = r.u8(p)
        ndim = r.u8(p + 1)
        if ver == 1:
            q = p + 8
        elif ver == 2:
            if r.u8(p + 3) == 2:
                return None  # null dataspace
            q = p + 4
        else:
            raise NotImplementedError(f"HDF5 dataspace version {ver}")
        return tuple(r.length(q + r.sl * i) for i in range(ndim))

    def _filters(self, p):
        r = self._r
        ver = r.u8(p)
        n = r.u8(p + 1)
        q = p + (8 if ver == 1 else 2)
        out = []
        for _ in range(n):
            fid = r.u16(q)
            q += 2
            nlen = 0
            if ver == 1 or fid >= 256:
                nlen = r.u16(q)
                q += 2
            q += 2  # flags
            nval = r.u16(q)
            q += 2
            if ver == 1:
                q += (nlen + 7) // 8 * 8
            else:
                q += nlen
            vals = [r.u32(q + 4 * i) for i in range(nval)]
            q += 4 * nval
            if ver == 1 and nval % 2:
                q += 4
            out.append((fid, vals))
        return out

    # -- groups
    def _symbol_table(self, btree, heap):
        r = self._r
        h = r.base + heap
        assert r.b[h:h + 4] == b"HEAP", "bad local heap"
        data = r.base + r.off(h + 8 + 2 * r.sl)
        out = {}

        def visit(node):
            a = r.base + node
            assert r.b[a:a + 4] == b"TREE", "bad group B-tree node"
            level = r.u8(a + 5)
            used = r.u16(a + 6)
            q = a + 8 + 2 * r.so + r.sl
            for _ in range(used):
                child = r.off(q)
                q += r.so + r.sl
                if level > 0:
                    visit(child)
                else:
                    snod(child)

        def snod(node):
            a = r.base + node
            assert r.b[a:a + 4] == b"SNOD", "bad symbol-table node"
            n = r.u16(a + 6)
            q = a + 8
            for _ in range(n):
                name = r.cstr(data + r.off(q))
                out[name] = r.off(q + r.so)
                q += 2 * r.so + 24

        visit(btree)
        return out

    def _link(self, p):
        r = self._r
        fl = r.u8(p + 1)
        q = p + 2
        ltype = 0
        if fl & 0x08:
            ltype = r.u8(q)
            q += 1
        if fl & 0x04:
            q += 8
        if fl & 0x10:
            q += 1
        nb = 1 << (fl & 3)
        nlen = r.uint(q, nb)
        q += nb
        name = r.b[q:q + nlen].decode("utf-8")
        q += nlen
        return name, (r.off(q) if ltype == 0 else None)

    def _link_info_dense(self, p):
        r = self._r
        fl = r.u8(p + 1)
        q = p + 2 + (8 if fl & 1 else 0)
        return not r.undef(r.off(q))


# ---------------------------------------------------------------------------- writer
_UNDEF8 = b"\xff" * 8


def _pad8(b: bytes) -> bytes:
    return b + bytes((-len(b)) % 8)


def _dtype_msg(dt: np.dtype) -> bytes:
    """Datatype message (version 1 encodings) for numeric numpy dtypes and complex."""
    dt = np.dtype(dt)
    if dt.kind == "c":
        half = np.dtype(f"<f{dt.itemsize // 2}")
        members = b""
        for name, off in (("r", 0), ("i", half.itemsize)):
            members += _pad8(name.encode() + b"\0") + struct.pack("<IB3xI4x16x", off, 0, 0) + _dtype_msg(half)
        return struct.pack("<BBBBI", 0x16, 2, 0, 0, dt.itemsize) + members
    if dt.kind == "f":
        prec = dt.itemsize * 8
        eloc, esize, msize, bias = {4: (23, 8, 23, 127), 8: (52, 11, 52, 1023)}[dt.itemsize]
        return struct.pack("<BBBBIHHBBBBI", 0x11, 0x20, prec - 1, 0, dt.itemsize, 0, prec, eloc, esize, 0, msize, bias)
    if dt.kind in "iu":
        return struct.pack("<BBBBIHH", 0x10, 0x08 if dt.kind == "i" else 0, 0, 0, dt.itemsize, 0, dt.itemsize * 8)
    if dt.kind == "b":
        return _dtype_msg(np.dtype("u1"))
    if dt.kind == "S":
        return struct.pack("<BBBBI", 0x13, 0, 0, 0, dt.itemsize)
    raise NotImplementedError(f"writing dtype {dt}")


def _message(mtype: int, data: bytes, flags: int = 0) -> bytes:
    data = _pad8(data)
    return struct.pack("<HHB3x", mtype, len(data), flags) + data


def _object_header(msgs: list) -> bytes:
    body = b"".join(msgs)
    return struct.pack("<BBHII4x", 1, 0, len(msgs), 1, len(body)) + body


class _Writer:
    def __init__(self, leaf_k):
        self.buf = bytearray()
        self.leaf_k = leaf_k
        self.internal_k = 16

    def alloc(self, n: int) -> int:
        a = len(self.buf)
        self.buf += bytes(n + ((-n) % 8))
        return a

    def put(self, addr: int, data: bytes):
        self.buf[addr:addr + len(data)] = data

    def dataset(self, arr: np.ndarray) -> int:
        arr = np.asarray(arr)
        if arr.dtype.kind == "U":
            arr = arr.astype("S")
        if arr.dtype.kind in "iufcb":
            arr = arr.astype(arr.dtype.newbyteorder("<"))
        if arr.dtype.kind == "c":
            raw = np.ascontiguousarray(arr).view(np.dtype(f"<f{arr.dtype.itemsize // 2}")).tobytes()
        else:
            raw = np.ascontiguousarray(arr).tobytes()
        if arr.ndim == 0:
            space = struct.pack("<BBBB", 2, 0, 0, 0)
        else:
            space = struct.pack("<BBBB", 2, arr.ndim, 0, 1) + b"".join(struct.pack("<Q", d) for d in arr.shape)
        daddr = self.alloc(len(raw)) if raw else None
        if raw:
            self.put(daddr, raw)
        layout = struct.pack("<BB", 3, 1) + (struct.pack("<Q", daddr) if raw else _UNDEF8) + struct.pack("<Q", len(raw))
        fill = struct.pack("<BBBB", 2, 2, 0, 0)  # version 2, late allocation, fill at allocation, undefined
        hdr = _object_header([_message(0x0001, space), _message(0x0003, _dtype_msg(arr.dtype), 1),
                              _message(0x0005, fill, 1), _message(0x0008, layout)])
        a = self.alloc(len(hdr))
        self.put(a, hdr)
        return a

    def group(self, tree: dict):
        """Returns (object header address, B-tree address, heap address)."""
        items = sorted(tree.items(), key=lambda kv: kv[0].encode())
        if len(items) > 2 * self.leaf_k:
            raise ValueError("group larger than one symbol-table node")
        children = []
        for name, val in items:
            if isinstance(val, dict):
                oh, bt, hp = self.group(val)
                children.append((name, oh, (bt, hp)))
            else:
                children.append((name, self.dataset(val), None))
        # local heap: offset 0 is the empty name
        names = b"\0" * 8
        offs = []
        for name, _, _ in children:
            offs.append(len(names))
            names += _pad8(name.encode() + b"\0")
        hdata = self.alloc(len(names))
        self.put(hdata, names)
        heap = self.alloc(32)
        self.put(heap, b"HEAP" + struct.pack("<B3xQ", 0, len(names)) + _UNDEF8 + struct.pack("<Q", hdata))
        # one symbol-table node of full capacity
        snod = self.alloc(8 + 2 * self.leaf_k * 40)
        ents = b""
        for (name, oh, cache), off in zip(children, offs):
            if cache is None:
                ents += struct.pack("<QQII16x", off, oh, 0, 0)
            else:
                ents += struct.pack("<QQII", off, oh, 1, 0) + struct.pack("<QQ", *cache)
        self.put(snod, b"SNOD" + struct.pack("<BBH", 1, 0, len(children)) + ents)
        # B-tree leaf (type 0) of full capacity: key 0, child, key = last name
        bt = self.alloc(8 + 16 + (2 * self.internal_k + 1) * 8 + 2 * self.internal_k * 8)
        if children:
            body = struct.pack("<QQQ", 0, snod, offs[-1])
            self.put(bt, b"TREE" + struct.pack("<BBH", 0, 0, 1) + _UNDEF8 + _UNDEF8 + body)
        else:
            self.put(bt, b"TREE" + struct.pack("<BBH", 0, 0, 0) + _UNDEF8 + _UNDEF8 + struct.pack("<Q", 0))
        hdr = _object_header([_message(0x0011, struct.pack("<QQ", bt, heap))])
        oh = self.alloc(len(hdr))
        self.put(oh, hdr)
        return oh, bt, heap


def _max_group(tree: dict) -> int:
    n = len(tree)
    for v in tree.values():
        if isinstance(v, dict):
            n = max(n, _max_group(v))
    return n


def write_file(path, tree: dict):
    """Write a nested dict (names -> numpy arrays, scalars or dicts) as an HDF5 file."""
    tree = {k: (v if isinstance(v, dict) else np.asarray(v)) for k, v in tree.items()}
    w = _Writer(leaf_k=max(4, (_max_group(tree) + 1) // 2))
    w.alloc(96)  # superblock 0 with the root symbol-table entry
    oh, bt, heap = w.group(tree)
    sb = SIGNATURE + struct.pack("<BBBBBBBBHHI", 0, 0, 0, 0, 0, 8, 8, 0, w.leaf_k, w.internal_k, 0)
    sb += struct.pack("<Q", 0) + _UNDEF8 + struct.pack("<Q", len(w.buf)) + _UNDEF8
    sb += struct.pack("<QQII", 0, oh, 1, 0) + struct.pack("<QQ", bt, heap)
    w.put(0, sb)
    with open(path, "wb") as fh:
        fh.write(bytes(w.buf))
