"""A small HDF5 reader/writer for snapshot files, used by ``H5Saver`` when
h5py is not importable.

It implements the part of the published HDF5 file format (HDF Group, "HDF5
File Format Specification", version 2 / 3 documents) that snapshot files
need, with an h5py-like surface (``File``, ``Group``, ``Dataset``,
``attrs``):

* writes the classic layout every HDF5 library reads: superblock version 0,
  version-1 object headers, symbol-table groups (version-1 B-tree of type 0,
  symbol-table nodes, a local heap of names), attributes (version-1 messages),
  datasets with version-1 dataspace and numeric datatype messages and a
  version-3 layout (contiguous, or one chunk with the deflate filter, as
  ``compression="gzip"`` asks);
* reads the same, plus what h5py writes by default: continuation messages,
  attribute messages 1-3, dataspace 1-2, chunked datasets indexed by a
  version-1 B-tree of type 1 with deflate / shuffle filters, compact link
  messages of version-2 object headers.

Writes are append-only: every flush writes the new objects and a new root
group at the end of the file and then rewrites the 96-byte superblock, so
existing snapshot data is never copied.  A deleted link leaves its objects
as unreachable bytes, as in HDF5 itself.
"""
import os
import struct
import zlib

import numpy as np

SIG = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF
FREE_NULL = 1          # end of a local heap's free list on disk
K_LEAF, K_INT = 32, 64  # symbol-table node capacity 2*K_LEAF, B-tree fan-out 2*K_INT (written files)
K_CHUNK = 32            # chunk B-tree K of a version-0 superblock (fixed by the format)
MSG_NIL, MSG_SPACE, MSG_LINKINFO, MSG_TYPE, MSG_FILL, MSG_LINK, MSG_LAYOUT = 0, 1, 2, 3, 5, 6, 8
MSG_FILTER, MSG_ATTR, MSG_CONT, MSG_STAB = 11, 12, 16, 17


def _pad8(b):
    return b + b"\0" * (-len(b) % 8)


# ----------------------------------------------------------------- datatypes
def _encode_dtype(dt):
    dt = np.dtype(dt)
    big = dt.byteorder == ">"
    if dt.kind == "f" and dt.itemsize in (4, 8):
        if dt.itemsize == 8:
            props = struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
        else:
            props = struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
        return struct.pack("<BBBBI", 0x11, 0x20 | int(big), 8 * dt.itemsize - 1, 0, dt.itemsize) + props
    if dt.kind in "iu":
        bits0 = (0x08 if dt.kind == "i" else 0) | int(big)
        return struct.pack("<BBBBI", 0x10, bits0, 0, 0, dt.itemsize) + struct.pack("<HH", 0, 8 * dt.itemsize)
    if dt.kind == "S":
        return struct.pack("<BBBBI", 0x13, 0, 0, 0, dt.itemsize)  # null-terminated ASCII
    raise TypeError(f"h5lite cannot store dtype {dt}")


def _decode_dtype(b):
    cls, ver = b[0] & 0x0F, b[0] >> 4
    bits = b[1] | (b[2] << 8) | (b[3] << 16)
    size = struct.unpack_from("<I", b, 4)[0]
    order = ">" if bits & 1 else "<"
    if cls == 0:
        return np.dtype(f"{order}{'i' if bits & 8 else 'u'}{size}")
    if cls == 1:
        return np.dtype(f"{order}f{size}")
    if cls == 3:
        return np.dtype(f"S{size}")
    raise NotImplementedError(f"HDF5 datatype class {cls} (version {ver})")


# ----------------------------------------------------------------- messages
def _space_msg(shape):
    return struct.pack("<BBBB4x", 1, len(shape), 0, 0) + b"".join(struct.pack("<Q", d) for d in shape)


def _decode_space(b):
    ver, rank, flags = b[0], b[1], b[2]
    off = 8 if ver == 1 else 4
    if ver == 2 and b[3] == 2:
        return None  # null dataspace
    return tuple(struct.unpack_from(f"<{rank}Q", b, off)) if rank else ()


def _ohdr(msgs):
    """Version-1 object header: (type, flags, data) messages, 8-byte aligned."""
    body = b""
    for t, fl, data in msgs:
        data = _pad8(data)
        body += struct.pack("<HHB3x", t, len(data), fl) + data
    return struct.pack("<BBHII4x", 1, 0, len(msgs), 1, len(body)) + body


def _attr_msg(name, value):
    v = np.asarray(value)
    if v.dtype.kind == "U":
        v = np.asarray(v.astype("S"))
    if v.dtype.kind == "b":
        v = v.astype(np.int8)
    if v.dtype.byteorder == "=":
        v = v.astype(v.dtype.newbyteorder("<"))
    nm = name.encode() + b"\0"
    dt, sp = _encode_dtype(v.dtype), _space_msg(v.shape)
    return (struct.pack("<BBHHH", 1, 0, len(nm), len(dt), len(sp)) + _pad8(nm) + _pad8(dt) + _pad8(sp)
            + np.ascontiguousarray(v).tobytes())


def _decode_attr(b):
    ver = b[0]
    nlen, tlen, slen = struct.unpack_from("<HHH", b, 2)
    off = 8 if ver != 3 else 9
    pad = _pad8 if ver == 1 else (lambda x: x)
    name = b[off:off + nlen].split(b"\0", 1)[0].decode()
    off += len(pad(b"\0" * nlen))
    dt = _decode_dtype(b[off:off + tlen])
    off += len(pad(b"\0" * tlen))
    shape = _decode_space(b[off:off + slen])
    off += len(pad(b"\0" * slen))
    n = int(np.prod(shape)) if shape else 1
    arr = np.frombuffer(b, dtype=dt, count=n, offset=off).reshape(shape if shape else ())
    val = arr.astype(dt.newbyteorder("=")) if dt.kind in "iuf" else arr
    return name, (val[()] if val.ndim == 0 else val.copy())


def _filter_msg_deflate(level):
    name = _pad8(b"deflate\0")
    return (struct.pack("<BB6x", 1, 1) + struct.pack("<HHHH", 1, len(name), 1, 1) + name
            + struct.pack("<I4x", level))


def _decode_filters(b):
    ver, n = b[0], b[1]
    off = 8 if ver == 1 else 2
    out = []
    for _ in range(n):
        fid = struct.unpack_from("<H", b, off)[0]
        if ver == 1 or fid >= 256:
            nlen, flags, ncd = struct.unpack_from("<HHH", b, off + 2)
            off += 8
        else:
            nlen = 0
            flags, ncd = struct.unpack_from("<HH", b, off + 2)
            off += 6
        off += len(_pad8(b"\0" * nlen)) if ver == 1 else nlen
        cd = struct.unpack_from(f"<{ncd}I", b, off)
        off += 4 * ncd + (4 if ver == 1 and ncd % 2 else 0)
        out.append((fid, cd))
    return out


# ----------------------------------------------------------------- reading
class _Reader:
    def __init__(self, f):
        self.f = f
        f.seek(0)
        sb = f.read(128)
        if sb[:8] != SIG:
            raise OSError("not an HDF5 file (no signature at offset 0)")
        ver = sb[8]
        if ver not in (0, 1):
            raise NotImplementedError(f"HDF5 superblock version {ver}")
        if sb[13] != 8 or sb[14] != 8:
            raise NotImplementedError("HDF5 offsets / lengths other than 8 bytes")
        off = 24 + (4 if ver == 1 else 0)
        self.eof = struct.unpack_from("<Q", sb, off + 16)[0]
        self.root_addr = struct.unpack_from("<Q", sb, off + 32 + 8)[0]

    def read(self, addr, n):
        self.f.seek(addr)
        b = self.f.read(n)
        if len(b) != n:
            raise OSError(f"truncated HDF5 file at {addr}")
        return b

    def messages(self, addr):
        """[(type, data)] of the object header at addr (versions 1 and 2)."""
        head = self.read(addr, 16)
        out, blocks = [], []
        if head[:4] == b"OHDR":
            flags = head[5]
            off = 6 + (16 if flags & 0x20 else 0) + (4 if flags & 0x10 else 0)
            w = 1 << (flags & 3)
            size = int.from_bytes(self.read(addr + off, w), "little")
            blocks.append((addr + off + w, size, 2, flags))  # chunk 0: messages only
        elif head[0] == 1:
            size = struct.unpack_from("<I", head, 8)[0]
            blocks.append((addr + 16, size, 1, 0))
        else:
            raise NotImplementedError(f"HDF5 object header version {head[0]}")
        while blocks:
            start, size, ver, flags = blocks.pop(0)
            b = self.read(start, size)
            p, end = 0, size
            if ver == 2 and b[:4] == b"OCHK":  # continuation: signature ... checksum
                p, end = 4, size - 4
            while p + (4 if ver == 2 else 8) <= end:
                if ver == 1:
                    t, n = struct.unpack_from("<HH", b, p)
                    p += 8
                else:
                    t, n = b[p], struct.unpack_from("<H", b, p + 1)[0]
                    p += 4 + (2 if flags & 0x04 else 0)
                data = b[p:p + n]
                p += n
                if t == MSG_CONT:
                    caddr, clen = struct.unpack_from("<QQ", data)
                    blocks.append((caddr, clen, ver, flags))
                elif t != MSG_NIL:
                    out.append((t, data))
        return out

    def heap_name(self, heap_addr, off):
        h = self.read(heap_addr, 32)
        if h[:4] != b"HEAP":
            raise OSError("bad local heap")
        data_addr = struct.unpack_from("<Q", h, 24)[0]
        self.f.seek(data_addr + off)
        s = b""
        while b"\0" not in s:
            s += self.f.read(64)
        return s.split(b"\0", 1)[0].decode()

    def stab_links(self, btree, heap):
        links = {}
        stack = [btree]
        while stack:
            a = stack.pop()
            h = self.read(a, 24)
            if h[:4] != b"TREE" or h[4] != 0:
                raise OSError("bad group B-tree node")
            level, n = h[5], struct.unpack_from("<H", h, 6)[0]
            body = self.read(a + 24, n * 16 + 8)
            kids = [struct.unpack_from("<Q", body, 8 + 16 * i)[0] for i in range(n)]
            if level > 0:
                stack.extend(kids)
                continue
            for s in kids:
                sh = self.read(s, 8)
                if sh[:4] != b"SNOD":
                    raise OSError("bad symbol table node")
                nsym = struct.unpack_from("<H", sh, 6)[0]
                ent = self.read(s + 8, 40 * nsym)
                for i in range(nsym):
                    noff, oaddr = struct.unpack_from("<QQ", ent, 40 * i)
                    links[self.heap_name(heap, noff)] = oaddr
        return links

    def chunks(self, btree, ndims):
        """[(offsets, size, filter_mask, address)] of a chunk B-tree (type 1)."""
        ks = 8 + 8 * ndims
        out, stack = [], [btree]
        while stack:
            a = stack.pop()
            h = self.read(a, 24)
            if h[:4] != b"TREE" or h[4] != 1:
                raise OSError("bad chunk B-tree node")
            level, n = h[5], struct.unpack_from("<H", h, 6)[0]
            body = self.read(a + 24, n * (ks + 8) + ks)
            for i in range(n):
                p = i * (ks + 8)
                size, mask = struct.unpack_from("<II", body, p)
                offs = struct.unpack_from(f"<{ndims}Q", body, p + 8)
                child = struct.unpack_from("<Q", body, p + ks)[0]
                if level > 0:
                    stack.append(child)
                else:
                    out.append((offs, size, mask, child))
        return out


class Dataset:
    def __init__(self, file, addr, msgs):
        self.file, self.addr = file, addr
        self._msgs = msgs
        self.attrs = {}
        self.shape, self.dtype, self._layout, self._filters = (), None, None, []
        for t, d in msgs:
            if t == MSG_SPACE:
                self.shape = _decode_space(d)
            elif t == MSG_TYPE:
                self.dtype = _decode_dtype(d)
            elif t == MSG_LAYOUT:
                self._layout = d
            elif t == MSG_FILTER:
                self._filters = _decode_filters(d)
            elif t == MSG_ATTR:
                k, v = _decode_attr(d)
                self.attrs[k] = v

    def _read(self):
        d, rd = self._layout, self.file._r
        if d is None or d[0] != 3:
            raise NotImplementedError("HDF5 data layout other than version 3")
        cls = d[1]
        n = int(np.prod(self.shape)) if self.shape else 1
        nbytes = n * self.dtype.itemsize
        if cls == 0:
            size = struct.unpack_from("<H", d, 2)[0]
            raw = d[4:4 + size]
        elif cls == 1:
            addr, size = struct.unpack_from("<QQ", d, 2)
            raw = rd.read(addr, nbytes) if addr != UNDEF else b"\0" * nbytes
        elif cls == 2:
            ndims = d[2]
            bt = struct.unpack_from("<Q", d, 3)[0]
            cdims = struct.unpack_from(f"<{ndims}I", d, 11)[:-1]
            out = np.zeros(self.shape, dtype=self.dtype)
            if bt != UNDEF:
                for offs, size, mask, caddr in rd.chunks(bt, ndims):
                    buf = rd.read(caddr, size)
                    for i, (fid, cd) in reversed(list(enumerate(self._filters))):
                        if mask & (1 << i):
                            continue
                        if fid == 1:
                            buf = zlib.decompress(buf)
                        elif fid == 2:
                            es = self.dtype.itemsize
                            buf = np.frombuffer(buf, np.uint8).reshape(es, -1).T.tobytes()
                        else:
                            raise NotImplementedError(f"HDF5 filter {fid}")
                    c = np.frombuffer(buf, dtype=self.dtype, count=int(np.prod(cdims))).reshape(cdims)
                    dst = tuple(slice(o, min(o + cd, s)) for o, cd, s in zip(offs, cdims, self.shape))
                    out[dst] = c[tuple(slice(0, sl.stop - sl.start) for sl in dst)]
            return out.astype(self.dtype.newbyteorder("=")) if self.dtype.kind in "iuf" else out
        else:
            raise NotImplementedError(f"HDF5 layout class {cls}")
        a = np.frombuffer(raw, dtype=self.dtype, count=n).reshape(self.shape)
        return a.astype(self.dtype.newbyteorder("=")) if self.dtype.kind in "iuf" else a.copy()

    def __getitem__(self, idx):
        return self._read()[idx]

    def __array__(self, dtype=None, copy=None):
        a = self._read()
        return a if dtype is None else a.astype(dtype)

    def __len__(self):
        return self.shape[0]


def _decode_link(b):
    """(name, address) of a hard link message (version 1), else (name, None)."""
    flags = b[1]
    p = 2
    ltype = 0
    if flags & 0x08:
        ltype = b[p]
        p += 1
    if flags & 0x04:
        p += 8
    if flags & 0x10:
        p += 1
    w = 1 << (flags & 3)
    n = int.from_bytes(b[p:p + w], "little")
    p += w
    name = b[p:p + n].decode()
    p += n
    return name, (struct.unpack_from("<Q", b, p)[0] if ltype == 0 else None)


class Group:
    """A group: ``keys()``, ``[name]``, ``in``, ``attrs``, ``create_group``,
    ``create_dataset``, ``del``.  Groups read from a file are read-only
    except the root, whose links may be added or deleted."""

    def __init__(self, file, addr=None, name="/"):
        self.file, self.addr, self.name = file, addr, name
        self.attrs = {}
        self._links = {}     # name -> address (on disk) or a new Group / _NewDataset
        self._new = addr is None
        if addr is not None:
            for t, d in file._r.messages(addr):
                if t == MSG_STAB:
                    bt, heap = struct.unpack_from("<QQ", d)
                    self._links.update(file._r.stab_links(bt, heap))
                elif t == MSG_LINK:
                    k, a = _decode_link(d)
                    if a is not None:
                        self._links[k] = a
                elif t == MSG_LINKINFO:
                    fh = struct.unpack_from("<Q", d, 2 + (8 if d[1] & 1 else 0))[0]
                    if fh != UNDEF:
                        raise NotImplementedError("HDF5 dense link storage (fractal heap)")
                elif t == MSG_ATTR:
                    k, v = _decode_attr(d)
                    self.attrs[k] = v

    def _writable(self):
        if self.file.mode == "r":
            raise OSError("file is open read-only")
        if not (self._new or self is self.file._root):
            raise NotImplementedError("h5lite modifies only new groups and the root group")

    def keys(self):
        return list(self._links.keys())

    def __iter__(self):
        return iter(self.keys())

    def __len__(self):
        return len(self._links)

    def __contains__(self, name):
        return name in self._links

    def __getitem__(self, name):
        obj = self._links[name]
        if isinstance(obj, int):
            msgs = self.file._r.messages(obj)
            if any(t == MSG_LAYOUT for t, _ in msgs):
                return Dataset(self.file, obj, msgs)
            return Group(self.file, obj, name)
        return obj

    def __delitem__(self, name):
        self._writable()
        del self._links[name]
        self.file._dirty = True

    def create_group(self, name):
        self._writable()
        if name in self._links:
            raise ValueError(f"name already exists: {name}")
        g = Group(self.file, None, name)
        self._links[name] = g
        self.file._dirty = True
        return g

    def create_dataset(self, name, data=None, compression=None, compression_opts=None, **kw):
        self._writable()
        if name in self._links:
            raise ValueError(f"name already exists: {name}")
        d = _NewDataset(np.asarray(data), compression, compression_opts)
        self._links[name] = d
        self.file._dirty = True
        return d


class _NewDataset:
    def __init__(self, data, compression, level):
        if compression not in (None, "gzip"):
            raise NotImplementedError(f"compression {compression!r} (h5lite writes gzip or none)")
        a = np.ascontiguousarray(data)
        if a.dtype.kind in "iuf" and a.dtype.byteorder not in ("<", "|") and a.dtype.itemsize > 1:
            a = a.astype(a.dtype.newbyteorder("<"))
        self.data, self.compression = a, compression
        self.level = 4 if level is None else int(level)
        self.attrs = {}
        self.shape, self.dtype = a.shape, a.dtype

    def __getitem__(self, idx):
        return self.data[idx]

    def __array__(self, dtype=None, copy=None):
        return self.data if dtype is None else self.data.astype(dtype)


class File(Group):
    """``File(path, mode)`` with mode ``r``, ``r+``, ``a``, ``w``; a context
    manager; ``flush()`` writes pending objects, ``close()`` flushes."""

    def __init__(self, path, mode="r"):
        self.path, self.mode = os.fspath(path), mode
        exists = os.path.exists(self.path)
        if mode == "w" or (mode == "a" and not exists):
            self._fh = open(self.path, "w+b")
            self._fh.write(b"\0" * 96)
            self._end = 96
            self._r = None
            Group.__init__(self, self, None, "/")
            self._root = self
            self._dirty = True
            self.flush()
        else:
            if mode not in ("r", "r+", "a"):
                raise ValueError(f"mode {mode!r}")
            self._fh = open(self.path, "rb" if mode == "r" else "r+b")
            self._r = _Reader(self._fh)
            self._fh.seek(0, os.SEEK_END)
            self._end = max(self._fh.tell(), self._r.eof)
            Group.__init__(self, self, self._r.root_addr, "/")
            self._root = self
            self._new = False
            self._dirty = False
        self.file = self

    # ------------------------------------------------------------ writing
    def _append(self, b, align=8):
        self._end += -self._end % align
        addr = self._end
        self._fh.seek(addr)
        self._fh.write(b)
        self._end += len(b)
        return addr

    def _write_obj(self, obj):
        if isinstance(obj, int):
            return obj
        if isinstance(obj, _NewDataset):
            return self._write_dataset(obj)
        links = {k: self._write_obj(v) for k, v in obj._links.items()}
        addr = self._write_group(links, obj.attrs)[0]
        obj.addr, obj._links, obj._new = addr, links, False
        return addr

    def _write_dataset(self, d):
        a = d.data
        msgs = [(MSG_SPACE, 0, _space_msg(a.shape)), (MSG_TYPE, 1, _encode_dtype(a.dtype))]
        chunked = (d.compression == "gzip" and a.ndim > 0 and a.size > 0 and a.nbytes < 2 ** 32)
        if not chunked:
            addr = self._append(a.tobytes()) if a.size else UNDEF
            msgs += [(MSG_FILL, 1, bytes([2, 2, 2, 0])),
                     (MSG_LAYOUT, 0, struct.pack("<BBQQ", 3, 1, addr, a.nbytes))]
        else:
            comp = zlib.compress(a.tobytes(), d.level)
            caddr = self._append(comp)
            nd = a.ndim + 1
            ks = 8 + 8 * nd
            node = (b"TREE" + bytes([1, 0]) + struct.pack("<HQQ", 1, UNDEF, UNDEF)
                    + struct.pack(f"<II{nd}Q", len(comp), 0, *([0] * nd)) + struct.pack("<Q", caddr)
                    + struct.pack(f"<II{nd}Q", 0, 0, *(list(a.shape) + [0])))
            node += b"\0" * (24 + 2 * K_CHUNK * 8 + (2 * K_CHUNK + 1) * ks - len(node))
            bt = self._append(node)
            msgs += [(MSG_FILL, 1, bytes([2, 3, 2, 0])),
                     (MSG_LAYOUT, 0, struct.pack(f"<BBBQ{nd}I", 3, 2, nd, bt, *(list(a.shape) + [a.itemsize]))),
                     (MSG_FILTER, 0, _filter_msg_deflate(d.level))]
        msgs += [(MSG_ATTR, 0, _attr_msg(k, v)) for k, v in d.attrs.items()]
        return self._append(_ohdr(msgs))

    def _write_group(self, links, attrs):
        names = sorted(links, key=lambda n: n.encode())
        heap, offs = b"\0" * 8, {}
        for n in names:
            offs[n] = len(heap)
            heap += _pad8(n.encode() + b"\0")
        hdata = self._append(heap)
        haddr = self._append(b"HEAP" + bytes(4) + struct.pack("<QQQ", len(heap), FREE_NULL, hdata))
        cap = 2 * K_LEAF
        chunks = [names[i:i + cap] for i in range(0, len(names), cap)]
        if len(chunks) > 2 * K_INT:
            raise NotImplementedError(f"h5lite groups hold at most {2 * K_INT * cap} links")
        snods = []
        for ch in chunks:
            ent = b"".join(struct.pack("<QQII16x", offs[n], links[n], 0, 0) for n in ch)
            snods.append(self._append(b"SNOD" + bytes([1, 0]) + struct.pack("<H", len(ch)) + ent
                                      + b"\0" * (40 * (cap - len(ch)))))
        body = struct.pack("<Q", 0)
        for ch, sa in zip(chunks, snods):
            body += struct.pack("<QQ", sa, offs[ch[-1]])
        node = b"TREE" + bytes([0, 0]) + struct.pack("<HQQ", len(chunks), UNDEF, UNDEF) + body
        node += b"\0" * (24 + 2 * K_INT * 8 + (2 * K_INT + 1) * 8 - len(node))
        bt = self._append(node)
        msgs = [(MSG_STAB, 0, struct.pack("<QQ", bt, haddr))]
        msgs += [(MSG_ATTR, 0, _attr_msg(k, v)) for k, v in attrs.items()]
        return self._append(_ohdr(msgs)), bt, haddr

    def flush(self):
        if self.mode == "r" or not self._dirty:
            return
        links = {k: self._write_obj(v) for k, v in self._links.items()}
        self._links = links
        root, bt, heap = self._write_group(links, self.attrs)
        self._end += -self._end % 8
        sb = (SIG + struct.pack("<8BHHI", 0, 0, 0, 0, 0, 8, 8, 0, K_LEAF, K_INT, 0)
              + struct.pack("<QQQQ", 0, UNDEF, self._end, UNDEF)
              + struct.pack("<QQII", 0, root, 1, 0) + struct.pack("<QQ", bt, heap))
        assert len(sb) == 96
        self._fh.seek(0, os.SEEK_END)
        if self._fh.tell() < self._end:  # the file reaches the end address
            self._fh.seek(self._end - 1)
            self._fh.write(b"\0")
        self._fh.seek(0)
        self._fh.write(sb)
        self._fh.flush()
        self.addr = root
        self._r = _Reader(self._fh)
        self._dirty = False

    def close(self):
        if self._fh is None:
            return
        try:
            self.flush()
        finally:
            self._fh.close()
            self._fh = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
