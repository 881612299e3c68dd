"""HDF5 files without libhdf5: a reader and an append-only writer for the
structures bfps' files use, written from the published HDF5 file format
specification (superblock version 0, version-1 object headers, symbol-table
groups with a version-1 B-tree and a local heap, contiguous and chunked
datasets without filters, fixed-point / floating-point / compound (complex)
/ string / variable-length-string datatypes).

The reference writes its files through libhdf5 and h5py:
  parameters and statistics        bfps/_code.py write_par, bfps/DNS.py:372-452
  fields (checkpoints)             bfps/cpp/field.cpp:167-356
  tracer state / rhs               bfps/cpp/particles/particles_output_hdf5.hpp:54-312
  sampled velocity / acceleration  bfps/cpp/particles/particles_output_sampling_hdf5.hpp
  growth of the statistics         bfps/cpp/hdf5_tools.cpp:74-92
and reads them back with the same paths (dataset names are the iteration
numbers under each group).  This module reads such files by their structure
and writes files of the same shape: superblock version 0 with 8-byte offsets
and lengths, which is what libhdf5 writes by default.

Public surface (a small subset of h5py's):
  File(path, mode)          mode 'r', 'w' (truncate), 'a' (append, create if absent)
  f[path] -> Dataset | Group;  path in f;  f.keys() / group.keys()
  f[path] = array           create a contiguous dataset (and missing groups)
  f.create_group(path)
  f.create_dataset(path, shape, dtype, chunks=None, maxshape=None, data=None)
  Dataset: shape, dtype, read() / [()] / [slices], write(array) for contiguous,
           resize(n) along axis 0 and write_rows(start, rows) for chunked
  close(), context manager
"""
import os
import struct

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF

# message types
MSG_NIL, MSG_DATASPACE, MSG_LINKINFO, MSG_DATATYPE = 0x0, 0x1, 0x2, 0x3
MSG_FILL_OLD, MSG_FILL, MSG_LINK, MSG_LAYOUT = 0x4, 0x5, 0x6, 0x8
MSG_FILTERS, MSG_ATTRIBUTE, MSG_CONT, MSG_STAB = 0xB, 0xC, 0x10, 0x11
MSG_MTIME = 0x12

# node capacities this writer uses (stored in the superblock, read back
# from it by every reader): one symbol-table node holds 2 * LEAF_K links
LEAF_K = 64
INTERNAL_K = 16
CHUNK_K = 32     # chunk B-tree: 2 * CHUNK_K chunks per node (superblock v0 default)


class H5Error(Exception):
    pass


def _pad8(n):
    return (n + 7) & ~7


# ------------------------------------------------------------ datatypes --
def _float_dt(size, order):
    return np.dtype(("<" if order == 0 else ">") + "f%d" % size)


def _parse_datatype(b, o=0):
    """(numpy dtype or 'vlen-str', bytes consumed) of a datatype message."""
    cv = b[o]
    cls, ver = cv & 0x0F, cv >> 4
    bits = b[o + 1] | (b[o + 2] << 8) | (b[o + 3] << 16)
    size = struct.unpack_from("<I", b, o + 4)[0]
    p = o + 8
    if cls == 0:  # fixed point
        order = bits & 1
        signed = (bits >> 3) & 1
        return np.dtype(("<" if order == 0 else ">") + ("i" if signed else "u") + str(size)), 12
    if cls == 1:  # floating point
        return _float_dt(size, bits & 1), 20
    if cls == 3:  # fixed-length string
        return np.dtype("S%d" % size), 8
    if cls == 6:  # compound
        nmemb = bits & 0xFFFF
        names, formats, offsets = [], [], []
        for _ in range(nmemb):
            end = b.index(b"\0", p)
            name = b[p:end].decode()
            if ver in (1, 2):
                p = p + _pad8(end - p + 1)
                off = struct.unpack_from("<I", b, p)[0]
                p += 4 + 1 + 3 + 4 + 4 + 16  # offset, ndims, reserved, perm, reserved, dims
            else:
                p = end + 1
                nb = 1 if size < 256 else (2 if size < 65536 else (3 if size < (1 << 24) else 4))
                off = int.from_bytes(b[p:p + nb], "little")
                p += nb
            mdt, used = _parse_datatype(b, p)
            p += used
            names.append(name)
            formats.append(mdt)
            offsets.append(off)
        dt = np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": size})
        return dt, p - o
    if cls == 9:  # variable length
        base, used = _parse_datatype(b, p)
        return ("vlen-str" if (bits & 0xF) == 1 else ("vlen-seq", base)), 8 + used
    raise H5Error("unsupported datatype class %d" % cls)


def _complex_of(dt):
    """complex dtype for a compound {r, i} of two equal floats, else None."""
    if isinstance(dt, np.dtype) and dt.names and len(dt.names) == 2:
        a, b = (dt.fields[n] for n in dt.names)
        if a[0] == b[0] and a[0].kind == "f" and a[1] == 0 and b[1] == a[0].itemsize:
            return np.dtype(a[0].byteorder.replace("=", "<") + "c%d" % (2 * a[0].itemsize))
    return None


def _encode_datatype(dt):
    """Datatype message body for a numpy dtype (little endian)."""
    dt = np.dtype(dt)
    if dt.kind == "c":
        half = dt.itemsize // 2
        memb = b""
        for name, off in (("r", 0), ("i", half)):
            nb = name.encode() + b"\0"
            memb += nb + b"\0" * (_pad8(len(nb)) - len(nb))
            memb += struct.pack("<IB3xI4x16x", off, 0, 0)
            memb += _encode_datatype(np.dtype("<f%d" % half))
        return struct.pack("<B3sI", 0x16, (2).to_bytes(3, "little"), dt.itemsize) + memb
    if dt.kind == "f":
        if dt.itemsize == 4:
            props = struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
        else:
            props = struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
        bits = 0x20 | ((dt.itemsize * 8 - 1) << 8)   # implied msb normalisation, sign bit
        return struct.pack("<B3sI", 0x11, bits.to_bytes(3, "little"), dt.itemsize) + props
    if dt.kind in "iu":
        bits = 0x08 if dt.kind == "i" else 0
        return (struct.pack("<B3sI", 0x10, bits.to_bytes(3, "little"), dt.itemsize) +
                struct.pack("<HH", 0, dt.itemsize * 8))
    if dt.kind == "S":
        return struct.pack("<B3sI", 0x13, (0).to_bytes(3, "little"), dt.itemsize)
    if dt.kind == "b":
        return _encode_datatype(np.dtype("i1"))
    raise H5Error("cannot store dtype %s" % dt)


# ------------------------------------------------------------- objects --
class Group:
    def __init__(self, f, name, addr):
        self.file, self.name, self.addr = f, name, addr

    def _links(self):
        return self.file._group_links(self.addr)

    def keys(self):
        return sorted(self._links())

    def __iter__(self):
        return iter(self.keys())

    def __contains__(self, path):
        return self.file._lookup(self._abs(path)) is not None

    def _abs(self, path):
        return path if path.startswith("/") else self.name.rstrip("/") + "/" + path

    def __getitem__(self, path):
        return self.file[self._abs(path)]

    def __setitem__(self, path, value):
        self.file[self._abs(path)] = value

    def create_group(self, path):
        return self.file.create_group(self._abs(path))

    def create_dataset(self, path, *a, **kw):
        return self.file.create_dataset(self._abs(path), *a, **kw)


class Dataset:
    def __init__(self, f, name, addr, info):
        self.file, self.name, self.addr = f, name, addr
        self._info = info

    @property
    def shape(self):
        return tuple(self._info["dims"])

    @property
    def maxshape(self):
        return tuple(self._info["maxdims"]) if self._info["maxdims"] is not None else self.shape

    @property
    def dtype(self):
        return self._info["dtype"]

    @property
    def chunks(self):
        return self._info.get("chunks")

    def read(self):
        return self.file._read_dataset(self._info)

    def __getitem__(self, key):
        a = self.read()
        return a if key == () or key is Ellipsis else a[key]

    def __len__(self):
        return self.shape[0] if self.shape else 0

    def write(self, data):
        self.file._write_contiguous(self, data)

    def resize(self, n0):
        self.file._resize_chunked(self, n0)

    def write_rows(self, start, rows):
        self.file._write_rows(self, start, rows)


# --------------------------------------------------------------- file --
class File:
    def __init__(self, path, mode="r"):
        if mode not in ("r", "w", "a", "r+"):
            raise H5Error("mode must be r, r+, w or a")
        self.path = path
        self.mode = mode
        exists = os.path.exists(path)
        if mode == "w" or (mode == "a" and not exists):
            self._fh = open(path, "w+b")
            self._create_empty()
        else:
            if not exists:
                raise FileNotFoundError(path)
            self._fh = open(path, "rb" if mode == "r" else "r+b")
        self._read_superblock()

    # ------------------------------------------------------ low level
    def _rd(self, addr, n):
        self._fh.seek(addr)
        b = self._fh.read(n)
        if len(b) != n:
            raise H5Error("short read at %d" % addr)
        return b

    def _append(self, data, align=8):
        self._fh.seek(0, 2)
        end = self._fh.tell()
        pad = (-end) % align
        if pad:
            self._fh.write(b"\0" * pad)
            end += pad
        self._fh.write(data)
        self._set_eof(end + len(data))
        return end

    def _wr(self, addr, data):
        self._fh.seek(addr)
        self._fh.write(data)

    def _writable(self):
        if self.mode == "r":
            raise H5Error("file opened read-only")

    # ------------------------------------------------------ superblock
    def _read_superblock(self):
        b = self._rd(0, 96)
        if b[:8] != SIGNATURE:
            raise H5Error("not an HDF5 file (or a user block precedes the superblock)")
        ver = b[8]
        if ver not in (0, 1):
            raise H5Error("superblock version %d not supported" % ver)
        self._so, self._sl = b[13], b[14]
        if (self._so, self._sl) != (8, 8):
            raise H5Error("only 8-byte offsets and lengths are supported")
        self._leaf_k, self._int_k = struct.unpack_from("<HH", b, 16)
        # version 1 adds the chunk B-tree K and two reserved bytes
        p = 24 if ver == 0 else 28
        self._chunk_k = CHUNK_K if ver == 0 else struct.unpack_from("<H", b, 24)[0]
        b = self._rd(0, p + 72)
        base, _freespace, eof, _driver = struct.unpack_from("<QQQQ", b, p)
        if base != 0:
            raise H5Error("base address %d not supported" % base)
        self._eof = eof
        self._eof_addr_pos = p + 16
        self._root_entry_pos = p + 32
        _name_off, self._root = struct.unpack_from("<QQ", b, self._root_entry_pos)

    def _set_eof(self, end):
        if end > self._eof:
            self._eof = end
            self._fh.seek(self._eof_addr_pos)
            self._fh.write(struct.pack("<Q", end))

    def _create_empty(self):
        sb = bytearray(96)
        sb[:8] = SIGNATURE
        sb[8:16] = bytes([0, 0, 0, 0, 0, 8, 8, 0])
        struct.pack_into("<HHI", sb, 16, LEAF_K, INTERNAL_K, 0)
        struct.pack_into("<QQQQ", sb, 24, 0, UNDEF, 96, UNDEF)
        self._fh.write(bytes(sb))
        self._eof = 96
        self._eof_addr_pos = 40
        btree, heap = self._new_group_storage([])
        hdr = self._write_object_header([(MSG_STAB, struct.pack("<QQ", btree, heap))], nil_pad=0)
        # root symbol table entry: cache type 1 keeps the B-tree and heap addresses
        struct.pack_into("<QQII QQ", sb, 56, 0, hdr, 1, 0, btree, heap)
        self._wr(0, bytes(sb))
        self._set_eof(self._fh.seek(0, 2))

    # ------------------------------------------------------ object headers
    def _messages(self, addr):
        """[(type, flags, body bytes, absolute body address)] of an object header."""
        b = self._rd(addr, 16)
        ver = b[0]
        if ver != 1:
            if b[:4] == b"OHDR":
                raise H5Error("version-2 object headers are not supported")
            raise H5Error("bad object header at %d" % addr)
        nmsg = struct.unpack_from("<H", b, 2)[0]
        size = struct.unpack_from("<I", b, 8)[0]
        out = []
        blocks = [(addr + 16, size)]
        while blocks and len(out) < nmsg:
            start, length = blocks.pop(0)
            data = self._rd(start, length)
            p = 0
            while p + 8 <= length and len(out) < nmsg:
                mtype, msize, flags = struct.unpack_from("<HHB", data, p)
                body = data[p + 8:p + 8 + msize]
                if mtype == MSG_CONT:
                    caddr, clen = struct.unpack_from("<QQ", body, 0)
                    blocks.append((caddr, clen))
                out.append((mtype, flags, body, start + p + 8))
                p += 8 + msize
        return out

    def _write_object_header(self, msgs, nil_pad=0):
        """Append a version-1 object header holding msgs [(type, body)] or
        [(type, body, flags)] (flag 1: constant message)."""
        body = b""
        for m in msgs:
            mtype, data = m[0], m[1]
            flags = m[2] if len(m) > 2 else 0
            data = data + b"\0" * (_pad8(len(data)) - len(data))
            body += struct.pack("<HHB3x", mtype, len(data), flags) + data
        n = len(msgs)
        if nil_pad:
            body += struct.pack("<HHB3x", MSG_NIL, nil_pad, 0) + b"\0" * nil_pad
            n += 1
        hdr = struct.pack("<BBHII", 1, 0, n, 1, len(body)) + b"\0" * 4
        return self._append(hdr + body)

    # ------------------------------------------------------ groups
    def _group_storage(self, addr):
        for mtype, _f, body, _a in self._messages(addr):
            if mtype == MSG_STAB:
                return struct.unpack_from("<QQ", body, 0) + (_a,)
            if mtype in (MSG_LINK, MSG_LINKINFO):
                raise H5Error("link-message (new style) groups are not supported")
        return None

    def _heap(self, heap_addr):
        b = self._rd(heap_addr, 32)
        if b[:4] != b"HEAP":
            raise H5Error("bad local heap at %d" % heap_addr)
        size, _free, data_addr = struct.unpack_from("<QQQ", b, 8)
        return self._rd(data_addr, size)

    def _group_links(self, addr, cached=None):
        """{name: object header address} of a group; names whose entries
        cache the child group's B-tree and heap (cache type 1) go into
        `cached` when a set is given."""
        st = self._group_storage(addr)
        if st is None:
            raise H5Error("object at %d is not a group" % addr)
        btree, heap_addr, _ = st
        heap = self._heap(heap_addr)
        links = {}
        self._walk_group_btree(btree, heap, links, cached)
        return links

    def _walk_group_btree(self, node, heap, links, cached=None):
        b = self._rd(node, 24)
        if b[:4] != b"TREE" or b[4] != 0:
            raise H5Error("bad group B-tree node at %d" % node)
        level, used = b[5], struct.unpack_from("<H", b, 6)[0]
        body = self._rd(node + 24, (2 * used + 1) * 8)
        children = [struct.unpack_from("<Q", body, 8 + 16 * i)[0] for i in range(used)]
        for c in children:
            if level > 0:
                self._walk_group_btree(c, heap, links, cached)
            else:
                sb = self._rd(c, 8)
                if sb[:4] != b"SNOD":
                    raise H5Error("bad symbol table node at %d" % c)
                nsym = struct.unpack_from("<H", sb, 6)[0]
                ents = self._rd(c + 8, 40 * nsym)
                for i in range(nsym):
                    noff, oaddr, ctype = struct.unpack_from("<QQI", ents, 40 * i)
                    end = heap.index(b"\0", noff)
                    name = heap[noff:end].decode()
                    links[name] = oaddr
                    if cached is not None and ctype == 1:
                        cached.add(name)

    def _new_group_storage(self, entries):
        """Write a local heap, one symbol-table node and a one-level B-tree
        for entries [(name, object header address)]; returns (btree, heap)."""
        entries = sorted(entries, key=lambda e: e[0].encode())
        if len(entries) > 2 * LEAF_K * 2 * INTERNAL_K:
            raise H5Error("too many links in one group")
        heap = bytearray(b"\0" * 8)   # offset 0: the empty name
        offs = []
        for name, _a in entries:
            nb = name.encode() + b"\0"
            offs.append(len(heap))
            heap += nb + b"\0" * (_pad8(len(nb)) - len(nb))
        # the heap is written whole for every change, so it keeps no free list
        data_addr = self._append(bytes(heap))
        heap_addr = self._append(b"HEAP" + bytes([0, 0, 0, 0]) +
                                 struct.pack("<QQQ", len(heap), UNDEF, data_addr))
        # symbol-table nodes of up to 2K entries each
        snods, keys = [], [0]
        cap = 2 * LEAF_K
        groups = [entries[i:i + cap] for i in range(0, len(entries), cap)] or [[]]
        gi = 0
        for grp in groups:
            body = bytearray(b"SNOD" + bytes([1, 0]) + struct.pack("<H", len(grp)))
            for name, oaddr in grp:
                body += struct.pack("<QQII16x", offs[gi], oaddr, 0, 0)
                gi += 1
            body += b"\0" * (8 + 40 * cap - len(body))
            snods.append(self._append(bytes(body)))
            keys.append(offs[gi - 1] if grp else 0)
        n = len(snods) if entries else 0
        node = bytearray(b"TREE" + bytes([0, 0]) + struct.pack("<H", n) + struct.pack("<QQ", UNDEF, UNDEF))
        for i in range(n):
            node += struct.pack("<QQ", keys[i], snods[i])
        node += struct.pack("<Q", keys[n] if n else 0)
        node += b"\0" * (24 + (2 * 2 * INTERNAL_K + 1) * 8 - len(node))
        return self._append(bytes(node)), heap_addr

    def _set_group_links(self, gaddr, links, gpath):
        """New storage for the group at gpath, pointed to by its symbol-table
        message.  libhdf5 also caches a group's B-tree and heap addresses in
        its parent's entry (and the superblock caches the root's): the root
        cache is rewritten, and a parent whose entry for this group carries a
        cache gets new storage itself (entries without caches), up the path."""
        btree, heap = self._new_group_storage(list(links.items()))
        _b, _h, body_at = self._group_storage(gaddr)
        self._wr(body_at, struct.pack("<QQ", btree, heap))
        if gaddr == self._root:
            self._wr(self._root_entry_pos + 24, struct.pack("<QQ", btree, heap))
            return
        ppath, _, name = gpath.rstrip("/").rpartition("/")
        ppath = ppath or "/"
        paddr = self._lookup(ppath)
        cached = set()
        plinks = self._group_links(paddr, cached)
        if name in cached:
            self._set_group_links(paddr, plinks, ppath)

    # ------------------------------------------------------ lookup
    def _lookup(self, path):
        addr = self._root
        for part in [p for p in path.split("/") if p]:
            if self._group_storage(addr) is None:
                return None
            links = self._group_links(addr)
            if part not in links:
                return None
            addr = links[part]
        return addr

    def _obj(self, path, addr):
        if self._group_storage(addr) is not None:
            return Group(self, path, addr)
        return Dataset(self, path, addr, self._dataset_info(addr))

    def __getitem__(self, path):
        path = "/" + path.strip("/")
        addr = self._lookup(path)
        if addr is None:
            raise KeyError(path)
        return self._obj(path, addr)

    def __contains__(self, path):
        return self._lookup("/" + path.strip("/")) is not None

    def keys(self):
        return Group(self, "/", self._root).keys()

    def __iter__(self):
        return iter(self.keys())

    # ------------------------------------------------------ datasets
    def _dataset_info(self, addr):
        info = {"dims": None, "maxdims": None, "dtype": None, "layout": None, "filters": False}
        for mtype, _f, body, at in self._messages(addr):
            if mtype == MSG_DATASPACE:
                ver, rank, flags = body[0], body[1], body[2]
                p = 8 if ver == 1 else 4
                dims = list(struct.unpack_from("<%dQ" % rank, body, p))
                p += 8 * rank
                maxd = None
                if flags & 1:
                    maxd = [None if m == UNDEF else m for m in struct.unpack_from("<%dQ" % rank, body, p)]
                if ver == 2 and body[3] == 2:
                    dims = [0]
                info.update(dims=dims, maxdims=maxd, dataspace_at=at)
            elif mtype == MSG_DATATYPE:
                dt, _ = _parse_datatype(body)
                info["raw_dtype"] = dt
                c = _complex_of(dt)
                info["dtype"] = c if c is not None else dt
            elif mtype == MSG_LAYOUT:
                ver = body[0]
                if ver == 3:
                    cls = body[1]
                    if cls == 0:
                        size = struct.unpack_from("<H", body, 2)[0]
                        info["layout"] = ("compact", bytes(body[4:4 + size]))
                    elif cls == 1:
                        a, s = struct.unpack_from("<QQ", body, 2)
                        info["layout"] = ("contiguous", a, s)
                    elif cls == 2:
                        nd = body[2]
                        a = struct.unpack_from("<Q", body, 3)[0]
                        cd = list(struct.unpack_from("<%dI" % nd, body, 11))
                        info["layout"] = ("chunked", a, cd)
                        info["chunks"] = tuple(cd[:-1])
                        info["layout_at"] = at
                    else:
                        raise H5Error("layout class %d not supported" % cls)
                elif ver in (1, 2):
                    nd, cls = body[1], body[2]
                    p = 8
                    a = struct.unpack_from("<Q", body, p)[0] if cls != 0 else None
                    p += 8 if cls != 0 else 0
                    cd = list(struct.unpack_from("<%dI" % nd, body, p))
                    if cls == 1:
                        info["layout"] = ("contiguous", a, int(np.prod(cd)) if cd else 0)
                    elif cls == 2:
                        info["layout"] = ("chunked", a, cd)
                        info["chunks"] = tuple(cd[:-1])
                    else:
                        raise H5Error("compact layout version %d not supported" % ver)
                else:
                    raise H5Error("layout message version %d not supported" % ver)
            elif mtype == MSG_FILTERS:
                info["filters"] = True
        if info["layout"] is None or info["dtype"] is None:
            raise H5Error("object at %d is neither a group nor a dataset" % addr)
        return info

    def _element_dtype(self, info):
        dt = info["dtype"]
        if dt == "vlen-str" or isinstance(dt, tuple):
            return np.dtype("<u4,<u8,<u4")   # length, collection address, index
        return dt

    def _read_dataset(self, info):
        dims = info["dims"]
        dt = self._element_dtype(info)
        n = int(np.prod(dims)) if dims else 1
        lay = info["layout"]
        if lay[0] == "compact":
            raw = lay[1][:n * dt.itemsize]
        elif lay[0] == "contiguous":
            if lay[1] == UNDEF:
                raw = b"\0" * (n * dt.itemsize)
            else:
                raw = self._rd(lay[1], n * dt.itemsize)
        else:
            if info["filters"]:
                raise H5Error("filtered (compressed) chunks are not supported")
            return self._read_chunked(info, dt)
        a = np.frombuffer(raw, dtype=dt).reshape(dims if dims else ())
        if info["dtype"] == "vlen-str":
            return self._vlen_strings(a)
        return a.copy()

    def _chunk_entries(self, node, rank1):
        """[(chunk offsets, size, address)] under a chunk B-tree node."""
        if node == UNDEF:
            return []
        b = self._rd(node, 24)
        if b[:4] != b"TREE" or b[4] != 1:
            raise H5Error("bad chunk B-tree node at %d" % node)
        level, used = b[5], struct.unpack_from("<H", b, 6)[0]
        ksz = 8 + 8 * rank1
        body = self._rd(node + 24, used * (ksz + 8) + ksz)
        out = []
        for i in range(used):
            k = i * (ksz + 8)
            size, _mask = struct.unpack_from("<II", body, k)
            offs = struct.unpack_from("<%dQ" % rank1, body, k + 8)
            child = struct.unpack_from("<Q", body, k + ksz)[0]
            if level > 0:
                out += self._chunk_entries(child, rank1)
            else:
                out.append((offs[:-1], size, child))
        return out

    def _read_chunked(self, info, dt):
        dims = info["dims"]
        _, bt, cd = info["layout"]
        cdims = cd[:-1]
        out = np.zeros(dims, dtype=dt)
        for offs, size, addr in self._chunk_entries(bt, len(cd)):
            nb = int(np.prod(cdims)) * dt.itemsize
            c = np.frombuffer(self._rd(addr, nb), dtype=dt).reshape(cdims)
            sl_out = tuple(slice(o, min(o + s, d)) for o, s, d in zip(offs, cdims, dims))
            sl_in = tuple(slice(0, s.stop - s.start) for s in sl_out)
            if all(s.stop > s.start for s in sl_out):
                out[sl_out] = c[sl_in]
        return out

    def _vlen_strings(self, a):
        out = np.empty(a.shape, dtype=object)
        cache = {}
        for idx in np.ndindex(a.shape):
            ln, coll, oid = (int(x) for x in a[idx])
            if coll not in cache:
                cache[coll] = self._global_heap(coll)
            out[idx] = cache[coll].get(oid, b"")[:ln].decode()
        return out if a.shape else out[()]

    def _global_heap(self, addr):
        b = self._rd(addr, 16)
        if b[:4] != b"GCOL":
            raise H5Error("bad global heap at %d" % addr)
        size = struct.unpack_from("<Q", b, 8)[0]
        data = self._rd(addr, size)
        objs, p = {}, 16
        while p + 16 <= size:
            oid, _ref = struct.unpack_from("<HH", data, p)
            osz = struct.unpack_from("<Q", data, p + 8)[0]
            if oid == 0:
                break
            objs[oid] = data[p + 16:p + 16 + osz]
            p += 16 + _pad8(osz)
        return objs

    # ------------------------------------------------------ writing
    def _require_group(self, path):
        addr = self._root
        cur = ""
        for part in [p for p in path.split("/") if p]:
            parent = cur or "/"
            cur += "/" + part
            links = self._group_links(addr)
            if part in links:
                addr = links[part]
                if self._group_storage(addr) is None:
                    raise H5Error("%s is a dataset" % cur)
            else:
                btree, heap = self._new_group_storage([])
                new = self._write_object_header([(MSG_STAB, struct.pack("<QQ", btree, heap))])
                links[part] = new
                self._set_group_links(addr, links, parent)
                addr = new
        return addr

    def create_group(self, path):
        self._writable()
        path = "/" + path.strip("/")
        if self._lookup(path) is not None:
            raise H5Error("%s exists" % path)
        return Group(self, path, self._require_group(path))

    def require_group(self, path):
        self._writable()
        path = "/" + path.strip("/")
        return Group(self, path, self._require_group(path))

    def _link(self, path, addr):
        parent, _, name = ("/" + path.strip("/")).rpartition("/")
        paddr = self._require_group(parent or "/")
        links = self._group_links(paddr)
        if name in links:
            raise H5Error("%s exists" % path)
        links[name] = addr
        self._set_group_links(paddr, links, parent or "/")

    @staticmethod
    def _dataspace(shape, maxshape=None):
        rank = len(shape)
        flags = 1 if maxshape is not None else 0
        b = struct.pack("<BBBB4x", 1, rank, flags, 0) + struct.pack("<%dQ" % rank, *shape)
        if maxshape is not None:
            b += struct.pack("<%dQ" % rank, *[UNDEF if m is None else m for m in maxshape])
        return b

    def create_dataset(self, path, shape=None, dtype=None, chunks=None, maxshape=None, data=None):
        self._writable()
        path = "/" + path.strip("/")
        if data is not None:
            data = np.asarray(data)
            if data.dtype.kind == "U":
                data = np.char.encode(data, "utf-8")
            shape = data.shape if shape is None else tuple(shape)
            dtype = data.dtype if dtype is None else np.dtype(dtype)
            data = np.ascontiguousarray(data, dtype=np.dtype(dtype).newbyteorder("<"))
        dtype = np.dtype(dtype).newbyteorder("<") if np.dtype(dtype).itemsize > 1 else np.dtype(dtype)
        shape = tuple(int(s) for s in shape)
        n = int(np.prod(shape)) if shape else 1
        # fill value message, version 2: allocation late (contiguous) or
        # incremental (chunked), fill written if set, the default (zero)
        # fill value -- the form libhdf5 writes for h5py datasets
        fill = struct.pack("<BBBBI", 2, 2 if chunks is None else 3, 2, 1, 0)
        dtmsg = (MSG_DATATYPE, _encode_datatype(dtype), 1)
        if chunks is None:
            raw = (data.tobytes() if data is not None else b"\0" * (n * dtype.itemsize))
            addr = self._append(raw) if n else UNDEF
            layout = struct.pack("<BBQQ", 3, 1, addr, n * dtype.itemsize)
            msgs = [(MSG_DATASPACE, self._dataspace(shape, shape)), dtmsg,
                    (MSG_FILL, fill, 1), (MSG_LAYOUT, layout, 1)]
        else:
            chunks = tuple(int(c) for c in chunks)
            if maxshape is None:
                maxshape = shape
            cd = list(chunks) + [dtype.itemsize]
            layout = struct.pack("<BBBQ", 3, 2, len(cd), UNDEF) + struct.pack("<%dI" % len(cd), *cd)
            msgs = [(MSG_DATASPACE, self._dataspace(shape, maxshape)), dtmsg,
                    (MSG_FILL, fill, 1), (MSG_LAYOUT, layout, 1)]
        hdr = self._write_object_header(msgs)
        self._link(path, hdr)
        ds = self[path]
        if chunks is not None and data is not None:
            ds.write_rows(0, data)
        return ds

    def __setitem__(self, path, value):
        self.create_dataset(path, data=np.asarray(value))

    def _write_contiguous(self, ds, data):
        self._writable()
        lay = ds._info["layout"]
        if lay[0] != "contiguous":
            raise H5Error("write() needs a contiguous dataset; use write_rows")
        data = np.ascontiguousarray(np.asarray(data), dtype=ds.dtype).reshape(ds.shape)
        self._wr(lay[1], data.tobytes())

    def _resize_chunked(self, ds, n0):
        self._writable()
        info = ds._info
        if info["layout"][0] != "chunked":
            raise H5Error("only chunked datasets can be resized")
        mx = info["maxdims"]
        if mx is not None and mx[0] is not None and n0 > mx[0]:
            raise H5Error("resize beyond the maximum shape")
        dims = [n0] + list(info["dims"][1:])
        self._wr(info["dataspace_at"] + 8, struct.pack("<%dQ" % len(dims), *dims))
        info["dims"] = dims

    def _write_rows(self, ds, start, rows):
        """Write rows [start, start + len(rows)) of a chunked dataset (the
        dataset grows along axis 0 if needed); chunks are allocated whole."""
        self._writable()
        info = ds._info
        _, bt, cd = info["layout"]
        cdims = cd[:-1]
        rows = np.ascontiguousarray(np.asarray(rows), dtype=ds.dtype)
        if list(rows.shape[1:]) != list(info["dims"][1:]):
            raise H5Error("row shape mismatch")
        if any(c < d for c, d in zip(cdims[1:], info["dims"][1:])):
            raise H5Error("chunks must span every axis but the first")
        end = start + rows.shape[0]
        if end > info["dims"][0]:
            self._resize_chunked(ds, end)
        entries = {tuple(o): (s, a) for o, s, a in self._chunk_entries(bt, len(cd))}
        c0 = cdims[0]
        nb = int(np.prod(cdims)) * rows.dtype.itemsize
        changed = False
        for ci in range(start // c0, (end - 1) // c0 + 1):
            key = tuple([ci * c0] + [0] * (len(cdims) - 1))
            if key not in entries:
                entries[key] = (nb, self._append(b"\0" * nb))
                changed = True
            _s, addr = entries[key]
            lo, hi = max(start, ci * c0), min(end, (ci + 1) * c0)
            blk = np.frombuffer(self._rd(addr, nb), dtype=rows.dtype).reshape(cdims).copy()
            blk[lo - ci * c0:hi - ci * c0] = rows[lo - start:hi - start]
            self._wr(addr, blk.tobytes())
        if changed:
            if len(entries) > 2 * CHUNK_K:
                raise H5Error("more chunks than one B-tree node holds")
            ordered = sorted(entries.items())
            rank1 = len(cd)
            node = bytearray(b"TREE" + bytes([1, 0]) + struct.pack("<H", len(ordered)) +
                             struct.pack("<QQ", UNDEF, UNDEF))
            for (offs, (size, addr)) in ordered:
                node += struct.pack("<II", size, 0) + struct.pack("<%dQ" % rank1, *(list(offs) + [0]))
                node += struct.pack("<Q", addr)
            last = list(ordered[-1][0])
            last[0] += c0
            node += struct.pack("<II", 0, 0) + struct.pack("<%dQ" % rank1, *(last + [0]))
            ksz = 8 + 8 * rank1
            node += b"\0" * (24 + 2 * CHUNK_K * (ksz + 8) + ksz - len(node))
            new_bt = self._append(bytes(node))
            self._wr(info["layout_at"] + 3, struct.pack("<Q", new_bt))
            info["layout"] = ("chunked", new_bt, cd)

    def flush(self):
        self._fh.flush()

    def close(self):
        if getattr(self, "_fh", None):
            self._fh.close()
            self._fh = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
