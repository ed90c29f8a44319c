"""REST's HDF5 guess and checkpoint files, read and written without libhdf5.

REST hands densities and orbitals between runs through two HDF5 files:

* the external initial guess (``initial_guess_from_hdf5guess``,
  src/initial_guess/mod.rs:71-83): dataset ``init_guess`` at the root, read
  raw as f64; spin s is the column-major n x n density at raw elements
  [s n^2, (s + 1) n^2);
* the restart chkfile (``initial_guess_from_hdf5chk``, :85-124, written by
  ``save_chkfile``, src/post_scf_analysis/mod.rs:47-103): group ``scf`` with
  the scalar ``e_tot``, ``mo_coeff`` read raw per spin as a row-major
  (num_basis x num_state) block -- i.e. C[mu, i] at mu * num_state + i -- and
  ``mo_energy`` (num_state per spin).

Neither h5py nor libhdf5 is available here, so this module implements the
part of the public HDF5 file format these files use: superblock version 0
with 8-byte offsets and lengths, version-1 object headers (with continuation
blocks), groups as symbol tables (version-1 B-tree of group nodes, symbol
table nodes, local heap), dataspace messages of version 1 and 2, IEEE
little-endian floating-point and integer datatypes, and data layout version 3
(contiguous and compact).  The reader is pinned against files that libhdf5
wrote (REST's example chkfiles, tests/test_chkfile.py); the writer produces
the same structures libhdf5 writes for such files, so that REST's reader
(the ``hdf5`` crate over libhdf5) opens them.

The learned initial guess uses ``write_init_guess`` to hand its density to
REST's own guess path (``external_init_guess = true``, ``guessfile_type =
"hdf5"``) as a drop-in.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

SIGNATURE = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF

# message types of version-1 object headers
MSG_NIL, MSG_DATASPACE, MSG_DATATYPE, MSG_FILL, MSG_LAYOUT, MSG_CONT, MSG_STAB = 0x0, 0x1, 0x3, 0x5, 0x8, 0x10, 0x11


class HDF5FormatError(ValueError):
    pass


# ---------------------------------------------------------------------------
# reader
# ---------------------------------------------------------------------------
@dataclass
class _Object:
    messages: list  # (type, flags, bytes)


class H5Reader:
    """Read-only view of an HDF5 file with a version-0 superblock."""

    def __init__(self, data: bytes):
        self.b = data
        if data[:8] != SIGNATURE:
            raise HDF5FormatError("not an HDF5 file (signature)")
        ver = data[8]
        if ver not in (0, 1):
            raise HDF5FormatError(f"superblock version {ver} not supported (0 and 1 are)")
        so, sl = data[13], data[14]
        if so != 8 or sl != 8:
            raise HDF5FormatError(f"offset/length sizes {so}/{sl} not supported (8/8 are)")
        p = 24 + (4 if ver == 1 else 0)  # version 1 adds indexed-storage K + reserved
        self.base = self._q(p)
        root_entry = p + 32  # base, free-space, EOF, driver addresses
        self.root = self._q(root_entry + 8)

    @classmethod
    def open(cls, path) -> "H5Reader":
        with open(path, "rb") as f:
            return cls(f.read())

    def _q(self, off):
        return struct.unpack_from("<Q", self.b, off)[0]

    def _addr(self, a):
        return self.base + a

    # object headers ----------------------------------------------------------
    def _object(self, addr) -> _Object:
        b = self.b
        a = self._addr(addr)
        if b[a] != 1:
            raise HDF5FormatError(f"object header version {b[a]} at {addr} not supported (1 is)")
        nmsg, _refc, hsize = struct.unpack_from("<HII", b, a + 2)
        blocks = [(a + 16, hsize)]
        msgs = []
        while blocks:
            p, size = blocks.pop(0)
            end = p + size
            while p + 8 <= end and len(msgs) < nmsg:
                mtype, msize, mflags = struct.unpack_from("<HHB", b, p)
                body = b[p + 8:p + 8 + msize]
                if mtype == MSG_CONT:
                    caddr, clen = struct.unpack_from("<QQ", body)
                    blocks.append((self._addr(caddr), clen))
                msgs.append((mtype, mflags, body))
                p += 8 + msize
        return _Object(msgs)

    # groups ------------------------------------------------------------------
    def _group_entries(self, obj: _Object) -> dict:
        stab = [m for m in obj.messages if m[0] == MSG_STAB]
        if not stab:
            raise HDF5FormatError("object is not a group (no symbol table message)")
        btree, heap = struct.unpack_from("<QQ", stab[0][2])
        h = self._addr(heap)
        if self.b[h:h + 4] != b"HEAP":
            raise HDF5FormatError("local heap signature")
        _dsize, _free, data_addr = struct.unpack_from("<QQQ", self.b, h + 8)
        heap_data = self._addr(data_addr)
        out = {}
        self._walk_btree(btree, heap_data, out)
        return out

    def _walk_btree(self, addr, heap_data, out):
        b = self.b
        a = self._addr(addr)
        if b[a:a + 4] != b"TREE":
            raise HDF5FormatError("B-tree signature")
        ntype, level, nent = struct.unpack_from("<BBH", b, a + 4)
        if ntype != 0:
            raise HDF5FormatError("expected a group B-tree node")
        p = a + 24
        for _ in range(nent):
            child = struct.unpack_from("<Q", b, p + 8)[0]  # skip key i
            p += 16
            if level > 0:
                self._walk_btree(child, heap_data, out)
                continue
            s = self._addr(child)
            if b[s:s + 4] != b"SNOD":
                raise HDF5FormatError("symbol table node signature")
            nsym = struct.unpack_from("<H", b, s + 6)[0]
            q = s + 8
            for _ in range(nsym):
                name_off, ohdr = struct.unpack_from("<QQ", b, q)
                start = heap_data + name_off
                name = b[start:b.index(b"\0", start)].decode()
                out[name] = ohdr
                q += 40

    def _resolve(self, path: str) -> int:
        addr = self.root
        for part in [x for x in path.strip("/").split("/") if x]:
            ent = self._group_entries(self._object(addr))
            if part not in ent:
                raise KeyError(f"{path!r}: no member {part!r}")
            addr = ent[part]
        return addr

    def keys(self, path: str = "/") -> list:
        return sorted(self._group_entries(self._object(self._resolve(path))))

    # datasets ----------------------------------------------------------------
    def dataset(self, path: str) -> np.ndarray:
        obj = self._object(self._resolve(path))
        msg = {m[0]: m[2] for m in obj.messages}
        for need in (MSG_DATASPACE, MSG_DATATYPE, MSG_LAYOUT):
            if need not in msg:
                raise HDF5FormatError(f"{path!r} is not a dataset (message {need:#x} missing)")
        shape = _parse_dataspace(msg[MSG_DATASPACE])
        dtype = _parse_datatype(msg[MSG_DATATYPE])
        lay = msg[MSG_LAYOUT]
        if lay[0] != 3:
            raise HDF5FormatError(f"layout message version {lay[0]} not supported (3 is)")
        count = int(np.prod(shape)) if shape else 1
        nbytes = count * dtype.itemsize
        if lay[1] == 1:  # contiguous
            addr, size = struct.unpack_from("<QQ", lay, 2)
            if addr == UNDEF:
                raw = b"\0" * nbytes  # never written: the fill value (zero)
            else:
                if size < nbytes:
                    raise HDF5FormatError("contiguous storage smaller than the dataspace")
                a = self._addr(addr)
                raw = self.b[a:a + nbytes]
        elif lay[1] == 0:  # compact
            size = struct.unpack_from("<H", lay, 2)[0]
            raw = lay[4:4 + size][:nbytes]
        else:
            raise HDF5FormatError("chunked storage not supported")
        return np.frombuffer(raw, dtype=dtype, count=count).reshape(shape).copy()


def _parse_dataspace(m: bytes) -> tuple:
    ver, rank, flags = m[0], m[1], m[2]
    if ver == 1:
        off = 8
    elif ver == 2:
        if m[3] == 2:  # null dataspace
            return (0,)
        off = 4
    else:
        raise HDF5FormatError(f"dataspace version {ver} not supported")
    return tuple(struct.unpack_from(f"<{rank}Q", m, off)) if rank else ()


def _parse_datatype(m: bytes) -> np.dtype:
    cls, ver = m[0] & 0x0F, m[0] >> 4
    bits = m[1] | (m[2] << 8) | (m[3] << 16)
    size = struct.unpack_from("<I", m, 4)[0]
    big = bool(bits & 1)
    if cls == 1:  # floating point
        if size not in (4, 8):
            raise HDF5FormatError(f"float of {size} bytes not supported")
        return np.dtype((">" if big else "<") + ("f8" if size == 8 else "f4"))
    if cls == 0:  # fixed point
        signed = bool(bits & 8)
        return np.dtype((">" if big else "<") + ("i" if signed else "u") + str(size))
    raise HDF5FormatError(f"datatype class {cls} (version {ver}) not supported")


# ---------------------------------------------------------------------------
# writer
# ---------------------------------------------------------------------------
GROUP_LEAF_K = 4       # symbol table node capacity 2K entries (libhdf5's default)
GROUP_INTERNAL_K = 16  # group B-tree node capacity 2K children (libhdf5's default)


@dataclass
class _Group:
    children: dict = field(default_factory=dict)  # name -> _Group | np.ndarray


class H5Writer:
    """Builds an HDF5 file of groups and contiguous little-endian datasets in
    the layout libhdf5 writes with its default settings: superblock version 0,
    version-1 object headers, one symbol table (B-tree leaf + symbol table
    node + local heap) per group."""

    def __init__(self):
        self.root = _Group()

    def create_dataset(self, path: str, data) -> None:
        arr = np.array(data, order="C")  # keeps a 0-d array 0-d (a scalar dataspace)
        if arr.dtype.kind not in "fiu":
            raise TypeError("only numeric datasets are written")
        arr = arr.astype(arr.dtype.newbyteorder("<"), copy=False)
        g, name = self._parent(path, create=True)
        if name in g.children:
            raise ValueError(f"{path!r} exists")
        g.children[name] = arr

    def _parent(self, path, create):
        parts = [x for x in path.strip("/").split("/") if x]
        g = self.root
        for p in parts[:-1]:
            nxt = g.children.get(p)
            if nxt is None and create:
                nxt = g.children[p] = _Group()
            if not isinstance(nxt, _Group):
                raise ValueError(f"{p!r} is not a group")
            g = nxt
        return g, parts[-1]

    # layout --------------------------------------------------------------------
    def tobytes(self) -> bytes:
        self._buf = bytearray(96)  # superblock, filled in last
        root_ohdr, root_btree, root_heap = self._emit_group(self.root)
        eof = len(self._buf)
        sb = bytearray(SIGNATURE)
        sb += bytes([0, 0, 0, 0, 0, 8, 8, 0])  # versions, sizes of offsets / lengths
        sb += struct.pack("<HHI", GROUP_LEAF_K, GROUP_INTERNAL_K, 0)
        sb += struct.pack("<QQQQ", 0, UNDEF, eof, UNDEF)
        sb += _symbol_entry(0, root_ohdr, cache=(root_btree, root_heap))
        assert len(sb) == 96
        self._buf[:96] = sb
        return bytes(self._buf)

    def save(self, path) -> None:
        with open(path, "wb") as f:
            f.write(self.tobytes())

    def _alloc(self, nbytes, align=8) -> int:
        pad = (-len(self._buf)) % align
        self._buf += b"\0" * pad
        at = len(self._buf)
        self._buf += b"\0" * nbytes
        return at

    def _put(self, at, data: bytes):
        self._buf[at:at + len(data)] = data

    def _emit_group(self, g: _Group):
        names = sorted(g.children)  # symbol table entries are kept in name order
        if len(names) > 2 * GROUP_LEAF_K:
            raise ValueError(f"a group holds at most {2 * GROUP_LEAF_K} members here")
        # object header: one symbol table message
        ohdr = self._alloc(16 + 8 + 16)
        btree = self._alloc(24 + (2 * GROUP_INTERNAL_K + 1) * 8 + 2 * GROUP_INTERNAL_K * 8)
        # local heap: the empty name at 0, then every name, 8-byte aligned
        heap_data = bytearray(8)
        name_off = {}
        for nm in names:
            name_off[nm] = len(heap_data)
            enc = nm.encode() + b"\0"
            heap_data += enc + b"\0" * ((-len(enc)) % 8)
        heap_data += b"\0" * max(0, 88 - len(heap_data))  # room libhdf5 leaves for more names
        heap = self._alloc(32)
        heap_at = self._alloc(len(heap_data))
        self._put(heap_at, heap_data)
        free = UNDEF
        last = 8 + sum(len(nm.encode()) + 1 + (-(len(nm.encode()) + 1)) % 8 for nm in names)
        if last + 16 <= len(heap_data):  # the unused tail is one free block (next = 1: the last)
            free = last
            self._put(heap_at + last, struct.pack("<QQ", 1, len(heap_data) - last))
        self._put(heap, b"HEAP" + bytes([0, 0, 0, 0]) + struct.pack("<QQQ", len(heap_data), free, heap_at))
        # children, then the symbol table node that lists them
        entries = []
        for nm in names:
            ch = g.children[nm]
            if isinstance(ch, _Group):
                c_ohdr, c_bt, c_hp = self._emit_group(ch)
                entries.append(_symbol_entry(name_off[nm], c_ohdr, cache=(c_bt, c_hp)))
            else:
                entries.append(_symbol_entry(name_off[nm], self._emit_dataset(ch)))
        snod = self._alloc(8 + 2 * GROUP_LEAF_K * 40)
        node = bytearray(b"SNOD" + bytes([1, 0]) + struct.pack("<H", len(entries)))
        for e in entries:
            node += e
        self._put(snod, node)
        # B-tree leaf: key 0 = the empty name, key 1 = the last name of the child
        tree = bytearray(b"TREE" + bytes([0, 0]) + struct.pack("<H", 1 if names else 0))
        tree += struct.pack("<QQ", UNDEF, UNDEF)
        if names:
            tree += struct.pack("<QQQ", 0, snod, name_off[names[-1]])
        else:
            tree += struct.pack("<Q", 0)
        self._put(btree, tree)
        msg = _message(MSG_STAB, struct.pack("<QQ", btree, heap))
        self._put(ohdr, struct.pack("<BBHII", 1, 0, 1, 1, len(msg)) + b"\0" * 4 + msg)
        return ohdr, btree, heap

    def _emit_dataset(self, arr: np.ndarray) -> int:
        msgs = [
            _message(MSG_DATASPACE, _dataspace_v1(arr.shape)),
            _message(MSG_DATATYPE, _datatype(arr.dtype), flags=1),
            _message(MSG_FILL, bytes([2, 2, 2, 1, 0, 0, 0, 0]), flags=1),
        ]
        data_at_placeholder = len(msgs)
        msgs.append(b"")  # layout, once the data address is known
        size = sum(len(m) for m in msgs) + 8 + 24
        ohdr = self._alloc(16 + size)
        data_at = self._alloc(arr.nbytes if arr.nbytes else 0)
        self._put(data_at, arr.tobytes())
        msgs[data_at_placeholder] = _message(MSG_LAYOUT, struct.pack("<BBQQ", 3, 1, data_at, arr.nbytes))
        body = b"".join(msgs)
        self._put(ohdr, struct.pack("<BBHII", 1, 0, len(msgs), 1, len(body)) + b"\0" * 4 + body)
        return ohdr


def _message(mtype: int, body: bytes, flags: int = 0) -> bytes:
    body = body + b"\0" * ((-len(body)) % 8)
    return struct.pack("<HHB3x", mtype, len(body), flags) + body


def _symbol_entry(name_off: int, ohdr: int, cache=None) -> bytes:
    if cache is None:
        return struct.pack("<QQII", name_off, ohdr, 0, 0) + b"\0" * 16
    return struct.pack("<QQIIQQ", name_off, ohdr, 1, 0, cache[0], cache[1])


def _dataspace_v1(shape) -> bytes:
    rank = len(shape)
    out = struct.pack("<BBBB4x", 1, rank, 1 if rank else 0, 0)
    if rank:
        out += struct.pack(f"<{rank}Q", *shape) + struct.pack(f"<{rank}Q", *shape)
    return out


def _datatype(dt: np.dtype) -> bytes:
    size = dt.itemsize
    if dt.kind == "f":
        if size == 8:
            props = struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
            bits = (0x20, 0x3F, 0x00)
        elif size == 4:
            props = struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
            bits = (0x20, 0x1F, 0x00)
        else:
            raise TypeError(f"float of {size} bytes")
        return bytes([0x11, *bits]) + struct.pack("<I", size) + props
    signed = dt.kind == "i"
    return bytes([0x10, 0x08 if signed else 0x00, 0, 0]) + struct.pack("<IHH", size, 0, 8 * size)


# ---------------------------------------------------------------------------
# REST's files
# ---------------------------------------------------------------------------
def rest_ao_order(shells) -> np.ndarray:
    """Index map from this library's AO order to REST's.

    Both order shells alike and the functions of a shell by m = -l..l, except
    for p shells: here the real solid harmonics S_1,-1 S_1,0 S_1,1 = (y, z, x),
    in REST (libcint's spherical functions) (x, y, z).  REST function i is this
    library's function perm[i]: ``m_rest = m[np.ix_(perm, perm)]``,
    ``c_rest = c[perm]``.  (Checked on REST's Cu2 example chkfile, s to f
    shells: its orbitals are orthonormal under this library's overlap after
    this map.)"""
    perm, off = [], 0
    for l in np.asarray(shells.l):
        w = 2 * int(l) + 1
        perm += [off + 2, off, off + 1] if int(l) == 1 else list(range(off, off + w))
        off += w
    return np.asarray(perm, dtype=np.int64)


def _to_rest(m, perm, cols_too=True):
    if perm is None:
        return m
    return m[np.ix_(perm, perm)] if cols_too else m[perm]


def _from_rest(m, perm, cols_too=True):
    if perm is None:
        return m
    inv = np.argsort(perm)
    return m[np.ix_(inv, inv)] if cols_too else m[inv]


def write_init_guess(path, densities, shells=None) -> None:
    """The external initial guess REST reads (src/initial_guess/mod.rs:71-83):
    dataset ``init_guess`` whose raw f64 elements are the column-major n x n
    density of each spin, spin after spin (shape (n, n) for one spin, as
    PySCF writes it, (2, n, n) for two).  With ``shells`` (the AO basis) the
    densities are taken in this library's AO order and written in REST's."""
    perm = None if shells is None else rest_ao_order(shells)
    dms = [_to_rest(np.asarray(d, dtype=np.float64), perm) for d in densities]
    n = dms[0].shape[0]
    if any(d.shape != (n, n) for d in dms) or len(dms) not in (1, 2):
        raise ValueError("one or two n x n densities")
    raw = np.concatenate([d.ravel(order="F") for d in dms])
    w = H5Writer()
    w.create_dataset("init_guess", raw.reshape((n, n) if len(dms) == 1 else (2, n, n)))
    w.save(path)


def read_init_guess(path, num_basis: int, spin_channel: int = 1, shells=None) -> list:
    """REST's initial_guess_from_hdf5guess: per spin a column-major n x n
    density (in this library's AO order when ``shells`` is given)."""
    raw = H5Reader.open(path).dataset("init_guess").ravel()
    n2 = num_basis * num_basis
    if raw.size < spin_channel * n2:
        raise HDF5FormatError(f"init_guess holds {raw.size} values, {spin_channel * n2} needed")
    perm = None if shells is None else rest_ao_order(shells)
    return [np.asfortranarray(_from_rest(raw[s * n2:(s + 1) * n2].reshape((num_basis, num_basis), order="F"), perm))
            for s in range(spin_channel)]


def write_chkfile(path, e_tot: float, mo_coeff, mo_energy, mo_occ=None, shells=None) -> None:
    """REST's restart chkfile (save_chkfile, src/post_scf_analysis/mod.rs:47-103):
    group ``scf`` with ``e_tot`` (scalar), ``mo_coeff`` and ``mo_energy``
    (``mo_occ`` optional).  mo_coeff: per spin the n x num_state coefficient
    matrix; stored row-major so that REST's reader, which takes each spin's raw
    block as a column-major (num_state x n) matrix and transposes it, gets it
    back.  With ``shells`` the rows are taken in this library's AO order and
    written in REST's."""
    perm = None if shells is None else rest_ao_order(shells)
    cs = [_to_rest(np.asarray(c, dtype=np.float64), perm, cols_too=False) for c in mo_coeff]
    es = [np.asarray(e, dtype=np.float64) for e in mo_energy]
    w = H5Writer()
    w.create_dataset("scf/e_tot", np.float64(e_tot))
    w.create_dataset("scf/mo_coeff", cs[0] if len(cs) == 1 else np.stack(cs))
    w.create_dataset("scf/mo_energy", es[0] if len(es) == 1 else np.stack(es))
    if mo_occ is not None:
        os_ = [np.asarray(o, dtype=np.float64) for o in mo_occ]
        w.create_dataset("scf/mo_occ", os_[0] if len(os_) == 1 else np.stack(os_))
    w.save(path)


def read_chkfile(path, num_basis: int, num_state: int, spin_channel: int = 1, shells=None):
    """REST's initial_guess_from_hdf5chk: (e_tot, eigenvectors, eigenvalues),
    eigenvectors per spin as n x num_state (rows in this library's AO order
    when ``shells`` is given), eigenvalues num_state per spin."""
    r = H5Reader.open(path)
    e_tot = float(r.dataset("scf/e_tot").ravel()[0])
    c = r.dataset("scf/mo_coeff").ravel()
    e = r.dataset("scf/mo_energy").ravel()
    blk = num_basis * num_state
    perm = None if shells is None else rest_ao_order(shells)
    vecs = [np.asfortranarray(_from_rest(c[s * blk:(s + 1) * blk].reshape(num_basis, num_state), perm, False))
            for s in range(spin_channel)]
    vals = [e[s * num_state:(s + 1) * num_state].copy() for s in range(spin_channel)]
    return e_tot, vecs, vals
