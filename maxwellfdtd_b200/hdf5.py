"""A minimal HDF5 writer (and a reader of what it writes), for the reference's output file.

The reference saves its results with HDF5.jl (src/outputs.jl:33-65, 120-179, 437-472;
monitors.jl write_monitor): coordinate vectors, the PML indices, the material map, the
field snapshots under "fields", the running sums Sa/E2, rho_end and JE, and every monitor
under "monitors/<n>/...".  Neither h5py nor libhdf5 is available to this package, so it
writes the subset of the HDF5 file format (version 1.10 specification) such a file needs:

- superblock version 2 (checksummed);
- groups as version 2 object headers holding their links in Link messages ("compact"
  new-style groups: Link Info and Group Info messages, no heaps or B-trees);
- datasets as version 2 object headers with a version 2 Dataspace message, a Datatype
  message (IEEE little-endian float32/float64, signed little-endian int8..int64, unsigned
  uint8, and complex128 as the compound {"r": float64, "i": float64} that HDF5.jl uses for
  ComplexF64), a version 3 Fill Value message and a version 3 contiguous Data Layout message;
- every checksum is Jenkins' lookup3 hashlittle with initial value 0, as the format requires.

Array layout: a Julia array of size (n1, n2, ..., nk) is column-major, and HDF5.jl stores it
as the HDF5 dataspace (nk, ..., n2, n1) with the same bytes; the C-ordered numpy arrays of
this package ([t][z][y][x] for a field, x fastest) are therefore written as they are, which
is the dataspace the reference's file has.  Booleans (a monitor's issum) are written as
uint8 0/1 and monitor indices as an int64 array of 1-based (i, j, k) rows.
"""
import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
SIGNATURE = b"\x89HDF\r\n\x1a\n"


# ------------------------------------------------------------------------------------------
# Jenkins lookup3 hashlittle (Bob Jenkins, 2006, public domain), byte-wise form
# ------------------------------------------------------------------------------------------
def _rot(x, k):
    return ((x << k) | (x >> (32 - k))) & 0xFFFFFFFF


def lookup3(data, initval=0):
    """hashlittle(key, length, initval) of the lookup3 hash."""
    data = bytes(data)
    n = len(data)
    M = 0xFFFFFFFF
    a = b = c = (0xDEADBEEF + n + initval) & M
    i = 0
    while n > 12:
        a = (a + int.from_bytes(data[i:i + 4], "little")) & M
        b = (b + int.from_bytes(data[i + 4:i + 8], "little")) & M
        c = (c + int.from_bytes(data[i + 8:i + 12], "little")) & M
        a = (a - c) & M; a ^= _rot(c, 4); c = (c + b) & M
        b = (b - a) & M; b ^= _rot(a, 6); a = (a + c) & M
        c = (c - b) & M; c ^= _rot(b, 8); b = (b + a) & M
        a = (a - c) & M; a ^= _rot(c, 16); c = (c + b) & M
        b = (b - a) & M; b ^= _rot(a, 19); a = (a + c) & M
        c = (c - b) & M; c ^= _rot(b, 4); b = (b + a) & M
        n -= 12
        i += 12
    if n == 0:
        return c
    tail = data[i:i + n] + bytes(12 - n)
    a = (a + int.from_bytes(tail[0:4], "little")) & M
    b = (b + int.from_bytes(tail[4:8], "little")) & M
    c = (c + int.from_bytes(tail[8:12], "little")) & M
    c ^= b; c = (c - _rot(b, 14)) & M
    a ^= c; a = (a - _rot(c, 11)) & M
    b ^= a; b = (b - _rot(a, 25)) & M
    c ^= b; c = (c - _rot(b, 16)) & M
    a ^= c; a = (a - _rot(c, 4)) & M
    b ^= a; b = (b - _rot(a, 14)) & M
    c ^= b; c = (c - _rot(b, 24)) & M
    return c


# ------------------------------------------------------------------------------------------
# messages
# ------------------------------------------------------------------------------------------
def _float_type(size):
    """Datatype message body: IEEE little-endian floating point of 4 or 8 bytes."""
    sign, exp_loc, exp_size, man_size, bias = (31, 23, 8, 23, 127) if size == 4 else (63, 52, 11, 52, 1023)
    head = bytes([0x11, 0x20, sign, 0x00]) + struct.pack("<I", size)   # class 1, version 1; normalisation 2
    props = struct.pack("<HHBBBBI", 0, 8 * size, exp_loc, exp_size, 0, man_size, bias)
    return head + props


def _int_type(size, signed):
    head = bytes([0x10, 0x08 if signed else 0x00, 0x00, 0x00]) + struct.pack("<I", size)   # class 0, version 1
    return head + struct.pack("<HH", 0, 8 * size)


def _complex_type():
    """Compound {"r": float64 at 0, "i": float64 at 8}, datatype version 3."""
    f64 = _float_type(8)
    members = b"".join(name + b"\x00" + bytes([off]) + f64 for name, off in ((b"r", 0), (b"i", 8)))
    return bytes([0x36, 2, 0, 0]) + struct.pack("<I", 16) + members


def _datatype(dt):
    dt = np.dtype(dt)
    if dt == np.float32 or dt == np.float64:
        return _float_type(dt.itemsize)
    if dt == np.complex128:
        return _complex_type()
    if dt.kind in "iu":
        return _int_type(dt.itemsize, dt.kind == "i")
    raise TypeError(f"no HDF5 datatype for {dt}")


def _message(mtype, body):
    return struct.pack("<BHB", mtype, len(body), 0) + body


def _object_header(messages):
    """Version 2 object header, chunk size field of 4 bytes, no times, then the checksum."""
    body = b"".join(messages)
    head = b"OHDR" + bytes([2, 0x02]) + struct.pack("<I", len(body))
    block = head + body
    return block + struct.pack("<I", lookup3(block))


def _group_header(links):
    """links: [(name bytes, object header address)]."""
    msgs = [_message(0x02, bytes([0, 0]) + struct.pack("<QQ", UNDEF, UNDEF)),   # Link Info
            _message(0x0A, bytes([0, 0]))]                                      # Group Info
    for name, addr in links:
        if len(name) > 255:
            raise ValueError("link name longer than 255 bytes")
        msgs.append(_message(0x06, bytes([1, 0, len(name)]) + name + struct.pack("<Q", addr)))   # hard link
    return _object_header(msgs)


def _dataset_header(shape, dt, data_addr, nbytes):
    rank = len(shape)
    space = bytes([2, rank, 0, 1 if rank else 0]) + b"".join(struct.pack("<Q", int(n)) for n in shape)
    fill = bytes([3, 0x09])                      # allocated early, written if set, no value defined
    layout = bytes([3, 1]) + struct.pack("<QQ", data_addr if nbytes else UNDEF, nbytes)
    return _object_header([_message(0x01, space), _message(0x03, _datatype(dt)), _message(0x05, fill),
                           _message(0x08, layout)])


def _header_len(obj):
    """Length of an object's header, which does not depend on the addresses it holds."""
    if isinstance(obj, dict):
        return len(_group_header([(k.encode(), 0) for k in obj]))
    a = obj
    return len(_dataset_header(a.shape, a.dtype, 0, 1))


def _as_array(v):
    a = np.asarray(v)
    if a.dtype == np.bool_:
        a = a.astype(np.uint8)
    if a.dtype.byteorder == ">":
        a = a.astype(a.dtype.newbyteorder("<"))
    return a if a.flags["C_CONTIGUOUS"] else a.copy(order="C")   # keeps a scalar 0-d


def write(path, tree):
    """Write `tree` (a dict: name -> numpy array / scalar, or name -> dict for a group) as an
    HDF5 file.  Objects are laid out as: superblock, every object header (depth first), then
    every dataset's data, contiguous and 8-byte aligned."""
    def norm(t):
        return {str(k): (norm(v) if isinstance(v, dict) else _as_array(v)) for k, v in t.items()}
    root = norm(tree)
    order = []            # depth-first list of objects (the root first)

    def walk(obj):
        order.append(obj)
        if isinstance(obj, dict):
            for v in obj.values():
                walk(v)
    walk(root)
    addr = {}
    pos = 48
    for obj in order:
        addr[id(obj)] = pos
        pos += _header_len(obj)
    data_addr = {}
    for obj in order:
        if not isinstance(obj, dict) and obj.nbytes:
            pos = (pos + 7) // 8 * 8
            data_addr[id(obj)] = pos
            pos += obj.nbytes
    eof = pos
    with open(path, "wb") as f:
        sb = SIGNATURE + bytes([2, 8, 8, 0]) + struct.pack("<QQQQ", 0, UNDEF, eof, addr[id(root)])
        f.write(sb + struct.pack("<I", lookup3(sb)))
        for obj in order:
            if isinstance(obj, dict):
                h = _group_header([(k.encode(), addr[id(v)]) for k, v in obj.items()])
            else:
                h = _dataset_header(obj.shape, obj.dtype, data_addr.get(id(obj), 0), obj.nbytes)
            assert f.tell() == addr[id(obj)] and len(h) == _header_len(obj)
            f.write(h)
        for obj in order:
            if id(obj) in data_addr:
                f.write(bytes(data_addr[id(obj)] - f.tell()))
                obj.tofile(f)
        assert f.tell() == eof


# ------------------------------------------------------------------------------------------
# reader of the subset above (every checksum verified)
# ------------------------------------------------------------------------------------------
def _parse_type(b, off):
    """(numpy dtype, length of the datatype message) at b[off:]."""
    cls, ver = b[off] & 0x0F, b[off] >> 4
    size = struct.unpack_from("<I", b, off + 4)[0]
    if cls == 1:
        return np.dtype("<f%d" % size), 20
    if cls == 0:
        return np.dtype(("<i%d" if b[off + 1] & 0x08 else "<u%d") % size), 12
    if cls == 6 and ver == 3:
        n = b[off + 1] | (b[off + 2] << 8)
        p = off + 8
        names = []
        for _ in range(n):
            end = b.index(b"\x00", p)
            names.append(b[p:end].decode())
            p = end + 2                       # the name's null and a 1-byte offset (size 16)
            _, ln = _parse_type(b, p)
            p += ln
        if names == ["r", "i"] and size == 16:
            return np.dtype(np.complex128), p - off
    raise ValueError("datatype outside the written subset")


def _read_object(b, f, at):
    if b[at:at + 4] != b"OHDR" or b[at + 4] != 2:
        raise ValueError("not a version 2 object header")
    flags = b[at + 5]
    if flags & 0x30 or flags & 0x03 != 0x02:
        raise ValueError("object header outside the written subset")
    n = struct.unpack_from("<I", b, at + 6)[0]
    end = at + 10 + n
    if lookup3(b[at:end]) != struct.unpack_from("<I", b, end)[0]:
        raise ValueError("object header checksum mismatch")
    p = at + 10
    links, shape, dt, layout = {}, None, None, None
    while p + 4 <= end:
        mtype, size, _ = struct.unpack_from("<BHB", b, p)
        body = p + 4
        if mtype == 0x06:
            ln = b[body + 2]
            name = b[body + 3:body + 3 + ln].decode()
            links[name] = struct.unpack_from("<Q", b, body + 3 + ln)[0]
        elif mtype == 0x01:
            rank = b[body + 1]
            shape = tuple(struct.unpack_from("<%dQ" % rank, b, body + 4)) if rank else ()
        elif mtype == 0x03:
            dt, _ = _parse_type(b, body)
        elif mtype == 0x08:
            layout = struct.unpack_from("<QQ", b, body + 2)
        p = body + size
    if shape is None:
        return {k: _read_object(b, f, a) for k, a in links.items()}
    a_data, nbytes = layout
    count = int(np.prod(shape)) if shape else 1
    if nbytes == 0:
        return np.zeros(shape, dtype=dt)
    f.seek(a_data)
    return np.fromfile(f, dtype=dt, count=count).reshape(shape)


def read(path):
    """The tree of a file written by write()."""
    with open(path, "rb") as f:
        sb = f.read(48)
        if sb[:8] != SIGNATURE or sb[8] != 2 or lookup3(sb[:44]) != struct.unpack_from("<I", sb, 44)[0]:
            raise ValueError("not a version 2 superblock written by this module")
        eof, root = struct.unpack_from("<QQ", sb, 28)
        f.seek(0)
        head = f.read(min(eof, 1 << 26))
        return _read_object(head, f, root)
