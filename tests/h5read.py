"""A small HDF5 reader written from the HDF5 file format specification, for
the tests of the CXI files the library writes (no HDF5 library is available
here).  It follows the structures independently of the writer: version 0
superblock, version 1 object headers, groups as symbol tables (version 1
B-tree of node type 0 -> symbol table nodes, names in a local heap),
contiguous datasets of little-endian IEEE floats, signed integers and
compounds of floats.  read(path) returns {"/group/dataset": numpy array}.
"""
import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF


class H5Error(ValueError):
    pass


def _u(buf, at, n):
    return int.from_bytes(buf[at:at + n], "little")


def _messages(buf, addr):
    """(type, body bytes) of a version 1 object header's messages."""
    if buf[addr] != 1:
        raise H5Error("object header at %d: version %d" % (addr, buf[addr]))
    nmsg = _u(buf, addr + 2, 2)
    size = _u(buf, addr + 8, 4)
    at, end, out = addr + 16, addr + 16 + size, []
    while len(out) < nmsg and at < end:
        mtype, msize = _u(buf, at, 2), _u(buf, at + 2, 2)
        out.append((mtype, buf[at + 8:at + 8 + msize]))
        at += 8 + msize
    if len(out) != nmsg:
        raise H5Error("object header at %d: %d of %d messages" % (addr, len(out), nmsg))
    return out


def _heap_name(buf, heap, off):
    if buf[heap:heap + 4] != b"HEAP":
        raise H5Error("no local heap at %d" % heap)
    size, data = _u(buf, heap + 8, 8), _u(buf, heap + 24, 8)
    if off >= size:
        raise H5Error("name offset %d beyond the heap's %d bytes" % (off, size))
    end = buf.index(b"\0", data + off)
    return buf[data + off:end].decode()


def _group(buf, btree, heap):
    """(name, object header address) of a group's members, from its B-tree."""
    if buf[btree:btree + 4] != b"TREE" or buf[btree + 4] != 0:
        raise H5Error("no group B-tree at %d" % btree)
    level, used = buf[btree + 5], _u(buf, btree + 6, 2)
    members = []
    for k in range(used):
        child = _u(buf, btree + 24 + 8 + 16 * k, 8)
        if level > 0:
            members += _group(buf, child, heap)
            continue
        if buf[child:child + 4] != b"SNOD":
            raise H5Error("no symbol table node at %d" % child)
        for e in range(_u(buf, child + 6, 2)):
            at = child + 8 + 40 * e
            members.append((_heap_name(buf, heap, _u(buf, at, 8)), _u(buf, at + 8, 8)))
    names = [m[0] for m in members]
    if names != sorted(names):
        raise H5Error("group members not in name order: %s" % names)
    return members


def _float_type(body):
    cls, size = body[0] & 0x0F, _u(body, 4, 4)
    if cls != 1 or body[1] & 1:
        raise H5Error("not a little-endian float")
    return {4: "<f4", 8: "<f8"}[size]


def _dtype(body):
    cls = body[0] & 0x0F
    size = _u(body, 4, 4)
    if cls == 1:
        return np.dtype(_float_type(body))
    if cls == 0:
        if body[1] & 1:
            raise H5Error("big-endian integer")
        return np.dtype(("<i" if body[1] & 0x08 else "<u") + str(size))
    if cls == 6:
        if body[0] >> 4 != 1:
            raise H5Error("compound datatype version %d" % (body[0] >> 4))
        n, at, fields = _u(body, 1, 2), 8, []
        for _ in range(n):
            end = body.index(b"\0", at)
            name = body[at:end].decode()
            at += (end - at + 8) // 8 * 8
            off, ndim = _u(body, at, 4), body[at + 4]
            if ndim:
                raise H5Error("array members are not read")
            mt = body[at + 32:]
            fields.append((name, _float_type(mt), off))
            at += 32 + 20
        return np.dtype({"names": [f[0] for f in fields], "formats": [f[1] for f in fields],
                         "offsets": [f[2] for f in fields], "itemsize": size})
    raise H5Error("datatype class %d" % cls)


def _dataset(buf, msgs):
    shape = dt = layout = None
    for mtype, body in msgs:
        if mtype == 0x0001:
            if body[0] != 1:
                raise H5Error("dataspace version %d" % body[0])
            shape = tuple(_u(body, 8 + 8 * k, 8) for k in range(body[1]))
        elif mtype == 0x0003:
            dt = _dtype(body)
        elif mtype == 0x0008:
            if body[0] != 3 or body[1] != 1:
                raise H5Error("layout version %d class %d (contiguous version 3 read)" % (body[0], body[1]))
            layout = (_u(body, 2, 8), _u(body, 10, 8))
    if shape is None or dt is None or layout is None:
        raise H5Error("dataset without dataspace, datatype or layout")
    count = int(np.prod(shape)) if shape else 1
    if layout[1] != count * dt.itemsize:
        raise H5Error("layout size %d for %d elements of %d bytes" % (layout[1], count, dt.itemsize))
    return np.frombuffer(buf, dt, count, layout[0]).reshape(shape).copy()


def read(path):
    buf = open(path, "rb").read()
    if buf[:8] != b"\x89HDF\r\n\x1a\n":
        raise H5Error("no HDF5 signature")
    if buf[8] != 0 or buf[13] != 8 or buf[14] != 8:
        raise H5Error("superblock version %d, offsets %d, lengths %d" % (buf[8], buf[13], buf[14]))
    if _u(buf, 40, 8) != len(buf):
        raise H5Error("end-of-file address %d, file size %d" % (_u(buf, 40, 8), len(buf)))
    root = _u(buf, 64, 8)
    out = {}

    def walk(addr, path):
        msgs = _messages(buf, addr)
        stab = [b for t, b in msgs if t == 0x0011]
        if stab:
            for name, child in _group(buf, _u(stab[0], 0, 8), _u(stab[0], 8, 8)):
                walk(child, path + "/" + name)
        else:
            out[path] = _dataset(buf, msgs)

    walk(root, "")
    return out


def complex_of(a):
    """A {r, i} compound array as complex64."""
    return (a["r"] + 1j * a["i"]).astype(np.complex64)
