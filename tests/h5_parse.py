"""A small reader of HDF5 files, written from the HDF5 file format specification, for
checking the matrix dumps in the tests (libhdf5 and h5py are not available here).

It follows what a conforming reader does for a version-0 superblock: root group
symbol-table entry -> root object header -> symbol-table message -> v1 B-tree (group
nodes) -> symbol-table nodes -> names in the local heap -> the dataset's object
header (dataspace, datatype, layout messages) -> contiguous raw data.  Every
structure is validated (signatures, versions, sizes) on the way."""
import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF


class H5Error(ValueError):
    pass


def _u(buf, off, n):
    return int.from_bytes(buf[off:off + n], "little")


def _object_header_messages(buf, addr):
    if buf[addr] != 1:
        raise H5Error(f"object header version {buf[addr]} at {addr}")
    nmsg = _u(buf, addr + 2, 2)
    size = _u(buf, addr + 8, 4)
    msgs, off, end = [], addr + 16, addr + 16 + size
    while off < end and len(msgs) < nmsg:
        mtype, msize = _u(buf, off, 2), _u(buf, off + 2, 2)
        if msize % 8:
            raise H5Error("v1 message size not a multiple of 8")
        msgs.append((mtype, buf[off + 8:off + 8 + msize]))
        off += 8 + msize
    if len(msgs) != nmsg or off != end:
        raise H5Error("object header message count or size mismatch")
    return msgs


def _heap(buf, addr):
    if buf[addr:addr + 4] != b"HEAP" or buf[addr + 4] != 0:
        raise H5Error("bad local heap")
    size, free, data = _u(buf, addr + 8, 8), _u(buf, addr + 16, 8), _u(buf, addr + 24, 8)
    seg = buf[data:data + size]
    # walk the free list: offsets are multiples of 8 and end at 1
    while free != 1:
        if free >= size or free % 8:
            raise H5Error("bad heap free list")
        nxt, fsize = _u(seg, free, 8), _u(seg, free + 8, 8)
        if free + fsize > size:
            raise H5Error("free block past the heap")
        free = nxt
    return seg


def _name(seg, off):
    end = seg.index(b"\0", off)
    return seg[off:end].decode()


def read_datasets(path):
    """{name: numpy array} of the datasets in the root group."""
    buf = open(path, "rb").read()
    if buf[:8] != b"\x89HDF\r\n\x1a\n":
        raise H5Error("not an HDF5 file")
    if buf[8] != 0 or buf[13] != 8 or buf[14] != 8:
        raise H5Error("expected superblock version 0 with 8-byte offsets and lengths")
    leaf_k, internal_k = _u(buf, 16, 2), _u(buf, 18, 2)
    eof = _u(buf, 40, 8)
    if eof != len(buf):
        raise H5Error(f"end-of-file address {eof} != file size {len(buf)}")
    root_oh = _u(buf, 56 + 8, 8)
    cache_type = _u(buf, 56 + 16, 4)
    msgs = dict(_object_header_messages(buf, root_oh))
    if 0x0011 not in msgs:
        raise H5Error("root group has no symbol-table message")
    btree, heap = struct.unpack("<QQ", msgs[0x0011][:16])
    if cache_type == 1 and (_u(buf, 56 + 24, 8), _u(buf, 56 + 32, 8)) != (btree, heap):
        raise H5Error("superblock scratch-pad disagrees with the root symbol-table message")
    seg = _heap(buf, heap)
    if buf[btree:btree + 4] != b"TREE" or buf[btree + 4] != 0:
        raise H5Error("bad group B-tree node")
    level, used = buf[btree + 5], _u(buf, btree + 6, 2)
    if level != 0:
        raise H5Error("only leaf group B-trees are read here")
    node_size = 24 + 2 * internal_k * 8 + (2 * internal_k + 1) * 8
    if btree + node_size > len(buf):
        raise H5Error("B-tree node truncated")
    out = {}
    for c in range(used):
        child = _u(buf, btree + 24 + 8 + 16 * c, 8)
        if buf[child:child + 4] != b"SNOD" or buf[child + 4] != 1:
            raise H5Error("bad symbol-table node")
        if child + 8 + 2 * leaf_k * 40 > len(buf):
            raise H5Error("symbol-table node truncated")
        for e in range(_u(buf, child + 6, 2)):
            ent = child + 8 + 40 * e
            name = _name(seg, _u(buf, ent, 8))
            out[name] = _dataset(buf, _u(buf, ent + 8, 8))
    return out


def _dataset(buf, addr):
    msgs = dict(_object_header_messages(buf, addr))
    sp = msgs[0x0001]
    if sp[0] != 1:
        raise H5Error("dataspace version")
    rank = sp[1]
    dims = [_u(sp, 8 + 8 * d, 8) for d in range(rank)]
    ty = msgs[0x0003]
    if ty[0] != 0x11:
        raise H5Error("expected a version-1 floating-point datatype")
    size = _u(ty, 4, 4)
    if ty[1] & 1:
        raise H5Error("big-endian data")
    dtype = {4: np.float32, 8: np.float64}[size]
    if (_u(ty, 10, 2), ty[13], _u(ty, 16, 4)) != ((32, 8, 127) if size == 4 else (64, 11, 1023)):
        raise H5Error("not an IEEE float layout")
    lay = msgs[0x0008]
    if lay[0] != 3 or lay[1] != 1:
        raise H5Error("expected a version-3 contiguous layout")
    daddr, nbytes = struct.unpack("<QQ", lay[2:18])
    if nbytes != int(np.prod(dims)) * size or daddr + nbytes > len(buf):
        raise H5Error("data size mismatch")
    return np.frombuffer(buf[daddr:daddr + nbytes], dtype).reshape(dims)
