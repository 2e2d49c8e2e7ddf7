"""Minimal read-only HDF5 reader for the ChronusQ golden files.

Test infrastructure only: it is used by ``make_golden.py`` to turn the
reference's HDF5 test data (``tests/func/reference/contract.hdf5``,
``tests/scf/reference/*.bin.ref``) into small ``.npz`` fixtures.  There is no
h5py / libhdf5 in this image.

Supported subset (what ChronusQ's ``SafeFile`` writes through the HDF5 C++ API,
``include/util/files.hpp:64-339``):

* superblock version 0 (8-byte offsets and lengths),
* old-style groups: symbol-table message -> v1 B-tree + SNOD nodes + local heap,
* version-1 object headers with continuation blocks,
* dataspace messages v1/v2, datatype classes float (class 1) and compound
  (class 6, the ``{r,i}`` complex type of ``files.hpp:64-77``), fixed-point ints,
* contiguous and compact data layouts (message versions 1-3).

Datasets written from column-major N x N buffers come back as C-order arrays of
shape (N, N), i.e. transposed; callers transpose with ``.T``.
"""
import struct

import numpy as np


class H5Error(RuntimeError):
    pass


def _u(fmt, buf, off):
    return struct.unpack_from("<" + fmt, buf, off)


class H5File:
    def __init__(self, path):
        with open(path, "rb") as f:
            self.d = f.read()
        d = self.d
        if d[:8] != b"\x89HDF\r\n\x1a\n":
            raise H5Error("not an HDF5 file: %s" % path)
        if d[8] != 0:
            raise H5Error("only superblock version 0 is supported")
        if d[13] != 8 or d[14] != 8:
            raise H5Error("only 8-byte offsets/lengths are supported")
        # root group symbol-table entry starts at byte 56
        self.root = self._sym_entry(56)

    # -- low-level structures -------------------------------------------------
    def _sym_entry(self, off):
        name_off, ohdr, cache = _u("QQI", self.d, off)
        scratch = self.d[off + 24: off + 40]
        ent = {"name_off": name_off, "ohdr": ohdr, "cache": cache}
        if cache == 1:
            ent["btree"], ent["heap"] = struct.unpack("<QQ", scratch)
        return ent

    def _heap_data(self, addr):
        d = self.d
        if d[addr:addr + 4] != b"HEAP":
            raise H5Error("bad local heap at %d" % addr)
        size, _free, data = _u("QQQ", d, addr + 8)
        return data, size

    def _cstr(self, off):
        end = self.d.index(b"\0", off)
        return self.d[off:end].decode()

    def _group_entries(self, btree, heap):
        hdata, _ = self._heap_data(heap)
        out = {}
        self._walk_btree(btree, hdata, out)
        return out

    def _walk_btree(self, addr, hdata, out):
        d = self.d
        if d[addr:addr + 4] != b"TREE":
            raise H5Error("bad B-tree node at %d" % addr)
        ntype, level, used = d[addr + 4], d[addr + 5], _u("H", d, addr + 6)[0]
        if ntype != 0:
            raise H5Error("expected a group B-tree")
        p = addr + 24  # signature, type, level, used, left, right
        children = []
        for i in range(used):
            p += 8  # key i (heap offset)
            children.append(_u("Q", d, p)[0])
            p += 8
        for c in children:
            if level > 0:
                self._walk_btree(c, hdata, out)
            else:
                self._walk_snod(c, hdata, out)

    def _walk_snod(self, addr, hdata, out):
        d = self.d
        if d[addr:addr + 4] != b"SNOD":
            raise H5Error("bad symbol-table node at %d" % addr)
        nsym = _u("H", d, addr + 6)[0]
        for i in range(nsym):
            e = self._sym_entry(addr + 8 + 40 * i)
            out[self._cstr(hdata + e["name_off"])] = e

    def _messages(self, addr):
        d = self.d
        if d[addr] != 1:
            raise H5Error("only v1 object headers are supported (addr %d)" % addr)
        nmsg, _ref, hsize = _u("HII", d, addr + 2)
        blocks = [(addr + 16, hsize)]
        msgs = []
        while blocks and len(msgs) < nmsg:
            start, size = blocks.pop(0)
            p = start
            while p + 8 <= start + size and len(msgs) < nmsg:
                mtype, msize, _flags = _u("HHB", d, p)
                body = p + 8
                if mtype == 0x10:  # continuation
                    caddr, clen = _u("QQ", d, body)
                    blocks.append((caddr, clen))
                msgs.append((mtype, body, msize))
                p = body + msize
        return msgs

    # -- decoding of dataset metadata -----------------------------------------
    def _dataspace(self, off):
        d = self.d
        ver, ndim, flags = d[off], d[off + 1], d[off + 2]
        if ver == 1:
            p = off + 8
        elif ver == 2:
            p = off + 4
        else:
            raise H5Error("dataspace version %d" % ver)
        return tuple(_u("Q", d, p + 8 * i)[0] for i in range(ndim))

    def _datatype(self, off):
        d = self.d
        cv = d[off]
        cls, ver = cv & 0x0F, cv >> 4
        bits = d[off + 1] | (d[off + 2] << 8) | (d[off + 3] << 16)
        size = _u("I", d, off + 4)[0]
        if cls == 1:
            if bits & 1:
                raise H5Error("big-endian floats not supported")
            return np.dtype("<f%d" % size)
        if cls == 0:
            signed = bool(bits & 0x8)
            return np.dtype(("<i%d" if signed else "<u%d") % size)
        if cls == 6:
            nmemb = bits & 0xFFFF
            p = off + 8
            names, offs, types = [], [], []
            for _ in range(nmemb):
                name = self._cstr(p)
                if ver < 3:
                    p += (len(name) + 1 + 7) // 8 * 8
                    moff = _u("I", d, p)[0]
                    p += 4 + 1 + 3 + 4 + 4 + 16 if ver == 1 else 4
                else:
                    p += len(name) + 1
                    nb = 1 if size < 256 else 2 if size < 65536 else 4
                    moff = int.from_bytes(d[p:p + nb], "little")
                    p += nb
                mt, mlen = self._datatype_len(p)
                names.append(name)
                offs.append(moff)
                types.append(mt)
                p += mlen
            if names == ["r", "i"] and types[0] == types[1] == np.dtype("<f8") \
                    and offs == [0, 8] and size == 16:
                return np.dtype("<c16")
            return np.dtype({"names": names, "formats": types,
                             "offsets": offs, "itemsize": size})
        raise H5Error("datatype class %d not supported" % cls)

    def _datatype_len(self, off):
        cls = self.d[off] & 0x0F
        dt = self._datatype(off)
        if cls in (0, 1):
            plen = 4 if cls == 0 else 12
            return dt, 8 + plen
        raise H5Error("nested compound members not supported")

    def _layout(self, off):
        d = self.d
        ver = d[off]
        if ver == 3:
            cls = d[off + 1]
            if cls == 1:
                addr, size = _u("QQ", d, off + 2)
                return ("contig", addr, size)
            if cls == 0:
                size = _u("H", d, off + 2)[0]
                return ("compact", off + 4, size)
            raise H5Error("chunked layout not supported")
        if ver in (1, 2):
            ndim, cls = d[off + 1], d[off + 2]
            p = off + 8
            if cls == 1:
                addr = _u("Q", d, p)[0]
                return ("contig", addr, None)
            if cls == 0:
                p += 4 * ndim
                size = _u("I", d, p)[0]
                return ("compact", p + 4, size)
            raise H5Error("chunked layout not supported")
        raise H5Error("layout version %d" % ver)

    # -- public API ------------------------------------------------------------
    def _lookup(self, path):
        ent = self.root
        for part in [p for p in path.strip("/").split("/") if p]:
            if "btree" not in ent:
                ent = self._resolve_group(ent)
            kids = self._group_entries(ent["btree"], ent["heap"])
            if part not in kids:
                raise KeyError(path)
            ent = kids[part]
        return ent

    def _resolve_group(self, ent):
        for mtype, body, _ in self._messages(ent["ohdr"]):
            if mtype == 0x11:
                bt, hp = _u("QQ", self.d, body)
                return dict(ent, btree=bt, heap=hp)
        raise H5Error("object is not a group")

    def keys(self, path="/"):
        ent = self._lookup(path)
        if "btree" not in ent:
            ent = self._resolve_group(ent)
        return sorted(self._group_entries(ent["btree"], ent["heap"]).keys())

    def read(self, path):
        ent = self._lookup(path)
        shape = dtype = layout = None
        for mtype, body, _ in self._messages(ent["ohdr"]):
            if mtype == 0x01:
                shape = self._dataspace(body)
            elif mtype == 0x03:
                dtype = self._datatype(body)
            elif mtype == 0x08:
                layout = self._layout(body)
        if shape is None or dtype is None or layout is None:
            raise H5Error("%s is not a dataset" % path)
        n = int(np.prod(shape)) if shape else 1
        kind, addr, _size = layout
        nbytes = n * dtype.itemsize
        if addr == 0xFFFFFFFFFFFFFFFF:
            return np.zeros(shape, dtype)
        buf = self.d[addr:addr + nbytes]
        return np.frombuffer(buf, dtype=dtype, count=n).reshape(shape).copy()

    def walk(self, path="/"):
        """Yield every dataset path below ``path``."""
        for k in self.keys(path):
            sub = path.rstrip("/") + "/" + k
            ent = self._lookup(sub)
            is_group = "btree" in ent or any(
                m[0] == 0x11 for m in self._messages(ent["ohdr"]))
            if is_group:
                yield from self.walk(sub)
            else:
                yield sub
