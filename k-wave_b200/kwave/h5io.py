"""k-Wave HDF5 files without libhdf5.

``write_input_file`` restates the reference's file writers
(``k-Wave/private/kspaceFirstOrder_saveToDisk.m:452-485``,
``k-Wave/writeMatrix.m:56-213``, ``k-Wave/writeAttributes.m:56-70``): every
float dataset is single precision, every integer dataset uint64, each with
``data_type`` / ``domain_type`` string attributes, dataset dimensions in
MATLAB order reversed (x fastest), plus the root attributes of a version 1.2
input file.  ``read`` loads a dataset from any file this package, the
solver binary or MATLAB's HDF5 library writes (superblock 0-3, object
header 1-2, symbol-table or compact-link groups, contiguous / compact /
chunked B-tree-v1 storage, deflate and shuffle filters).

The on-disk structures follow the published HDF5 File Format
Specification; the metadata checksum is Bob Jenkins' lookup3 hashlittle.
"""
from __future__ import annotations

import datetime
import mmap
import struct
import warnings
import zlib

import numpy as np

SIG = b"\x89HDF\r\n\x1a\n"
UNDEF = 0xFFFFFFFFFFFFFFFF


# ---------------------------------------------------------------------------
# lookup3
# ---------------------------------------------------------------------------
def lookup3(data: bytes, initval: int = 0) -> int:
    """Bob Jenkins' lookup3 hashlittle() (public domain)."""
    M = 0xFFFFFFFF

    def rot(x, k):
        return ((x << k) | (x >> (32 - k))) & M

    n = len(data)
    a = b = c = (0xDEADBEEF + n + initval) & M
    k = 0
    while n > 12:
        a = (a + int.from_bytes(data[k:k + 4], "little")) & M
        b = (b + int.from_bytes(data[k + 4:k + 8], "little")) & M
        c = (c + int.from_bytes(data[k + 8:k + 12], "little")) & M
        a = (a - c) & M; a ^= rot(c, 4); c = (c + b) & M
        b = (b - a) & M; b ^= rot(a, 6); a = (a + c) & M
        c = (c - b) & M; c ^= rot(b, 8); b = (b + a) & M
        a = (a - c) & M; a ^= rot(c, 16); c = (c + b) & M
        b = (b - a) & M; b ^= rot(a, 19); a = (a + c) & M
        c = (c - b) & M; c ^= rot(b, 4); b = (b + a) & M
        n -= 12
        k += 12
    if n == 0:
        return c
    tail = data[k:k + n] + bytes(12 - n)
    a = (a + int.from_bytes(tail[0:4], "little")) & M
    b = (b + int.from_bytes(tail[4:8], "little")) & M
    c = (c + int.from_bytes(tail[8:12], "little")) & M
    c ^= b; c = (c - rot(b, 14)) & M
    a ^= c; a = (a - rot(c, 11)) & M
    b ^= a; b = (b - rot(a, 25)) & M
    c ^= b; c = (c - rot(b, 16)) & M
    a ^= c; a = (a - rot(c, 4)) & M
    b ^= a; b = (b - rot(a, 14)) & M
    c ^= b; c = (c - rot(b, 24)) & M
    return c


# ---------------------------------------------------------------------------
# writer (superblock 2, object header 2, compact links, contiguous data)
# ---------------------------------------------------------------------------
def _msg(mtype, body: bytes) -> bytes:
    return struct.pack("<BHB", mtype, len(body), 0) + body


def _ohdr(msgs: bytes) -> bytes:
    h = b"OHDR" + struct.pack("<BBI", 2, 0x02, len(msgs)) + msgs
    return h + struct.pack("<I", lookup3(h))


def _attr(name: str, value: str) -> bytes:
    v = value.encode() + b"\0"
    dt = struct.pack("<BBBBI", 0x13, 0, 0, 0, len(v))
    ds = struct.pack("<BBBB", 2, 0, 0, 0)
    nm = name.encode() + b"\0"
    return _msg(0x0C, struct.pack("<BBHHHB", 3, 0, len(nm), len(dt), len(ds), 0) + nm + dt + ds + v)


def _dtype(arr: np.ndarray) -> bytes:
    if arr.dtype == np.float32:
        return struct.pack("<BBBBIHHBBBBI", 0x11, 0x20, 31, 0, 4, 0, 32, 23, 8, 0, 23, 127)
    if arr.dtype == np.float64:
        return struct.pack("<BBBBIHHBBBBI", 0x11, 0x20, 63, 0, 8, 0, 64, 52, 11, 0, 52, 1023)
    if arr.dtype == np.uint64:
        return struct.pack("<BBBBIHH", 0x10, 0, 0, 0, 8, 0, 64)
    raise TypeError(arr.dtype)


class _Node:
    def __init__(self, group=True):
        self.group = group
        self.children = {}
        self.attrs = {}
        self.arr = None
        self.addr = 0
        self.data_addr = 0


class Writer:
    def __init__(self):
        self.root = _Node()

    def dataset(self, path, arr, attrs=None):
        """`arr` is stored with its C-order shape as the HDF5 dimensions."""
        parts = [p for p in path.split("/") if p]
        g = self.root
        for p in parts[:-1]:
            g = g.children.setdefault(p, _Node())
        n = _Node(group=False)
        n.arr = np.ascontiguousarray(arr)
        n.attrs = dict(attrs or {})
        g.children[parts[-1]] = n

    def attribute(self, name, value):
        self.root.attrs[name] = value

    def _header(self, n):
        m = b""
        if n.group:
            m += _msg(0x02, struct.pack("<BBQQ", 0, 0, UNDEF, UNDEF))
            m += _msg(0x0A, struct.pack("<BB", 0, 0))
            for name, ch in n.children.items():
                nm = name.encode()
                m += _msg(0x06, struct.pack("<BBB", 1, 0, len(nm)) + nm + struct.pack("<Q", ch.addr))
        else:
            a = n.arr
            m += _msg(0x01, struct.pack("<BBBB", 2, a.ndim, 0, 1) + b"".join(struct.pack("<Q", d) for d in a.shape))
            m += _msg(0x03, _dtype(a))
            m += _msg(0x05, struct.pack("<BBBB", 2, 1, 1, 0))
            m += _msg(0x08, struct.pack("<BBQQ", 3, 1, n.data_addr, a.nbytes))
        for k, v in n.attrs.items():
            m += _attr(k, v)
        return _ohdr(m)

    def write(self, path):
        nodes = []

        def collect(n):
            nodes.append(n)
            for ch in n.children.values():
                collect(ch)

        collect(self.root)
        cur = 48
        sizes = []
        for n in nodes:
            s = len(self._header(n))
            sizes.append(s)
            n.addr = cur
            cur += s
        for n in nodes:
            if not n.group:
                cur = (cur + 7) // 8 * 8
                n.data_addr = cur
                cur += n.arr.nbytes
        eof = cur
        sb = SIG + struct.pack("<BBBBQQQQ", 2, 8, 8, 0, 0, UNDEF, eof, self.root.addr)
        sb += struct.pack("<I", lookup3(sb))
        with open(path, "wb") as f:
            f.write(sb)
            for n, s in zip(nodes, sizes):
                h = self._header(n)
                assert len(h) == s
                f.write(h)
            pos = f.tell()
            for n in nodes:
                if n.group:
                    continue
                f.write(bytes(n.data_addr - pos))
                f.write(n.arr.tobytes())
                pos = n.data_addr + n.arr.nbytes


FLOAT_VARS = ("dx", "dy", "dz", "pml_x_alpha", "pml_y_alpha", "pml_z_alpha", "dt", "c0", "c_ref", "rho0",
              "rho0_sgx", "rho0_sgy", "rho0_sgz", "BonA", "alpha_coeff", "alpha_power", "p_source_input",
              "ux_source_input", "uy_source_input", "uz_source_input", "p0_source_input",
              "transducer_source_input")
INT_VARS = ("Nx", "Ny", "Nz", "Nt", "p_source_flag", "p0_source_flag", "ux_source_flag", "uy_source_flag",
            "uz_source_flag", "sxx_source_flag", "syy_source_flag", "szz_source_flag", "sxy_source_flag",
            "sxz_source_flag", "syz_source_flag", "transducer_source_flag", "nonuniform_grid_flag",
            "nonlinear_flag", "absorbing_flag", "elastic_flag", "axisymmetric_flag", "sensor_mask_type",
            "pml_x_size", "pml_y_size", "pml_z_size", "p_source_mode", "p_source_many", "p_source_index",
            "u_source_mode", "u_source_many", "u_source_index", "sensor_mask_index", "sensor_mask_corners",
            "delay_mask")


def _matlab_dims(v):
    """HDF5 (C-order) dimensions of a MATLAB array: its 3D size reversed."""
    v = np.asarray(v)
    shape = list(v.shape) + [1] * (3 - v.ndim) if v.ndim <= 3 else list(v.shape)
    if v.ndim == 0:
        shape = [1, 1, 1]
    return tuple(reversed(shape))


def write_input_file(path, inp: dict, description="input written by kwave.h5io"):
    """Write the datasets of ``prepare()``'s input dict as a k-Wave v1.2
    input file.  Arrays are given in MATLAB axis order (x first).

    A transducer's transmit apodization has no dataset in the format (the
    reference's writer, kspaceFirstOrder_saveToDisk.m:289-293, 339-343,
    drops it too); it is left out with a warning unless it is all ones."""
    if inp.get("sensor_interp_index") is not None:
        raise ValueError("the input file format has no interpolated Cartesian sensors: use cart_interp='nearest'")
    apod = inp.get("transducer_source_apodization")
    if apod is not None and np.any(np.asarray(apod) != 1):
        warnings.warn("the input file format has no transmit apodization: it is dropped", stacklevel=2)
    w = Writer()
    dim3 = int(inp["Nz"]) > 1
    flags = {k: 0 for k in INT_VARS if k.endswith("_flag")}
    flags["sensor_mask_type"] = 0
    full = dict(flags)
    full.update(inp)
    for k, v in full.items():
        if not dim3 and "z" in k and k not in ("Nz", "pml_z_size") and k in FLOAT_VARS:
            continue  # saveToDisk.m:421-427 drops z variables in 2D
        if k in FLOAT_VARS:
            a = np.asarray(v, dtype=np.float32)
            w.dataset("/" + k, np.asfortranarray(a).reshape(-1, order="F").reshape(_matlab_dims(a)),
                      {"data_type": "float", "domain_type": "real"})
        elif k in INT_VARS:
            a = np.asarray(v, dtype=np.uint64)
            w.dataset("/" + k, a.reshape(-1, order="F").reshape(_matlab_dims(a)),
                      {"data_type": "long", "domain_type": "real"})
    for k, v in (("created_by", "k-Wave B200 host package"), ("creation_date",
                 datetime.datetime.now().strftime("%d-%b-%Y-%H-%M-%S")), ("file_description", description),
                 ("file_type", "input"), ("major_version", "1"), ("minor_version", "2")):
        w.attribute(k, v)
    w.write(path)


# ---------------------------------------------------------------------------
# reader
# ---------------------------------------------------------------------------
class File:
    def __init__(self, path):
        self._f = open(path, "rb")
        self.m = mmap.mmap(self._f.fileno(), 0, access=mmap.ACCESS_READ)
        off = 0
        while off + 8 <= len(self.m):
            if self.m[off:off + 8] == SIG:
                break
            off = 512 if off == 0 else off * 2
        else:
            raise ValueError("no HDF5 superblock")
        self.base = off
        v = self.m[off + 8]
        if v in (0, 1):
            self.so, self.sl = self.m[off + 13], self.m[off + 14]
            q = off + 24 + (4 if v == 1 else 0)
            ba = self.u(q, self.so, absolute=True)
            if ba not in (0, off):
                self.base = ba
            self.root = self.u(q + 5 * self.so, self.so, absolute=True)
        elif v in (2, 3):
            self.so, self.sl = self.m[off + 9], self.m[off + 10]
            q = off + 12
            ba = self.u(q, self.so, absolute=True)
            if ba not in (0, off):
                self.base = ba
            self.root = self.u(q + 3 * self.so, self.so, absolute=True)
        else:
            raise ValueError(f"superblock version {v}")

    def close(self):
        self.m.close()
        self._f.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def u(self, addr, n, absolute=False):
        o = addr if absolute else self.base + addr
        return int.from_bytes(self.m[o:o + n], "little")

    def b(self, addr, n):
        o = self.base + addr
        return self.m[o:o + n]

    def undef(self, a):
        return a == (1 << (8 * self.so)) - 1

    def messages(self, addr):
        out = []
        if self.b(addr, 4) == b"OHDR":
            flags = self.b(addr, 6)[5]
            off = 6 + (16 if flags & 0x20 else 0) + (4 if flags & 0x10 else 0)
            nb = 1 << (flags & 3)
            blocks = [(addr + off + nb, self.u(addr + off, nb), True)]
            crt = 2 if flags & 0x04 else 0
            i = 0
            while i < len(blocks):
                a, ln, first = blocks[i]
                end = a + ln
                if not first:
                    a += 4
                    end -= 4
                while a + 4 <= end:
                    t = self.b(a, 1)[0]
                    size = self.u(a + 1, 2)
                    d = a + 4 + crt
                    if d + size > end:
                        break
                    if t == 0x10:
                        blocks.append((self.u(d, self.so), self.u(d + self.so, self.sl), False))
                    elif t:
                        out.append((t, d, size))
                    a = d + size
                i += 1
        else:
            nmsg = self.u(addr + 2, 2)
            blocks = [(addr + 16, self.u(addr + 8, 4))]
            count = 0
            i = 0
            while i < len(blocks) and count < nmsg:
                a, ln = blocks[i]
                end = a + ln
                while a + 8 <= end and count < nmsg:
                    t, size = self.u(a, 2), self.u(a + 2, 2)
                    count += 1
                    if t == 0x10:
                        blocks.append((self.u(a + 8, self.so), self.u(a + 8 + self.so, self.sl)))
                    elif t:
                        out.append((t, a + 8, size))
                    a += 8 + size
                i += 1
        return out

    def children(self, oh):
        res = {}
        for t, d, size in self.messages(oh):
            if t == 0x11:
                self._symtab(self.u(d, self.so), self.u(d + self.so, self.so), res)
            elif t == 0x06:
                flags = self.b(d + 1, 1)[0]
                off = 2
                lt = 0
                if flags & 0x08:
                    lt = self.b(d + off, 1)[0]
                    off += 1
                off += 8 if flags & 0x04 else 0
                off += 1 if flags & 0x10 else 0
                nb = 1 << (flags & 3)
                ln = self.u(d + off, nb)
                off += nb
                name = bytes(self.b(d + off, ln)).decode()
                if lt == 0:
                    res[name] = self.u(d + off + ln, self.so)
        return res

    def _symtab(self, btree, heap, res):
        seg_size = self.u(heap + 8, self.sl)
        seg = self.u(heap + 8 + 2 * self.sl, self.so)
        names = bytes(self.b(seg, seg_size))

        def walk(node):
            level = self.b(node + 5, 1)[0]
            n = self.u(node + 6, 2)
            q = node + 8 + 2 * self.so
            for i in range(n):
                child = self.u(q + self.sl + i * (self.sl + self.so), self.so)
                if level:
                    walk(child)
                    continue
                ns = self.u(child + 6, 2)
                esz = 2 * self.so + 24
                for j in range(ns):
                    e = child + 8 + j * esz
                    no = self.u(e, self.so)
                    res[names[no:names.index(b"\0", no)].decode()] = self.u(e + self.so, self.so)

        walk(btree)

    def lookup(self, path):
        oh = self.root
        for p in [p for p in path.split("/") if p]:
            ch = self.children(oh)
            if p not in ch:
                raise KeyError(path)
            oh = ch[p]
        return oh

    def __contains__(self, path):
        try:
            self.lookup(path)
            return True
        except KeyError:
            return False

    def attrs(self, path="/"):
        res = {}
        for t, d, size in self.messages(self.lookup(path)):
            if t != 0x0C:
                continue
            ver = self.b(d, 1)[0]
            nsz, tsz, ssz = self.u(d + 2, 2), self.u(d + 4, 2), self.u(d + 6, 2)
            pad = (lambda v: (v + 7) // 8 * 8) if ver == 1 else (lambda v: v)
            off = d + (9 if ver == 3 else 8)
            name = bytes(self.b(off, nsz)).split(b"\0")[0].decode()
            off += pad(nsz)
            tcls = self.b(off, 1)[0] & 0x0F
            tlen = self.u(off + 4, 4)
            off += pad(tsz) + pad(ssz)
            if tcls == 3:
                res[name] = bytes(self.b(off, tlen)).split(b"\0")[0].decode().rstrip()
        return res

    def read(self, path):
        dims = dt = lay = None
        filters = []
        for t, d, size in self.messages(self.lookup(path)):
            if t == 0x01:
                ver, rank = self.b(d, 2)
                q = d + (8 if ver == 1 else 4)
                dims = [self.u(q + i * self.sl, self.sl) for i in range(rank)]
            elif t == 0x03:
                c0, b0 = self.b(d, 2)
                cls, size_b = c0 & 0x0F, self.u(d + 4, 4)
                be = ">" if b0 & 1 else "<"
                if cls == 1:
                    dt = np.dtype(f"{be}f{size_b}")
                elif cls == 0:
                    dt = np.dtype(f"{be}{'i' if b0 & 0x08 else 'u'}{size_b}")
                else:
                    raise TypeError(f"{path}: unsupported datatype class {cls}")
            elif t == 0x08:
                ver = self.b(d, 1)[0]
                if ver in (1, 2):
                    nd, cls = self.b(d + 1, 2)
                    off = d + 8
                    addr = 0
                    if cls != 0:
                        addr = self.u(off, self.so)
                        off += self.so
                    dd = [self.u(off + 4 * i, 4) for i in range(nd)]
                    off += 4 * nd
                    if cls == 0:
                        lay = ("compact", off + 4, self.u(off, 4))
                    elif cls == 1:
                        lay = ("contig", addr, 0)
                    else:
                        lay = ("chunk", addr, dd[:-1])
                    continue
                if ver != 3:
                    raise ValueError(f"{path}: data layout version {ver}")
                cls = self.b(d + 1, 1)[0]
                if cls == 0:
                    lay = ("compact", d + 4, self.u(d + 2, 2))
                elif cls == 1:
                    lay = ("contig", self.u(d + 2, self.so), self.u(d + 2 + self.so, self.sl))
                else:
                    nd = self.b(d + 2, 1)[0]
                    addr = self.u(d + 3, self.so)
                    cd = [self.u(d + 3 + self.so + 4 * i, 4) for i in range(nd - 1)]
                    lay = ("chunk", addr, cd)
            elif t == 0x0B:
                ver, n = self.b(d, 2)
                off = d + (8 if ver == 1 else 2)
                for _ in range(n):
                    fid = self.u(off, 2)
                    off += 2
                    nlen = 0
                    if ver == 1 or fid >= 256:
                        nlen = self.u(off, 2)
                        off += 2
                    off += 2
                    ncd = self.u(off, 2)
                    off += 2
                    if ver == 1:
                        nlen = (nlen + 7) // 8 * 8
                    off += nlen
                    cd = [self.u(off + 4 * i, 4) for i in range(ncd)]
                    off += 4 * ncd + (4 if ver == 1 and ncd % 2 else 0)
                    filters.append((fid, cd))
        if dims is None or dt is None or lay is None:
            raise ValueError(f"{path} is not a dataset")
        n = int(np.prod(dims)) if dims else 1
        if lay[0] == "compact":
            return np.frombuffer(bytes(self.b(lay[1], lay[2])), dt, count=n).reshape(dims)
        if lay[0] == "contig":
            if self.undef(lay[1]):
                return np.zeros(dims, dt)
            return np.frombuffer(bytes(self.b(lay[1], n * dt.itemsize)), dt).reshape(dims)
        out = np.zeros(dims, dt)
        cd = lay[2]
        cn = int(np.prod(cd))

        def walk(node):
            level = self.b(node + 5, 1)[0]
            ne = self.u(node + 6, 2)
            ksz = 8 + 8 * (len(dims) + 1)
            q = node + 8 + 2 * self.so
            for i in range(ne):
                key = q + i * (ksz + self.so)
                child = self.u(key + ksz, self.so)
                if level:
                    walk(child)
                    continue
                csize, mask = self.u(key, 4), self.u(key + 4, 4)
                off = [self.u(key + 8 + 8 * r, 8) for r in range(len(dims))]
                raw = bytes(self.b(child, csize))
                for fi in range(len(filters) - 1, -1, -1):
                    if mask & (1 << fi):
                        continue
                    fid, fcd = filters[fi]
                    if fid == 1:
                        raw = zlib.decompress(raw)
                    elif fid == 2:
                        es = fcd[0] if fcd else dt.itemsize
                        raw = np.frombuffer(raw, np.uint8).reshape(es, -1).T.tobytes()
                    elif fid == 3:
                        raw = raw[:-4]
                    else:
                        raise ValueError(f"filter {fid}")
                blk = np.frombuffer(raw, dt, count=cn).reshape(cd)
                sl_out = tuple(slice(o, min(o + c, dd)) for o, c, dd in zip(off, cd, dims))
                sl_in = tuple(slice(0, s.stop - s.start) for s in sl_out)
                out[sl_out] = blk[sl_in]

        if not self.undef(lay[1]):
            walk(lay[1])
        return out


def read(path, name):
    with File(path) as f:
        return f.read(name)


def read_matlab(path, name):
    """A dataset as MATLAB's h5read returns it: dimensions reversed."""
    a = read(path, name)
    return np.asarray(a).transpose(tuple(range(a.ndim))[::-1])


def read_output_file(path, dim):
    """The datasets of a solver output file in the layout kwave._lib.solve
    returns: time series (Ns, Nt_rec), per-point (Ns,), grid arrays (Nx, Ny[, Nz]);
    cuboid outputs as a list of arrays, one per cuboid, [x, y, (z,) t]."""
    res = {}
    with File(path) as f:
        names = f.children(f.root)
        for k in names:
            if k in ("Nx", "Ny", "Nz", "Nt", "pml_x_size", "pml_y_size", "pml_z_size"):
                continue
            sub = f.children(names[k])
            if sub:  # one dataset per cuboid, MATLAB order [x, y, (z,) t]
                blocks = [f.read(f"/{k}/{i}") for i in sorted(sub, key=int)]
                res[k] = [b.transpose(tuple(range(b.ndim))[::-1]) for b in blocks]
                continue
            a = f.read("/" + k)
            m = a.transpose(tuple(range(a.ndim))[::-1])
            if k.endswith("_all") or k.endswith("_final"):
                res[k] = m if dim == 3 else m[:, :, 0]
            elif k in ("p", "ux", "uy", "uz") or k.endswith("_non_staggered"):
                res[k] = m[:, :, 0]
            else:
                res[k] = m.reshape(-1)
    return res
