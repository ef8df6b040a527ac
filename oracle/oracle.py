"""ctypes bindings for the CPU oracle and the CPU baseline.

TEST / BENCHMARK INFRASTRUCTURE ONLY.  Only tests/, ``__graft_entry__.smoke()``
and bench.py's CPU-baseline leg import this module, as the checker.  The
product path (``openfpm_data_b200``) never imports it.

``OracleGrid`` mirrors the reference's block map (sorted chunk keys, SoA chunk
data with a trailing background chunk, one mask byte per point) and exposes
the restated flush / findNeighbours / tagBoundaries / stencil semantics of
``oracle/sgb_oracle.cpp``.  ``CpuSgrid`` is the sgrid_cpu-style baseline of
``oracle/sgrid_cpu_baseline.cpp``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")

T_F32, T_I32, T_F64, T_U8 = 0, 1, 2, 3
OP_NONE, OP_RIGHT, OP_LEFT, OP_ADD, OP_MAX, OP_MIN, OP_OR = range(7)
NN_STAR, NN_FULL = 0, 1
_NP = {T_F32: np.float32, T_I32: np.int32, T_F64: np.float64, T_U8: np.uint8}


def build(force: bool = False) -> None:
    """Compile the oracle libraries with the committed Makefile."""
    need = force or not all(
        os.path.exists(os.path.join(BUILD, f)) for f in ("libsgb_oracle.so", "libsgrid_cpu.so")
    )
    if need:
        subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None
_cpu = None


def _load():
    global _lib, _cpu
    if _lib is None:
        build()
        _lib = C.CDLL(os.path.join(BUILD, "libsgb_oracle.so"))
        _cpu = C.CDLL(os.path.join(BUILD, "libsgrid_cpu.so"))
        vp, i64, i32 = C.c_void_p, C.c_int64, C.c_int
        _lib.sgo_create.restype = vp
        _lib.sgo_create.argtypes = [i32, i32, vp, i32, vp]
        _lib.sgo_destroy.argtypes = [vp]
        _lib.sgo_set_background.argtypes = [vp, i32, vp]
        _lib.sgo_nchunks.restype = i64
        _lib.sgo_nchunks.argtypes = [vp]
        _lib.sgo_lin_ids.argtypes = [vp, i64, vp, vp]
        _lib.sgo_inv_lin.argtypes = [vp, i64, vp, vp]
        _lib.sgo_load_map.argtypes = [vp, i64, vp, vp, vp]
        _lib.sgo_export_map.argtypes = [vp, vp, vp, vp]
        _lib.sgo_flush_chunks.argtypes = [vp, i64, vp, vp, vp, vp]
        _lib.sgo_flush_points.argtypes = [vp, i64, vp, vp, vp, vp]
        _lib.sgo_find_neighbours.restype = i32
        _lib.sgo_find_neighbours.argtypes = [vp, i32, vp]
        _lib.sgo_tag_boundaries.argtypes = [vp, i32]
        _lib.sgo_remove_boxes.argtypes = [vp, i64, vp]
        f = C.c_float
        _lib.sgo_heat7.argtypes = [vp, i32, i32, f, vp]
        _lib.sgo_gs7.argtypes = [vp, i32, i32, i32, i32, f, f, f, f, f, vp]
        _lib.sgo_gs7_steps.argtypes = [vp, i32, i32, i32, i32, f, f, f, f, f, i32, i32]
        _lib.sgo_heat7_steps.argtypes = [vp, i32, i32, f, i32, i32]
        _lib.sgo_box27.argtypes = [vp, i32, i32, vp, vp]
        _lib.sgo_box27_ns.argtypes = [vp, i32, i32, vp, vp]
        _lib.sgo_set_zorder.argtypes = [vp, i32]
        d = C.c_double
        _lib.sgo_heat7_f64.argtypes = [vp, vp, vp, d, d, i32]
        _lib.sgo_gs7_f64.argtypes = [vp, vp, vp, vp, vp, d, d, d, d, d, d, d, i32]
        _lib.sgo_gs7_f64_mt.argtypes = [vp, vp, vp, vp, vp, d, d, d, d, d, d, d, i32, i32]
        _cpu.cpub_create.restype = vp
        _cpu.cpub_create.argtypes = [vp, i32, vp]
        _cpu.cpub_destroy.argtypes = [vp]
        _cpu.cpub_nchunks.restype = C.c_int32
        _cpu.cpub_nchunks.argtypes = [vp]
        _cpu.cpub_insert.argtypes = [vp, i64, vp, vp]
        _cpu.cpub_get.argtypes = [vp, i64, vp, i32, vp]
        _cpu.cpub_heat.restype = i32
        _cpu.cpub_heat.argtypes = [vp, i32, i32, f, i32, i32]
        _cpu.cpub_gs.restype = i32
        _cpu.cpub_gs.argtypes = [vp, i32, i32, i32, i32, f, f, f, f, f, i32, i32]
    return _lib, _cpu


def _up8(n: int) -> int:
    return (n + 7) & ~7


def _pad8(b: bytes) -> bytes:
    return b + bytes(_up8(len(b)) - len(b))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _ptr_array(arrs):
    return (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


class OracleGrid:
    """CPU restatement of one SparseGridGpu block map."""

    def __init__(self, size, edge=8, ptypes=(T_F32,), dim=None, zorder=False):
        lib, _ = _load()
        self.zorder = bool(zorder)
        self.dim = dim if dim is not None else len(size)
        self.edge = edge
        self.bs = edge ** self.dim
        self.size = tuple(int(s) for s in size) + (1,) * (3 - len(size))
        self.ptypes = list(ptypes)
        sz = np.array(self.size, dtype=np.int64)
        pt = np.array(self.ptypes, dtype=np.int32)
        self._h = lib.sgo_create(self.dim, edge, _ptr(sz), len(self.ptypes), _ptr(pt))
        if self.zorder:
            lib.sgo_set_zorder(self._h, 1)

    # -- chunk ids (grid_smb: block x fastest; grid_zmb: Morton code, src/util/zmorton.hpp) --
    def _bsz(self):
        return [(int(s) + self.edge - 1) // self.edge for s in self.size]

    def block_key(self, bc):
        """Chunk ids of non-negative block coordinates [m, 3]."""
        bc = np.asarray(bc, dtype=np.int64).reshape(-1, 3)
        if not self.zorder:
            b = self._bsz()
            return bc[:, 0] + b[0] * (bc[:, 1] + b[1] * bc[:, 2])
        k = np.zeros(len(bc), dtype=np.uint64)
        for i in range(21):
            for d in range(3):
                k |= ((bc[:, d].astype(np.uint64) >> np.uint64(i)) & np.uint64(1)) << np.uint64(3 * i + d)
        return k.astype(np.int64)

    def block_coords(self, keys, size=None):
        """Block coordinates [m, 3] of chunk ids (size: the grid size the ids were made for)."""
        keys = np.asarray(keys, dtype=np.int64)
        if not self.zorder:
            b = self._bsz() if size is None else [(int(s) + self.edge - 1) // self.edge for s in size]
            return np.stack([keys % b[0], (keys // b[0]) % b[1], keys // (b[0] * b[1])], axis=1)
        u = keys.astype(np.uint64)
        bc = np.zeros((len(keys), 3), dtype=np.int64)
        for i in range(21):
            for d in range(3):
                bc[:, d] |= (((u >> np.uint64(3 * i + d)) & np.uint64(1)).astype(np.int64)) << i
        return bc

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.sgo_destroy(self._h)
            self._h = None

    # -- layout ------------------------------------------------------------
    def set_background(self, p, value):
        v = np.array([value], dtype=_NP[self.ptypes[p]])
        _lib.sgo_set_background(self._h, p, _ptr(v))

    @property
    def nchunks(self) -> int:
        return int(_lib.sgo_nchunks(self._h))

    def lin_ids(self, coords) -> np.ndarray:
        c = np.ascontiguousarray(coords, dtype=np.int64).reshape(-1, self.dim)
        out = np.empty(len(c), dtype=np.int64)
        _lib.sgo_lin_ids(self._h, len(c), _ptr(c), _ptr(out))
        return out

    def inv_lin(self, lin) -> np.ndarray:
        l = np.ascontiguousarray(lin, dtype=np.int64)
        out = np.empty((len(l), self.dim), dtype=np.int64)
        _lib.sgo_inv_lin(self._h, len(l), _ptr(l), _ptr(out))
        return out

    def load_map(self, keys, data, mask):
        keys = np.ascontiguousarray(keys, dtype=np.int64)
        data = [np.ascontiguousarray(d, dtype=_NP[t]) for d, t in zip(data, self.ptypes)]
        mask = np.ascontiguousarray(mask, dtype=np.uint8)
        _lib.sgo_load_map(self._h, len(keys), _ptr(keys), _ptr_array(data), _ptr(mask))

    def export(self):
        """(keys[n], [data_p[(n+1)*bs]], mask[(n+1)*bs]) including the background chunk."""
        n = self.nchunks
        keys = np.empty(n, dtype=np.int64)
        data = [np.empty((n + 1) * self.bs, dtype=_NP[t]) for t in self.ptypes]
        mask = np.empty((n + 1) * self.bs, dtype=np.uint8)
        _lib.sgo_export_map(self._h, _ptr(keys), _ptr_array(data), _ptr(mask))
        return keys, data, mask

    # -- flush -------------------------------------------------------------
    def flush_chunks(self, slot_keys, slot_data, slot_mask, ops):
        k = np.ascontiguousarray(slot_keys, dtype=np.int64)
        d = [np.ascontiguousarray(x, dtype=_NP[t]) for x, t in zip(slot_data, self.ptypes)]
        m = np.ascontiguousarray(slot_mask, dtype=np.uint8)
        o = np.array(ops, dtype=np.int32)
        _lib.sgo_flush_chunks(self._h, len(k), _ptr(k), _ptr_array(d), _ptr(m), _ptr(o))

    def flush_points(self, lin, vals, ops, pmask=None):
        l = np.ascontiguousarray(lin, dtype=np.int64)
        v = [np.ascontiguousarray(x, dtype=_NP[t]) for x, t in zip(vals, self.ptypes)]
        o = np.array(ops, dtype=np.int32)
        pm = None if pmask is None else np.ascontiguousarray(pmask, dtype=np.uint8)
        _lib.sgo_flush_points(self._h, len(l), _ptr(l), _ptr_array(v),
                              None if pm is None else _ptr(pm), _ptr(o))

    def insert_flush(self, coords, vals, ops):
        self.flush_points(self.lin_ids(coords), vals, ops)

    # -- neighbours / tag --------------------------------------------------
    def find_neighbours(self, kind=NN_STAR) -> np.ndarray:
        k = (1 << self.dim) if kind == NN_STAR else 3 ** self.dim
        out = np.empty(self.nchunks * k, dtype=np.int64)
        _lib.sgo_find_neighbours(self._h, kind, _ptr(out))
        return out.reshape(self.nchunks, k)

    def tag_boundaries(self, kind=NN_STAR):
        _lib.sgo_tag_boundaries(self._h, kind)

    def remove_boxes(self, boxes):
        """remove(box) for each box + removePoints; boxes [k, 6] = lo[3], hi[3] inclusive."""
        b = np.ascontiguousarray(np.asarray(boxes, dtype=np.int64).reshape(-1, 6))
        _lib.sgo_remove_boxes(self._h, len(b), _ptr(b))

    def existing_points(self, box=None):
        """Coordinates [k, 3] of the existing points in (chunk position, offset in the chunk)
        order, optionally only those inside an inclusive box (lo, hi): the order of the
        reference's SparseGridGpu iterators after deviceToHost."""
        keys, _, mask = self.export()
        n = len(keys)
        idx = np.nonzero(mask[: n * self.bs] & 1)[0]
        lin = keys[idx // self.bs] * self.bs + idx % self.bs
        c = self.inv_lin(lin)
        if box is not None:
            lo, hi = np.asarray(box[0]), np.asarray(box[1])
            c = c[np.all((c >= lo) & (c <= hi), axis=1)]
        return c

    # -- pack / unpack (SparseGridGpu.hpp:3041-3210 packRequest/packCalculate,
    #    3244-3300 pack, 1293-1408 pack_sg_implement, 1420-1615 unpack) -----
    def pack(self, boxes, props) -> bytes:
        """The packed boxes back to back.  Per box (every section padded to 8 bytes):
        uint64 n_cnk, int32 start[3] (box lower corner), int32 size[3] (grid size),
        int64 chunk ids, uint32 scan[n_cnk + 1], per property its n_pnt values,
        int16 offsets, uint8 masks (SparseGridGpu.hpp:3192-3200 size formula;
        SparseGridGpu_kernels.cuh:1658-1697 pack_data).  Points: the existing points
        inside the inclusive box (Box<dim,int>::isInside, kernels.cuh:1388-1399), chunks
        in index order, points in offset order inside a chunk."""
        keys, data, mask = self.export()
        n = len(keys)
        idx = np.nonzero(mask[: n * self.bs] & 1)[0]
        lin = keys[idx // self.bs] * self.bs + idx % self.bs
        c = self.inv_lin(lin) if len(lin) else np.zeros((0, 3), dtype=np.int64)
        out = bytearray()
        for b in np.asarray(boxes, dtype=np.int64).reshape(-1, 6):
            sel = np.all((c >= b[:3]) & (c <= b[3:]), axis=1)
            pidx = idx[sel]
            cpos = pidx // self.bs
            ids, first = np.unique(cpos, return_index=True)
            n_cnk, n_pnt = len(ids), len(pidx)
            sec = [np.array([n_cnk], dtype="<u8").tobytes(),
                   np.array(list(b[:3]) + list(self.size), dtype="<i4").tobytes(),
                   keys[ids].astype("<i8").tobytes(),
                   _pad8(np.array(list(first) + [n_pnt], dtype="<u4").tobytes()),
                   _pad8(b"".join(data[p][pidx].tobytes() for p in props)),
                   _pad8((pidx % self.bs).astype("<i2").tobytes()),
                   _pad8(mask[pidx].tobytes())]
            out += b"".join(sec)
        return bytes(out)

    def unpack(self, buf, props, starts=None):
        """Parse the packed boxes of buf (packed with props) and return, per box, the
        points at packed coordinate - packed start + starts[k] (starts None: in place)
        and their values: [(coords [m, 3], [values_p])]."""
        es = [np.dtype(_NP[self.ptypes[p]]).itemsize for p in props]
        res, pos, k = [], 0, 0
        buf = bytes(buf)
        while pos < len(buf):
            n_cnk = int(np.frombuffer(buf, "<u8", 1, pos)[0])
            hdr = np.frombuffer(buf, "<i4", 6, pos + 8).astype(np.int64)
            q = pos + 32
            ids = np.frombuffer(buf, "<i8", n_cnk, q)
            q += 8 * n_cnk
            scan = np.frombuffer(buf, "<u4", n_cnk + 1, q)
            n_pnt = int(scan[-1])
            q += _up8(4 * (n_cnk + 1))
            vals = []
            for p, e in zip(props, es):
                vals.append(np.frombuffer(buf, _NP[self.ptypes[p]], n_pnt, q).copy())
                q += n_pnt * e
            q = pos + 32 + 8 * n_cnk + _up8(4 * (n_cnk + 1)) + _up8(n_pnt * sum(es))
            offs = np.frombuffer(buf, "<i2", n_pnt, q).astype(np.int64)
            q += _up8(2 * n_pnt)
            q += _up8(n_pnt)
            chunk = np.repeat(np.arange(n_cnk), np.diff(scan.astype(np.int64)))
            org = self.block_coords(ids[chunk], size=hdr[3:]) * self.edge
            e = self.edge
            coords = org + np.stack([offs % e, (offs // e) % e, offs // (e * e)], axis=1)
            if starts is not None:
                coords = coords - hdr[:3] + np.asarray(starts[k], dtype=np.int64)
            res.append((coords, vals))
            pos, k = q, k + 1
        return res

    # -- multi-resolution links (SparseGridGpu.hpp:2113-2262, kernels
    #    SparseGridGpu_kernels.cuh:775-1000) ---------------------------------
    def _other_exists(self, c):
        """SparseGridGpu_ker::get<pMask>(coord) & 1 for int64 coords [m, 3]: grid_smb::LinId
        with C (truncating) division and no bounds checks, cast to unsigned int, then the
        chunk looked up (absent: the background chunk).  Returns (exists, pos, off)."""
        keys, _, mask = self.export()
        e = self.edge
        bsz = [(s + e - 1) // e for s in self.size]
        q = lambda a: np.sign(a) * (np.abs(a) // e)  # noqa: E731  (truncating division by e)
        r = lambda a: a - q(a) * e  # noqa: E731
        if self.zorder:
            # Morton ids: a negative coordinate is absent (its id lies above every chunk's)
            neg = np.any(c < 0, axis=1)
            cc = np.where(neg[:, None], 0, c)
            blk = self.block_key(cc // e)
            loc = cc[:, 0] % e + e * (cc[:, 1] % e + e * (cc[:, 2] % e))
            blk = np.where(neg, -1, blk)
        else:
            blk, loc = q(c[:, 2]), r(c[:, 2])
            for d in (1, 0):
                blk = blk * bsz[d] + q(c[:, d])
                loc = loc * e + r(c[:, d])
        lin = np.where(blk < 0, -1, (blk * self.bs + loc) & 0xFFFFFFFF) if self.zorder else \
            (blk * self.bs + loc) & 0xFFFFFFFF
        b, off = lin // self.bs, lin % self.bs
        pos = np.searchsorted(keys, b)
        found = (pos < len(keys)) & (keys[np.minimum(pos, max(len(keys) - 1, 0))] == b) if len(keys) else \
            np.zeros(len(b), bool)
        pos = np.where(found, pos, len(keys))
        ex = (mask[pos * self.bs + off] & 1) != 0
        return ex, pos, off

    def construct_links(self, other, box, shift, up):
        """Padding points inside the inclusive box in (chunk, offset) order, and their links
        to `other`: down (up=False) to the existing points at 2p + shift + (j&1, j>>1&1,
        j>>2&1) for j < 6, up to the existing point at (p - shift) / 2 truncated."""
        keys, _, mask = self.export()
        n = len(keys)
        idx = np.nonzero(mask[: n * self.bs] & 2)[0]
        lin = keys[idx // self.bs] * self.bs + idx % self.bs
        p = self.inv_lin(lin) if len(lin) else np.zeros((0, 3), np.int64)
        lo, hi = np.asarray(box[0]), np.asarray(box[1])
        sel = np.all((p >= lo) & (p <= hi), axis=1)
        idx, p = idx[sel], p[sel]
        sh = np.asarray(shift, dtype=np.int64)
        if up:
            t = p - sh
            cands = [np.sign(t) * (np.abs(t) // 2)]
        else:
            cands = [p * 2 + sh + np.array([(j >> d) & 1 for d in range(3)]) for j in range(6)]
        hits = [other._other_exists(c) for c in cands]
        ex = np.stack([h[0] for h in hits], axis=1)     # [npad, candidates]
        pos = np.stack([h[1] for h in hits], axis=1)
        off = np.stack([h[2] for h in hits], axis=1)
        offsets = np.concatenate([[0], np.cumsum(ex.sum(axis=1))]).astype(np.int64)
        # links point by point, candidates in loop order inside a point
        return {"pad_pos": idx // self.bs, "pad_off": idx % self.bs, "offsets": offsets,
                "link_pos": pos[ex].astype(np.int64), "link_off": off[ex].astype(np.int64)}

    # -- stencils ----------------------------------------------------------


    @staticmethod
    def _box(box):
        if box is None:
            return None
        b = np.array(list(box[0]) + list(box[1]) + [0] * (6 - 2 * len(box[0])), dtype=np.int64)
        return b

    def heat7(self, src, dst, dt, box=None):
        b = self._box(box)
        _lib.sgo_heat7(self._h, src, dst, dt, None if b is None else _ptr(b))

    def gs7(self, pu, pv, pu2, pv2, Du, Dv, F, k, dt, box=None):
        b = self._box(box)
        _lib.sgo_gs7(self._h, pu, pv, pu2, pv2, Du, Dv, F, k, dt, None if b is None else _ptr(b))

    def gs7_steps(self, pu, pv, pu2, pv2, Du, Dv, F, k, dt, steps, threads=None):
        """`steps` gs7 calls ping-ponging (pu, pv) <-> (pu2, pv2), the chunks of each step shared
        out over host threads (the same bits as the serial calls)."""
        _lib.sgo_gs7_steps(self._h, pu, pv, pu2, pv2, Du, Dv, F, k, dt, steps, threads or (os.cpu_count() or 1))

    def heat7_steps(self, src, dst, dt, steps, threads=None):
        """`steps` heat7 calls ping-ponging src <-> dst over host threads (the same bits as the
        serial calls)."""
        _lib.sgo_heat7_steps(self._h, src, dst, dt, steps, threads or (os.cpu_count() or 1))

    def box27(self, src, dst, coeff, box=None):
        c = np.ascontiguousarray(coeff, dtype=np.float32).reshape(27)
        b = self._box(box)
        _lib.sgo_box27(self._h, src, dst, _ptr(c), None if b is None else _ptr(b))

    def box27_noshared(self, src, dst, coeff, box=None):
        """Conv3x3x3_noshared through applyStencilInPlaceNoShared: coeff[i][j][k], i along z."""
        c = np.ascontiguousarray(coeff, dtype=np.float32).reshape(27)
        b = self._box(box)
        _lib.sgo_box27_ns(self._h, src, dst, _ptr(c), None if b is None else _ptr(b))

    def heat7_f64(self, field, dt, bck, steps):
        a = np.ascontiguousarray(field, dtype=np.float64).copy()
        b = a.copy()
        _lib.sgo_heat7_f64(self._h, _ptr(a), _ptr(b), dt, bck, steps)
        return a

    def gs7_f64(self, u, v, Du, Dv, F, k, dt, bcku, bckv, steps, threads=1):
        u = np.ascontiguousarray(u, dtype=np.float64).copy()
        v = np.ascontiguousarray(v, dtype=np.float64).copy()
        u2, v2 = u.copy(), v.copy()
        _lib.sgo_gs7_f64_mt(self._h, _ptr(u), _ptr(v), _ptr(u2), _ptr(v2), Du, Dv, F, k, dt, bcku, bckv, steps,
                            int(threads))
        return u, v

    # -- point access (host get<p>(coord), BlockMapGpu.hpp:108-126) --------
    def get(self, p, coords):
        keys, data, mask = self.export()
        lin = self.lin_ids(coords)
        bkey, off = lin // self.bs, lin % self.bs
        pos = np.searchsorted(keys, bkey)
        pos = np.where((pos < len(keys)) & (keys[np.minimum(pos, len(keys) - 1)] == bkey), pos, len(keys))
        idx = pos * self.bs + off
        vals = data[p][idx]
        bck = data[p][len(keys) * self.bs]
        return np.where(mask[idx] & 1, vals, bck)

    def mask_at(self, coords):
        keys, _, mask = self.export()
        lin = self.lin_ids(coords)
        bkey, off = lin // self.bs, lin % self.bs
        pos = np.searchsorted(keys, bkey)
        found = (pos < len(keys)) & (keys[np.minimum(pos, max(len(keys) - 1, 0))] == bkey)
        return np.where(found, mask[np.where(found, pos, len(keys)) * self.bs + off], 0)


class CpuSgrid:
    """sgrid_cpu-style CPU baseline (16^3 hashed chunks)."""

    def __init__(self, size, nprop, bck):
        _, cpu = _load()
        sz = np.array(size, dtype=np.int64)
        b = np.array(bck, dtype=np.float32)
        self.nprop = nprop
        self._h = cpu.cpub_create(_ptr(sz), nprop, _ptr(b))

    def __del__(self):
        if getattr(self, "_h", None) and _cpu is not None:
            _cpu.cpub_destroy(self._h)
            self._h = None

    @property
    def nchunks(self):
        return int(_cpu.cpub_nchunks(self._h))

    def insert(self, coords, vals):
        c = np.ascontiguousarray(coords, dtype=np.int64).reshape(-1, 3)
        v = [np.ascontiguousarray(x, dtype=np.float32) for x in vals]
        _cpu.cpub_insert(self._h, len(c), _ptr(c), _ptr_array(v))

    def get(self, p, coords):
        c = np.ascontiguousarray(coords, dtype=np.int64).reshape(-1, 3)
        out = np.empty(len(c), dtype=np.float32)
        _cpu.cpub_get(self._h, len(c), _ptr(c), p, _ptr(out))
        return out

    def heat(self, src, dst, dt, steps, threads=1) -> int:
        return int(_cpu.cpub_heat(self._h, src, dst, dt, steps, threads))

    def gs(self, pu, pv, pu2, pv2, Du, Dv, F, k, dt, steps, threads=1) -> int:
        return int(_cpu.cpub_gs(self._h, pu, pv, pu2, pv2, Du, Dv, F, k, dt, steps, threads))
