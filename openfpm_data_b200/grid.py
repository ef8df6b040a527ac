"""Python host mirror of SparseGridGpu<3, aggregate<...>, edge> over the C ABI.

Method names follow the reference class (src/SparseGridGpu/SparseGridGpu.hpp);
device data is exchanged as torch CUDA tensors (torch is plumbing here: device
memory and streams; every computation runs in libsgb200.so).
"""
from __future__ import annotations

import ctypes as C
from typing import Iterable, Optional, Sequence

import numpy as np
import torch

from . import _lib as L

_TYPES = {"f32": L.F32, "float32": L.F32, "i32": L.I32, "int32": L.I32, "f64": L.F64, "float64": L.F64,
          "u8": L.U8, "uint8": L.U8}
_NP = {L.F32: np.float32, L.I32: np.int32, L.F64: np.float64, L.U8: np.uint8}
_TORCH = {L.F32: torch.float32, L.I32: torch.int32, L.F64: torch.float64, L.U8: torch.uint8}
_TS = {L.F32: "<f4", L.I32: "<i4", L.F64: "<f8", L.U8: "|u1"}

# reference reduction names -> sgb_op
OPS = {"sRight_": L.OP_RIGHT, "sLeft_": L.OP_LEFT, "sadd_": L.OP_ADD, "smax_": L.OP_MAX, "smin_": L.OP_MIN,
       "sBitwiseOr_": L.OP_OR, None: L.OP_NONE, "none": L.OP_NONE}


class _Links(C.Structure):
    """sgb_links of include/sgb200.h."""
    _fields_ = [("npad", C.c_int64), ("pad_pos", C.c_void_p), ("pad_off", C.c_void_p), ("offsets", C.c_void_p),
                ("nlinks", C.c_int64), ("link_pos", C.c_void_p), ("link_off", C.c_void_p)]


class _View(C.Structure):
    """sgb_view of include/sgb200.h."""
    _fields_ = [("n", C.c_int64), ("edge", C.c_int), ("bs", C.c_int), ("nprop", C.c_int), ("nn_kind", C.c_int),
                ("size", C.c_int64 * 3), ("bsz", C.c_int64 * 3), ("keys", C.c_void_p), ("data", C.c_void_p * 8),
                ("mask", C.c_void_p), ("nn", C.c_void_p), ("zorder", C.c_int)]


def _stream(stream=None) -> int:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)


def _i32arr(vals):
    return (C.c_int * len(vals))(*vals)


class _DevView:
    """Zero-copy torch view of a device buffer owned by the library."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


class SparseGridGpu:
    """SparseGridGpu(size, props, edge): a 3-D sparse block grid on one GPU."""

    def __init__(self, size: Sequence[int], props: Sequence[str] = ("f32",), edge: int = 8, device: int = 0,
                 linearizer: str = "smb"):
        """linearizer "smb" (grid_smb, block x fastest) or "zmb" (grid_zmb Morton chunk ids,
        SparseGridGpu_z)."""
        lib = L.load()
        self.size = tuple(int(s) for s in size)
        self.edge = int(edge)
        self.bs = self.edge ** 3
        self.ptypes = [_TYPES[p] if isinstance(p, str) else int(p) for p in props]
        self.device = device
        sz = (C.c_int64 * 3)(*self.size)
        pt = _i32arr(self.ptypes)
        h = C.c_void_p()
        L.check(lib.sgb_create(C.byref(h), 3, self.edge, sz, len(self.ptypes), pt, device), "sgb_create")
        self._h = h
        self._lib = lib
        self.bck = [0] * len(self.ptypes)
        self.linearizer = linearizer
        if linearizer not in ("smb", "zmb"):
            raise ValueError("linearizer is 'smb' or 'zmb'")
        if linearizer == "zmb":
            L.check(lib.sgb_set_linearizer(h, L.LIN_ZMB), "sgb_set_linearizer")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.sgb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # ---------------------------------------------------------------- setup
    def setBackgroundValue(self, p: int, value) -> None:
        v = np.array([value], dtype=_NP[self.ptypes[p]])
        L.check(self._lib.sgb_set_background(self._h, p, v.ctypes.data_as(C.c_void_p)), "sgb_set_background")
        self.bck[p] = value

    def setLaunchConfig(self, ctas_per_sm: int = 0, stages: int = 0) -> None:
        L.check(self._lib.sgb_set_launch_config(self._h, ctas_per_sm, stages), "sgb_set_launch_config")

    # ---------------------------------------------------------------- insert / flush
    def _values(self, values):
        ptrs = (C.c_void_p * len(self.ptypes))()
        keep = []
        for p, t in enumerate(self.ptypes):
            v = None if values is None else values[p] if p < len(values) else None
            if v is None:
                ptrs[p] = None
                continue
            v = v.to(device=f"cuda:{self.device}", dtype=_TORCH[t]).contiguous()
            keep.append(v)
            ptrs[p] = v.data_ptr()
        return ptrs, keep

    def insert(self, coords: torch.Tensor, values: Sequence[Optional[torch.Tensor]], stream=None) -> None:
        """Stage points (int32 [n,3] on the device) with one value per property."""
        c = coords.to(device=f"cuda:{self.device}", dtype=torch.int32).contiguous()
        ptrs, keep = self._values(values)
        L.check(self._lib.sgb_insert(self._h, c.shape[0], c.data_ptr(), ptrs, _stream(stream)), "sgb_insert")
        self._keep = (c, keep)  # the staging copy is stream ordered; keep inputs alive until then

    def insert_lin(self, lin: torch.Tensor, values, stream=None) -> None:
        l = lin.to(device=f"cuda:{self.device}", dtype=torch.int64).contiguous()
        ptrs, keep = self._values(values)
        L.check(self._lib.sgb_insert_lin(self._h, l.shape[0], l.data_ptr(), ptrs, _stream(stream)), "sgb_insert_lin")
        self._keep = (l, keep)

    def insert_pools(self, counts: torch.Tensor, lin: torch.Tensor, values, stream=None) -> None:
        """Stage per-CTA insert pools (setGPUInsertBuffer + insert<p> + flush_block_insert):
        counts int32 [npools], lin int64 [npools, nslot], values[p] [npools, nslot] or None."""
        dev = f"cuda:{self.device}"
        cnt = counts.to(device=dev, dtype=torch.int32).contiguous()
        l = lin.to(device=dev, dtype=torch.int64).contiguous()
        npools, nslot = l.shape
        ptrs, keep = self._values(values)
        L.check(self._lib.sgb_insert_pools(self._h, npools, nslot, cnt.data_ptr(), l.data_ptr(), ptrs,
                                           _stream(stream)), "sgb_insert_pools")
        self._keep = (cnt, l, keep)

    def insert_blocks(self, counts: torch.Tensor, keys: torch.Tensor, values, masks: torch.Tensor,
                      stream=None) -> None:
        """Stage chunk slots written through insertBlock: counts int32 [npools], keys int64
        [npools, nslot], values[p] [npools, nslot, bs] or None, masks uint8 [npools, nslot, bs]."""
        dev = f"cuda:{self.device}"
        cnt = counts.to(device=dev, dtype=torch.int32).contiguous()
        k = keys.to(device=dev, dtype=torch.int64).contiguous()
        m = masks.to(device=dev, dtype=torch.uint8).contiguous()
        npools, nslot = k.shape
        ptrs, keep = self._values(values)
        L.check(self._lib.sgb_insert_blocks(self._h, npools, nslot, cnt.data_ptr(), k.data_ptr(), ptrs, m.data_ptr(),
                                            _stream(stream)), "sgb_insert_blocks")
        self._keep_blocks = (cnt, k, m, keep)

    def view(self, nn: int = L.NN_STAR, stream=None) -> dict:
        """Device view for user kernels (toKernel): sizes and raw device pointers (sgb_get_view)."""
        v = _View()
        L.check(self._lib.sgb_get_view(self._h, nn, C.byref(v), _stream(stream)), "sgb_get_view")
        return {"n": v.n, "edge": v.edge, "bs": v.bs, "nprop": v.nprop, "nn_kind": v.nn_kind,
                "size": tuple(v.size), "bsz": tuple(v.bsz), "keys": v.keys or 0,
                "data": [v.data[p] or 0 for p in range(v.nprop)], "mask": v.mask or 0, "nn": v.nn or 0,
                "zorder": v.zorder}

    def flush(self, ops: Iterable, stream=None) -> None:
        """flush<ops...>: one reduction per property (sgb_op ids or reference names)."""
        o = [OPS[x] if (isinstance(x, str) or x is None) else int(x) for x in ops]
        o += [L.OP_NONE] * (len(self.ptypes) - len(o))
        L.check(self._lib.sgb_flush(self._h, _i32arr(o), _stream(stream)), "sgb_flush")

    # ---------------------------------------------------------------- neighbours / tag
    def findNeighbours(self, nn: int = L.NN_STAR, stream=None) -> None:
        L.check(self._lib.sgb_find_neighbours(self._h, nn, _stream(stream)), "sgb_find_neighbours")

    def neighbour_table(self, nn: int = L.NN_STAR, stream=None) -> np.ndarray:
        k = 8 if nn == L.NN_STAR else 27
        out = np.empty(self.nchunks * k, dtype=np.int64)
        L.check(self._lib.sgb_neighbour_table(self._h, nn, out.ctypes.data_as(C.c_void_p), _stream(stream)),
                "sgb_neighbour_table")
        return out.reshape(self.nchunks, k)

    def tagBoundaries(self, nn: int = L.NN_STAR, calculate_existing_points: bool = False, stream=None) -> None:
        """tagBoundaries<NN>(ctx, No_check(), opt); calculate_existing_points builds the
        existing-point list (tag_boundaries::CALCULATE_EXISTING_POINTS)."""
        L.check(self._lib.sgb_tag_boundaries(self._h, nn, _stream(stream)), "sgb_tag_boundaries")
        if calculate_existing_points:
            self.calc_existing_points(stream)

    def calc_existing_points(self, stream=None) -> int:
        cnt = C.c_int64()
        L.check(self._lib.sgb_calc_existing_points(self._h, C.byref(cnt), _stream(stream)),
                "sgb_calc_existing_points")
        return cnt.value

    def existing_point_list(self, stream=None) -> torch.Tensor:
        """The e_points list: int64 copy of the uint32 ids chunk position * bs + offset."""
        p, cnt = C.c_void_p(), C.c_int64()
        L.check(self._lib.sgb_existing_point_list(self._h, C.byref(p), C.byref(cnt), _stream(stream)),
                "sgb_existing_point_list")
        if cnt.value == 0:
            return torch.empty(0, dtype=torch.int64, device=f"cuda:{self.device}")
        v = torch.as_tensor(_DevView(p.value, (cnt.value,), "<i4"), device=f"cuda:{self.device}")
        return v.to(torch.int64) & 0xFFFFFFFF

    # ---------------------------------------------------------------- stencils
    @staticmethod
    def _box(box):
        if box is None:
            return None
        lo, hi = box
        return (C.c_int64 * 6)(*(list(lo) + list(hi)))

    def applyStencils(self, kind: int, src: Sequence[int], dst: Sequence[int], params: Sequence[float],
                      box=None, stream=None, tiled: bool = False) -> None:
        prm = (C.c_float * len(params))(*params)
        fn = self._lib.sgb_apply_stencil_tiled if tiled else self._lib.sgb_apply_stencil
        L.check(fn(self._h, kind, _i32arr(src), _i32arr(dst), prm, len(params), self._box(box), _stream(stream)),
                "sgb_apply_stencil")

    def run_steps(self, kind: int, src, dst, params, nsteps: int, use_graph: bool = True, stream=None) -> bool:
        """nsteps ping-pong applications; returns True when the result is in dst."""
        prm = (C.c_float * len(params))(*params)
        fin = C.c_int(0)
        L.check(self._lib.sgb_run_steps(self._h, kind, _i32arr(src), _i32arr(dst), prm, len(params), nsteps,
                                        int(use_graph), C.byref(fin), _stream(stream)), "sgb_run_steps")
        return bool(fin.value)

    def check_device_errors(self, stream=None) -> None:
        L.check(self._lib.sgb_check_device_errors(self._h, _stream(stream)), "device error word")

    # ---------------------------------------------------------------- data access
    @property
    def nchunks(self) -> int:
        n = C.c_int64()
        L.check(self._lib.sgb_nchunks(self._h, C.byref(n)), "sgb_nchunks")
        return n.value

    def private_get_index_array(self) -> torch.Tensor:
        p = C.c_void_p()
        L.check(self._lib.sgb_index_buffer(self._h, C.byref(p)), "sgb_index_buffer")
        return torch.as_tensor(_DevView(p.value or 0, (self.nchunks,), "<i8"), device=f"cuda:{self.device}")

    def private_get_data_array(self, prop: int) -> torch.Tensor:
        """Chunk data of one property, (nchunks + 1) * bs elements, background chunk last."""
        p = C.c_void_p()
        L.check(self._lib.sgb_data_buffer(self._h, prop, C.byref(p)), "sgb_data_buffer")
        return torch.as_tensor(_DevView(p.value, ((self.nchunks + 1) * self.bs,), _TS[self.ptypes[prop]]),
                               device=f"cuda:{self.device}")

    def private_get_mask_array(self) -> torch.Tensor:
        p = C.c_void_p()
        L.check(self._lib.sgb_mask_buffer(self._h, C.byref(p)), "sgb_mask_buffer")
        return torch.as_tensor(_DevView(p.value, ((self.nchunks + 1) * self.bs,), "|u1"), device=f"cuda:{self.device}")

    def load_map(self, keys: np.ndarray, data: Sequence[np.ndarray], mask: np.ndarray, stream=None) -> None:
        """hostToDevice of a whole block map (sorted keys, chunk data without
        background); a None entry fills that property with its background."""
        keys = np.ascontiguousarray(keys, dtype=np.int64)
        data = [None if d is None else np.ascontiguousarray(d, dtype=_NP[t]) for d, t in zip(data, self.ptypes)]
        data += [None] * (len(self.ptypes) - len(data))
        mask = np.ascontiguousarray(mask, dtype=np.uint8)
        ptrs = (C.c_void_p * len(data))(*[None if d is None else d.ctypes.data for d in data])
        L.check(self._lib.sgb_load_map(self._h, len(keys), keys.ctypes.data_as(C.c_void_p), ptrs,
                                       mask.ctypes.data_as(C.c_void_p), _stream(stream)), "sgb_load_map")

    def load_map_dev(self, keys: torch.Tensor, data: Sequence[torch.Tensor], mask: torch.Tensor, stream=None) -> None:
        ptrs = (C.c_void_p * len(data))(*[d.data_ptr() for d in data])
        L.check(self._lib.sgb_load_map_dev(self._h, keys.shape[0], keys.data_ptr(), ptrs, mask.data_ptr(),
                                           _stream(stream)), "sgb_load_map_dev")

    def deviceToHost(self, stream=None):
        """(keys[n], [data_p[(n+1)*bs]], mask[(n+1)*bs]) as numpy arrays."""
        n = self.nchunks
        keys = np.empty(n, dtype=np.int64)
        data = [np.empty((n + 1) * self.bs, dtype=_NP[t]) for t in self.ptypes]
        mask = np.empty((n + 1) * self.bs, dtype=np.uint8)
        ptrs = (C.c_void_p * len(data))(*[d.ctypes.data for d in data])
        L.check(self._lib.sgb_download_map(self._h, keys.ctypes.data_as(C.c_void_p), ptrs,
                                           mask.ctypes.data_as(C.c_void_p), _stream(stream)), "sgb_download_map")
        return keys, data, mask

    # ---------------------------------------------------------------- VTK output
    _VTK_TYPES = {L.F32: ("float", ">f4"), L.I32: ("int", ">i4"), L.F64: ("double", ">f8"),
                  L.U8: ("unsigned_char", "u1")}

    def write(self, output: str, spacing=(1.0, 1.0, 1.0), offset=(0.0, 0.0, 0.0), names=None) -> bool:
        """write / write_with_spacing_offset (src/SparseGridGpu/SparseGridGpu.hpp:3844-3903): every
        point whose mask byte is not 0, at coord * spacing + offset * spacing (float32), with all
        properties and the mask byte as point data, as a binary legacy VTK poly-data file of
        vertices.  The reference hands the same points and values to openfpm_io's VTKWriter
        (VECTOR_POINTS), which is not part of this project; the file layout here is the VTK
        legacy format's."""
        keys, data, mask = self.deviceToHost()
        n = len(keys)
        idx = np.nonzero(mask[: n * self.bs])[0]
        coords = self.existing_coords_of(keys, idx)
        sp = np.asarray(spacing, dtype=np.float64)
        pos = (coords * sp + np.asarray(offset, dtype=np.float64) * sp).astype(">f4")
        m = len(idx)
        names = list(names) if names else [f"attr{p}" for p in range(len(self.ptypes))]
        with open(output, "wb") as f:
            f.write(b"# vtk DataFile Version 3.0\nsparse_grid\nBINARY\nDATASET POLYDATA\n")
            f.write(f"POINTS {m} float\n".encode())
            f.write(pos.tobytes())
            f.write(f"\nVERTICES {m} {2 * m}\n".encode())
            f.write(np.stack([np.ones(m, ">i4"), np.arange(m, dtype=">i4")], axis=1).tobytes())
            f.write(f"\nPOINT_DATA {m}\n".encode())
            for p, t in enumerate(self.ptypes):
                vt, dt = self._VTK_TYPES[t]
                f.write(f"SCALARS {names[p]} {vt}\nLOOKUP_TABLE default\n".encode())
                f.write(data[p][idx].astype(dt).tobytes())
                f.write(b"\n")
            f.write(b"SCALARS mask unsigned_char\nLOOKUP_TABLE default\n")
            f.write(mask[idx].astype("u1").tobytes())
            f.write(b"\n")
        return True

    def existing_coords_of(self, keys: np.ndarray, idx: np.ndarray) -> np.ndarray:
        """Coordinates [m, 3] of chunk-data positions idx (chunk position * bs + offset)."""
        e = self.edge
        key = keys[idx // self.bs]
        off = idx % self.bs
        if self.linearizer == "zmb":
            u = key.astype(np.uint64)
            bc = np.zeros((len(key), 3), dtype=np.int64)
            for i in range(21):
                for d in range(3):
                    bc[:, d] |= ((u >> np.uint64(3 * i + d)) & np.uint64(1)).astype(np.int64) << i
        else:
            b = [(s + e - 1) // e for s in self.size]
            bc = np.stack([key % b[0], (key // b[0]) % b[1], key // (b[0] * b[1])], axis=1)
        return bc * e + np.stack([off % e, (off // e) % e, off // (e * e)], axis=1)

    # ---------------------------------------------------------------- remove / iterate
    def remove(self, box) -> None:
        """remove(box): queue an inclusive box ((lo), (hi)) of points to remove at removePoints()."""
        lo, hi = box
        self._rem = getattr(self, "_rem", []) + [list(lo) + list(hi)]

    def removePoints(self, stream=None) -> None:
        """Remove the existing points inside the queued boxes (chunks stay) and clear the queue."""
        rem = getattr(self, "_rem", [])
        self._rem = []
        if not rem:
            return
        b = np.ascontiguousarray(np.asarray(rem, dtype=np.int64).reshape(-1, 6))
        L.check(self._lib.sgb_remove_boxes(self._h, len(b), b.ctypes.data_as(C.c_void_p), _stream(stream)),
                "sgb_remove_boxes")

    def existing_points(self, box=None, stream=None) -> torch.Tensor:
        """int32 [k, 3] device tensor of the existing points (inside the inclusive box
        ((lo), (hi)) if given), in chunk order then offset order."""
        bx = None
        if box is not None:
            bx = np.ascontiguousarray(np.asarray(list(box[0]) + list(box[1]), dtype=np.int64))
        bptr = None if bx is None else bx.ctypes.data_as(C.c_void_p)
        cnt = C.c_int64()
        L.check(self._lib.sgb_existing_points(self._h, bptr, None, 0, C.byref(cnt), _stream(stream)),
                "sgb_existing_points")
        out = torch.empty((cnt.value, 3), dtype=torch.int32, device=f"cuda:{self.device}")
        if cnt.value:
            L.check(self._lib.sgb_existing_points(self._h, bptr, out.data_ptr(), cnt.value, C.byref(cnt),
                                                  _stream(stream)), "sgb_existing_points")
        return out

    def getIterator(self, start=None, stop=None):
        """Host iteration over the existing points (inside [start, stop] when given), as
        (x, y, z) tuples in the reference iterator's order."""
        box = None if start is None else (start, stop)
        for p in self.existing_points(box).cpu().numpy():
            yield tuple(int(v) for v in p)

    # ---------------------------------------------------------------- multi-resolution links
    def construct_link_dw(self, grid_dw: "SparseGridGpu", box, p_dw=(0, 0, 0), stream=None) -> None:
        """Links from the padding points inside box ((lo), (hi)) to the finer grid grid_dw."""
        b = (C.c_int64 * 6)(*(list(box[0]) + list(box[1])))
        sh = (C.c_int64 * 3)(*[int(v) for v in p_dw])
        L.check(self._lib.sgb_construct_link_dw(self._h, grid_dw._h, b, sh, _stream(stream)), "sgb_construct_link_dw")

    def construct_link_up(self, grid_up: "SparseGridGpu", box, p_up=(0, 0, 0), stream=None) -> None:
        """Links from the padding points inside box to the coarser grid grid_up."""
        b = (C.c_int64 * 6)(*(list(box[0]) + list(box[1])))
        sh = (C.c_int64 * 3)(*[int(v) for v in p_up])
        L.check(self._lib.sgb_construct_link_up(self._h, grid_up._h, b, sh, _stream(stream)), "sgb_construct_link_up")

    def _links(self, up: int) -> dict:
        v = _Links()
        L.check(self._lib.sgb_get_links(self._h, up, C.byref(v)), "sgb_get_links")
        dev = f"cuda:{self.device}"

        def arr(ptr, n, ts):
            if n == 0 or not ptr:
                return torch.empty(0, dtype=torch.int64, device=dev)
            return torch.as_tensor(_DevView(ptr, (n,), ts), device=dev).to(torch.int64)
        offs = arr(v.offsets, v.npad + 1, "<i4") & 0xFFFFFFFF if v.offsets else torch.zeros(1, dtype=torch.int64)
        return {"pad_pos": arr(v.pad_pos, v.npad, "<i4"), "pad_off": arr(v.pad_off, v.npad, "<i2"),
                "offsets": offs, "link_pos": arr(v.link_pos, v.nlinks, "<i4"),
                "link_off": arr(v.link_off, v.nlinks, "<i2")}

    def getDownLinks(self) -> dict:
        """Padding points, per-point link offsets (npad + 1) and links (chunk position, offset)."""
        return self._links(0)

    def getUpLinks(self) -> dict:
        return self._links(1)

    # ---------------------------------------------------------------- pack / unpack
    def packReset(self) -> None:
        """Forget the queued pack boxes."""
        self._pack = []

    def packRequest(self, box) -> None:
        """Queue an inclusive box ((lo), (hi)) to pack (packRequest(sub_it, req))."""
        lo, hi = box
        self._pack = getattr(self, "_pack", []) + [list(lo) + list(hi)]

    def packCalculate(self, props: Sequence[int], stream=None) -> int:
        """Bytes needed to pack the queued boxes with the listed properties."""
        return int(sum(self.pack_sizes(getattr(self, "_pack", []), props, stream)))

    def pack_sizes(self, boxes, props: Sequence[int], stream=None) -> list:
        b = np.ascontiguousarray(np.asarray(boxes, dtype=np.int64).reshape(-1, 6))
        out = np.zeros(len(b), dtype=np.int64)
        if len(b):
            L.check(self._lib.sgb_pack_request(self._h, len(b), b.ctypes.data_as(C.c_void_p), len(props),
                                               _i32arr(list(props)), out.ctypes.data_as(C.c_void_p),
                                               _stream(stream)), "sgb_pack_request")
        return [int(x) for x in out]

    def packFinalize(self, buf: torch.Tensor, props: Sequence[int], stream=None) -> int:
        """Pack the queued boxes into the uint8 device tensor buf; returns the bytes written."""
        boxes = getattr(self, "_pack", [])
        return self.pack_boxes(boxes, props, buf, stream)

    def pack_boxes(self, boxes, props: Sequence[int], buf: Optional[torch.Tensor] = None, stream=None):
        """Pack the inclusive boxes [k, 6] (lo, hi) into buf (allocated when None; then the tensor
        is returned, else the bytes written)."""
        b = np.ascontiguousarray(np.asarray(boxes, dtype=np.int64).reshape(-1, 6))
        ret_buf = buf is None
        if buf is None:
            buf = torch.empty(sum(self.pack_sizes(b, props, stream)), dtype=torch.uint8,
                              device=f"cuda:{self.device}")
        written = C.c_int64(0)
        L.check(self._lib.sgb_pack(self._h, len(b), b.ctypes.data_as(C.c_void_p), len(props),
                                   _i32arr(list(props)), buf.data_ptr() if buf.numel() else None, buf.numel(),
                                   C.byref(written), _stream(stream)), "sgb_pack")
        return buf if ret_buf else written.value

    def unpack(self, buf: torch.Tensor, props: Sequence[int], start=None, offset: int = 0, stream=None) -> int:
        """unpack one packed box at byte offset of buf into the box starting at start (None: its
        packed place); the points are staged until removeAddUnpackFinalize.  Returns the offset
        of the next box (Unpack_stat)."""
        st = None if start is None else (C.c_int64 * 3)(*[int(v) for v in start])
        used = C.c_int64(0)
        L.check(self._lib.sgb_unpack(self._h, buf.data_ptr() + offset, buf.numel() - offset, len(props),
                                     _i32arr(list(props)), st, C.byref(used), _stream(stream)), "sgb_unpack")
        return offset + used.value

    def unpack_boxes(self, buf: torch.Tensor, props: Sequence[int], starts=None, nboxes: Optional[int] = None,
                     offset: int = 0, stream=None) -> int:
        """unpack of nboxes consecutive packed boxes (len(starts) when starts are given) in one call;
        returns the offset after them."""
        if nboxes is None:
            if starts is None:
                raise ValueError("give starts or nboxes")
            nboxes = len(starts)
        st = None
        if starts is not None:
            st = np.ascontiguousarray(np.asarray(starts, dtype=np.int64).reshape(-1, 3))
            assert len(st) == nboxes
        used = C.c_int64(0)
        L.check(self._lib.sgb_unpack_boxes(self._h, buf.data_ptr() + offset, buf.numel() - offset, len(props),
                                           _i32arr(list(props)), nboxes,
                                           None if st is None else st.ctypes.data_as(C.c_void_p), C.byref(used),
                                           _stream(stream)), "sgb_unpack_boxes")
        return offset + used.value

    def removeAddUnpackReset(self) -> None:
        self._rem = []

    def removeAddUnpackFinalize(self, props: Sequence[int], stream=None) -> None:
        """Apply the queued removals, then merge the unpacked points: their unpacked properties are
        overwritten, the others keep their values (background for new points)."""
        self.removePoints(stream)
        ops = [L.OP_NONE] * len(self.ptypes)
        for p in props:
            ops[p] = L.OP_RIGHT
        self.flush(ops, stream)

    def measureBlockOccupancy(self, memory: bool = False):
        """(mean, sample standard deviation) over the chunks of the fraction of active points
        (existing and not padding; existing points with memory=True) -- measureBlockOccupancy /
        measureBlockOccupancyMemory (src/SparseGridGpu/SparseGridGpu.hpp:2485-2554)."""
        keys, _, mask = self.deviceToHost()
        n = len(keys)
        m = mask[: n * self.bs].reshape(n, self.bs)
        sel = (m & 1) != 0 if memory else (m & 3) == 1
        occ = sel.sum(axis=1) / self.bs
        return float(occ.mean()), float(occ.std(ddof=1)) if n > 1 else float("nan")

    def removeUnusedBuffers(self) -> None:
        """Free the temporary device buffers (removeUnusedBuffers)."""
        L.check(self._lib.sgb_release_scratch(self._h), "sgb_release_scratch")

    def countExistingElements(self, stream=None) -> int:
        e = C.c_int64()
        L.check(self._lib.sgb_count_existing(self._h, C.byref(e), None, _stream(stream)), "sgb_count_existing")
        return e.value

    def countBoundaryElements(self, stream=None) -> int:
        p = C.c_int64()
        L.check(self._lib.sgb_count_existing(self._h, None, C.byref(p), _stream(stream)), "sgb_count_existing")
        return p.value

    def build_balls(self, balls: np.ndarray, init: int, seed: int, props: Sequence[int], stream=None) -> None:
        """Replace the block map by a union of balls [k,4] = (cx, cy, cz, r) (sgb_build_balls)."""
        b = np.ascontiguousarray(balls, dtype=np.float32).reshape(-1, 4)
        L.check(self._lib.sgb_build_balls(self._h, len(b), b.ctypes.data_as(C.c_void_p), int(init),
                                          C.c_uint64(int(seed) & (2 ** 64 - 1)), _i32arr(list(props)),
                                          _stream(stream)), "sgb_build_balls")

    def existing_offsets(self, stream=None) -> torch.Tensor:
        """int64 [nchunks + 1]: existing points before each chunk, total last."""
        out = torch.empty(self.nchunks + 1, dtype=torch.int64, device=f"cuda:{self.device}")
        L.check(self._lib.sgb_existing_offsets(self._h, out.data_ptr(), _stream(stream)), "sgb_existing_offsets")
        return out

    def get(self, prop: int, coords: torch.Tensor, stream=None) -> torch.Tensor:
        c = coords.to(device=f"cuda:{self.device}", dtype=torch.int32).contiguous()
        out = torch.empty(c.shape[0], dtype=_TORCH[self.ptypes[prop]], device=f"cuda:{self.device}")
        L.check(self._lib.sgb_get(self._h, c.shape[0], c.data_ptr(), prop, out.data_ptr(), _stream(stream)), "sgb_get")
        return out

    def device_bytes(self) -> int:
        b = C.c_int64()
        L.check(self._lib.sgb_device_bytes(self._h, C.byref(b)), "sgb_device_bytes")
        return b.value


class Batch:
    """Many grids advanced by one persistent launch per step (sgb_batch_*)."""

    def __init__(self, device: int = 0):
        lib = L.load()
        h = C.c_void_p()
        L.check(lib.sgb_batch_create(C.byref(h), device), "sgb_batch_create")
        self._h, self._lib = h, lib

    def close(self):
        if getattr(self, "_h", None):
            self._lib.sgb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_launch_config(self, ctas_per_sm: int = 0, stages: int = 0):
        L.check(self._lib.sgb_batch_set_launch_config(self._h, ctas_per_sm, stages), "sgb_batch_set_launch_config")

    def add(self, g: SparseGridGpu, kind: int, src, dst, params, nsteps: int, stream=None) -> int:
        prm = (C.c_float * len(params))(*params)
        slot = C.c_int(-1)
        L.check(self._lib.sgb_batch_add(self._h, g.handle, kind, _i32arr(src), _i32arr(dst), prm, len(params),
                                        int(nsteps), C.byref(slot), _stream(stream)), "sgb_batch_add")
        return slot.value

    def remove(self, slot: int, stream=None):
        L.check(self._lib.sgb_batch_remove(self._h, slot, _stream(stream)), "sgb_batch_remove")

    def step(self, nsteps: int = 1, use_graph: bool = True, stream=None):
        L.check(self._lib.sgb_batch_step(self._h, nsteps, int(use_graph), _stream(stream)), "sgb_batch_step")

    def slot_steps(self, slot: int) -> int:
        d = C.c_int64()
        L.check(self._lib.sgb_batch_slot_steps(self._h, slot, C.byref(d)), "sgb_batch_slot_steps")
        return d.value

    def extract(self, slot: int, g: SparseGridGpu, stream=None) -> bool:
        fin = C.c_int(0)
        L.check(self._lib.sgb_batch_extract(self._h, slot, g.handle, C.byref(fin), _stream(stream)),
                "sgb_batch_extract")
        return bool(fin.value)

    def nchunks(self, slot: int) -> int:
        n = C.c_int64()
        L.check(self._lib.sgb_batch_read(self._h, slot, None, None, None, C.byref(n), None), "sgb_batch_read")
        return n.value

    def read(self, slot: int, nfields: int, bs: int = 512, stream=None, staged: bool = False):
        """(keys, mask, [fields]) of a slot's current state as numpy arrays.

        staged=True reads into a grow-only pinned host buffer owned by the
        batch (fast device-to-host copies) and returns views of it, valid
        until the next staged read."""
        n = self.nchunks(slot)
        if staged:
            need = n * 8 + n * bs + nfields * n * bs * 4
            buf = getattr(self, "_pinned", None)
            if buf is None or buf.numel() < need:
                buf = torch.empty(max(need, 1 << 20), dtype=torch.uint8).pin_memory()
                self._pinned = buf
            raw = buf.numpy()
            keys = raw[: n * 8].view(np.int64)
            mask = raw[n * 8: n * 8 + n * bs]
            o = n * 8 + n * bs
            fields = [raw[o + j * n * bs * 4: o + (j + 1) * n * bs * 4].view(np.float32) for j in range(nfields)]
        else:
            keys = np.empty(n, np.int64)
            mask = np.empty(n * bs, np.uint8)
            fields = [np.empty(n * bs, np.float32) for _ in range(nfields)]
        ptrs = (C.c_void_p * nfields)(*[f.ctypes.data for f in fields])
        L.check(self._lib.sgb_batch_read(self._h, slot, keys.ctypes.data_as(C.c_void_p),
                                         mask.ctypes.data_as(C.c_void_p), ptrs, None, _stream(stream)),
                "sgb_batch_read")
        return keys, mask, fields

    def read_async(self, slot: int, nfields: int, bs: int = 512, stream=None):
        """Queue the copy of a slot's state into fresh pinned host tensors on `stream` and return
        (keys, mask, [fields], event): the arrays hold the state once `event` has completed."""
        n = self.nchunks(slot)
        keys = torch.empty(max(n, 1), dtype=torch.int64).pin_memory()
        mask = torch.empty(max(n * bs, 1), dtype=torch.uint8).pin_memory()
        fields = [torch.empty(max(n * bs, 1), dtype=torch.float32).pin_memory() for _ in range(nfields)]
        ptrs = (C.c_void_p * nfields)(*[f.data_ptr() for f in fields])
        L.check(self._lib.sgb_batch_read_async(self._h, slot, keys.data_ptr(), mask.data_ptr(), ptrs, None,
                                               _stream(stream)), "sgb_batch_read_async")
        ev = torch.cuda.Event()
        ev.record(stream if stream is not None else torch.cuda.current_stream())
        return keys.numpy()[:n], mask.numpy()[: n * bs], [f.numpy()[: n * bs] for f in fields], ev

    def info(self):
        ng, nc, nb = C.c_int(), C.c_int64(), C.c_int64()
        L.check(self._lib.sgb_batch_info(self._h, C.byref(ng), C.byref(nc), C.byref(nb)), "sgb_batch_info")
        return ng.value, nc.value, nb.value
