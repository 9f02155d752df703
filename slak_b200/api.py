"""Python mirror of the reference's scheme API on top of the C ABI.

``CatmullClark.subdivideIteratively`` and ``LAKCatmullClark.subdivideIteratively``
keep the reference's call shape (``LibInclude/CatmullClark.h:163-164``,
``LibInclude/LAKCatmullClark.h:165-166``): a device-resident control mesh in,
a target level, a refined device mesh out.  ``Plan`` exposes the
allocation-free execution used for timing and CUDA-graph replay, and
``subdivide`` is a host-to-host convenience.  Device memory and streams come
from PyTorch; every computation runs in ``libslak_b200.so``.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import List, Optional

import numpy as np

from . import _abi
from .mesh import LAK, QUAD, SLAK, Mesh


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("slak_b200 needs a CUDA device (no CPU fallback)")
    return torch


class _CudaArray:
    """Zero-copy handle for a raw device pointer (``__cuda_array_interface__``)."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr,
                                         "data": (int(ptr), False), "version": 3, "strides": None}


def device_view(ptr: int, shape, dtype: str):
    """Torch view of device memory the library owns (valid while the owner lives)."""
    torch = _torch()
    if not ptr or int(np.prod(shape)) == 0:
        return torch.zeros(shape, dtype={"<i4": torch.int32, "<f4": torch.float32}[dtype], device="cuda")
    return torch.as_tensor(_CudaArray(ptr, shape, dtype), device="cuda")


def _stream_handle(stream) -> Optional[int]:
    torch = _torch()
    if stream is None:
        stream = torch.cuda.current_stream()
    return int(stream.cuda_stream) or None


@dataclasses.dataclass
class DeviceMesh:
    """``MeshInfo<int,int,int,float>`` with device arrays (torch tensors)."""
    type: int = QUAD
    nfaces: int = 0
    nverts: int = 0
    nnz: int = 0
    max_face_order: int = 0
    is_reduced: bool = False
    ptr: object = None
    ids: object = None
    vals: object = None
    verts: object = None
    _owner: object = None          # keeps library-owned memory alive

    @staticmethod
    def from_host(m: Mesh, device="cuda") -> "DeviceMesh":
        torch = _torch()
        t = lambda a: None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(device)
        return DeviceMesh(m.type, m.nfaces, m.nverts, m.nnz, m.max_face_order, m.is_reduced,
                          t(m.ptr), t(m.ids), t(m.vals), t(m.verts.reshape(-1).astype(np.float32)))

    def as_c(self) -> _abi.SlakMesh:
        import torch                    # dtypes only: the check itself needs no device
        for name, want, count in (("ptr", torch.int32, self.nfaces + 1), ("ids", torch.int32, self.nnz),
                                  ("vals", torch.int32, self.nnz), ("verts", torch.float32, 4 * self.nverts)):
            t = getattr(self, name)
            if t is None:
                continue
            # the C ABI takes the raw pointer: a tensor of another type, layout
            # or device would be reinterpreted, so it is refused here
            if t.dtype != want or not t.is_contiguous() or t.device.type != "cuda":
                raise TypeError(f"DeviceMesh.{name}: expected a contiguous CUDA {want} tensor, "
                                f"got {t.dtype} on {t.device}")
            if t.numel() < count:
                raise ValueError(f"DeviceMesh.{name}: {t.numel()} elements, the counts need {count}")
        c = _abi.SlakMesh()
        c.type, c.is_reduced = int(self.type), int(bool(self.is_reduced))
        c.nfaces, c.nverts, c.nnz, c.max_face_order = self.nfaces, self.nverts, self.nnz, self.max_face_order
        c.ptr = None if self.ptr is None else self.ptr.data_ptr()
        c.ids = None if self.ids is None else self.ids.data_ptr()
        c.vals = None if self.vals is None else self.vals.data_ptr()
        c.verts = None if self.verts is None else self.verts.data_ptr()
        return c

    def to_host(self) -> "HostResult":
        g = lambda t: None if t is None else t.detach().cpu().numpy().copy()
        verts = g(self.verts)
        return HostResult(self.type, self.nfaces, self.nverts, self.nnz, self.max_face_order, self.is_reduced,
                          g(self.ptr), g(self.ids), g(self.vals),
                          None if verts is None else verts.reshape(-1, 4))


@dataclasses.dataclass
class HostResult:
    type: int
    nfaces: int
    nverts: int
    nnz: int
    max_face_order: int
    is_reduced: bool
    ptr: Optional[np.ndarray]
    ids: np.ndarray
    vals: Optional[np.ndarray]
    verts: np.ndarray


def _wrap_c(c: _abi.SlakMesh, owner) -> DeviceMesh:
    return DeviceMesh(int(c.type), int(c.nfaces), int(c.nverts), int(c.nnz), int(c.max_face_order),
                      bool(c.is_reduced),
                      device_view(c.ptr, (c.nfaces + 1,), "<i4") if c.ptr else None,
                      device_view(c.ids, (c.nnz,), "<i4") if c.ids else None,
                      device_view(c.vals, (c.nnz,), "<i4") if c.vals else None,
                      device_view(c.verts, (4 * c.nverts,), "<f4") if c.verts else None, owner)


class _OwnedMesh:
    """Frees library-allocated output arrays (slak_mesh_free) when dropped."""

    def __init__(self, c: _abi.SlakMesh):
        self.c = c

    def __del__(self):
        try:
            _abi.lib().slak_mesh_free(ctypes.byref(self.c))
        except Exception:
            pass


class _Scheme:
    scheme = SLAK

    @classmethod
    def subdivideIteratively(cls, cmesh: DeviceMesh, rmesh: DeviceMesh, target_level: int, stream=None) -> None:
        cin = cmesh.as_c()
        cout = rmesh.as_c() if rmesh is not None else _abi.SlakMesh()
        rc = _abi.lib().slak_subdivide(ctypes.byref(cin), ctypes.byref(cout), int(target_level), cls.scheme,
                                       _stream_handle(stream))
        _abi.check(rc, "slak_subdivide")
        if not cout.ids:
            return      # nothing refined: rmesh untouched (QUAD input, target_level <= 0)
        r = _wrap_c(cout, _OwnedMesh(cout))
        for f in dataclasses.fields(DeviceMesh):
            setattr(rmesh, f.name, getattr(r, f.name))


class CatmullClark(_Scheme):
    """SLAK scheme (``struct CatmullClark``, LibInclude/CatmullClark.h:33-165)."""
    scheme = SLAK
    MeshInfo = DeviceMesh


class LAKCatmullClark(_Scheme):
    """LAK scheme (``struct LAKCatmullClark``, LibInclude/LAKCatmullClark.h:33-192)."""
    scheme = LAK
    MeshInfo = DeviceMesh


def _crease_tensors(creases):
    """(pairs, sharpness) as contiguous int32 (m, 2) and float32 (m,) CUDA tensors."""
    torch = _torch()
    pairs, sharp = creases
    pairs = torch.as_tensor(np.asarray(pairs) if not torch.is_tensor(pairs) else pairs)
    sharp = torch.as_tensor(np.asarray(sharp) if not torch.is_tensor(sharp) else sharp)
    pairs = pairs.to(device="cuda", dtype=torch.int32).reshape(-1, 2).contiguous()
    sharp = sharp.to(device="cuda", dtype=torch.float32).reshape(-1).contiguous()
    if pairs.shape[0] != sharp.shape[0]:
        raise ValueError("creases: one sharpness per vertex pair")
    return pairs, sharp


def _corner_tensors(corners):
    """(vertex ids, sharpness) as contiguous int32 (k,) and float32 (k,) CUDA tensors."""
    torch = _torch()
    kv, ks = corners
    kv = torch.as_tensor(np.asarray(kv) if not torch.is_tensor(kv) else kv)
    ks = torch.as_tensor(np.asarray(ks) if not torch.is_tensor(ks) else ks)
    kv = kv.to(device="cuda", dtype=torch.int32).reshape(-1).contiguous()
    ks = ks.to(device="cuda", dtype=torch.float32).reshape(-1).contiguous()
    if kv.shape[0] != ks.shape[0]:
        raise ValueError("corners: one sharpness per vertex")
    return kv, ks


class Plan:
    """Sized-once execution of ``levels`` subdivision levels (see slak_plan_create)."""

    def __init__(self, cmesh: DeviceMesh, levels: int, scheme: int, flags: int = 0, stream=None, creases=None,
                 corners=None):
        """``creases``: None, or (pairs, sharpness) -- an (m, 2) array of vertex
        ids and m sharpness values; ``corners``: None, or (vertex ids,
        sharpness).  Host arrays or device tensors (slak_plan_create_sharp; the
        plan keeps its own copy)."""
        self._cmesh = cmesh            # the plan reads these arrays on every execute
        self._cin = cmesh.as_c()
        h = ctypes.c_void_p()
        if creases is None and corners is None:
            rc = _abi.lib().slak_plan_create(ctypes.byref(self._cin), int(levels), int(scheme), int(flags),
                                             _stream_handle(stream), ctypes.byref(h))
            _abi.check(rc, "slak_plan_create")
        else:
            pairs, sharp = _crease_tensors(creases if creases is not None else (np.zeros((0, 2)), np.zeros(0)))
            kv, ks = _corner_tensors(corners if corners is not None else (np.zeros(0), np.zeros(0)))
            rc = _abi.lib().slak_plan_create_sharp(ctypes.byref(self._cin), int(levels), int(scheme), int(flags),
                                                   pairs.data_ptr() if pairs.numel() else None,
                                                   sharp.data_ptr() if sharp.numel() else None, int(sharp.numel()),
                                                   kv.data_ptr() if kv.numel() else None,
                                                   ks.data_ptr() if ks.numel() else None, int(ks.numel()),
                                                   _stream_handle(stream), ctypes.byref(h))
            _abi.check(rc, "slak_plan_create_sharp")
        self._h = h
        self.scheme = scheme

    def execute(self, stream=None) -> None:
        _abi.check(_abi.lib().slak_plan_execute(self._h, _stream_handle(stream)), "slak_plan_execute")

    def status(self, stream=None) -> int:
        return _abi.lib().slak_plan_status(self._h, _stream_handle(stream))

    def check(self, stream=None) -> None:
        _abi.check(self.status(stream), "device status")

    def output(self) -> DeviceMesh:
        c = _abi.SlakMesh()
        _abi.check(_abi.lib().slak_plan_output(self._h, ctypes.byref(c)), "slak_plan_output")
        return _wrap_c(c, self)

    @property
    def launches(self) -> int:
        return int(_abi.lib().slak_plan_launches(self._h))

    def kernel_timings(self) -> List[dict]:
        """Per-launch device times of the last execution (plan created with PLAN_TIMING)."""
        buf = (_abi.KernelTiming * 512)()
        n = _abi.lib().slak_plan_kernel_timings(self._h, buf, 512)
        if n < 0:
            _abi.check(-n, "slak_plan_kernel_timings")
        return [{"name": buf[i].name.decode(), "level": int(buf[i].level), "ms": float(buf[i].ms),
                 "algorithmic_bytes": int(buf[i].algorithmic_bytes)} for i in range(n)]

    def tuning(self) -> List[dict]:
        """Launch shapes of every level (slak_plan_tuning): state -1 for a
        general level, 0 default, 1 measured by this plan, 2 from the cache."""
        out = []
        for i in range(_abi.lib().slak_plan_num_levels(self._h)):
            t = _abi.Tuning()
            _abi.check(_abi.lib().slak_plan_tuning(self._h, i, ctypes.byref(t)), "slak_plan_tuning")
            out.append({"level": i, "state": int(t.state), "block": list(t.block),
                        "ms": [[float(t.ms[k][c]) for c in range(3)] for k in range(3)],
                        "key": t.key.decode()})
        return out

    def level_stats(self) -> List[dict]:
        out = []
        for i in range(_abi.lib().slak_plan_num_levels(self._h)):
            s = _abi.LevelStats()
            _abi.check(_abi.lib().slak_plan_level_stats(self._h, i, ctypes.byref(s)), "slak_plan_level_stats")
            out.append({f: int(getattr(s, f)) for f, _ in _abi.LevelStats._fields_})
        return out

    def close(self) -> None:
        if getattr(self, "_h", None):
            _abi.lib().slak_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:       # interpreter teardown: the library may already be unloaded
            pass


def subdivide(mesh: Mesh, levels: int, scheme: int = SLAK, flags: int = 0, creases=None,
              corners=None) -> HostResult:
    """Host mesh in, host refined mesh out (H2D, one plan execution, D2H).
    ``creases`` / ``corners``: None or (ids, sharpness), see Plan."""
    torch = _torch()
    dm = DeviceMesh.from_host(mesh)
    plan = Plan(dm, levels, scheme, flags, creases=creases, corners=corners)
    plan.execute()
    plan.check()
    out = plan.output().to_host()
    torch.cuda.synchronize()
    plan.close()
    return out


def subdivide_batched(meshes: List[DeviceMesh], levels: List[int], scheme: int, stream=None) -> List[DeviceMesh]:
    """slak_subdivide_batched: every mesh refined in one call; each result owns
    its device arrays (freed with the returned DeviceMesh)."""
    n = len(meshes)
    if len(levels) != n:
        raise ValueError(f"subdivide_batched: {n} meshes but {len(levels)} level counts")
    arr = (_abi.SlakMesh * max(n, 1))()
    for i, m in enumerate(meshes):
        arr[i] = m.as_c()
    lv = (ctypes.c_int * max(n, 1))(*[int(l) for l in levels])
    out = (_abi.SlakMesh * max(n, 1))()
    rc = _abi.lib().slak_subdivide_batched(arr, lv, n, int(scheme), out, _stream_handle(stream))
    _abi.check(rc, "slak_subdivide_batched")
    res = []
    for i in range(n):
        c = out[i]
        res.append(_wrap_c(c, _OwnedMesh(c)) if c.nfaces else DeviceMesh())
    return res


class Batch:
    """Many meshes, each with its own level count, in one call (slak_batch_*).

    ``meshes`` are DeviceMesh inputs; outputs are views into the batch's
    memory, valid while the Batch lives."""

    def __init__(self, meshes: List[DeviceMesh], levels: List[int], scheme: int, flags: int = 0, stream=None):
        self._meshes = list(meshes)
        n = len(self._meshes)
        if len(levels) != n:
            raise ValueError(f"Batch: {n} meshes but {len(levels)} level counts")
        self._arr = (_abi.SlakMesh * max(n, 1))()
        for i, m in enumerate(self._meshes):
            self._arr[i] = m.as_c()
        self._levels = (ctypes.c_int * max(n, 1))(*[int(l) for l in levels])
        h = ctypes.c_void_p()
        rc = _abi.lib().slak_batch_create(self._arr, self._levels, n, int(scheme), int(flags),
                                          _stream_handle(stream), ctypes.byref(h))
        _abi.check(rc, "slak_batch_create")
        self._h = h
        self.count = n

    def execute(self, stream=None) -> None:
        _abi.check(_abi.lib().slak_batch_execute(self._h, _stream_handle(stream)), "slak_batch_execute")

    def check(self, stream=None) -> None:
        _abi.check(_abi.lib().slak_batch_status(self._h, _stream_handle(stream)), "slak_batch_status")

    def output(self, i: int) -> Optional[DeviceMesh]:
        c = _abi.SlakMesh()
        _abi.check(_abi.lib().slak_batch_output(self._h, int(i), ctypes.byref(c)), "slak_batch_output")
        return _wrap_c(c, self) if c.ids else None

    @property
    def waves(self) -> int:
        return int(_abi.lib().slak_batch_num_waves(self._h))

    @property
    def groups(self) -> int:
        return int(_abi.lib().slak_batch_num_groups(self._h))

    @property
    def launches(self) -> int:
        return int(_abi.lib().slak_batch_launches(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            _abi.lib().slak_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:       # interpreter teardown: the library may already be unloaded
            pass
