"""Wavefront OBJ files <-> host meshes (slak_obj_read / slak_obj_write).

The arrays are the reference's CSCMesh layout (include/Mesh.h:153-176):
face offsets, 0-based corner ids, vals = 1-based corner position in its face,
positions (x, y, z, 1); the mesh type is TRI / QUAD / POLY from the face sizes.
The parse runs multi-threaded in the C++ library.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _abi
from .mesh import QUAD, TRI, Mesh


def read_obj(path: str) -> Mesh:
    return _read(path, None)


def read_obj_sharp(path: str):
    """(mesh, (pairs, sharpness), (corner ids, corner sharpness)) with the
    file's "t crease" and "t corner" tags."""
    cr = _abi.SlakCreases()
    ko = _abi.SlakCorners()
    mesh = _read(path, cr, ko)
    try:
        m, k = int(cr.count), int(ko.count)
        pairs = np.ctypeslib.as_array(cr.verts, shape=(2 * m,)).copy().reshape(m, 2) if m else np.zeros((0, 2), np.int32)
        sharp = np.ctypeslib.as_array(cr.sharpness, shape=(m,)).copy() if m else np.zeros(0, np.float32)
        kv = np.ctypeslib.as_array(ko.verts, shape=(k,)).copy() if k else np.zeros(0, np.int32)
        ks = np.ctypeslib.as_array(ko.sharpness, shape=(k,)).copy() if k else np.zeros(0, np.float32)
        return mesh, (pairs, sharp), (kv, ks)
    finally:
        _abi.lib().slak_obj_free_creases(ctypes.byref(cr))
        _abi.lib().slak_obj_free_corners(ctypes.byref(ko))


def read_obj_creased(path: str):
    """(mesh, (pairs, sharpness)) with the file's "t crease" tags as an (m, 2)
    int32 array of 0-based vertex ids and m float32 sharpness values."""
    cr = _abi.SlakCreases()
    mesh = _read(path, cr)
    try:
        m = int(cr.count)
        if m == 0:
            return mesh, (np.zeros((0, 2), np.int32), np.zeros(0, np.float32))
        pairs = np.ctypeslib.as_array(cr.verts, shape=(2 * m,)).copy().reshape(m, 2)
        sharp = np.ctypeslib.as_array(cr.sharpness, shape=(m,)).copy()
        return mesh, (pairs, sharp)
    finally:
        _abi.lib().slak_obj_free_creases(ctypes.byref(cr))


def _read(path, cr, ko=None) -> Mesh:
    c = _abi.SlakMesh()
    if cr is None:
        rc = _abi.lib().slak_obj_read(os.fsencode(path), ctypes.byref(c))
    elif ko is None:
        rc = _abi.lib().slak_obj_read_creased(os.fsencode(path), ctypes.byref(c), ctypes.byref(cr))
    else:
        rc = _abi.lib().slak_obj_read_sharp(os.fsencode(path), ctypes.byref(c), ctypes.byref(cr), ctypes.byref(ko))
    _abi.check(rc, f"slak_obj_read({path})")
    try:
        F, N, V = int(c.nfaces), int(c.nnz), int(c.nverts)
        arr = lambda p, n, t: np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(t)), shape=(n,)).copy()
        ptr = arr(c.ptr, F + 1, ctypes.c_int32)
        ids = arr(c.ids, N, ctypes.c_int32) if N else np.zeros(0, np.int32)
        vals = arr(c.vals, N, ctypes.c_int32) if N else np.zeros(0, np.int32)
        verts = arr(c.verts, 4 * V, ctypes.c_float).reshape(V, 4) if V else np.zeros((0, 4), np.float32)
        return Mesh(int(c.type), ids, verts, ptr, vals, F, int(c.max_face_order), True)
    finally:
        _abi.lib().slak_obj_free(ctypes.byref(c))


def write_obj(path: str, mesh, creases=None, corners=None) -> None:
    """Writes a host mesh (a Mesh, or any object with its fields, e.g. a
    refined HostResult); QUAD and TRI meshes need no face offsets.  With
    ``creases`` = (pairs, sharpness), one "t crease" tag per pair follows;
    with ``corners`` = (vertex ids, sharpness), one "t corner" tag each."""
    keep = []

    def p(a, dt):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data

    c = _abi.SlakMesh()
    c.type = int(mesh.type)
    c.nfaces, c.nverts, c.nnz = int(mesh.nfaces), int(mesh.nverts), int(mesh.nnz)
    c.ptr = p(None if mesh.type in (QUAD, TRI) else mesh.ptr, np.int32)
    c.ids = p(mesh.ids, np.int32)
    c.verts = p(np.asarray(mesh.verts, np.float32).reshape(-1), np.float32)
    if creases is None and corners is None:
        rc = _abi.lib().slak_obj_write(os.fsencode(path), ctypes.byref(c))
    else:
        cr = None
        if creases is not None:
            pairs = np.ascontiguousarray(np.asarray(creases[0], np.int32).reshape(-1, 2))
            sharp = np.ascontiguousarray(np.asarray(creases[1], np.float32).reshape(-1))
            keep += [pairs, sharp]
            cr = _abi.SlakCreases()
            cr.count = sharp.size
            cr.verts = pairs.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
            cr.sharpness = sharp.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        ko = None
        if corners is not None:
            kv = np.ascontiguousarray(np.asarray(corners[0], np.int32).reshape(-1))
            ks = np.ascontiguousarray(np.asarray(corners[1], np.float32).reshape(-1))
            keep += [kv, ks]
            ko = _abi.SlakCorners()
            ko.count = ks.size
            ko.verts = kv.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
            ko.sharpness = ks.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        rc = _abi.lib().slak_obj_write_sharp(os.fsencode(path), ctypes.byref(c),
                                             ctypes.byref(cr) if cr is not None else None,
                                             ctypes.byref(ko) if ko is not None else None)
    _abi.check(rc, f"slak_obj_write({path})")
