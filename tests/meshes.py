"""Small hand-built and seeded control meshes shared by the tests."""
import numpy as np

from slak_b200 import meshgen
from slak_b200.mesh import QUAD, Mesh, from_arrays


def cube() -> Mesh:
    V = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], dtype=np.float32)
    i = lambda x, y, z: ((x > 0) << 2) | ((y > 0) << 1) | (z > 0)
    faces = [[i(1, -1, -1), i(1, 1, -1), i(1, 1, 1), i(1, -1, 1)],
             [i(-1, -1, -1), i(-1, -1, 1), i(-1, 1, 1), i(-1, 1, -1)],
             [i(-1, 1, -1), i(-1, 1, 1), i(1, 1, 1), i(1, 1, -1)],
             [i(-1, -1, -1), i(1, -1, -1), i(1, -1, 1), i(-1, -1, 1)],
             [i(-1, -1, 1), i(1, -1, 1), i(1, 1, 1), i(-1, 1, 1)],
             [i(-1, -1, -1), i(-1, 1, -1), i(1, 1, -1), i(1, -1, -1)]]
    return from_arrays(np.arange(7) * 4, np.array(faces).reshape(-1), V)


def cube_quad_type() -> Mesh:
    """The cube as a QUAD mesh without ptr/vals (SLAK quad functions only)."""
    m = cube()
    return Mesh(QUAD, m.ids, m.verts, None, None, m.nfaces, 4, True)


def tetrahedron() -> Mesh:
    V = np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], dtype=np.float32)
    F = [[0, 1, 2], [0, 3, 1], [0, 2, 3], [1, 3, 2]]
    return from_arrays(np.arange(5) * 3, np.array(F).reshape(-1), V)


def pentagon_prism() -> Mesh:
    a = np.linspace(0, 2 * np.pi, 6)[:-1]
    V = np.concatenate([np.stack([np.cos(a), np.sin(a), -np.ones(5)], 1),
                        np.stack([np.cos(a), np.sin(a), np.ones(5)], 1)]).astype(np.float32)
    faces = [[4, 3, 2, 1, 0], [5, 6, 7, 8, 9]] + [[k, (k + 1) % 5, 5 + (k + 1) % 5, 5 + k] for k in range(5)]
    ptr = np.cumsum([0] + [len(f) for f in faces])
    return from_arrays(ptr, np.concatenate(faces), V)


def open_grid(nx=3, ny=2) -> Mesh:
    """Flat nx x ny quad patch with a boundary (SLAK/LAK boundary rules)."""
    xs, ys = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="ij")
    rng = np.random.default_rng(7)
    V = np.stack([xs.ravel(), ys.ravel(), 0.1 * rng.standard_normal(xs.size)], 1).astype(np.float32)
    vid = lambda i, j: i * (ny + 1) + j
    faces = [[vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)] for i in range(nx) for j in range(ny)]
    return from_arrays(np.arange(len(faces) + 1) * 4, np.array(faces).reshape(-1), V)


def fan_disk(n=7) -> Mesh:
    """Open triangle fan around a centre vertex plus one quad: polygon level with a boundary."""
    a = np.linspace(0, 2 * np.pi, n + 1)[:-1]
    V = np.concatenate([[[0, 0, 0.3]], np.stack([np.cos(a), np.sin(a), 0 * a], 1), [[2.0, 0.5, 0.0]]]).astype(np.float32)
    faces = [[0, 1 + k, 1 + (k + 1) % n] for k in range(n - 1)]
    faces.append([1, n + 1, 2, ])   # a triangle hanging off the rim
    ptr = np.cumsum([0] + [len(f) for f in faces])
    return from_arrays(ptr, np.concatenate(faces), V)


def small_set():
    """(name, mesh, levels) cases for exact parity checks."""
    return [
        ("cube", cube(), 3),
        ("cube_quadtype", cube_quad_type(), 2),
        ("tetra", tetrahedron(), 3),
        ("prism", pentagon_prism(), 3),
        ("grid", open_grid(), 3),
        ("fan", fan_disk(), 3),
        ("torus6x5", meshgen.torus(6, 5, seed=3), 3),
        ("ico2", meshgen.icosphere(2, 0.02, seed=4), 3),
        ("mixed12", meshgen.mixed_torus(12, 10, 0.1, 0.06, 0.005, seed=5), 3),
        ("cyl8x4", meshgen.capped_cylinder(8, 4, 0.001, seed=6), 3),
    ]


def closed(mesh) -> bool:
    ptr = mesh.ptr if mesh.ptr is not None else np.arange(mesh.nfaces + 1) * 4
    orders = np.diff(ptr)
    start = np.repeat(ptr[:-1], orders)
    end = np.repeat(ptr[1:], orders)
    c = np.arange(mesh.nnz)
    nxt = np.where(c + 1 < end, c + 1, start)
    a, b = mesh.ids.astype(np.int64), mesh.ids[nxt].astype(np.int64)
    return bool(np.isin(a * mesh.nverts + b, b * mesh.nverts + a).all())


def cut_mesh(mesh, keep_face) -> Mesh:
    """The faces of `mesh` where keep_face[f] is true, unused vertices dropped:
    an open mesh (boundaries where faces were removed)."""
    ptr = mesh.ptr if mesh.ptr is not None else np.arange(mesh.nfaces + 1, dtype=np.int64) * 4
    keep = np.flatnonzero(keep_face)
    orders = np.diff(ptr)[keep]
    corners = np.concatenate([np.arange(ptr[f], ptr[f + 1]) for f in keep])
    ids = mesh.ids[corners].astype(np.int64)
    used = np.unique(ids)
    remap = np.full(mesh.nverts, -1, np.int64)
    remap[used] = np.arange(used.size)
    nptr = np.concatenate([[0], np.cumsum(orders)])
    return from_arrays(nptr, remap[ids], np.asarray(mesh.verts, np.float32)[used, :3])


def open_mixed(W=64, H=48, seed=5) -> Mesh:
    """The mixed-polygon torus with a sector around the major axis removed:
    polygons of 3-8 sides and two boundary loops."""
    m = meshgen.mixed_torus(W, H, 0.05, 0.03, 0.005, seed=seed)
    ptr = m.ptr
    cx = np.add.reduceat(np.asarray(m.verts, np.float64)[m.ids, 0], ptr[:-1]) / np.diff(ptr)
    cy = np.add.reduceat(np.asarray(m.verts, np.float64)[m.ids, 1], ptr[:-1]) / np.diff(ptr)
    ang = np.arctan2(cy, cx)
    return cut_mesh(m, ~((ang > 0.0) & (ang < 1.2)))


def bowtie(n=4) -> Mesh:
    """Two open n x n grids sharing one corner vertex: a boundary vertex with
    two boundary loops through it (two out- and two in-boundary half-edges)."""
    a = open_grid(n, n)
    va = np.asarray(a.verts, np.float32)[:, :3]
    shared = n * (n + 1) + n                   # corner (n, n) of grid a
    vb = va + np.array([n, n, 0.5], np.float32)
    # grid b's corner (0, 0) (vertex 0) is grid a's corner (n, n)
    remap = np.arange(va.shape[0]) + va.shape[0] - 1
    remap[0] = shared
    ids = np.concatenate([a.ids, remap[a.ids]])
    verts = np.concatenate([va, vb[1:]])
    return from_arrays(np.arange(2 * a.nfaces + 1) * 4, ids, verts)
