"""slak_b200 -- B200-native Catmull-Clark subdivision as sparse linear algebra.

The compute path is ``lib/libslak_b200.so`` (hand-written sm_100a CUDA behind
the C ABI of ``include/slak_b200.h``).  This package is its host-side mirror:
the reference's ``CatmullClark`` / ``LAKCatmullClark`` entry points, plans,
the mesh container and the seeded workload generators.
"""
from .mesh import LAK, POLY, QUAD, SLAK, TRI, Mesh  # noqa: F401

__all__ = ["Mesh", "LAK", "SLAK", "TRI", "QUAD", "POLY", "api", "meshgen", "canon", "shard"]


def __getattr__(name):
    import importlib
    if name in ("api", "meshgen", "canon", "build", "_abi", "shard"):
        return importlib.import_module(f".{name}", __name__)
    raise AttributeError(name)
