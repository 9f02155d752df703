"""The grandparent-quad levels (SLAK_PLAN_GQ: k_g1 sums the columns of PP's
face and edge points, k_g3 only those of PP's old vertices) against the
slot-record path (the default), the general path and the oracle: bit for bit, on levels that
write the next level's state and on last levels, in both schemes, with and
without compensated sums.  Quad inputs reach GQ at level 2 (the input is the
grandparent), polygon inputs at level 3."""
import numpy as np
import pytest

import oracle
from slak_b200 import api, meshgen
from slak_b200.mesh import LAK, SLAK

pytestmark = pytest.mark.gpu

GQ = api._abi.PLAN_GQ


def _bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


CASES = [("torus", lambda: meshgen.torus(24, 20, seed=5), 3),            # level 2 last
         ("torus4", lambda: meshgen.torus(16, 12, seed=7), 4),           # level 2 state, level 3 last
         ("mixed", lambda: meshgen.mixed_torus(40, 32, 0.05, 0.03, 0.005, seed=3), 4),
         ("cylinder", lambda: meshgen.capped_cylinder(64, 32, 0.001, seed=15), 5),
         ("ico", lambda: meshgen.icosphere(3, 0.02, seed=9), 4)]


@pytest.mark.parametrize("scheme", [SLAK, LAK])
@pytest.mark.parametrize("name,make,levels", CASES, ids=[c[0] for c in CASES])
def test_gq_levels_equal_the_record_path_and_the_oracle(name, make, levels, scheme):
    m = make()
    if scheme == LAK and m.ptr is None:
        m = m.with_quad_ptr()
    gq = api.subdivide(m, levels, scheme, GQ)
    rec = api.subdivide(m, levels, scheme)
    ref = oracle.subdivide(m, levels, scheme)
    for other in (rec, ref):
        assert np.array_equal(gq.ids, other.ids)
        assert np.array_equal(_bits(gq.verts), _bits(other.verts))
    if scheme == LAK:
        assert np.array_equal(gq.ptr, ref.ptr) and np.array_equal(gq.vals, ref.vals)


@pytest.mark.parametrize("scheme", [SLAK, LAK])
def test_gq_compensated_and_graph(scheme):
    m = meshgen.capped_cylinder(64, 32, 0.001, seed=15)
    if scheme == LAK:
        m = m.with_quad_ptr() if m.ptr is None else m
    C = api._abi.PLAN_COMPENSATED
    a = api.subdivide(m, 5, scheme, C | GQ)
    b = api.subdivide(m, 5, scheme, C)
    g = api.subdivide(m, 5, scheme, C | api._abi.PLAN_GENERAL)
    assert np.array_equal(a.ids, b.ids) and np.array_equal(_bits(a.verts), _bits(b.verts))
    assert np.array_equal(a.ids, g.ids) and np.array_equal(_bits(a.verts), _bits(g.verts))
    r = api.subdivide(m, 5, scheme, api._abi.PLAN_GRAPH | GQ)
    assert np.array_equal(_bits(r.verts), _bits(api.subdivide(m, 5, scheme).verts))


def test_gq_level_kinds_in_the_tuning_key():
    """Which levels run GQ: the tuning key of a fast level names it."""
    m = meshgen.mixed_torus(40, 32, 0.05, 0.03, 0.005, seed=3)
    dm = api.DeviceMesh.from_host(m)
    p = api.Plan(dm, 4, SLAK, GQ)
    keys = [t["key"] for t in p.tuning() if t["state"] >= 0]
    p.close()
    assert "gquad" not in keys[0] and "gquad" not in keys[1]      # levels 1, 2: polygon grandparent
    assert "/gquad/" in keys[2]                                     # level 3: PP = level 1's quads
    # the last level takes its parent's state from the grandparent's (SG), so
    # level 2 writes none
    assert "/state/" in keys[0] and "/last/" in keys[1] and "/last-sg/" in keys[2]
