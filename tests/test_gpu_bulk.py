"""k_g3 with bulk-copied slot records (SLAK_PLAN_BULK_RECORDS): the block's
records reach shared memory by cp.async.bulk on an mbarrier.  Its results
must equal the default path's and the oracle's bit for bit; and its bounded
wait must end in SLAK_ERR_TIMEOUT, not a hang, when the poll budget is spent
(SLAK_BULK_WAIT_POLLS=0 at plan creation: the first poll is never made), with
the device still usable afterwards."""
import os

import numpy as np
import pytest

import oracle
from slak_b200 import _abi, api, meshgen
from slak_b200.mesh import LAK, SLAK

pytestmark = pytest.mark.gpu

BULK = api._abi.PLAN_BULK_RECORDS


def _bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


CASES = [("torus", lambda: meshgen.torus(40, 30, seed=5), 3),
         ("mixed", lambda: meshgen.mixed_torus(64, 48, 0.05, 0.03, 0.005, seed=8), 4),
         ("cylinder", lambda: meshgen.capped_cylinder(64, 32, 0.001, seed=15), 5),    # valence 64: warp columns
         ("ico", lambda: meshgen.icosphere(3, 0.02, seed=9), 4)]


@pytest.mark.parametrize("scheme", [SLAK, LAK])
@pytest.mark.parametrize("name,make,levels", CASES, ids=[c[0] for c in CASES])
def test_bulk_records_equal_default_and_oracle(name, make, levels, scheme):
    m = make()
    if scheme == LAK and m.ptr is None:
        m = m.with_quad_ptr()
    got = api.subdivide(m, levels, scheme, BULK)
    dflt = api.subdivide(m, levels, scheme)
    ref = oracle.subdivide(m, levels, scheme)
    for other in (dflt, ref):
        assert np.array_equal(got.ids, other.ids)
        assert np.array_equal(_bits(got.verts), _bits(other.verts))


@pytest.mark.parametrize("scheme", [SLAK, LAK])
def test_bulk_records_with_gq_and_compensated(scheme):
    m = meshgen.capped_cylinder(64, 32, 0.001, seed=15)
    if scheme == LAK and m.ptr is None:
        m = m.with_quad_ptr()
    C = api._abi.PLAN_COMPENSATED
    a = api.subdivide(m, 5, scheme, BULK | api._abi.PLAN_GQ | C)
    b = api.subdivide(m, 5, scheme, C)
    assert np.array_equal(a.ids, b.ids) and np.array_equal(_bits(a.verts), _bits(b.verts))


def test_bulk_wait_budget_spent_reports_timeout():
    m = meshgen.mixed_torus(64, 48, 0.05, 0.03, 0.005, seed=8)
    dm = api.DeviceMesh.from_host(m)
    os.environ["SLAK_BULK_WAIT_POLLS"] = "0"
    try:
        p = api.Plan(dm, 3, SLAK, BULK)
    finally:
        del os.environ["SLAK_BULK_WAIT_POLLS"]
    p.execute()
    with pytest.raises(_abi.SlakError) as e:
        p.check()
    assert e.value.code == 5                       # SLAK_ERR_TIMEOUT
    p.close()
    # the context is intact: the same plan kind with the default budget works
    got = api.subdivide(m, 3, SLAK, BULK)
    ref = oracle.subdivide(m, 3, SLAK)
    assert np.array_equal(got.ids, ref.ids) and np.array_equal(_bits(got.verts), _bits(ref.verts))
