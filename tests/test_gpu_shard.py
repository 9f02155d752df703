"""ShardedBatch on one GPU: the shares of two emulated ranks, each a batch of
its own (nothing waits on anything else), together give every mesh of the
whole batch, bit for bit what the one-rank batch gives."""
import numpy as np
import pytest

from slak_b200 import api, meshgen, shard
from slak_b200.mesh import LAK, SLAK

pytestmark = pytest.mark.gpu


def _meshes():
    return [meshgen.torus(24, 20, seed=1), meshgen.icosphere(3, 0.02, seed=2),
            meshgen.mixed_torus(40, 32, 0.05, 0.03, 0.005, seed=3), meshgen.capped_cylinder(16, 8, 0.001, seed=4),
            meshgen.open_grid(30, 17, seed=5), meshgen.torus(8, 6, seed=6)]


@pytest.mark.parametrize("scheme", [SLAK, LAK])
def test_two_shards_cover_the_batch(scheme):
    ms = _meshes()
    if scheme == LAK:
        ms = [m if m.ptr is not None else m.with_quad_ptr() for m in ms]
    levels = [3, 2, 2, 3, 2, 4]
    whole = shard.ShardedBatch(ms, levels, scheme, rank=0, world_size=1)
    whole.execute()
    whole.check()
    want = [whole.output(i).to_host() for i in range(len(ms))]
    got = {}
    for r in range(2):
        # meshes made on demand: only this rank's are built
        makers = [(lambda m=m: m) for m in ms]
        work = [shard.predicted_quads(m.nnz, l) for m, l in zip(ms, levels)]
        sb = shard.ShardedBatch(makers, levels, scheme, work=work, rank=r, world_size=2)
        assert sb.indices == shard.shard_indices(work, r, 2)
        sb.execute()
        sb.check()
        for i in range(len(ms)):
            o = sb.output(i)
            assert (o is None) == (i not in sb.indices)
            if o is not None:
                got[i] = o.to_host()
        sb.close()
    whole.close()
    assert sorted(got) == list(range(len(ms)))
    for i, w in enumerate(want):
        assert np.array_equal(got[i].ids, w.ids)
        assert np.array_equal(got[i].verts.view(np.uint32), w.verts.view(np.uint32))
