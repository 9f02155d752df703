"""The autotuner: measured launch shapes are valid, the results stay
bit-exact, a second plan with the same key takes the cached choice, and the
cache round-trips through SLAK_TUNE_FILE."""
import numpy as np
import pytest

import oracle
from slak_b200 import _abi, api, meshgen
from slak_b200.mesh import LAK, SLAK

pytestmark = pytest.mark.gpu


def _run(mesh, levels, scheme, flags):
    plan = api.Plan(api.DeviceMesh.from_host(mesh), levels, scheme, flags)
    plan.execute()
    plan.check()
    out = plan.output().to_host()
    tun = plan.tuning()
    plan.close()
    return out, tun


@pytest.mark.parametrize("scheme", [SLAK, LAK])
def test_autotune_measures_then_caches(scheme, tmp_path, monkeypatch):
    _abi.lib().slak_autotune_reset()
    mesh = meshgen.mixed_torus(64, 48, 0.05, 0.03, 0.005, seed=21)
    ref = oracle.subdivide(mesh, 4, scheme)
    out, tun = _run(mesh, 4, scheme, _abi.PLAN_AUTOTUNE)
    assert np.array_equal(out.ids, ref.ids)
    assert np.array_equal(np.asarray(out.verts, np.float32).view(np.uint32), ref.verts.view(np.uint32))
    assert tun[0]["state"] == -1                      # level 0 is a general level
    fast = [t for t in tun if t["state"] >= 0]
    assert len(fast) == 3 and all(t["state"] == 1 for t in fast)
    for t in fast:
        assert all(b in (128, 256, 512) for b in t["block"])
        for k in range(3):
            if k == 1 and t["level"] >= 2:       # quad parent: k_g1 does k_g2's work, nothing to measure
                assert t["ms"][k] == [0.0, 0.0, 0.0] and t["block"][k] == 256
                continue
            assert min(t["ms"][k]) > 0
            assert t["ms"][k][(128, 256, 512).index(t["block"][k])] == min(t["ms"][k])
    # same key again: no measurement, the cached shapes
    out2, tun2 = _run(mesh, 4, scheme, _abi.PLAN_AUTOTUNE)
    assert [t["state"] for t in tun2 if t["state"] >= 0] == [2, 2, 2]
    assert [t["block"] for t in tun2] == [t["block"] for t in tun]
    assert np.array_equal(out2.ids, ref.ids)


def test_tune_file_round_trip(tmp_path, monkeypatch):
    path = tmp_path / "tune.txt"
    monkeypatch.setenv("SLAK_TUNE_FILE", str(path))
    _abi.lib().slak_autotune_reset()
    mesh = meshgen.torus(40, 30, seed=3)
    # reset marks the file as read; a fresh measurement writes it
    _, tun = _run(mesh, 3, SLAK, _abi.PLAN_AUTOTUNE)
    lines = path.read_text().split("\n")
    keys = {t["key"] for t in tun if t["state"] == 1}
    assert keys and keys <= {ln.split()[0] for ln in lines if ln}
    for ln in lines:
        if ln:
            k, *b = ln.split()
            assert all(int(x) in (128, 256, 512) for x in b)
