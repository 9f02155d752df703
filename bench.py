"""Benchmark: refined faces/s of Catmull-Clark subdivision on one B200.

Default workload: the 512x512 mixed-polygon torus (262,144 faces, 5% of face
pairs merged, 3% of quads split), SLAK scheme, 4 levels (~67 M output quads).
One step = one full multi-level subdivision of that mesh.

  value   device time of a plan execution (CUDA graph replay), input and
          output resident in HBM, L2 flushed (256 MiB write) before every step
  e2e     the C-ABI call a user makes with host buffers: H2D of the input from
          pinned memory, slak_subdivide, D2H of the refined ids and positions
  roofline  dominant kernel: algorithmic bytes / its CUDA-event duration
  cpu_baseline  the CPU restatement (oracle) on a bounded sample, OpenMP
  secondary the other configurations, timed the same way: the large mesh in
          the other scheme, the capped cylinder (7 levels, both schemes), the
          32x32 torus and the icosphere
  batched the 2,000-mesh batch as one CUDA graph beside the per-mesh loop of
          plans and the per-mesh loop of slak_subdivide
  batched_small  2,000 small meshes, grouped launches against chains
          (--no-extras skips secondary, batched and batched_small)

--impl reference times the reference's own CUDA path (GPUPeople/SLAK compiled
from its sources for sm_100a, oracle/_ref) on the same workload.
Multi-GPU: replicas only (each rank subdivides its own copy, no collective on
the data path); value = all ranks' refined faces / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

HBM_FALLBACK_GBS = 6650.0

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per unit of work of a
# kernel, from one single-pass ncu capture of the bench workload itself
# (profiles/k_g1_k_g3_last_level_mixed512_slak.txt: k_g1 of the last level,
# SLAK, per quad of the level it refines, this build); times the units of the
# bench's launch.
TRAFFIC_PER_UNIT = {("k_g1", "slak", "last"): 174.88}
# B200 HBM3e datasheet bandwidth (DGX figure), reported beside the measured peak
HBM_NOMINAL_GBS = 8000.0


def _peaks():
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """SM clock and clock-event (throttle) samples while the timed region runs.

    Reads NVML directly every 2 ms (the device found by its UUID, so
    CUDA_VISIBLE_DEVICES does not matter), which gives tens of samples even in
    a region of ~12 ms; without NVML it falls back to nvidia-smi every 200 ms.
    Only reads: nothing here changes a GPU setting."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int):
        self.index = index
        self.rows = []          # (sm MHz, max sm MHz, set of reason names)
        self.source = None
        self._stop = threading.Event()
        self._t = None
        self._nvml = None
        self._handle = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(index).uuid)
            self._handle = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            self._nvml = pynvml
            self._bits = [pynvml.nvmlClocksEventReasonHwSlowdown, pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                          pynvml.nvmlClocksEventReasonSwThermalSlowdown, pynvml.nvmlClocksEventReasonSwPowerCap]
        except Exception:
            self._nvml = None

    def _run_nvml(self):
        n, h = self._nvml, self._handle
        mx = float(n.nvmlDeviceGetMaxClockInfo(h, n.NVML_CLOCK_SM))
        while not self._stop.is_set():
            try:
                sm = float(n.nvmlDeviceGetClockInfo(h, n.NVML_CLOCK_SM))
                r = n.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((sm, mx, {self.NAMES[i] for i, bit in enumerate(self._bits) if r & bit}))
            except Exception:
                pass
            self._stop.wait(0.002)

    def _run_smi(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    r = [x.strip() for x in out.split(",")]
                    if r[1].replace(".", "").isdigit() and r[2].replace(".", "").isdigit():
                        self.rows.append((float(r[1]), float(r[2]),
                                          {self.NAMES[i] for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"}))
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self.source = "nvml" if self._nvml is not None else "nvidia-smi"
        self._t = threading.Thread(target=self._run_nvml if self._nvml is not None else self._run_smi, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0, "source": self.source}
        sm = [r[0] for r in self.rows]
        return {"sm_mhz": statistics.median(sm), "sm_min_mhz": min(sm), "sm_max_mhz": max(r[1] for r in self.rows),
                "reasons": sorted(set().union(*[r[2] for r in self.rows])), "samples": len(self.rows),
                "source": self.source}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        return dist, dist.get_rank(), ws
    return None, 0, 1


def _max_over_ranks(dist, x: float) -> float:
    if dist is None:
        return x
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(dist):
    if dist is not None:
        dist.barrier()


def _workload(name):
    from slak_b200 import meshgen
    w = meshgen.workload(name)
    return w.mesh, w.levels


def _config(args, mesh, levels, faces, ws, creases=None):
    """The `config` object of the JSON line, the same dict in both arms."""
    return {"workload": f"{args.workload}: {mesh.nfaces} faces, {mesh.nverts} verts, {args.scheme.upper()}, "
                        f"{levels} levels -> {faces} quads", "scheme": args.scheme.upper(),
            "levels": levels, "refined_faces": faces, "l2": "flushed (256 MiB write) before every step",
            "parallelism": f"replicas x{ws}",
            **({"creases": f"{creases[1].size} crease edges ({args.crease_frac:g} of the edges), "
                           f"sharpness in {{0.5, 1, 2, 3, 5}}"} if creases is not None else {})}


def _spread(ms):
    return {"min": min(ms), "median": statistics.median(ms), "max": max(ms), "steps": len(ms)}


def cpu_baseline(mesh, levels, scheme, budget_s=20.0, single_budget_s=10.0, creases=None):
    """The oracle (CPU restatement, OpenMP) on the largest prefix of levels that
    fits the budget; refined faces of that sample per second.  A single-thread
    figure of the same restatement rides along under "single_thread".  With
    creases, the oracle levels plus the numpy crease restatement."""
    import oracle
    from oracle import creases as oc

    def run(lv):
        if creases is None:
            return oracle.subdivide(mesh, lv, scheme)
        return oc.subdivide_creased(mesh, lv, scheme, *creases)

    best = None
    for lv in range(1, levels + 1):
        t0 = time.perf_counter()
        r = run(lv)
        dt = time.perf_counter() - t0
        best = (lv, r.nfaces, dt)
        if dt * 4.5 > budget_s:
            break
    lv, faces, dt = best
    out = {"value": faces / dt, "unit": "refined_faces/s", "cores": oracle.num_threads(), "kind": "port",
           "sample": f"{lv} of {levels} levels of the same mesh ({faces} refined faces) in {dt:.2f} s"}
    if single_budget_s > 0:
        # the same restatement on one thread, on the prefix that fits its own budget
        oracle.set_threads(1)
        try:
            one = None
            for l1 in range(1, levels + 1):
                t0 = time.perf_counter()
                r = run(l1)
                d1 = time.perf_counter() - t0
                one = (l1, r.nfaces, d1)
                if d1 * 4.5 > single_budget_s:
                    break
        finally:
            oracle.set_threads(0)
        l1, f1, d1 = one
        out["single_thread"] = {"value": f1 / d1, "unit": "refined_faces/s", "cores": 1,
                                "sample": f"{l1} of {levels} levels ({f1} refined faces) in {d1:.2f} s"}
    return out


def _creases(mesh, frac, seed=11):
    """A seeded fraction of the mesh's edges as creases, sharpness drawn from
    {0.5, 1, 2, 3, 5} (live for up to five levels); None when frac <= 0."""
    if frac <= 0:
        return None
    ptr = mesh.ptr if mesh.ptr is not None else np.arange(mesh.nfaces + 1) * 4
    ids = np.asarray(mesh.ids, np.int64)
    c = np.arange(ids.size)
    face = np.repeat(np.arange(len(ptr) - 1), np.diff(ptr))
    nxt = np.where(c + 1 == np.asarray(ptr)[face + 1], np.asarray(ptr)[face], c + 1)
    e = np.unique(np.sort(np.stack([ids, ids[nxt]], 1), 1), axis=0)
    rng = np.random.default_rng(seed)
    pick = e[rng.random(e.shape[0]) < frac].astype(np.int32)
    sharp = rng.choice(np.array([0.5, 1.0, 2.0, 3.0, 5.0], np.float32), pick.shape[0])
    return pick, sharp


def run_ours(args, dist, rank, ws):
    import torch
    from slak_b200 import api
    from slak_b200.mesh import LAK, SLAK

    mesh, levels = _workload(args.workload)
    scheme = SLAK if args.scheme == "slak" else LAK
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dev = torch.cuda.current_device()
    stream = torch.cuda.Stream()
    dm = api.DeviceMesh.from_host(mesh)
    flags = api._abi.PLAN_GRAPH | (0 if args.no_tune else api._abi.PLAN_AUTOTUNE)
    creases = _creases(mesh, args.crease_frac)
    with torch.cuda.stream(stream):
        plan = api.Plan(dm, levels, scheme, flags, stream=stream, creases=creases)   # tuning runs here, untimed
    stats = plan.level_stats()
    tuning = []
    for t in plan.tuning():
        if t["state"] < 0:
            continue
        row = {"level": t["level"], "key": t["key"], "block": t["block"], "state": t["state"]}
        if t["state"] == 1:    # measured now: each kernel's ms at its choice and at the default 256
            row["ms_chosen"] = [t["ms"][k][(128, 256, 512).index(t["block"][k])] for k in range(3)]
            row["ms_block256"] = [t["ms"][k][1] for k in range(3)]
        tuning.append(row)
    faces = stats[-1]["out_faces"]
    alg_bytes = sum(s["algorithmic_bytes"] for s in stats)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            plan.execute(stream)
        plan.check(stream)
        torch.cuda.synchronize()
        _barrier(dist)
        with ClockSampler(dev) as clk:
            for i in range(args.steps):
                flush.fill_(float(i))          # L2 flush outside the timed events
                ev[i][0].record(stream)
                plan.execute(stream)
                ev[i][1].record(stream)
            torch.cuda.synchronize()
        _barrier(dist)
        st = plan.check(stream)
    ms = [a.elapsed_time(b) for a, b in ev]
    spread = _spread(ms)
    ms_step = _max_over_ranks(dist, statistics.mean(ms))
    value = faces * ws / (ms_step * 1e-3)
    launches = plan.launches * args.steps

    # dominant kernel: per-kernel events of instrumented eager executions
    kern, ktable = plan_kernel_profile(dm, levels, scheme, args.steps, stream, torch, flush, creases)
    tpu = TRAFFIC_PER_UNIT.get((kern["kernel"], args.scheme, "last" if kern["level"] == levels - 1 else "mid"))
    if tpu is not None:
        units = stats[kern["level"]]["nfaces"]
        kern["traffic"] = tpu * units
        kern["traffic_note"] = (f"{tpu} B per quad refined (ncu, one pass, mixed512 capture) x {units} quads; "
                                f"{tpu * units / kern['algorithmic_bytes_per_launch']:.2f}x the algorithmic bytes")

    # ms per level: the per-kernel event times summed by level, with the level's
    # compulsory bytes against the measured peak
    peak, _ = _peaks()
    per_level = []
    for lv in range(levels):
        ms_l = sum(t["ms"] for t in ktable if t["level"] == lv)
        b = stats[lv]["algorithmic_bytes"]
        per_level.append({"level": lv, "out_faces": stats[lv]["out_faces"], "ms": ms_l, "algorithmic_bytes": b,
                          "GB/s": b / (ms_l * 1e-3) / 1e9 if ms_l > 0 else None,
                          "frac": (b / (ms_l * 1e-3) / 1e9) / peak if ms_l > 0 else None})

    # e2e: host buffers, the C-ABI drop-in call
    e2e = run_e2e(mesh, levels, scheme, args, torch, dist, ws, creases)

    peak, peak_kind = _peaks()
    achieved = alg_bytes / (ms_step * 1e-3) / 1e9
    out = {
        "metric": "refined_faces_per_s", "value": value, "unit": "refined_faces/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
        "config": _config(args, mesh, levels, faces, ws, creases),
        "gpu_launches": launches,
        "ms_per_step_spread": spread,
        "roofline": kern,
        "kernels": ktable[:8],
        "levels": per_level,
        "tuning": tuning,
        "pipeline_roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                              "frac": achieved / peak, "peak_kind": peak_kind,
                              "frac_of_nominal": achieved / HBM_NOMINAL_GBS,
                              "algorithmic_bytes": alg_bytes},
        "e2e": e2e,
        "clocks": clk.summary(),
    }
    if rank == 0 and ws == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(mesh, levels, scheme, args.cpu_budget, creases=creases)
    plan.close()
    if ws == 1 and not args.no_extras and creases is None:
        # the survey's other configurations, then the batched form beside the
        # per-mesh loops (its outputs, 136 GB, need the memory the plan held)
        out["secondary"] = secondary_configs(args, torch, stream, flush)
        del flush
        torch.cuda.empty_cache()
        b = run_batch(args, torch, dist, rank, ws)
        b.pop("clocks", None)
        out["batched"] = b
        out["batched_small"] = run_small_batch(args, torch)
    return out


def run_small_batch(args, torch, count=2000, fmax=2000):
    """A batch of many small meshes (faces log-uniform in [100, fmax], levels
    1-4), where launches rather than bytes bound the time: grouped launches
    (the default) against every mesh in chains (SLAK_BATCH_GROUP_QUADS=0), one
    CUDA graph each, median device time of 7 executions."""
    from slak_b200 import _abi, api, meshgen
    from slak_b200.mesh import LAK, SLAK
    scheme = SLAK if args.scheme == "slak" else LAK
    items = [(meshgen.batch_mesh(it), it.levels) for it in meshgen.batch_specs(count, seed=5, fmin=100, fmax=fmax)]
    if scheme == LAK:
        items = [(m if m.ptr is not None else m.with_quad_ptr(), l) for m, l in items]
    dms = [api.DeviceMesh.from_host(m) for m, _ in items]
    stream = torch.cuda.Stream()
    res = {"meshes": count, "faces": f"log-uniform in [100, {fmax}]", "levels": "uniform in 1..4"}
    saved = os.environ.get("SLAK_BATCH_GROUP_QUADS")
    try:
        for name, gq in (("grouped", saved), ("chains", "0")):
            if gq is None:
                os.environ.pop("SLAK_BATCH_GROUP_QUADS", None)
            else:
                os.environ["SLAK_BATCH_GROUP_QUADS"] = gq
            with torch.cuda.stream(stream):
                b = api.Batch(dms, [l for _, l in items], scheme, _abi.PLAN_GRAPH, stream=stream)
                for _ in range(3):
                    b.execute(stream)
                b.check(stream)
                ms = []
                for _ in range(7):
                    a = torch.cuda.Event(enable_timing=True)
                    c = torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                    b.execute(stream)
                    c.record(stream)
                    c.synchronize()
                    ms.append(a.elapsed_time(c))
                b.check(stream)
                res[f"{name}_ms"] = statistics.median(ms)
                res[f"{name}_launches"] = b.launches
                res[f"{name}_groups"] = b.groups
                b.close()
    finally:
        if saved is None:
            os.environ.pop("SLAK_BATCH_GROUP_QUADS", None)
        else:
            os.environ["SLAK_BATCH_GROUP_QUADS"] = saved
    res["refined_faces"] = int(sum(m.nnz * 4 ** (l - 1) for m, l in items))
    res["speedup_grouped_vs_chains"] = res["chains_ms"] / res["grouped_ms"]
    return res


def plan_time(mesh, levels, scheme, steps, warmup, stream, torch, flush):
    """Device time of one plan execution (CUDA-graph replay, L2 flushed before
    each step, autotuned launch shapes), with the pipeline's compulsory bytes
    against the measured peak: the secondary configurations of the line."""
    from slak_b200 import api
    peak, _ = _peaks()
    dm = api.DeviceMesh.from_host(mesh)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    with torch.cuda.stream(stream):
        plan = api.Plan(dm, levels, scheme, api._abi.PLAN_GRAPH | api._abi.PLAN_AUTOTUNE, stream=stream)
        for _ in range(warmup):
            plan.execute(stream)
        plan.check(stream)
        for i in range(steps):
            flush.fill_(float(i))
            ev[i][0].record(stream)
            plan.execute(stream)
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        plan.check(stream)
        stats = plan.level_stats()
        launches = plan.launches
        plan.close()
    ms = [a.elapsed_time(b) for a, b in ev]
    t = statistics.mean(ms)
    faces = stats[-1]["out_faces"]
    alg = sum(x["algorithmic_bytes"] for x in stats)
    return {"refined_faces": faces, "ms_per_step": t, "value": faces / (t * 1e-3), "unit": "refined_faces/s",
            "ms_per_step_spread": _spread(ms), "launches_per_step": launches,
            "pipeline_roofline": {"achieved": alg / (t * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                                  "frac": alg / (t * 1e-3) / 1e9 / peak, "algorithmic_bytes": alg}}


def secondary_configs(args, torch, stream, flush):
    """The other configurations the survey names, measured the same way as the
    headline (device time, graph replay): the large mixed mesh under LAK, the
    capped cylinder (valence-64 poles) at 7 levels in both schemes, and the
    small configurations (torus 32x32 SLAK 3 levels, icosphere 4 levels)."""
    from slak_b200 import meshgen
    from slak_b200.mesh import LAK, SLAK
    out = {}
    other = "lak" if args.scheme == "slak" else "slak"
    m, lv = _workload(args.workload)
    if other == "lak" and m.ptr is None:
        m = m.with_quad_ptr()
    out[f"{args.workload}_{other}"] = plan_time(m, lv, LAK if other == "lak" else SLAK, args.steps, args.warmup,
                                                 stream, torch, flush)
    for name, schemes in (("cylinder", ("slak", "lak")), ("torus32", ("slak",)), ("icosphere", ("slak", "lak"))):
        w = meshgen.workload(name)
        for sc in schemes:
            mm = w.mesh if sc == "slak" or w.mesh.ptr is not None else w.mesh.with_quad_ptr()
            r = plan_time(mm, w.levels, LAK if sc == "lak" else SLAK, args.steps, args.warmup, stream, torch, flush)
            r["config"] = f"{name}: {w.mesh.nfaces} faces, {sc.upper()}, {w.levels} levels"
            out[f"{name}_{sc}"] = r
    return out


def plan_kernel_profile(dm, levels, scheme, steps, stream, torch, flush, creases=None):
    """Per-kernel device times from CUDA events recorded after every launch of an
    eager execution (SLAK_PLAN_TIMING), averaged over `steps` timed executions
    with the L2 flushed before each; returns the dominant kernel's roofline and
    the per-kernel table."""
    from slak_b200 import api
    peak, peak_kind = _peaks()
    with torch.cuda.stream(stream):
        plan = api.Plan(dm, levels, scheme, api._abi.PLAN_TIMING, stream=stream, creases=creases)
        plan.execute(stream)
        plan.check(stream)
        acc = {}
        for i in range(steps):
            flush.fill_(float(i))
            plan.execute(stream)
            for t in plan.kernel_timings():
                key = (t["name"], t["level"])
                a = acc.setdefault(key, [0.0, 0, t["algorithmic_bytes"]])
                a[0] += t["ms"]
                a[1] += 1
        plan.check(stream)
        plan.close()
    table = []
    for (name, level), (ms, cnt, b) in acc.items():
        avg = ms / cnt
        table.append({"kernel": name, "level": level, "ms": avg, "algorithmic_bytes": b,
                      "GB/s": (b / (avg * 1e-3) / 1e9) if b and avg > 0 else None})
    total = sum(t["ms"] for t in table)
    for t in table:
        t["share"] = t["ms"] / total if total else None
    dom = max(table, key=lambda t: t["ms"])
    achieved = dom["GB/s"] or 0.0
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "frac_of_nominal": achieved / HBM_NOMINAL_GBS, "traffic": None,
            "kernel": dom["kernel"], "level": dom["level"],
            "kernel_ms": dom["ms"], "kernel_share": dom["share"], "peak_kind": f"{peak_kind} (copy bandwidth)",
            "algorithmic_bytes_per_launch": dom["algorithmic_bytes"]}
    return roof, sorted(table, key=lambda t: -t["ms"])


def run_e2e(mesh, levels, scheme, args, torch, dist, ws, creases=None):
    import ctypes
    from slak_b200 import _abi, api
    lib = _abi.lib()
    # pinned host input and output buffers
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    h_ptr = pin(mesh.ptr) if mesh.ptr is not None else None
    h_ids, h_vals = pin(mesh.ids), pin(mesh.vals) if mesh.vals is not None else None
    h_verts = pin(mesh.verts.reshape(-1))
    d_ptr = torch.empty_like(h_ptr, device="cuda") if h_ptr is not None else None
    d_ids = torch.empty_like(h_ids, device="cuda")
    d_vals = torch.empty_like(h_vals, device="cuda") if h_vals is not None else None
    d_verts = torch.empty_like(h_verts, device="cuda")
    cm = api.DeviceMesh(mesh.type, mesh.nfaces, mesh.nverts, mesh.nnz, mesh.max_face_order, mesh.is_reduced,
                        d_ptr, d_ids, d_vals, d_verts)
    cin = cm.as_c()
    stream = torch.cuda.current_stream()
    sh = int(stream.cuda_stream) or None
    out_ids = out_verts = None
    times = []
    h_cp = pin(creases[0].reshape(-1)) if creases is not None else None
    h_cs = pin(creases[1]) if creases is not None else None
    d_cp = torch.empty_like(h_cp, device="cuda") if h_cp is not None else None
    d_cs = torch.empty_like(h_cs, device="cuda") if h_cs is not None else None
    h2d = sum(t.numel() * t.element_size() for t in (h_ptr, h_ids, h_vals, h_verts, h_cp, h_cs) if t is not None)
    d2h = 0
    n = max(2, args.steps)
    for i in range(args.warmup + n):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for h, d in ((h_ptr, d_ptr), (h_ids, d_ids), (h_vals, d_vals), (h_verts, d_verts), (h_cp, d_cp),
                     (h_cs, d_cs)):
            if h is not None:
                d.copy_(h, non_blocking=True)
        cout = _abi.SlakMesh()
        if creases is None:
            rc = lib.slak_subdivide(ctypes.byref(cin), ctypes.byref(cout), levels, scheme, sh)
        else:
            rc = lib.slak_subdivide_creased(ctypes.byref(cin), ctypes.byref(cout), levels, scheme, d_cp.data_ptr(),
                                            d_cs.data_ptr(), int(h_cs.numel()), sh)
        _abi.check(rc, "slak_subdivide")
        if out_ids is None:
            out_ids = torch.empty(cout.nnz, dtype=torch.int32).pin_memory()
            out_verts = torch.empty(4 * cout.nverts, dtype=torch.float32).pin_memory()
            d2h = out_ids.numel() * 4 + out_verts.numel() * 4
        out_ids.copy_(api.device_view(cout.ids, (cout.nnz,), "<i4"), non_blocking=True)
        out_verts.copy_(api.device_view(cout.verts, (4 * cout.nverts,), "<f4"), non_blocking=True)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        faces = cout.nfaces
        lib.slak_mesh_free(ctypes.byref(cout))       # outside the bracket, as for the reference arm
        if i >= args.warmup:
            times.append(dt)
    t = _max_over_ranks(dist, statistics.mean(times))
    tm = _max_over_ranks(dist, statistics.median(times))
    return {"value": faces * ws / t, "unit": "refined_faces/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": t * 1e3,
            "value_median": faces * ws / tm, "ms_per_step_median": tm * 1e3,
            "ms_spread": _spread([x * 1e3 for x in times])}


def batch_shard(count, rank=0, ws=1):
    """Specs of this rank's meshes of the 2,000-mesh batch (seeded kinds, sizes
    and level counts), in batch order: the library's partition
    (slak_b200.shard) by predicted output, faces x 4^(levels-1), so the specs
    are split before any geometry is generated."""
    from slak_b200 import meshgen, shard
    specs = meshgen.batch_specs(count)
    if ws == 1:
        return specs
    work = [it.faces * 4 ** (it.levels - 1) for it in specs]
    return [specs[k] for k in shard.shard_indices(work, rank, ws)]


def batch_workload(count, rank=0, ws=1):
    from slak_b200 import meshgen
    return [(meshgen.batch_mesh(it), it.levels) for it in batch_shard(count, rank, ws)]


def run_batch(args, torch, dist, rank, ws):
    """Batched form vs the plain per-mesh loop on the same meshes.

    plain   one slak_subdivide per mesh (the drop-in call, as a caller of the
            reference loops over meshes), outputs freed after each call;
            device-resident inputs; one CUDA-event bracket around the loop
    batched one slak_batch_* object for all meshes, executed as one CUDA graph
            (SLAK_PLAN_GRAPH); the inputs (1.7 GB) exceed L2, so no flush
    """
    import ctypes
    from slak_b200 import _abi, api
    from slak_b200.mesh import LAK, SLAK
    scheme = SLAK if args.scheme == "slak" else LAK
    t0 = time.perf_counter()
    items = batch_workload(args.batch_count, rank, ws)
    if scheme == LAK:
        items = [(m if m.ptr is not None else m.with_quad_ptr(), l) for m, l in items]
    gen_s = time.perf_counter() - t0
    dms = [api.DeviceMesh.from_host(m) for m, _ in items]
    stream = torch.cuda.Stream()
    lib = _abi.lib()
    sh = int(stream.cuda_stream)
    cins = [d.as_c() for d in dms]

    def plain_loop(count=None):
        faces = 0
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(stream)
        for cin, (_, lv) in list(zip(cins, items))[:count]:
            cout = _abi.SlakMesh()
            _abi.check(lib.slak_subdivide(ctypes.byref(cin), ctypes.byref(cout), lv, scheme, sh), "slak_subdivide")
            faces += cout.nfaces
            lib.slak_mesh_free(ctypes.byref(cout))
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b), faces

    def plan_loop():
        # the same per-mesh loop with each mesh's plan created (and its memory
        # allocated) outside the bracket: device time of the executions alone
        total = 0.0
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for d, (_, lv) in zip(dms, items):
            p = api.Plan(d, lv, scheme, 0, stream=stream)
            a.record(stream)
            p.execute(stream)
            b.record(stream)
            b.synchronize()
            total += a.elapsed_time(b)
            p.check(stream)
            p.close()
        return total

    with torch.cuda.stream(stream):
        plain_loop(50)                                    # warm-up
        plain = [plain_loop() for _ in range(max(1, args.batch_plain_reps))]
        plan_ms = plan_loop()
    plain_ms = _max_over_ranks(dist, statistics.mean(p[0] for p in plain))
    plan_ms = _max_over_ranks(dist, plan_ms)
    faces = plain[0][1]

    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        b = api.Batch(dms, [l for _, l in items], scheme,
                      api._abi.PLAN_GRAPH | (0 if args.no_tune else api._abi.PLAN_AUTOTUNE), stream=stream)
    create_s = time.perf_counter() - t0
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    dev = torch.cuda.current_device()
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            b.execute(stream)
        b.check(stream)
        torch.cuda.synchronize()
        _barrier(dist)
        with ClockSampler(dev) as clk:
            for i in range(args.steps):
                ev[i][0].record(stream)
                b.execute(stream)
                ev[i][1].record(stream)
            torch.cuda.synchronize()
        b.check(stream)
    batch_ms = _max_over_ranks(dist, statistics.mean(a.elapsed_time(c) for a, c in ev))
    out = {"meshes": len(items) * ws, "refined_faces": faces * ws,
           "plain_ms": plain_ms, "plain_value": faces * ws / (plain_ms * 1e-3),
           "batched_ms": batch_ms, "batched_value": faces * ws / (batch_ms * 1e-3),
           "speedup": plain_ms / batch_ms, "unit": "refined_faces/s",
           "plan_loop_ms": plan_ms, "plan_loop_value": faces * ws / (plan_ms * 1e-3),
           "speedup_vs_plan_loop": plan_ms / batch_ms,
           "waves": b.waves, "groups": b.groups, "launches_per_execution": b.launches,
           "create_s": create_s, "generate_s": gen_s, "clocks": clk.summary(),
           "plain": "slak_subdivide per mesh (allocates and frees its output per call)",
           "plan_loop": "per mesh: plan created untimed, one eager execution timed with CUDA events",
           "batched": "slak_batch, one CUDA graph per execution"}
    b.close()                                            # its outputs go before the one-call form's arrive

    # the one-call form (slak_subdivide_batched): creation, per-mesh output
    # allocations and one eager execution, wall clock like the plain loop's bracket
    n = len(cins)
    arr = (_abi.SlakMesh * n)(*cins)
    lvs = (ctypes.c_int * n)(*[l for _, l in items])
    res = (_abi.SlakMesh * n)()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _abi.check(lib.slak_subdivide_batched(arr, lvs, n, scheme, res, sh), "slak_subdivide_batched")
    torch.cuda.synchronize()
    one_ms = _max_over_ranks(dist, (time.perf_counter() - t0) * 1e3)
    for i in range(n):
        lib.slak_mesh_free(ctypes.byref(res[i]))     # elements share the array's memory
    out.update({"one_call_ms": one_ms, "one_call_value": faces * ws / (one_ms * 1e-3),
                "speedup_one_call_vs_plain": plain_ms / one_ms,
                "one_call": "slak_subdivide_batched: batch creation, per-mesh cudaMalloc of the outputs, one eager "
                            "execution (wall clock)"})
    return out


def run_batch_line(args, dist, rank, ws):
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    r = run_batch(args, torch, dist, rank, ws)
    peak, peak_kind = _peaks()
    return {
        "metric": "refined_faces_per_s", "value": r["batched_value"], "unit": "refined_faces/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["batched_ms"], "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
        "config": {"workload": f"batch{args.batch_count}: {r['meshes']} meshes, {args.scheme.upper()}, "
                               f"levels 1-4 -> {r['refined_faces']} quads",
                   "l2": "inputs 1.7 GB > L2", "parallelism": f"meshes split over {ws} ranks"},
        "gpu_launches": r["launches_per_execution"] * args.steps,
        "batched": r, "clocks": r["clocks"],
    }


def run_reference_batch(args, scheme):
    """The reference's per-mesh loop (one subdivideIteratively per mesh, as its
    config-file loop runs) over the batch's meshes in order, until the time
    budget is spent: a bounded sample of the 2,000-mesh workload."""
    from oracle import ref
    from slak_b200.mesh import LAK
    import torch
    items = batch_workload(args.batch_count)
    if scheme == LAK:
        items = [(m if m.ptr is not None else m.with_quad_ptr(), l) for m, l in items]
    ref.time(items[0][0], items[0][1], scheme, 1, 1)           # context and module load
    dev = torch.cuda.current_device()
    done, faces, ms_total = 0, 0, 0.0
    from slak_b200 import canon
    t0 = time.perf_counter()
    with ClockSampler(dev) as clk:
        for m, lv in items:
            ms, _ = ref.time(m, lv, scheme, 0, 1)
            ms_total += ms[0]
            faces += canon.level_sizes(m, lv)[-1][2]
            done += 1
            if time.perf_counter() - t0 > args.cpu_budget * 3:
                break
    value = faces / (ms_total * 1e-3)
    sample = f"first {done} of {len(items)} meshes ({faces} refined faces), per-mesh CUDA-event time summed"
    return {
        "impl": "reference", "metric": "refined_faces_per_s", "value": value, "unit": "refined_faces/s",
        "n_gpus": 1, "steps": 1, "warmup": 1, "ms_per_step": ms_total, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
        "config": {"workload": f"batch{args.batch_count}: per-mesh loop, {'SLAK' if scheme else 'LAK'}",
                   "parallelism": "replicas x1"},
        "path": "GPUPeople/SLAK's own CUDA path, one subdivideIteratively per mesh",
        "cpu_baseline": {"value": None, "unit": "refined_faces/s", "cores": 0, "kind": "reference",
                         "unavailable": "the reference has no CPU implementation of the path; this line times "
                                        "its CUDA path", "sample": sample},
        "e2e": {"value": value, "unit": "refined_faces/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "clocks": clk.summary(),
    }


def run_reference(args, dist, rank, ws):
    from oracle import ref
    from slak_b200.mesh import LAK, SLAK
    if rank != 0:
        return None
    scheme = SLAK if args.scheme == "slak" else LAK
    if not ref.available():
        return {"impl": "reference", "unavailable": "reference library oracle/_ref/libslak_ref.so not built"}
    if args.crease_frac > 0:
        return {"impl": "reference", "unavailable": "the reference does not implement creases "
                                                    "(handleCreases is commented out, CatmullClarkImpl.cu:94-96)"}
    if args.workload == "batch2000":
        return run_reference_batch(args, scheme)
    mesh, levels = _workload(args.workload)
    import torch
    dev = torch.cuda.current_device()
    with ClockSampler(dev) as clk:
        ms, self_ms = ref.time(mesh, levels, scheme, args.warmup, args.steps)
    from slak_b200 import canon
    sizes = canon.level_sizes(mesh, levels)
    faces = sizes[-1][2]
    ms_step = statistics.mean(ms)
    value = faces / (ms_step * 1e-3)
    # end to end through the reference's public call with host buffers: the
    # same pinned H2D of the input and D2H of the refined ids and positions,
    # over the same number of steps, as this repository's e2e figure
    e2e_ms, h2d, d2h = ref.time_e2e(mesh, levels, scheme, 1, max(2, args.steps))
    e2e_t, e2e_med = statistics.mean(e2e_ms), statistics.median(e2e_ms)
    return {
        "impl": "reference", "metric": "refined_faces_per_s", "value": value, "unit": "refined_faces/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generator)",
        "config": _config(args, mesh, levels, faces, ws),
        "reference_self_reported_ms": statistics.mean(self_ms) if self_ms else None,
        "ms_per_step_spread": _spread(ms),
        "path": "GPUPeople/SLAK's own CUDA path (subdivideIteratively, built for sm_100a from its sources), "
                "device-resident input",
        "cpu_baseline": {"value": None, "unit": "refined_faces/s", "cores": 0, "kind": "reference",
                         "unavailable": "the reference has no CPU implementation of the path; this line times "
                                        "its CUDA path (the CPU restatement is timed in the repository's arm)",
                         "sample": "none"},
        "e2e": {"value": faces / (e2e_t * 1e-3), "unit": "refined_faces/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_t,
                "value_median": faces / (e2e_med * 1e-3), "ms_per_step_median": e2e_med,
                "ms_spread": _spread(e2e_ms)},
        "clocks": clk.summary(),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mixed512")
    ap.add_argument("--scheme", default="slak", choices=["slak", "lak"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="default launch shapes (no autotuning)")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--crease-frac", type=float, default=0.0,
                    help="refine with this seeded fraction of the edges as semi-sharp creases")
    ap.add_argument("--batch-count", type=int, default=2000)
    ap.add_argument("--batch-plain-reps", type=int, default=1)
    ap.add_argument("--no-extras", action="store_true",
                    help="headline configuration only (no secondary configurations, no batch block)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    dist, rank, ws = _dist()
    if args.impl == "reference":
        out = run_reference(args, dist, rank, ws)
    elif args.workload == "batch2000":
        out = run_batch_line(args, dist, rank, ws)
    else:
        out = run_ours(args, dist, rank, ws)
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
