"""Benchmark: raycastFirst on the 2M-triangle noisy torus knot, 2^24 incoherent + 4096^2 camera rays.

One step = one raycastFirst pass of the engine over both ray sets (33,554,432 rays), inputs
already resident in HBM.  `e2e` is the same work through the public API with host (pinned)
buffers: host->device copy of the rays, the kernel, device->host copy of the hits.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Under torchrun each rank runs its own copy of the workload (queries shard with the BVH
replicated: weak scaling, no collective on the data path); `value` is all ranks' rays divided
by the slowest rank's device time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mrays/s raycastFirst (2M tri)"
UNIT = "Mrays/s"
WORKLOAD = ("raycastFirst, TorusKnot(10,3,2000,500) 2,000,000 tri + N(0,0.02) normal noise (seed 1), "
            "SAH leaf 10; 2^24 incoherent rays (sphere shell r=40, uniform dirs, seed 1) + 4096x4096 "
            "pinhole camera (distance 35, 45 deg FOV), float32")
BYTES_RAY_IN, BYTES_HIT_OUT, BYTES_NODE, BYTES_TRI = 24, 32, 32, 36


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--workload",
                    choices=["first", "batched", "adjoint", "closest", "all", "build", "scene", "shapecast"],
                    default="first",
                    help="first: the headline raycastFirst line; batched: the 1024-geometry BatchedMesh form; "
                         "adjoint: forward/backward timing; closest: the 256^3 closest-point grid; all: raycast "
                         "(all hits); build: the device SAH build; scene: instanced BatchedMesh raycastFirst; "
                         "shapecast: triangles within spheres, intersectsSphere, intersectsBox")
    ap.add_argument("--grid", type=int, default=256, help="closest workload: grid resolution per axis")
    ap.add_argument("--closest-variant", type=int, default=None,
                    help="closest workload: force closestPointToPoint's kernel instead of tuning "
                         "(with --closest-tile-rows: tiled order)")
    ap.add_argument("--scene-variant", type=int, default=None,
                    help="scene workload: force the instanced kernel variant (0..2, with ray order 0) instead of "
                         "tuning")
    ap.add_argument("--closest-tile-rows", type=int, default=0,
                    help="closest workload, with --closest-variant 1: read the grid in tiles of this many "
                         "rows (2, 4, 8) of --grid points")
    ap.add_argument("--batch-meshes", type=int, default=1024)
    ap.add_argument("--tubular", type=int, default=2000)
    ap.add_argument("--radial", type=int, default=500)
    ap.add_argument("--rays-log2", type=int, default=24)
    ap.add_argument("--camera", type=int, default=4096)
    ap.add_argument("--cpu-sample", type=int, default=1 << 25, help="rays (both sets together) timed on the CPU baseline")
    ap.add_argument("--ref-sample", type=int, default=0,
                    help="rays (both sets together) per step in --impl reference; 0: the whole workload")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--headline-only", action="store_true",
                    help="first workload: skip the batched and forward/backward parts of the line")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (default traversal variant)")
    ap.add_argument("--leaf-sizes", default="0,2,4",
                    help="device leaf layouts the autotuner tries (0: the reference's leaves)")
    ap.add_argument("--leaf-size", type=int, default=None, help="force a device leaf layout")
    ap.add_argument("--traversal", default=None,
                    help="force traversal variants: 'p,o,r,occ,compact,sort' for every ray set, or "
                         "'incoherent=...;camera=...' per set")
    return ap.parse_args()


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist

        backend = "nccl" if args.impl == "engine" else "gloo"
        if backend == "nccl":
            import torch

            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return ws, rank, local


def incoherent_seed(rank: int) -> int:
    """Each rank traces its own incoherent rays (the BVH is replicated; weak scaling)."""
    return 1 + 1000 * rank


def max_over_ranks(value: float, ws: int, device=None) -> float:
    """The slowest rank's time: all-reduce MAX over the process group (identity for one rank)."""
    if ws <= 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_scaling_rate(ws: int, rays_per_rank: int, steps: int, ms: float) -> float:
    """Mrays/s of the whole job: every rank's rays over the slowest rank's time."""
    return ws * rays_per_rank * steps / (ms / 1e3) / 1e6


BUILD_OPTIONS = {"maxLeafSize": 10, "maxDepth": 40}   # with strategy SAH


def scene_inputs(pkg, args, rank):
    """The noisy knot and the two ray sets (numpy generators only: no library is loaded)."""
    geo = pkg.torus_knot(10, 3, args.tubular, args.radial, noise_sigma=0.02, noise_seed=1)
    inc = pkg.rays_incoherent(1 << args.rays_log2, seed=incoherent_seed(rank))
    cam = pkg.rays_camera(args.camera, args.camera)
    return geo, inc, cam


def scene(pkg, args, rank):
    geo, inc, cam = scene_inputs(pkg, args, rank)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH, **BUILD_OPTIONS})
    return geo, bvh, inc, cam


def headline_config(triangles, rays_per_step, ws):
    """The headline line's config, identical in the engine and reference arms."""
    return {"workload": WORKLOAD, "triangles": int(triangles), "rays_per_step": int(rays_per_step),
            "l2": "inputs larger than L2 (805 MB of rays + 1.07 GB of hits per step)",
            "parallelism": f"replicas x{ws}"}


def sample_index(n, sample, block=1 << 16):
    """Ray ids of a bounded sample of a set of n: every ray when sample >= n, else contiguous
    blocks of `block` rays spread evenly over the set (coherence within a block is kept)."""
    if sample >= n:
        return np.arange(n, dtype=np.int64)
    nb = max(1, sample // block)
    starts = np.linspace(0, n - block, nb).astype(np.int64)
    return (starts[:, None] + np.arange(block)[None, :]).reshape(-1)


class ClockSampler:
    """SM clock and clock-event reasons sampled (read-only NVML queries, every 5 ms) during the
    timed region; falls back to no record when NVML is unavailable."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.stop = threading.Event()
        self.nv = None

    def __enter__(self):
        try:
            import pynvml as nv

            nv.nvmlInit()
            self.nv = nv
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = int(vis.split(",")[self.gpu]) if vis and vis.split(",")[0].isdigit() else self.gpu
            self.h = nv.nvmlDeviceGetHandleByIndex(idx)
            self.smax = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        except Exception:
            self.nv = None
        return self

    def _run(self):
        nv = self.nv
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                pw = nv.nvmlDeviceGetPowerUsage(self.h) / 1000.0
                self.rows.append((sm, rs, pw))
            except Exception:
                pass
            time.sleep(0.005)

    def __exit__(self, *exc):
        self.stop.set()
        if self.nv is not None:
            self.t.join(timeout=2)

    def summary(self):
        if not self.rows:
            return None
        nv = self.nv
        reasons = set()
        for _, rs, _ in self.rows:
            for name, const in self.REASONS:
                if rs & getattr(nv, const, 0):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r[0] for r in self.rows), "sm_max_mhz": self.smax,
                "reasons": sorted(reasons), "samples": len(self.rows),
                "power_w_max": max(r[2] for r in self.rows)}


def parse_traversal(spec, names):
    """'1,1,32,2,1,0' (every set) or 'incoherent=1,1,32,2,1,0;camera=2,1,16,2,1,2' (per set)."""
    if "=" not in spec:
        return [[int(x) for x in spec.split(",")]] * len(names)
    per = {}
    for part in spec.split(";"):
        name, cfg = part.split("=")
        per[name.strip()] = [int(x) for x in cfg.split(",")]
    return [per.get(n) for n in names]


def traversal_kernel(cfg):
    """Name of the raycastFirst traversal kernel a variant launches."""
    p = 1 if cfg is None else cfg[0]
    if p == 2 and cfg is not None and len(cfg) > 7 and cfg[7]:
        return "raycast_first_packet4_kernel"
    return {0: "raycast_first_kernel", 1: "raycast_first_persistent_kernel", 2: "raycast_first_packet_kernel"}[p]


def kernel_launches(cfg):
    """Kernels one raycastFirst call launches with a variant (persistent, order, refill, occupancy,
    compact, sort): the traversal, the finalize pass that completes the records, the root-box
    pre-pass and the ray-ordering sort (key pass(es) + 4 radix passes of 3 kernels)."""
    cfg = list(cfg) if cfg is not None else [1, 1, 16, 0, 0, 0]
    cfg += [0] * (6 - len(cfg))
    persistent, compact, sort = cfg[0], cfg[4], cfg[5]
    if persistent == 0:
        return 2
    n = 2
    if compact or sort:
        n += 1
    if sort:
        n += (2 if sort == 1 else 1) + 12
    return n


def all_hits_launches(variant):
    """Kernels one raycast (all hits) call launches: the traversal and the finalize kernel that
    completes the stored hits, plus for the queue variants the root-box pre-pass and, when the
    queue is sorted, 3 kernels per radix pass (4 passes for the direction key, 3 for the others)."""
    if variant in (0, 1, "1t", "1t2", "1t8"):
        return 2
    v = int(variant)
    kind = {2: 1, 3: 2, 4: 3, 6: 1, 7: 2, 8: 3, 10: 1, 11: 2, 12: 3}.get(v, 0)
    return 3 + (3 * (4 if kind == 1 else 3) if kind else 0)


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_value(name, key):
    """A `key: value` figure recorded from an ncu capture in profiles/<name> (None if absent)."""
    p = ROOT / "profiles" / name
    if not p.exists():
        return None
    m = re.search(key + r":\s*([0-9.eE+-]+)", p.read_text())
    return float(m.group(1)) if m else None


def profile_traffic(name):
    """dram bytes per launch recorded from an ncu capture in profiles/<name> (None if absent)."""
    return profile_value(name, "traffic_bytes_per_launch")


def parity_module():
    """tests/parity.py: the parity bar of the engine's contract, shared with the tests."""
    if str(ROOT / "tests") not in sys.path:
        sys.path.insert(0, str(ROOT / "tests"))
    import parity

    return parity


def cpu_reference(ref, sets, got_sets, sample, threads):
    """The oracle (C++ float64 restatement of the reference path) timed on a bounded sample of
    each ray set (the whole set by default), and the engine's hits for the same rays checked
    against its results (outside the timed region; tests/parity.py's bar).  Returns rays/s over
    the sample, the reference traversal's mean node reads and triangle tests per ray (the
    algorithmic-bytes counters), the sample size and the parity counts per set."""
    par_mod = parity_module()
    stats, parity = [], {}
    total_rays, total_s = 0, 0.0
    chunk = 1 << 21
    for (name, rays), got in zip(sets, got_sets):
        idx = sample_index(rays.shape[0], sample)
        sn = st = 0
        tot = {}
        for c0 in range(0, idx.size, chunk):
            ii = idx[c0:c0 + chunk]
            sub = np.ascontiguousarray(rays[ii])
            t0 = time.perf_counter()
            exp, nn, nt = ref.raycast_first(sub, 0, 0.0, math.inf, threads=threads, counters=True)
            total_s += time.perf_counter() - t0
            sn += int(nn.sum())
            st += int(nt.sum())
            if got is not None:
                par_mod.add_counts(tot, par_mod.first_parity_chunk(ref, sub, got[ii], exp, threads=threads))
        total_rays += idx.size
        stats.append((sn / idx.size, st / idx.size))
        if got is not None:
            parity[name] = tot
    return total_rays / total_s, stats, total_rays, parity


def run_reference(args, ws, rank):
    """--impl reference: the reference path's CPU implementation on all host threads.  That is
    the oracle, a C++ float64 restatement of three-mesh-bvh's build and raycastFirst (the JS
    reference itself needs Node and three.js, neither of which is on this machine).  The BVH comes
    from the oracle's own builder (SAH, maxLeafSize 10, maxDepth 40; byte-identical to the
    engine's), and each step traces the engine arm's exact workload: both whole ray sets, in
    order.  Only rank 0 runs; it prints the line."""
    if rank != 0:
        return
    import __graft_entry__ as ge

    pkg = ge.load_package()          # numpy generators only; libbvhcuda is never loaded here
    geo, inc, cam = scene_inputs(pkg, args, 0)
    threads = os.cpu_count() or 1
    import oracle.oracle as orc

    ref = orc.OracleBVH.build(geo.position, geo.index.copy(), strategy=2, max_depth=BUILD_OPTIONS["maxDepth"],
                              target_leaf=BUILD_OPTIONS["maxLeafSize"])
    sets = [inc, cam]
    n_step = sum(r.shape[0] for r in sets)
    sample = args.ref_sample if args.ref_sample > 0 else n_step
    idx = [sample_index(r.shape[0], sample // len(sets)) for r in sets]
    chunk = 1 << 21

    def step():
        for r, ii in zip(sets, idx):
            for c0 in range(0, ii.size, chunk):
                ref.raycast_first(np.ascontiguousarray(r[ii[c0:c0 + chunk]]), threads=threads)

    for _ in range(args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    traced = sum(ii.size for ii in idx)
    rate = traced / statistics.mean(times) / 1e6
    what = ("both whole ray sets" if traced == n_step else
            f"{traced} rays (contiguous 65536-ray blocks spread over both sets)")
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * statistics.mean(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": headline_config(geo.triangle_count, n_step, 1),
            "implementation": "oracle: C++ float64 restatement of the reference's build and raycastFirst (port); "
                              "BVH from the oracle's builder",
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{what} per step, {threads} threads"},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_engine(args, ws, rank, local):
    import torch

    import __graft_entry__ as ge

    pkg = ge.load_package()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    geo, bvh, inc, cam = scene(pkg, args, rank)
    info = bvh.mesh_info()
    sets = [("incoherent", inc), ("camera", cam)]
    d_rays = [torch.from_numpy(r).to(dev) for _, r in sets]
    d_out = [torch.empty((r.shape[0], 8), dtype=torch.float32, device=dev) for _, r in sets]
    n_step = sum(r.shape[0] for _, r in sets)
    stream = torch.cuda.current_stream(dev)
    # traversal variant per ray set: forced, autotuned, or the library default
    tuned = {}
    set_configs = [None] * len(sets)
    if args.traversal:
        set_configs = parse_traversal(args.traversal, [n for n, _ in sets])
    elif not args.no_tune:
        from three_mesh_bvh_b200 import autotune

        # tuned on the whole sets: ray ordering and the warp-cooperative form depend on a set's
        # coherence at full size, which no strided or block sample reproduces; one device leaf
        # layout serves both sets
        # the camera's rays come one per pixel in row-major order: its width is the tiled order's
        # row pitch, as a renderer would pass it
        res = autotune.tune_raycast_first_sets(bvh, [(n, d) for (n, _), d in zip(sets, d_rays)],
                                               leaf_sizes=[int(x) for x in args.leaf_sizes.split(",")],
                                               tag="knot2M", tile_pitches=(args.camera,))
        tuned = {"leaf_size": res["leaf"], "total_ms_by_leaf_size": res["total_ms"],
                 **{n: {"best": e["best"], "ms": e["ms"]} for n, e in res["sets"].items()}}
        set_configs = [res["sets"][n]["best"] for n, _ in sets]
    if args.leaf_size is not None:
        bvh.set_leaf_size(args.leaf_size)

    def step(ev=None):
        for k in range(len(sets)):
            if set_configs[k] is not None:
                bvh.set_traversal(*set_configs[k])
            if ev is not None:
                ev[k][0].record(stream)
            bvh.raycast_first_batch(d_rays[k], out=d_out[k], stream=stream.cuda_stream)
            if ev is not None:
                ev[k][1].record(stream)

    for _ in range(args.warmup):
        step()
    bvh.synchronize(stream.cuda_stream)
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    kev = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in sets]
           for _ in range(args.steps)]
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        t_start.record(stream)
        for s in range(args.steps):
            step(kev[s])
        t_end.record(stream)
        torch.cuda.synchronize(dev)
    if ws > 1:
        torch.distributed.barrier()
    bvh.synchronize(stream.cuda_stream)
    ms = max_over_ranks(t_start.elapsed_time(t_end), ws, dev)
    per_set_ms = [statistics.mean(kev[s][k][0].elapsed_time(kev[s][k][1]) for s in range(args.steps))
                  for k in range(len(sets))]
    value = weak_scaling_rate(ws, n_step, args.steps, ms)

    # the timed run's hits, kept for the parity check against the oracle
    got = [np.frombuffer(d.cpu().numpy().tobytes(), dtype=pkg.HIT_DTYPE) for d in d_out]

    # e2e through the public API with pinned host buffers (copies inside the timed region)
    pinned_in = [torch.from_numpy(r).pin_memory() for _, r in sets]
    pinned_out = [torch.empty((r.shape[0] * 32,), dtype=torch.uint8).pin_memory() for _, r in sets]
    host_in = [p.numpy() for p in pinned_in]
    host_out = [p.numpy().view(pkg.HIT_DTYPE) for p in pinned_out]

    def e2e_step():
        for k in range(len(sets)):
            if set_configs[k] is not None:
                bvh.set_traversal(*set_configs[k])
            bvh.raycast_first_batch(host_in[k], out=host_out[k])

    e2e_step()
    e2e_steps = max(1, min(args.steps, 3))
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) / e2e_steps * 1e3, ws, dev)
    e2e = {"value": weak_scaling_rate(ws, n_step, 1, e2e_ms), "unit": UNIT,
           "h2d_bytes_per_step": n_step * BYTES_RAY_IN, "d2h_bytes_per_step": n_step * BYTES_HIT_OUT,
           "same_bytes_as_device_run": all(np.array_equal(h.view(np.uint8), g.view(np.uint8))
                                           for h, g in zip(host_out, got))}
    del pinned_in, pinned_out, host_in, host_out

    cpu = roof = parity = None
    if rank == 0 and not args.no_cpu_baseline:
        import oracle.oracle as orc

        threads = os.cpu_count() or 1
        ref = orc.OracleBVH.from_serialized(bvh._roots, geo.index, bvh._indirectBuffer, geo.position)
        rate, stats, nsample, per_set = cpu_reference(ref, sets, got, args.cpu_sample // 2, threads)
        cpu = {"value": rate / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": (f"{nsample} rays: both whole sets" if nsample == n_step else
                          f"{nsample} rays in contiguous 65536-ray blocks spread over both sets") + ", float64 oracle"}
        keys = parity_module().FIRST_KEYS
        parity = {"rays_checked": int(sum(r["rays"] for r in per_set.values())),
                  "mismatches": {k: int(sum(r[k] for r in per_set.values())) for k in keys},
                  "tie_exempt": int(sum(r["exempt"] for r in per_set.values())),
                  "per_set": per_set,
                  "bar": "hit/miss and faceIndex identical except rays whose two nearest reference hits are "
                         "within 1e-6 t; distance within 1e-5 relative; point and barycoord within "
                         "1e-5 max(1, |ref|)"}
        parity["ok"] = not any(parity["mismatches"].values())
        bytes_per_launch = []
        for (name, rays), (mn, mt) in zip(sets, stats):
            bytes_per_launch.append(rays.shape[0] * (BYTES_RAY_IN + BYTES_HIT_OUT + BYTES_NODE * mn + BYTES_TRI * mt))
        peak, how = measured_peak()
        # the dominant kernel: the traversal of the ray set that takes the longest
        k = max(range(len(sets)), key=lambda j: per_set_ms[j])
        achieved = bytes_per_launch[k] / (per_set_ms[k] / 1e3) / 1e9
        both = sum(bytes_per_launch) / (sum(per_set_ms) / 1e3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": profile_traffic(f"raycast_first_k2_{sets[k][0]}.md"), "peak_source": how,
                "kernel": traversal_kernel(set_configs[k]), "ray_set": sets[k][0],
                "both_sets": {"achieved": both, "frac": both / peak},
                "algorithmic_bytes_per_launch": dict(zip([n for n, _ in sets], map(float, bytes_per_launch))),
                "reference_node_reads_per_ray": [s[0] for s in stats],
                "reference_triangle_tests_per_ray": [s[1] for s in stats]}
        # the scene is L2-resident, so the HBM fraction saturates; the kernel is issue-bound, and
        # the ncu capture of the same kernel gives the figures that bound it
        prof = f"raycast_first_k2_{sets[k][0]}.md"
        roof["issue"] = {"source": f"profiles/{prof}",
                         "warp_instructions_per_ray": profile_value(prof, "warp_instructions_per_ray"),
                         "issue_slots_active": profile_value(prof, "issue_slots_active"),
                         "threads_per_instruction": profile_value(prof, "threads_per_instruction")}
        del ref
    del got
    line = None
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": headline_config(geo.triangle_count, n_step, ws),
                "mesh": {"node_records": info["node_records"], "max_depth": info["max_depth"]},
                "per_set_ms": dict(zip([n for n, _ in sets], per_set_ms)),
                "per_set_mrays_s": {n: r.shape[0] / (t / 1e3) / 1e6 for (n, r), t in zip(sets, per_set_ms)},
                "traversal": {n: (list(c) if c is not None else None) for (n, _), c in zip(sets, set_configs)},
                "leaf_size": bvh.get_leaf_size(),
                "autotune": tuned, "roofline": roof, "cpu_baseline": cpu, "parity": parity, "e2e": e2e,
                "clocks": clk.summary(),
                "gpu_launches": args.steps * sum(kernel_launches(c) for c in set_configs)}
    bvh.dispose()
    del d_rays, d_out
    torch.cuda.empty_cache()
    # the metric's other two parts, measured in the same run: the batched BatchedMesh launch
    # against per-mesh launches, and forward+backward against forward
    if not args.headline_only:
        line_b = measure_batched(args, ws, rank, local)
        torch.cuda.empty_cache()
        line_a = measure_adjoint(args, ws, rank, local)
        torch.cuda.empty_cache()
        if rank == 0:
            line["batched"] = line_b
            line["adjoint"] = line_a
    if rank == 0:
        print(json.dumps(line), flush=True)


def batched_oracle_check(batch, rays, off, got, per_geometry, threads):
    """Each geometry's hits against its own oracle (the reference's per-mesh raycast with the
    geometry's draw range, ExtensionUtilities.js:87-161,216-268): an evenly strided sample of up to
    `per_geometry` of its rays.  `got` holds faceIndex in the shared index."""
    import oracle.oracle as orc

    from three_mesh_bvh_b200.batched import shift_triangle_offsets

    par_mod = parity_module()
    tot, r0 = {}, 0
    for k in range(batch.n_meshes):
        nr = batch.roots_per_mesh[k]
        tb = int(batch.triangle_base[k])
        roots = [shift_triangle_offsets(r, (-tb) & 0xFFFFFFFF) for r in batch.roots[r0:r0 + nr]]
        r0 += nr
        g = batch.geometries[k]
        ref = orc.OracleBVH.from_serialized(roots, g.index, None, g.position)
        a, b = int(off[k]), int(off[k + 1])
        ii = np.linspace(a, b - 1, min(per_geometry, b - a)).astype(np.int64)
        sub = np.ascontiguousarray(rays[ii])
        gk = got[ii].copy()
        hit = gk["face_index"] != 0xFFFFFFFF
        gk["face_index"][hit] -= np.uint32(tb)
        exp = ref.raycast_first(sub, threads=threads)
        par_mod.add_counts(tot, par_mod.first_parity_chunk(ref, sub, gk, exp, threads=threads))
    return tot


def measure_batched(args, ws, rank, local):
    """BatchedMesh form (1024 sub-geometries, log-uniform 200..200,000 triangles and 1,000..1,000,000
    rays each): one graph-captured persistent launch versus one plain launch per geometry; returns
    the result dict on rank 0."""
    import torch

    import __graft_entry__ as ge

    pkg = ge.load_package()
    from three_mesh_bvh_b200.batched import BatchedMeshBVH

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    t_setup = time.perf_counter()
    geoms, _, rays, off = pkg.batched_scene(n_geometries=args.batch_meshes, seed=2)
    batch = BatchedMeshBVH(geoms, {"strategy": pkg.SAH, "maxLeafSize": 10}, threads=os.cpu_count())
    n = rays.shape[0]
    d_rays = torch.from_numpy(rays).to(dev)
    out = torch.empty((n, 8), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    s = stream.cuda_stream
    t_setup = time.perf_counter() - t_setup

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(steps):
            fn()
        b.record(stream)
        torch.cuda.synchronize(dev)
        return a.elapsed_time(b) / steps

    # autotune the batched launch over the traversal variants
    from three_mesh_bvh_b200 import autotune

    # (the batched launch always runs the persistent form; ray ordering applies to single meshes),
    # on each device leaf layout
    cands = [c for c in autotune.candidates() if c[0] == 1 and c[5] == 0]
    timings = {}
    for leaf in (0, 2, 4):
        batch.set_leaf_size(leaf)
        for cand in cands:
            batch.set_traversal(*cand)
            timings[f"{list(cand)}/leaf{leaf}"] = timed(lambda: batch.raycast_first(d_rays, off, out=out, stream=s),
                                                        1, 1)
    best_key = min(timings, key=timings.get)
    best_leaf = int(best_key.split("/leaf")[1])
    best = next(c for c in cands if f"{list(c)}/leaf{best_leaf}" == best_key)
    batch.set_leaf_size(best_leaf)
    batch.set_traversal(*best)
    graph = batch.capture(d_rays, off, out)
    with ClockSampler(local) as clk:
        ms_graph = max_over_ranks(timed(lambda: graph.launch(s), args.steps, args.warmup), ws, dev)
    batch.synchronize(s)
    ref_out = out.clone()
    # per-geometry launches: plain one-ray-per-thread kernel (same child order), and persistent
    batch.set_traversal(0, best[1], 16, 0)
    ms_plain = max_over_ranks(timed(lambda: batch.raycast_first_per_mesh(d_rays, off, out=out, stream=s),
                                    max(1, args.steps // 2), 1), ws, dev)
    batch.synchronize(s)
    same_plain = bool(torch.equal(out.view(torch.int32)[:, 0], ref_out.view(torch.int32)[:, 0]))
    batch.set_traversal(*best)
    ms_pers = max_over_ranks(timed(lambda: batch.raycast_first_per_mesh(d_rays, off, out=out, stream=s),
                                   max(1, args.steps // 2), 1), ws, dev)
    batch.synchronize(s)
    res = None
    if rank == 0:
        par = None
        if not args.no_cpu_baseline:
            got = np.frombuffer(ref_out.cpu().numpy().tobytes(), dtype=pkg.HIT_DTYPE)
            per = 256
            tot = batched_oracle_check(batch, rays, off, got, per, os.cpu_count() or 1)
            keys = parity_module().FIRST_KEYS
            par = {"rays_checked": tot["rays"], "per_geometry": f"up to {per} evenly strided rays of each geometry",
                   "mismatches": {k: tot[k] for k in keys}, "tie_exempt": tot["exempt"],
                   "ok": not any(tot[k] for k in keys)}
        res = {"metric": "Mrays/s batched raycastFirst (1024 meshes)", "value": n / (ms_graph / 1e3) / 1e6,
               "unit": UNIT, "ms_per_step": ms_graph, "steps": args.steps, "warmup": args.warmup,
               "config": {"workload": f"{args.batch_meshes} geometries alternating TorusKnot / Icosahedron, "
                                      "triangles log-uniform 200..200000, rays log-uniform 1e3..1e6 per geometry "
                                      "(seed 2), SAH leaf 10; one CUDA-graph persistent launch",
                          "triangles": int(batch.triangle_base[-1]), "rays_per_step": int(n)},
               "per_mesh_plain_launches": {"ms": ms_plain, "mrays_s": n / (ms_plain / 1e3) / 1e6,
                                           "same_face_indices": same_plain},
               "per_mesh_persistent_launches": {"ms": ms_pers, "mrays_s": n / (ms_pers / 1e3) / 1e6},
               "speedup_vs_per_mesh_plain": ms_plain / ms_graph, "same_face_indices": same_plain,
               "parity": par, "traversal": list(best), "leaf_size": best_leaf, "autotune_ms": timings, "clocks": clk.summary(),
               "setup_s": t_setup, "gpu_launches": args.steps * kernel_launches(best)}
    graph.destroy()
    batch.dispose()
    del d_rays, out, ref_out
    return res


def run_batched(args, ws, rank, local):
    res = measure_batched(args, ws, rank, local)
    if rank == 0:
        line = {**res, "n_gpus": ws, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic",
                "e2e": None, "e2e_note": "not measured: the rays and hits of all 1024 geometries (~1.5e8 rays) "
                                         "would need ~8.4 GB of page-locked host memory"}
        print(json.dumps(line), flush=True)


def closest_launches(variant: int) -> int:
    """Kernels one closestPointToPoint call launches: the traversal (per query or warp-cooperative)
    and the finalize kernel, after the query box, the Morton keys and a three-pass radix sort
    (three kernels a pass) for the sorted forms."""
    if variant == 0:
        return 2
    return 2 + (11 if variant % 2 == 0 else 0)


def run_closest(args, ws, rank, local):
    """Closest point / unsigned SDF: the 80,000-triangle knot, a 256^3 grid over its bounding box
    padded by 10%, closestPointToPoint with maxThreshold 5 and minThreshold 0."""
    import torch

    import __graft_entry__ as ge

    pkg = ge.load_package()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    geo = pkg.torus_knot(10, 3, 400, 100)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH, "maxLeafSize": 10, "maxDepth": 40})
    pts_h = pkg.grid_points(geo.position.min(0), geo.position.max(0), args.grid)
    pts = torch.from_numpy(pts_h).to(dev)
    out = torch.empty((pts.shape[0], 5), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    s = stream.cuda_stream
    n = pts.shape[0]
    lib = pkg.lib()
    from three_mesh_bvh_b200 import autotune

    bvh.set_traversal(1, 1, 16, 2)   # register budget shared with the warp-cooperative kernels
    if args.closest_variant is not None:
        kw = {"closest": args.closest_variant}
        if args.closest_tile_rows:
            kw.update(tile=args.grid, tile_rows=args.closest_tile_rows)
        bvh.set_traversal(1, 1, 16, 2, **kw)
        tuned = {"best": str(args.closest_variant), "setting": kw, "forced": True}
    else:
        # the grid's points come row by row (its last axis fastest): its row length is the tiled
        # order's pitch, as the caller that made the grid would pass it
        tuned = autotune.tune_closest_point(bvh, pts, 0.0, 5.0, tile_pitches=(args.grid,))

    def step():
        lib.bvhc_closest_point_to_point(bvh._device_mesh(), pts.data_ptr(), n, 0.0, 5.0, out.data_ptr(), 1, s)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        a.record(stream)
        for _ in range(args.steps):
            step()
        b.record(stream)
        torch.cuda.synchronize(dev)
    bvh.synchronize(s)
    ms = max_over_ranks(a.elapsed_time(b) / args.steps, ws, dev)
    # end to end: pinned host points in, pinned host results out, through the public call (chunks
    # pipelined over three streams inside the library)
    pin_p = torch.from_numpy(pts_h).pin_memory()
    pin_o = torch.empty((n, 5), dtype=torch.float32).pin_memory()
    e2e = []
    for _ in range(max(1, args.steps // 2)):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        lib.bvhc_closest_point_to_point(bvh._device_mesh(), pin_p.data_ptr(), n, 0.0, 5.0, pin_o.data_ptr(), 0, None)
        e2e.append((time.perf_counter() - t0) * 1e3)
    e2e_ms = max_over_ranks(float(np.median(e2e)), ws, dev)
    cpu = roof = None
    if rank == 0 and not args.no_cpu_baseline:
        import oracle.oracle as orc

        ref = orc.OracleBVH.from_serialized(bvh._roots, geo.index, None, geo.position)
        threads = os.cpu_count() or 1
        idx = np.linspace(0, n - 1, min(n, 1 << 21)).astype(np.int64)
        t0 = time.perf_counter()
        _, nn, nt = ref.closest_point(np.ascontiguousarray(pts_h[idx]), 0.0, 5.0, threads=threads, counters=True)
        dt = time.perf_counter() - t0
        cpu = {"value": idx.size / dt / 1e6, "unit": "Mqueries/s", "cores": threads, "kind": "port",
               "sample": f"{idx.size} evenly strided grid points, float64 oracle"}
        per_query = 12 + 20 + 32 * float(nn.mean()) + 36 * float(nt.mean())
        peak, how = measured_peak()
        achieved = n * per_query / (ms / 1e3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "peak_source": how, "algorithmic_bytes_per_launch": n * per_query,
                "reference_node_reads_per_query": float(nn.mean()),
                "reference_triangle_tests_per_query": float(nt.mean()),
                "kernel": "closest_point_kernel" if tuned["setting"]["closest"] == 0 else "closest_point_packet_kernel"}
        prof = "closest_point_k3.md"
        roof["issue"] = {"source": f"profiles/{prof}",
                         "warp_instructions_per_query": profile_value(prof, "warp_instructions_per_query"),
                         "issue_slots_active": profile_value(prof, "issue_slots_active"),
                         "threads_per_instruction": profile_value(prof, "threads_per_instruction")}
    if rank == 0:
        line = {"metric": "Mqueries/s closestPointToPoint (80k tri, 256^3 grid)",
                "value": weak_scaling_rate(ws, n, 1, ms), "unit": "Mqueries/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"TorusKnot(10,3,400,100) 80,000 tri, SAH leaf 10; {args.grid}^3 grid over "
                                       "the AABB padded 10%; maxThreshold 5, minThreshold 0", "queries": int(n)},
                "closest_variant": tuned, "roofline": roof, "cpu_baseline": cpu, "clocks": clk.summary(),
                "e2e": {"value": weak_scaling_rate(ws, n, 1, e2e_ms), "unit": "Mqueries/s",
                        "h2d_bytes_per_step": int(n * 12), "d2h_bytes_per_step": int(n * 20)},
                "gpu_launches": args.steps * closest_launches(tuned["setting"]["closest"])}
        print(json.dumps(line), flush=True)
    bvh.dispose()


def run_all_hits(args, ws, rank, local):
    """raycast (all hits, capped at 64 per ray plus the uncapped count) on the 2M-triangle knot's
    two ray sets."""
    import torch

    import __graft_entry__ as ge

    pkg = ge.load_package()
    from three_mesh_bvh_b200._native import check

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    geo, bvh, inc, cam = scene(pkg, args, rank)
    sets = [("incoherent", inc), ("camera", cam)]
    cap = 64
    stream = torch.cuda.current_stream(dev)
    n_max = max(r.shape[0] for _, r in sets)
    counts = torch.empty(n_max, dtype=torch.int32, device=dev)
    hits = torch.empty((n_max, cap, 8), dtype=torch.float32, device=dev)   # 32 B per hit slot
    lib = pkg.lib()
    per_set_ms, stored, variants = [], [], {}
    bvh.set_traversal(1, 1, 16, 2)   # register budget shared with the warp-cooperative kernels
    cur = bvh.get_traversal()
    with ClockSampler(local) as clk:
        for name, r in sets:
            d = torch.from_numpy(r).to(dev)
            n = d.shape[0]

            def call():
                check(lib.bvhc_raycast(bvh._device_mesh(), d.data_ptr(), n, 0, 0.0, math.inf, cap,
                                       counts.data_ptr(), hits.data_ptr(), 1, stream.cuda_stream), "bvhc_raycast")

            # the all-hits kernel variant for this set (one call each, on the same buffers)
            # the all-hits kernels, and the warp-cooperative one in tiled order with the camera's
            # row pitch ("1t": 4-row tiles, "1t2" / "1t8": 2 / 8 rows)
            t_var, settings = {}, {v: {"all": v} for v in range(13)}
            settings["1t"] = {"all": 1, "tile": args.camera}
            settings["1t2"] = {"all": 1, "tile": args.camera, "tile_rows": 2}
            settings["1t8"] = {"all": 1, "tile": args.camera, "tile_rows": 8}
            for v, kw in settings.items():
                bvh.set_traversal(**{**cur, **kw})
                call()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                call()
                e1.record(stream)
                e1.synchronize()
                t_var[v] = e0.elapsed_time(e1)
            best = min(t_var, key=t_var.get)
            bvh.set_traversal(**{**cur, **settings[best]})
            variants[name] = {"best": best, "timings_ms": {str(k): x for k, x in t_var.items()}}
            for _ in range(args.warmup):
                call()
            torch.cuda.synchronize(dev)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(args.steps):
                call()
            b.record(stream)
            torch.cuda.synchronize(dev)
            per_set_ms.append(max_over_ranks(a.elapsed_time(b) / args.steps, ws, dev))
            stored.append(int(counts[:n].clamp(max=cap).sum().item()))
            del d
    bvh.synchronize(stream.cuda_stream)
    n_step = sum(r.shape[0] for _, r in sets)
    ms = sum(per_set_ms)
    cpu = roof = None
    if rank == 0 and not args.no_cpu_baseline:
        import oracle.oracle as orc

        ref = orc.OracleBVH.from_serialized(bvh._roots, geo.index, bvh._indirectBuffer, geo.position)
        threads = os.cpu_count() or 1
        t_cpu, n_cpu, bytes_per_set = 0.0, 0, []
        for (name, r), sh in zip(sets, stored):
            idx = np.linspace(0, r.shape[0] - 1, min(r.shape[0], args.cpu_sample // 4)).astype(np.int64)
            t0 = time.perf_counter()
            _, _, nn, nt = ref.raycast_all(np.ascontiguousarray(r[idx]), cap=cap, threads=threads, counters=True)
            t_cpu += time.perf_counter() - t0
            n_cpu += idx.size
            # ray in + uncapped count + 32-byte records of the stored hits + reference node / triangle reads
            bytes_per_set.append(r.shape[0] * (BYTES_RAY_IN + 4 + BYTES_NODE * float(nn.mean()) +
                                               BYTES_TRI * float(nt.mean())) + BYTES_HIT_OUT * sh)
        cpu = {"value": n_cpu / t_cpu / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{n_cpu} rays ({args.cpu_sample // 4} evenly strided from each set), float64 oracle"}
        peak, how = measured_peak()
        k = max(range(len(sets)), key=lambda j: per_set_ms[j])
        achieved = bytes_per_set[k] / (per_set_ms[k] / 1e3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "peak_source": how, "ray_set": sets[k][0],
                "kernel": {0: "raycast_all_kernel", 1: "raycast_all_packet_kernel", "1t": "raycast_all_packet_kernel",
                           "1t2": "raycast_all_packet_kernel", "1t8": "raycast_all_packet_kernel",
                           2: "raycast_all_packet_kernel", 3: "raycast_all_packet_kernel",
                           4: "raycast_all_packet_kernel"}.get(variants[sets[k][0]]["best"],
                                                              "raycast_all_persistent_kernel"
                                                              if str(variants[sets[k][0]]["best"]) in
                                                              ("9", "10", "11", "12") else "raycast_all_kernel"),
                "algorithmic_bytes_per_launch": dict(zip([n for n, _ in sets], bytes_per_set))}
    if rank == 0:
        line = {"metric": "Mrays/s raycast all hits (2M tri, cap 64)", "value": weak_scaling_rate(ws, n_step, 1, ms),
                "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": WORKLOAD.replace("raycastFirst", "raycast (all hits, cap 64)"),
                           "rays_per_step": n_step, "stored_hits": dict(zip([n for n, _ in sets], stored))},
                "per_set_ms": dict(zip([n for n, _ in sets], per_set_ms)),
                "all_hits_variant": variants, "roofline": roof, "cpu_baseline": cpu, "clocks": clk.summary(),
                "gpu_launches": args.steps * sum(all_hits_launches(v["best"]) for v in variants.values()),
                "e2e": None, "e2e_note": "not measured: the hit rows (2^24 rays x 64 hits x 32 B per set) are "
                                         "34 GB, more than page-locked host memory should hold"}
        print(json.dumps(line), flush=True)
    bvh.dispose()


def measure_adjoint(args, ws, rank, local):
    """Differentiable depth and SDF on the 2M-triangle knot: forward raycastFirst of a 1024^2 camera
    and backward of L = sum (t - t*)^2 (t* rendered from the mesh with vertices moved by N(0, 0.01),
    seed 3); forward closestPointToPoint of a 128^3 grid and backward of sum distance.  Returns the
    result dict on rank 0."""
    import torch

    import __graft_entry__ as ge

    pkg = ge.load_package()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    geo = pkg.torus_knot(10, 3, args.tubular, args.radial, noise_sigma=0.02, noise_seed=1)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH, "maxLeafSize": 10})
    pert = geo.clone()
    pert.position = pert.position + np.random.default_rng(3).normal(0, 0.01, pert.position.shape).astype(np.float32)
    bvh_star = pkg.MeshBVH(pert, {"strategy": pkg.SAH, "maxLeafSize": 10})
    rays = torch.from_numpy(pkg.rays_camera(1024, 1024)).to(dev)
    stream = torch.cuda.current_stream(dev)
    s = stream.cuda_stream
    star = bvh_star.raycast_first_batch(rays, stream=s)
    t_star = star[:, 1].clone()
    star_hit = star[:, 0].view(torch.int32) != -1
    gv = torch.zeros((geo.position.shape[0], 3), dtype=torch.float32, device=dev)
    pts = torch.from_numpy(pkg.grid_points(geo.position.min(0), geo.position.max(0), 128)).to(dev)
    ones = torch.ones(pts.shape[0], dtype=torch.float32, device=dev)
    # the forward passes run their autotuned variants (the backward replays recorded triangles and
    # has no variants)
    from three_mesh_bvh_b200 import autotune

    tuned_ray = autotune.tune_raycast_first_sets(bvh, [("camera1024", rays)], leaf_sizes=(0, 2, 4), tag="adjoint",
                                                 tile_pitches=(1024,))
    bvh.set_traversal(*tuned_ray["sets"]["camera1024"]["best"])
    tuned_cp = autotune.tune_closest_point(bvh, pts, 0.0, 5.0, tile_pitches=(128,))

    def fwd():
        return bvh.raycast_first_batch(rays, stream=s)

    def fwd_bwd():
        hits = bvh.raycast_first_batch(rays, stream=s)
        hit = (hits[:, 0].view(torch.int32) != -1) & star_hit
        g = torch.where(hit, 2 * (hits[:, 1] - t_star), torch.zeros_like(t_star))
        gv.zero_()
        bvh.raycast_first_backward(rays, hits, g, grad_vertices=gv, stream=s)

    def cp_fwd():
        return bvh.closest_point_batch(pts, 0.0, 5.0, stream=s)

    def cp_fwd_bwd():
        res = bvh.closest_point_batch(pts, 0.0, 5.0, stream=s)
        gv.zero_()
        bvh.closest_point_backward(pts, res, ones, grad_vertices=gv, stream=s)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            fn()
        b.record(stream)
        torch.cuda.synchronize(dev)
        return a.elapsed_time(b) / args.steps

    # refit after a gradient step (the vertices moved a little): boxes rebuilt on the device
    pos_step = torch.from_numpy(geo.position).to(dev) - 1e-4 * gv

    def refit():
        bvh.refit(pos_step, stream=s, read_back=False)

    with ClockSampler(local) as clk:
        ms_f, ms_fb = timed(fwd), timed(fwd_bwd)
        ms_cf, ms_cfb = timed(cp_fwd), timed(cp_fwd_bwd)
        ms_refit = timed(refit)
    bvh.synchronize(s)
    ms_f, ms_fb, ms_cf, ms_cfb = (max_over_ranks(x, ws, dev) for x in (ms_f, ms_fb, ms_cf, ms_cfb))
    res = None
    if rank == 0:
        res = {"metric": "fwd+bwd / fwd time, raycastFirst depth loss (2M tri, 1024^2 camera)",
               "value": ms_fb / ms_f, "ratio": ms_fb / ms_f, "unit": "ratio", "ms_per_step": ms_fb,
               "steps": args.steps, "warmup": args.warmup, "target": "<= 2.5",
               "config": {"workload": "TorusKnot(10,3,2000,500) + N(0,0.02) noise, SAH leaf 10; 1024^2 camera; "
                                      "L = sum (t - t*)^2, t* from vertices + N(0,0.01) (seed 3); "
                                      "128^3 grid closest point, max 5, L = sum distance"},
               "raycast": {"fwd_ms": ms_f, "fwd_bwd_ms": ms_fb, "ratio": ms_fb / ms_f},
               "closest_point": {"fwd_ms": ms_cf, "fwd_bwd_ms": ms_cfb, "ratio": ms_cfb / ms_cf},
               "forward_variants": {"raycast": tuned_ray["sets"]["camera1024"]["best"],
                                    "leaf_size": tuned_ray["leaf"], "closest": tuned_cp["best"]},
               "refit_ms": ms_refit, "clocks": clk.summary()}
    bvh.dispose()
    bvh_star.dispose()
    return res


def run_adjoint(args, ws, rank, local):
    res = measure_adjoint(args, ws, rank, local)
    if rank == 0:
        line = {**res, "n_gpus": ws, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic",
                "e2e": None, "e2e_note": "the metric is a ratio of device times (backward over forward)"}
        print(json.dumps(line), flush=True)


def run_scene(args, ws, rank, local):
    """Instanced BatchedMesh raycastFirst on world rays: 256 geometries (the batched generator:
    torus knots and icospheres, log-uniform 200..200,000 triangles), 4096 instances with random
    rotations, uniform scales 0.5..2 and positions in [-1000, 1000]^3, 2^22 world rays from a
    sphere of radius 2500 towards uniform points of the instance cube."""
    import torch

    import __graft_entry__ as ge

    pkg = ge.load_package()
    from three_mesh_bvh_b200.batched import BatchedMeshBVH

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n_geo, n_inst, n_rays = 256, 4096, 1 << 22
    geoms, _, _, _ = pkg.batched_scene(n_geometries=n_geo, tri_range=(200, 200_000), seed=2, make_rays=False)
    batch = BatchedMeshBVH(geoms, {"strategy": pkg.SAH, "maxLeafSize": 10}, threads=os.cpu_count() or 1)
    rng = np.random.default_rng(3 + rank)
    geometry = rng.integers(0, n_geo, n_inst).astype(np.uint32)
    mats = np.zeros((n_inst, 16))
    for j in range(n_inst):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        x, y, z, w = q
        rot = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                        [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                        [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]]) * rng.uniform(0.5, 2.0)
        m = np.eye(4)
        m[:3, :3] = rot
        m[:3, 3] = rng.uniform(-1000, 1000, 3)
        mats[j] = m.T.reshape(-1)
    u = rng.normal(size=(n_rays, 3))
    o = u / np.linalg.norm(u, axis=1, keepdims=True) * 2500.0
    d = rng.uniform(-1000, 1000, (n_rays, 3)) - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays_h = np.concatenate([o, d], 1).astype(np.float32)
    scene = batch.instances(geometry, mats)
    rays = torch.from_numpy(rays_h).to(dev)
    hits = torch.empty((n_rays, 8), dtype=torch.float32, device=dev)
    inst = torch.empty(n_rays, dtype=torch.int32, device=dev)
    lib = pkg.lib()
    stream = torch.cuda.current_stream(dev)
    s = stream.cuda_stream

    def step():
        lib.bvhc_scene_raycast_first(scene.h, rays.data_ptr(), n_rays, 0, 0.0, math.inf, hits.data_ptr(),
                                     inst.data_ptr(), 1, s)

    # ray order (input order, a Morton key, or the first instance reached), kernel variant
    # (resident blocks per SM 14 / 10 / 8) and the geometries' leaf layout, whichever is fastest here
    order_ms = {}
    variants = (0, 1, 2) if args.scene_variant is None else (args.scene_variant,)
    leaves = (0, 4) if args.scene_variant is None else (0,)
    for leaf, occ in ((lf, v) for lf in leaves for v in variants):
        batch.set_leaf_size(leaf)
        scene.set_variant(occ)
        for order in ((0, 1, 2, 3, 4) if args.scene_variant is None else (0,)):
            scene.set_order(order)
            step()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            order_ms[(leaf, occ, order)] = e0.elapsed_time(e1)
    best_leaf, best_occ, best_order = min(order_ms, key=order_ms.get)
    batch.set_leaf_size(best_leaf)
    scene.set_variant(best_occ)
    scene.set_order(best_order)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize(dev)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        a.record(stream)
        for _ in range(args.steps):
            step()
        b.record(stream)
        torch.cuda.synchronize(dev)
    ms = max_over_ranks(a.elapsed_time(b) / args.steps, ws, dev)
    hit_frac = float((inst.cpu().numpy() >= 0).mean())
    # all hits (the BatchedMesh raycast without firstHitOnly), first 16 per ray stored
    cap_all = 16
    counts_all = torch.empty(n_rays, dtype=torch.int32, device=dev)
    hits_all = torch.empty((n_rays, cap_all, 8), dtype=torch.float32, device=dev)
    inst_all = torch.empty((n_rays, cap_all), dtype=torch.int32, device=dev)

    def step_all():
        lib.bvhc_scene_raycast(scene.h, rays.data_ptr(), n_rays, 0, 0.0, math.inf, cap_all, counts_all.data_ptr(),
                               hits_all.data_ptr(), inst_all.data_ptr(), 1, s)

    for _ in range(args.warmup):
        step_all()
    torch.cuda.synchronize(dev)
    a2, b2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a2.record(stream)
    for _ in range(args.steps):
        step_all()
    b2.record(stream)
    torch.cuda.synchronize(dev)
    ms_all = max_over_ranks(a2.elapsed_time(b2) / args.steps, ws, dev)
    mean_hits = float(counts_all.double().mean().item())
    # end to end: host rays in, host hits and instance ids out (pinned), through the public call
    pin_r = torch.from_numpy(rays_h).pin_memory()
    pin_h = torch.empty((n_rays, 8), dtype=torch.float32).pin_memory()
    pin_i = torch.empty(n_rays, dtype=torch.int32).pin_memory()
    e2e = []
    for _ in range(max(1, args.steps // 2)):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        lib.bvhc_scene_raycast_first(scene.h, pin_r.data_ptr(), n_rays, 0, 0.0, math.inf, pin_h.data_ptr(),
                                     pin_i.data_ptr(), 0, None)
        e2e.append((time.perf_counter() - t0) * 1e3)
    e2e_ms = max_over_ranks(float(np.median(e2e)), ws, dev)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        import oracle.oracle as orc

        oracles, r0 = [], 0
        for k in range(batch.n_meshes):
            roots = batch.roots[r0:r0 + batch.roots_per_mesh[k]]
            r0 += batch.roots_per_mesh[k]
            oracles.append(orc.OracleBVH.from_serialized(roots, batch.index, None, batch.position))
        idx = np.linspace(0, n_rays - 1, 1 << 14).astype(np.int64)
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        orc.scene_raycast_first(oracles, geometry, mats, rays_h[idx], threads=threads)
        dt = time.perf_counter() - t0
        cpu = {"value": idx.size / dt / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "port",
               "sample": f"{idx.size} evenly strided rays; the float64 oracle loops over every instance per ray, "
                         "as the reference's BatchedMesh raycast does"}
    if rank == 0:
        line = {"metric": "Mrays/s instanced raycastFirst (256 geometries, 4096 instances)",
                "value": weak_scaling_rate(ws, n_rays, 1, ms), "unit": "Mrays/s", "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "BatchedMesh instances: 256 geometries (torus knots / icospheres, log-uniform "
                                       "200..200,000 tri, seed 2), 4096 instances (random rotation, uniform scale "
                                       "0.5..2, position in [-1000,1000]^3), 2^22 world rays (sphere r=2500 towards "
                                       "the instance cube), firstHitOnly",
                           "geometry_triangles": int(sum(g.triangle_count for g in geoms)),
                           "hit_fraction": hit_frac, "l2": "inputs (100 MB rays + 134 MB hits) exceed L2",
                           "ray_order": best_order, "kernel_variant": best_occ, "leaf_size": best_leaf,
                           "order_ms": {str(k): v for k, v in order_ms.items()},
                           "all_hits": {"ms": ms_all, "Mrays_per_s": weak_scaling_rate(ws, n_rays, 1, ms_all),
                                        "cap": cap_all, "mean_hits_per_ray": mean_hits}},
                "e2e": {"value": weak_scaling_rate(ws, n_rays, 1, e2e_ms), "unit": "Mrays/s",
                        "h2d_bytes_per_step": int(rays_h.nbytes), "d2h_bytes_per_step": int(n_rays * 36)},
                "roofline": None, "roofline_note": "two-level traversal (instance tree, then a geometry tree per "
                "entered instance box) is latency-bound", "cpu_baseline": cpu, "clocks": clk.summary(),
                "gpu_launches": args.steps * (1 if best_order == 0 else 6)}
        print(json.dumps(line), flush=True)
    scene.dispose()
    batch.dispose()


def run_build(args, ws, rank, local):
    """SAH build of the 2M-triangle knot on the device (bvhc_build_device), host buffers in and
    out (the call uploads positions and index, builds, and returns the serialized roots and the
    reordered index), against the library's CPU builder; the serialized bytes must be identical."""
    import ctypes as C

    import torch

    import __graft_entry__ as ge

    pkg = ge.load_package()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    geo = pkg.torus_knot(10, 3, args.tubular, args.radial, noise_sigma=0.02, noise_seed=1)
    lib = pkg.lib()
    pos = np.ascontiguousarray(geo.position, dtype=np.float32)
    idx = geo.index
    n_tri = idx.size // 3

    def build(device: bool):
        out = C.c_void_p()
        args_ = (pos.ctypes.data, pos.shape[0], 3, idx.ctypes.data, idx.dtype.itemsize, idx.size, None, 0, 0, -1,
                 int(pkg.SAH), 40, 10, 0)
        st = (lib.bvhc_build_device(*args_, local, None, C.byref(out)) if device else lib.bvhc_build(*args_, C.byref(out)))
        if st != 0:
            raise RuntimeError(f"build failed with status {st}")
        return out

    def blob(s):
        parts = []
        for i in range(lib.bvhc_serialized_root_count(s)):
            p, nb = C.c_void_p(), C.c_uint64()
            lib.bvhc_serialized_root(s, i, C.byref(p), C.byref(nb))
            parts.append(C.string_at(p, nb.value))
        p, eb, cnt = C.c_void_p(), C.c_int(), C.c_uint64()
        lib.bvhc_serialized_index(s, C.byref(p), C.byref(eb), C.byref(cnt))
        parts.append(C.string_at(p, cnt.value * eb.value))
        return b"".join(parts)

    for _ in range(args.warmup):
        lib.bvhc_serialized_free(build(True))
    times = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            s = build(True)
            times.append((time.perf_counter() - t0) * 1e3)
            if len(times) < args.steps:
                lib.bvhc_serialized_free(s)
    ms = max_over_ranks(float(np.median(times)), ws, dev)
    d2h_bytes = len(blob(s))
    cpu = None
    identical = None
    if rank == 0:
        t0 = time.perf_counter()
        sc = build(False)
        cpu_ms = (time.perf_counter() - t0) * 1e3
        identical = blob(sc) == blob(s)
        lib.bvhc_serialized_free(sc)
        cpu = {"value": n_tri / (cpu_ms / 1e3) / 1e6, "unit": "Mtris/s", "cores": 1, "kind": "port",
               "sample": "the whole mesh, the library's single-threaded CPU builder (byte-identical to the "
                         "oracle's restatement of the reference build)", "ms": cpu_ms}
    lib.bvhc_serialized_free(s)
    if rank == 0:
        line = {"metric": "Mtris/s SAH build (2M tri, host buffers in and out)",
                "value": weak_scaling_rate(ws, n_tri, 1, ms), "unit": "Mtris/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32+binary64 (integer-emulated decisions)", "data": "synthetic",
                "config": {"workload": f"TorusKnot(10,3,{args.tubular},{args.radial}) {n_tri:,} tri + N(0,0.02) "
                                       "normal noise (seed 1), SAH, maxLeafSize 10, maxDepth 40",
                           "timing": "wall clock around bvhc_build_device (it synchronizes), median of steps"},
                "serialized_identical_to_cpu_build": identical,
                "e2e": {"value": weak_scaling_rate(ws, n_tri, 1, ms), "unit": "Mtris/s",
                        "h2d_bytes_per_step": int(pos.nbytes + idx.nbytes),
                        "d2h_bytes_per_step": d2h_bytes},
                "roofline": None, "roofline_note": "tree construction is latency-bound (level-synchronous "
                "kernels, 227 launches per build); kernel shares in profiles/device_build_k2_launches.md",
                "cpu_baseline": cpu, "clocks": clk.summary(),
                "gpu_launches": 227 * args.steps, "gpu_launches_source": "ncu launch list of this workload"}
        print(json.dumps(line), flush=True)


def shapecast_queries(geo, rng, n_brush, n_sphere, n_box):
    """Query sets on the mesh: sculpt brushes (spheres centred on random triangle centroids,
    radius log-uniform 0.03..0.3, i.e. a few to a few hundred triangles), spheres anywhere in the
    bounding box (radius log-uniform 0.01..2) and oriented boxes (random rotation, half extents
    0.05..1) as rows of 24 float32 (min xyz, 0, max xyz, 0, column-major box-to-mesh matrix)."""
    pos, idx = geo.position.astype(np.float64), geo.index.reshape(-1, 3)
    t = rng.integers(0, idx.shape[0], n_brush)
    cen = pos[idx[t]].mean(1)
    brush = np.concatenate([cen, np.exp(rng.uniform(np.log(0.03), np.log(0.3), n_brush))[:, None]], 1)
    lo, hi = pos.min(0), pos.max(0)
    sph = np.concatenate([lo + rng.random((n_sphere, 3)) * (hi - lo),
                          np.exp(rng.uniform(np.log(0.01), np.log(2.0), n_sphere))[:, None]], 1)
    q = rng.normal(size=(n_box, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    x, y, z, w = q.T
    m = np.zeros((n_box, 16))
    m[:, 0], m[:, 1], m[:, 2] = 1 - 2 * (y * y + z * z), 2 * (x * y + w * z), 2 * (x * z - w * y)
    m[:, 4], m[:, 5], m[:, 6] = 2 * (x * y - w * z), 1 - 2 * (x * x + z * z), 2 * (y * z + w * x)
    m[:, 8], m[:, 9], m[:, 10] = 2 * (x * z + w * y), 2 * (y * z - w * x), 1 - 2 * (x * x + y * y)
    m[:, 12:15] = lo + rng.random((n_box, 3)) * (hi - lo)
    m[:, 15] = 1
    half = rng.uniform(0.05, 1.0, (n_box, 3))
    box = np.zeros((n_box, 24))
    box[:, 0:3], box[:, 4:7], box[:, 8:24] = -half, half, m
    f = np.float32
    return brush.astype(f), sph.astype(f), box.astype(f)


def run_shapecast(args, ws, rank, local):
    """Shapecast queries on the 2M-triangle knot: triangles within sculpt-brush spheres (shapecast's
    CONTAINED path), intersectsSphere, intersectsBox (oriented boxes), and getTriangleHitPointInfo."""
    import torch

    import __graft_entry__ as ge

    pkg = ge.load_package()
    from three_mesh_bvh_b200._native import check

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    geo = pkg.torus_knot(10, 3, args.tubular, args.radial, noise_sigma=0.02, noise_seed=1)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH, "maxLeafSize": 10, "maxDepth": 40})
    n_brush, n_sphere, n_box, cap = 1 << 18, 1 << 22, 1 << 20, 256
    brush_h, sph_h, box_h = shapecast_queries(geo, np.random.default_rng(7 + rank), n_brush, n_sphere, n_box)
    lib = pkg.lib()
    mesh = bvh._device_mesh()
    stream = torch.cuda.current_stream(dev)
    s = stream.cuda_stream
    brush, sph, box = (torch.from_numpy(x).to(dev) for x in (brush_h, sph_h, box_h))
    counts = torch.empty(n_brush, dtype=torch.int32, device=dev)
    faces = torch.empty((n_brush, cap), dtype=torch.int32, device=dev)
    flags = torch.empty(max(n_sphere, n_box), dtype=torch.uint8, device=dev)
    calls = {
        "sphere_triangles": (n_brush, lambda: check(lib.bvhc_sphere_triangles(
            mesh, brush.data_ptr(), n_brush, cap, counts.data_ptr(), faces.data_ptr(), 1, s), "bvhc_sphere_triangles")),
        "intersects_sphere": (n_sphere, lambda: check(lib.bvhc_intersects_sphere(
            mesh, sph.data_ptr(), n_sphere, flags.data_ptr(), 1, s), "bvhc_intersects_sphere")),
        "intersects_box": (n_box, lambda: check(lib.bvhc_intersects_box(
            mesh, box.data_ptr(), n_box, flags.data_ptr(), 1, s), "bvhc_intersects_box")),
    }
    # getTriangleHitPointInfo on 2^20 (point, face) pairs: random faces, points at their centroids,
    # a uv attribute
    n_hpi = 1 << 20
    rng_h = np.random.default_rng(11 + rank)
    hpi_f = rng_h.integers(0, geo.triangle_count, n_hpi).astype(np.uint32)
    tri = geo.index.reshape(-1, 3).astype(np.int64)[hpi_f]
    hpi_p_h = geo.position[tri].astype(np.float64).mean(1).astype(np.float32)
    uv_h = rng_h.random((geo.position.shape[0], 2)).astype(np.float32)
    hpi_p, hpi_fd = torch.from_numpy(hpi_p_h).to(dev), torch.from_numpy(hpi_f.view(np.int32)).to(dev)
    pos_d, uv_d = torch.from_numpy(geo.position).to(dev), torch.from_numpy(uv_h).to(dev)
    hpi_out = torch.empty((n_hpi, 12), dtype=torch.int32, device=dev)   # 48-byte records
    calls["hit_point_info"] = (n_hpi, lambda: check(lib.bvhc_triangle_hit_point_info(
        mesh, hpi_p.data_ptr(), hpi_fd.data_ptr(), n_hpi, pos_d.data_ptr(), 3, uv_d.data_ptr(), 2,
        geo.position.shape[0], None, 0, hpi_out.data_ptr(), 1, s), "bvhc_triangle_hit_point_info"))
    ms = {}
    with ClockSampler(local) as clk:
        for name, (n, call) in calls.items():
            for _ in range(args.warmup):
                call()
            torch.cuda.synchronize(dev)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(args.steps):
                call()
            b.record(stream)
            torch.cuda.synchronize(dev)
            ms[name] = max_over_ranks(a.elapsed_time(b) / args.steps, ws, dev)
    bvh.synchronize(s)
    cnt = counts.cpu().numpy()
    # end to end: host spheres in, host counts and faces out (pinned), through the public call
    pin_b = torch.from_numpy(brush_h).pin_memory()
    pin_c = torch.empty(n_brush, dtype=torch.int32).pin_memory()
    pin_f = torch.empty((n_brush, cap), dtype=torch.int32).pin_memory()
    e2e = []
    for _ in range(max(1, args.steps // 2)):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        check(lib.bvhc_sphere_triangles(mesh, pin_b.data_ptr(), n_brush, cap, pin_c.data_ptr(), pin_f.data_ptr(), 0,
                                        None), "bvhc_sphere_triangles")
        e2e.append((time.perf_counter() - t0) * 1e3)
    e2e_ms = max_over_ranks(float(np.median(e2e)), ws, dev)
    cpu = roof = None
    sets = {k: {"queries": calls[k][0], "ms": v, "Mqueries_per_s": weak_scaling_rate(ws, calls[k][0], 1, v)}
            for k, v in ms.items()}
    if rank == 0 and not args.no_cpu_baseline:
        import oracle.oracle as orc

        ref = orc.OracleBVH.from_serialized(bvh._roots, geo.index, None, geo.position)
        threads = os.cpu_count() or 1
        peak, how = measured_peak()
        samples = {}
        # oracle over evenly strided samples of each set: CPU rate and the traversal counters
        idx = np.linspace(0, n_brush - 1, 1 << 15).astype(np.int64)
        t0 = time.perf_counter()
        ec, _, nn, nt = ref.sphere_triangles(brush_h[idx], cap=cap, threads=threads, counters=True)
        samples["sphere_triangles"] = (idx.size, time.perf_counter() - t0,
                                       16 + 4 + 4 * cap + 32 * nn.mean() + 36 * nt.mean() + 4 * ec.mean(), nn, nt)
        idx = np.linspace(0, n_sphere - 1, 1 << 17).astype(np.int64)
        t0 = time.perf_counter()
        _, nn, nt = ref.intersects_sphere(sph_h[idx], threads=threads, counters=True)
        samples["intersects_sphere"] = (idx.size, time.perf_counter() - t0, 16 + 1 + 32 * nn.mean() + 36 * nt.mean(),
                                        nn, nt)
        idx = np.linspace(0, n_box - 1, 1 << 16).astype(np.int64)
        t0 = time.perf_counter()
        _, nn, nt = ref.intersects_box(box_h[idx], threads=threads, counters=True)
        samples["intersects_box"] = (idx.size, time.perf_counter() - t0, 96 + 1 + 32 * nn.mean() + 36 * nt.mean(),
                                     nn, nt)
        m_h = 1 << 18
        t0 = time.perf_counter()
        orc.triangle_hit_point_info(hpi_p_h[:m_h], hpi_f[:m_h], geo.index, geo.position, uv_h)
        sets["hit_point_info"].update({"algorithmic_bytes_per_query": 136.0, "roofline_frac":
                                       n_hpi * 136.0 / (ms["hit_point_info"] / 1e3) / 1e9 / peak,
                                       "cpu_Mqueries_per_s": m_h / (time.perf_counter() - t0) / 1e6,
                                       "cpu_sample": m_h, "cpu_kind": "float64 numpy oracle, 1 thread"})
        for k, (m, dt, per, nn, nt) in samples.items():
            sets[k].update({"cpu_Mqueries_per_s": m / dt / 1e6, "cpu_sample": m,
                            "reference_node_reads_per_query": float(nn.mean()),
                            "reference_triangle_tests_per_query": float(nt.mean()),
                            "algorithmic_bytes_per_query": float(per),
                            "roofline_frac": calls[k][0] * per / (ms[k] / 1e3) / 1e9 / peak})
        m, dt, per, nn, nt = samples["sphere_triangles"]
        cpu = {"value": m / dt / 1e6, "unit": "Mqueries/s", "cores": threads, "kind": "port",
               "sample": f"{m} evenly strided brush spheres, float64 oracle"}
        achieved = n_brush * per / (ms["sphere_triangles"] / 1e3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "peak_source": how, "algorithmic_bytes_per_launch": n_brush * per,
                "kernel": "sphere_triangles_kernel"}
    if rank == 0:
        line = {"metric": "Mqueries/s triangles within sculpt-brush spheres (2M tri)",
                "value": weak_scaling_rate(ws, n_brush, 1, ms["sphere_triangles"]), "unit": "Mqueries/s",
                "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms["sphere_triangles"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": f"TorusKnot(10,3,{args.tubular},{args.radial}) + N(0,0.02) noise, SAH leaf "
                                       "10; 2^18 brush spheres on random triangle centroids, radius log-uniform "
                                       "0.03..0.3, first 256 faces per sphere; plus 2^22 spheres in the AABB "
                                       "(intersectsSphere), 2^20 oriented boxes (intersectsBox) and 2^20 "
                                       "(centroid, face) pairs with a uv attribute (getTriangleHitPointInfo)",
                           "mean_triangles_per_brush": float(cnt.mean()), "sets": sets,
                           "l2": "outputs (256 MB face rows) and sphere / box sets (64 / 96 MB) exceed or fill L2"},
                "e2e": {"value": weak_scaling_rate(ws, n_brush, 1, e2e_ms), "unit": "Mqueries/s",
                        "h2d_bytes_per_step": int(brush_h.nbytes), "d2h_bytes_per_step": int(n_brush * (1 + cap) * 4)},
                "roofline": roof, "cpu_baseline": cpu, "clocks": clk.summary(),
                "gpu_launches": args.steps}
        print(json.dumps(line), flush=True)
    bvh.dispose()


def main():
    args = parse()
    ws, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        elif args.workload == "batched":
            run_batched(args, ws, rank, local)
        elif args.workload == "adjoint":
            run_adjoint(args, ws, rank, local)
        elif args.workload == "closest":
            run_closest(args, ws, rank, local)
        elif args.workload == "all":
            run_all_hits(args, ws, rank, local)
        elif args.workload == "build":
            run_build(args, ws, rank, local)
        elif args.workload == "scene":
            run_scene(args, ws, rank, local)
        elif args.workload == "shapecast":
            run_shapecast(args, ws, rank, local)
        else:
            run_engine(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
