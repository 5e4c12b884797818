"""Benchmark of the 2 kHz soft-body substep on B200: node-substeps/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--workload fleet256|truss_car]

A step is one 60 Hz frame of 33 substeps (World::step_substeps(33)) over the whole workload. The default workload is
the batched fleet: 256 seeded lattice vehicles of log-normal size (500-20,000 nodes, median 3,000; about 0.9 M nodes
and 8.6 M beams) on four free-rolling wheel rings of 24 tyre nodes each, with collision skins, driving over a
2048^2-sample, 1 km^2 heightfield with contacts between the vehicles that meet - the fleet configuration's shape.
Under torchrun each rank steps its
own fleet (weak scaling, no data-path collective: vehicles that do not touch are independent islands).

Rank 0 prints one JSON line: value = node-substeps/s of all ranks with the state resident in HBM (CUDA events on the
world's stream, max over ranks); e2e = the same through the C ABI with the node state copied in from pinned host
memory and back out every frame; roofline = the dominant kernel's algorithmic bytes over its CUDA-event time in a
profiled frame of the timed region; cpu_baseline = the reference's own CPU step (compiled from its sources, all host
threads) on a bounded sample of the same workload.

--impl reference times the reference's CPU implementation alone (rank 0; other ranks exit at once).
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "node-substeps/s at 2 kHz, batched+learned vs plain GPU, residual<=1e-6"
UNIT = "node-substeps/s"
FRAME = 33
# algorithmic bytes of one substep (each array touched once): a beam reads its ends (8 B), L, k, d, max_pos, max_neg,
# strength (24 B), its type and flags (4 B) and writes its force's magnitude (stress, 4 B); a node reads p, v, 1/m
# (28 B) and writes p, v (24 B)
BYTES_PER_BEAM = 40
BYTES_PER_NODE = 52


def broadphase_bytes(rig: dict, pairs: int) -> dict:
    """Algorithmic bytes of one pair search (a contacter node: its position read, its cell key and id written and
    sorted, 12 + 12 + 4 x 2 x 12 = 120 B; a collision triangle: its 3 indices and 3 positions read, 48 B; a pair
    written, 12 B) and the searches a substep (the frame's first substep and every ceil(1 / (collision_hz dt)) after)."""
    import math
    contacters = sum(int(np.count_nonzero(np.asarray(b.get("node_flags", ()), np.int64) & 16)) for b in rig["bodies"])
    tris = sum(len(b.get("tris", ())) for b in rig["bodies"])
    st = rig.get("settings", {})
    dt, hz = float(st.get("dt", 0.0005)), float(st.get("collision_hz", 120.0))
    interval = max(1, math.ceil(1.0 / (max(hz, 1.0) * dt) - 1e-6))
    return {"bytes_per_search": 120 * contacters + 48 * tris + 12 * pairs, "contacter_nodes": contacters, "triangles": tris,
            "searches_per_substep": len(range(0, FRAME, interval)) / FRAME}


def workload(name: str, rank: int):
    from beamlab_b200 import rigs
    if name == "fleet256":
        rig = rigs.fleet(256, seed=3 + rank, layout="pairs")
        n, m = rigs.rig_counts(rig)
        nt = sum(len(b.get("tris", ())) for b in rig["bodies"])
        desc = (f"fleet256: 256 lattice vehicles ({n:,} nodes, {m:,} beams, {nt:,} collision triangles; log-normal "
                f"500-20,000 nodes, median 3,000), 2048^2-sample 1 km^2 heightfield (two octaves of value noise, 2 m), "
                f"5-30 m/s, laid out in 128 head-on pairs on random axes that crash within their first 0.12 s, "
                f"inter-vehicle node-triangle contacts (islands, pair search every 17 substeps); 4 wheel rings of 24 "
                f"tyre nodes a vehicle (free rolling, tyre patches sharing grip)")
    elif name == "plate64":
        rig = rigs.shell_plate(63, seed=1 + rank)
        n, m = rigs.rig_counts(rig)
        desc = ("plate64: co-rotational FEM shell plate, 64 x 64 nodes (4,096), 7,938 CST/DKT triangles, 1 m x 1 m, "
                "1.5 mm steel (E 210 GPa, nu 0.3, 7,850 kg/m^3), one edge clamped, a seeded 500 N point load, gravity; "
                "implicit step every substep: 64,411 off-diagonal 6x6 blocks, 1,359,082 block updates")
    elif name == "shellcar":
        rig = rigs.shell_body(50000, seed=1 + rank)
        n, m = rigs.rig_counts(rig)
        b = rig["bodies"][0]
        desc = (f"shellcar: a procedural box-and-pillar shell car body ({n:,} nodes, {len(b['fem_tris']):,} CST/DKT "
                f"triangles of 0.8-2.0 mm steel in six welded panels, {len(b['fem_members']):,} members: spot welds every "
                f"5 cm and tube pillars), floating under gravity and two point loads; implicit step every substep")
    elif name == "truss_car":
        rig = rigs.truss_car(1 + rank)
        n, m = rigs.rig_counts(rig)
        desc = f"truss_car: 20x4x5 lattice ({n} nodes, {m} beams) at 15 m/s into a rigid wall"
    else:
        raise SystemExit(f"unknown workload {name}")
    return rig, n, m, desc


class ClockSampler:
    """nvidia-smi samples of the GPU's clocks and throttle reasons every 200 ms while running."""

    FIELDS = ("clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.hw_slowdown",
              "clocks_event_reasons.hw_thermal_slowdown", "clocks_event_reasons.sw_thermal_slowdown",
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: str | None):
        self.gpu, self.lines, self.proc = gpu, [], None

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={','.join(self.FIELDS)}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.gpu:
            cmd += ["-i", self.gpu]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=lambda: self.lines.extend(iter(self.proc.stdout.readline, "")), daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def stop(self) -> dict | None:
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 7:
                continue
            try:
                sm.append(float(p[0]))
                smax = max(smax, float(p[1]))
            except ValueError:
                continue
            for nm, v in zip(names, p[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def fp64_peak(device: int) -> float:
    """The GPU's fp64 rate measured here (TFLOP/s): a cuBLAS DGEMM of 8192^3 through torch, CUDA events, best of 5."""
    import torch
    a = torch.randn(8192, 8192, dtype=torch.float64, device=f"cuda:{device}")
    b = torch.randn_like(a)
    best = float("inf")
    for _ in range(6):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2 * 8192 ** 3 / (best * 1e-3) / 1e12


def traffic_per_unit():
    """DRAM bytes per beam / per node of the two substep kernels from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    return json.load(open(path)) if os.path.exists(path) else {}


def cpu_reference(rig, n_nodes, budget_s=10.0, max_frames=100, warm=4, frame=FRAME):
    """The reference's own step (compiled from its sources, Release flags) on all host cores: node-substeps/s of a
    bounded sample (warm-up substeps, then frames of `frame` substeps of the same workload until about budget_s
    seconds have passed, at least 2 and at most max_frames)."""
    from oracle.oracle import RefWorld, build_world, ref_available, ref_jobs_init, ref_jobs_shutdown
    if not ref_available("timing"):
        return None
    cores = os.cpu_count() or 1
    threads = ref_jobs_init(max(0, cores - 1), "timing")
    w = build_world(RefWorld, rig, flavour="timing", multithreaded=True)
    w.step_substeps(warm)
    t0 = time.perf_counter()
    frames = 0
    while frames < 2 or (frames < max_frames and time.perf_counter() - t0 < budget_s):
        w.step_substeps(frame)
        frames += 1
    dt = time.perf_counter() - t0
    w.close()
    ref_jobs_shutdown("timing")
    return {"value": n_nodes * frame * frames / dt, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"the same workload, {frames} frames of {frame} substeps after {warm} warm-up substeps "
                      f"({frames * frame} substeps, {dt:.2f} s)"}


def fem_solvers(device: int, frames: int = 2, make=None, label: str = "shell_plate(63, seed=2)"):
    """The implicit step by each solver (include/beamlab_gpu.h: fem_solver), on a load the network was not trained on
    (make(seed 2); default the 64 x 64 plate): ms a substep (CUDA events of a profiled frame), CG iterations a solve,
    fallbacks, the largest relative residual of a solution the step took. The network is trained first on 200
    substeps of the Cholesky's solves of another load (make(seed 1); 12 epochs of Adam)."""
    from beamlab_b200 import rigs, world_from_rig
    make = make or (lambda seed: rigs.shell_plate(63, seed=seed))
    rec = world_from_rig(make(1), device=device)
    nf = len(rec.bodies()[0].fem()["node"])
    rec.mlp_record(200 * nf)
    for _ in range(10):
        rec.step_substeps(20)
    rec.mlp_record(0)
    t0 = time.perf_counter()
    rec.mlp_train(1, batch=4096, lr=2e-3, seed=0)
    loss = rec.mlp_train(12, batch=4096, lr=1e-3, seed=1)
    train_s = time.perf_counter() - t0
    weights = rec.mlp_weights()
    rec.close()
    out = {"load": label, "training": {"samples": 200 * nf, "epochs": 13, "loss": loss, "seconds": train_s}}
    for solver in ("cholesky", "pcg", "pcg_previous", "pcg_learned"):
        w = world_from_rig(make(2), device=device, fem_solver=solver, pcg_max_iters=3000, fem_check_residual=True)
        if solver == "pcg_learned":
            w.set_mlp_weights(weights)
        w.step_substeps(FRAME)  # (warm-up: the graph is captured)
        ms = 0.0
        for _ in range(frames):
            ms += w.profile_frame(FRAME)["frame_ms"]
        st = w.fem_stats()
        out[solver] = {"ms_per_substep": ms / (frames * FRAME), "max_residual": st["max_residual"],
                       "cg_iterations_per_solve": st["pcg_iterations"] / st["pcg_solves"] if st["pcg_solves"] else None,
                       "fallbacks": st["pcg_fallbacks"]}
        w.close()
    return out


def plain_gpu(rig, device: int, stream, sample_every: int = 8, frames: int = 3):
    """The plain per-instance GPU path the batched one is measured against: every sample_every-th vehicle of the
    workload in a World of its own (its own context, the same terrain), the worlds stepped one after another on one
    stream, each frame's kernels launched one by one (graphs off) - and, for reference, the same with each world's
    frame replayed as a CUDA graph. node-substeps/s of the sample (CUDA events on the stream)."""
    import torch
    from beamlab_b200 import world_from_rig
    sample = rig["bodies"][::sample_every]
    nodes = sum(len(b["mass"]) for b in sample)
    out = {"sample": f"{len(sample)} of the {len(rig['bodies'])} vehicles (every {sample_every}th: {nodes:,} nodes), "
                     f"{frames} frames of {FRAME} substeps each, a World per vehicle"}
    for key, graphs in (("launches", False), ("graphs", True)):
        worlds = [world_from_rig({"settings": rig["settings"], "statics": rig["statics"], "bodies": [b]}, device=device,
                                 graphs=graphs) for b in sample]
        for w in worlds:  # (warm-up: commits, and captures the graph where on)
            w.step_substeps(FRAME, stream)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(frames):
            for w in worlds:
                w.step_substeps(FRAME, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out[key] = {"value": nodes * FRAME * frames / (ms * 1e-3), "unit": UNIT, "ms_per_frame": ms / frames}
        for w in worlds:
            w.close()
    return out


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def aggregate(ms: float, ms_e2e: float, n_nodes: int, ws: int, device="cuda"):
    """The whole job's figures over the ranks: the slowest rank's timed regions (resident, end to end) and the nodes
    every rank stepped (each rank its own fleet: weak scaling, no data-path collective)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms, ms_e2e], dtype=torch.float64, device=device)
    units = torch.tensor([float(n_nodes)], dtype=torch.float64, device=device)
    if ws > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(units, op=dist.ReduceOp.SUM)
        dist.barrier()
    return float(t[0]), float(t[1]), float(units[0])


def run_reference(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return
    rig, n, m, desc = workload(args.workload, 0)
    from oracle.oracle import RefWorld, build_world, ref_available, ref_jobs_init, ref_jobs_shutdown
    base = {"metric": METRIC, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc, "frame_substeps": FRAME}}
    if not ref_available("timing"):
        print(json.dumps({"impl": "reference", "unavailable": "the reference's CPU build (oracle/_ref) is missing"}),
              flush=True)
        return
    cores = os.cpu_count() or 1
    threads = ref_jobs_init(max(0, cores - 1), "timing")
    w = build_world(RefWorld, rig, flavour="timing", multithreaded=True)
    frame = 1 if args.workload == "shellcar" else FRAME  # (the shell body's reference step takes seconds)
    for _ in range(args.warmup):
        w.step_substeps(frame)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        w.step_substeps(frame)
    dt = time.perf_counter() - t0
    v = n * frame * args.steps / dt
    w.close()
    ref_jobs_shutdown("timing")
    base.update({"value": v, "ms_per_step": dt * 1e3 / args.steps, "scaling": "weak", "vs_baseline": None,
                 "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                 "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "reference",
                                  "sample": f"the whole workload, {args.steps} frames of {frame} substeps"}})
    print(json.dumps(base), flush=True)


def run_gpu(args):
    import torch
    import torch.distributed as dist
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    from beamlab_b200 import NODE_DTYPE, world_from_rig
    rig, n, m, desc = workload(args.workload, rank)
    # two worlds of the same rig: `w` for the resident measurement, `we` for the end-to-end one; both are warmed up by
    # the same W frames, so the two measurements time the same K frames of the same simulation (in a crash the work
    # changes from frame to frame)
    w = world_from_rig(rig, device=local)
    we = world_from_rig(rig, device=local)
    stream = torch.cuda.Stream()
    K, W = args.steps, args.warmup

    # warm-up: every graph used below is captured here (plain frames, the profiled frame)
    for _ in range(max(W - 1, 0)):
        w.step_substeps(FRAME, stream)
        we.step_substeps(FRAME, stream)
    w.profile_frame(FRAME, stream)
    we.step_substeps(FRAME, stream)
    torch.cuda.synchronize()
    st0 = w.stats()

    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid)
    clocks.start()
    time.sleep(0.3)

    # ---- resident: K frames, the last one profiled (CUDA events between its kernels)
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(K - 1):
        w.step_substeps(FRAME, stream)
    prof = w.profile_frame(FRAME, stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    st1 = w.stats()

    # ---- end to end through the C ABI: the node state in from pinned host memory and out again every frame
    host = torch.empty(n * NODE_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True)
    hbuf = np.frombuffer(host.numpy(), dtype=NODE_DTYPE)
    we.download_all_nodes(hbuf, stream)
    stream.synchronize()
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(K):
        we.upload_all_nodes(hbuf, stream)
        we.step_substeps(FRAME, stream)
        we.download_all_nodes(hbuf, stream)
    f1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = f0.elapsed_time(f1)
    clk = clocks.stop()

    ms, ms_e2e, total_nodes = aggregate(ms, ms_e2e, n, ws, "cuda")
    if rank == 0:
        value = total_nodes * FRAME * K / (ms * 1e-3)
        e2e = total_nodes * FRAME * K / (ms_e2e * 1e-3)
        peak, pk_kind = peaks()
        per = {k: prof[f"{k}_ms"] / FRAME for k in ("search", "beams", "force", "contacts", "integrate", "fem")}
        # algorithmic bytes a launch (each array touched once): k_beams 40 B a beam; k_force reads a node's position
        # and mass and writes its force (32 B a node; the beams' scalars and the neighbours' positions it gathers are
        # the scratch and the L2-resident gathers of the substep); k_integrate reads p, v, 1/m, the force (44 B) and
        # writes p, v (24 B); the substep as a whole: 40 B a beam + 52 B a node (the force never leaving the chip)
        kern = {"k_beams": (BYTES_PER_BEAM * m, per["beams"], m, "beam"), "k_force": (32 * n, per["force"], n, "node"),
                "k_integrate": (68 * n, per["integrate"], n, "node")}
        fem_info = None
        if args.workload in ("plate64", "shellcar"):
            # the implicit FEM step: its factor (diagonal and off-diagonal 6x6 blocks of doubles) and right side each
            # read and written once a substep
            fs = w.fem_stats()
            fem_bytes = 2 * 8 * (36 * fs["columns"] + 36 * fs["blocks"] + 6 * fs["columns"])
            kern["fem_step"] = (fem_bytes, per["fem"], fs["columns"], "column")
            fp64 = fp64_peak(local)
            gf = fs["factor_flops"] / (per["fem"] * 1e-3) / 1e9
            fem_info = {"columns": fs["columns"], "blocks": fs["blocks"], "block_updates": fs["updates"],
                        "factorization": "multifrontal" if fs["fronts"] > 0 else "block columns",
                        "fronts": fs["fronts"], "levels": fs["levels"], "ms_per_substep": per["fem"],
                        "factor_gflop": fs["factor_flops"] / 1e9,
                        "gflops_fp64": gf, "fp64_peak_tflops": fp64, "fp64_frac": gf / (fp64 * 1e3),
                        "fp64_peak_source": "measured here: cuBLAS DGEMM 8192^3 (torch float64 matmul), CUDA events"}
        dom = max(kern, key=lambda k: kern[k][1])
        alg_bytes, kms, units_, unit_name = kern[dom]
        achieved = alg_bytes / (kms * 1e-3) / 1e9
        tr = traffic_per_unit().get(dom)
        traffic = tr[f"dram_bytes_per_{unit_name}"] * units_ if tr else None
        sub_ms = per["beams"] + per["force"] + per["integrate"]
        substep = {"algorithmic_bytes": BYTES_PER_BEAM * m + BYTES_PER_NODE * n, "ms": sub_ms,
                   "achieved_gbs": (BYTES_PER_BEAM * m + BYTES_PER_NODE * n) / (sub_ms * 1e-3) / 1e9}
        substep["frac"] = substep["achieved_gbs"] / peak
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": W,
            "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": desc, "frame_substeps": FRAME, "step": f"one frame of {FRAME} substeps",
                       "l2": "inputs larger than L2 (the fleet's device state is about 0.8 GB)",
                       "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                       "kernel_ms_per_substep": {"pair_search": per["search"], "k_beams": per["beams"], "k_force": per["force"],
                                                 "contacts": per["contacts"], "k_integrate": per["integrate"],
                                                 "fem": per["fem"],
                                                 "frame_begin_finish": (prof["begin_ms"] + prof["finish_ms"]) / FRAME}},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": n * NODE_DTYPE.itemsize,
                    "d2h_bytes_per_step": n * NODE_DTYPE.itemsize},
            "gpu_launches": int(st1["kernel_launches"] - st0["kernel_launches"]),
            "contacts": {"applied": int(st1["contacts"] - st0["contacts"]), "pair_searches": int(st1["pair_searches"] - st0["pair_searches"]),
                         "device_errors": int(st1["device_errors"])},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": f"{pk_kind} hbm_gbs",
                         "algorithmic_bytes_per_launch": alg_bytes, "traffic": traffic, "substep_kernels": substep},
            "clocks": clk,
        }
        if fem_info is not None:
            out["fem_step"] = fem_info
        if st1["contacts"] > st0["contacts"]:
            # the contacts between bodies: the narrow phase reads a node and its triangle's three nodes a pair (about
            # 64 B a pair a substep); the response runs each island's contacts level by level of their order (a level:
            # contacts that share no node), so its time is the deepest island's levels x one contact's dependent
            # arithmetic - latency-bound rather than HBM-bound
            pairs = len(w.pairs())
            frames_timed = K
            bp = broadphase_bytes(rig, pairs)
            search_gbs = (bp["bytes_per_search"] * bp["searches_per_substep"] / (per["search"] * 1e-3) / 1e9
                          if per["search"] > 0 else None)
            out["contacts_step"] = {
                "pairs_last_search": pairs, "contacts_per_substep": (st1["contacts"] - st0["contacts"]) / (frames_timed * FRAME),
                "ms_per_substep": per["contacts"], "pair_search_ms_per_substep": per["search"],
                "narrow_phase_bytes_per_substep": 64 * pairs,
                "achieved_gbs": 64 * pairs / (per["contacts"] * 1e-3) / 1e9 if per["contacts"] > 0 else None,
                "bound": "latency (the deepest island's levels of dependent contacts)",
                "pair_search": {**bp, "achieved_gbs": search_gbs,
                                "bound": "latency (an island's set-up in the reference's order, then every query at once)"}}
        if ws == 1 and args.workload == "plate64" and not args.no_solvers:
            out["fem_solvers"] = fem_solvers(local)
        if ws == 1 and args.workload == "shellcar" and not args.no_solvers:
            from beamlab_b200 import rigs as _rigs
            out["fem_solvers"] = fem_solvers(local, make=lambda seed: _rigs.shell_body(10000, seed=seed),
                                             label="shell_body(10000, seed=2)")
        if ws == 1 and args.workload == "fleet256" and not args.no_plain:
            pl = plain_gpu(rig, local, stream)
            pl["batched_over_plain"] = value / pl["launches"]["value"]
            out["plain_gpu"] = pl
        if ws == 1 and not args.no_cpu_baseline:
            # (the shell body's reference step takes seconds: a sample of single substeps)
            out["cpu_baseline"] = (cpu_reference(rig, n, warm=1, frame=1) if args.workload == "shellcar"
                                   else cpu_reference(rig, n))
        print(json.dumps(out), flush=True)
    if ws > 1:
        dist.destroy_process_group()
    w.close()
    we.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="fleet256", choices=["fleet256", "plate64", "shellcar", "truss_car"])
    ap.add_argument("--no-solvers", action="store_true", help="skip the shell car's comparison of FEM solvers")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain per-instance GPU path's measurement")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be at least 3")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
