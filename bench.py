#!/usr/bin/env python
"""Benchmark of the isosurface-extraction path on B200.

Workload (one step): the 1024^3 uint16 fBm ball (block 8^3) extracted at
isovalues 16384, 32768 and 49152 as three separate plain extractions, each
min/max + octree -> filter + compaction -> PMB count -> PMB emit, with the
volume already resident in HBM (2 GiB, larger than L2, so every extraction
streams it from DRAM).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mtx|reference]

With N > 1 it is launched by torchrun, one rank per GPU; every rank extracts
its own copy of the workload (independent replicas, weak scaling) and the
step time is the maximum over ranks.  `--impl reference` times the CPU
restatement of meshtrex's path (the oracle, all host threads) on a bounded
z-slab sample of the same workload.

Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402
import torch  # noqa: E402

METRIC = "Gvoxels/s + tris/s vs HBM roofline: plain vs batched; bwd/fwd time ratio"
N = 1024  # volume edge; --size changes it for profiling runs only
BLOCK = 8
ISOS = (16384.0, 32768.0, 49152.0)
def workload():
    return (f"plain {N}^3 uint16 fBm ball, block 8^3, isovalues 16384/32768/49152 as three "
            "separate plain extractions per step")
FALLBACK_HBM_GBS = 6650.0


# ------------------------------------------------------------------ infra
def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(t_local: float, ws: int, device: str = "cuda") -> float:
    """The step time of the whole job: the slowest rank's (one all-reduce; every
    rank calls it at the same point)."""
    if ws <= 1:
        return t_local
    import torch.distributed as dist
    tt = torch.tensor([t_local], device=device, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def job_throughput(units_per_rank: float, ws: int, t_max: float) -> float:
    """Whole-job throughput: every rank processed units_per_rank (replicas,
    weak scaling) in the slowest rank's time."""
    return ws * units_per_rank / t_max


def peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons over a window."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons, n = [], None, set(), 0
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax = float(parts[2])
                except ValueError:
                    continue
                n += 1
                for name, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(name)
        os.remove(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": n}


def relaunch_ranks(gpus: int, argv) -> int | None:
    """`--gpus N` (N > 1) run without torchrun around it: start N ranks of this
    script under torchrun on this node (rendezvous on 127.0.0.1), with the same
    arguments, and return their exit code.  None when there is nothing to do
    (N = 1, or already a rank of a torchrun job)."""
    if gpus <= 1 or os.environ.get("WORLD_SIZE"):
        return None
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + list(argv)
    try:
        return subprocess.run(cmd, timeout=3600).returncode
    except subprocess.TimeoutExpired:
        return 124


def nproc():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# --------------------------------------------------------------- CPU side
def bench_config(ws):
    """The workload description both arms print (the same keys and values)."""
    return {"workload": workload(), "volume": [N, N, N], "block": BLOCK, "isovalues": list(ISOS),
            "l2": "inputs larger than L2 (2 GiB volume streamed per extraction)",
            "parallelism": f"replicas x{ws}" if ws > 1 else "single device"}


def cpu_sample_volume(nz: int, device: str):
    """Middle z-slab of nz slices of the 1024^3 workload, as a host array."""
    from meshtrex_b200 import synth
    z0 = (N - nz) // 2
    t = synth.fbm_ball(N, seed=1, device=device, zslab=(z0, z0 + nz))
    return t.cpu().view(torch.int16).numpy().view(np.uint16), z0


def time_cpu_oracle(vol: np.ndarray, threads: int):
    """One step of meshtrex's CPU path as the oracle restates it, on `vol`:
    for each of the three isovalues, min/max over the (B+1)^3 blocks
    (testMinMax.h:28-135), ordered compaction (blockFilteringTestUtils.h:438-478)
    and PMB marching cubes with the vertex and index buffers written
    (extractionTestUtils.cpp:34-36 for the vertex placement).  Returns
    (seconds, triangles, meshes)."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    tris, meshes = 0, []
    for iso in ISOS:
        m = O.extract(vol, BLOCK, iso, nthreads=threads)
        tris += m.n_triangles
        meshes.append(m)
    return time.perf_counter() - t0, tris, meshes


def cpu_run(vol: np.ndarray, threads: int, target_s: float, what: str):
    """The oracle timed on `threads` host cores on `vol`, repeated to ~target_s."""
    secs, tris, reps = 0.0, 0, 0
    while reps == 0 or (secs < target_s and reps < 20):
        s, t, _ = time_cpu_oracle(vol, threads)
        secs += s
        tris += t
        reps += 1
    vox = 3 * vol.size * reps
    return {"value": vox / secs / 1e9, "unit": "Gvoxels/s", "cores": threads, "kind": "port",
            "sample": (f"{what}: {vol.shape[2]}x{vol.shape[1]}x{vol.shape[0]} uint16 at the three isovalues, "
                       f"min/max + compaction + marching cubes with vertices and indices written, "
                       f"{reps} repetition(s), {secs:.2f} s"),
            "tris_per_s": tris / secs}


def cpu_baselines(host: np.ndarray, dev: str):
    """All host threads on the whole volume, and one thread (meshtrex's CPU path
    is single-threaded) on a middle z-slab sized for about 10 s."""
    threads = nproc()
    allcore = cpu_run(host, threads, 10.0, "whole volume")
    probe, _ = cpu_sample_volume(32, dev)
    s1, _, _ = time_cpu_oracle(probe, 1)
    nz = int(max(16, min(N, 32 * 10.0 / max(s1, 1e-3))) // 8 * 8)
    slab, z0 = cpu_sample_volume(nz, dev)
    one = cpu_run(slab, 1, 10.0, f"middle z-slab z={z0}..{z0 + nz}")
    return allcore, one


def oracle_parity(host: np.ndarray, exts, threads: int):
    """The oracle's full mesh of every isovalue of the step, on the same host
    bytes as the GPU's volume, against the GPU's outputs bit for bit: active
    blocks, vertex and triangle counts, vertex bits and index buffers."""
    import hashlib
    from oracle import oracle as O
    per_iso = []
    ok = True
    for iso, e in zip(ISOS, exts):
        c = e.counters.cpu().numpy().view(np.uint32)
        V, T = int(c[0]), int(c[1]) // 3
        ref = O.extract(host, BLOCK, iso, nthreads=threads)
        gv = e.vertices[:V].cpu().numpy()
        gi = e.indices[:T].cpu().numpy().view(np.uint32)
        same = (int(c[4]) == 0 and int(c[3]) == len(ref.ids) and V == ref.n_vertices and T == ref.n_triangles
                and np.array_equal(gv.view(np.uint32), ref.xyz.view(np.uint32))
                and np.array_equal(gi, ref.indices))
        ok = ok and same
        h = hashlib.sha256()
        h.update(gv.tobytes())
        h.update(gi.tobytes())
        per_iso.append({"isovalue": iso, "active_blocks": int(c[3]), "vertices": V, "triangles": T,
                        "mesh_sha256": h.hexdigest()[:16], "match": bool(same)})
    return {"oracle_match": bool(ok), "per_isovalue": per_iso,
            "what": "oracle (CPU restatement, all host threads) on the same host bytes; active-block count, V, T, "
                    "vertex float bits and index buffer compared exactly"}


def run_reference(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    threads = nproc()
    # calibrate the sample so that one step is ~10 s of CPU work and the run ~150 s
    probe, _ = cpu_sample_volume(min(N, 64), dev)
    secs, _, _ = time_cpu_oracle(probe, threads)
    pz = probe.shape[0]
    total_steps = args.steps + args.warmup
    budget = 150.0  # seconds for the whole run
    nz = int(min(N, pz * 10.0 / max(secs, 1e-3), pz * budget / max(secs * total_steps, 1e-3)))
    nz = max(16, (nz // 8) * 8)
    vol, z0 = cpu_sample_volume(nz, dev)
    for _ in range(args.warmup):
        time_cpu_oracle(vol, threads)
    t_all, tris_all = 0.0, 0
    for _ in range(args.steps):
        s, t, _ = time_cpu_oracle(vol, threads)
        t_all += s
        tris_all += t
    vox = 3 * vol.size * args.steps
    value = vox / t_all / 1e9
    line = {"metric": METRIC, "impl": "reference", "value": value, "unit": "Gvoxels/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * t_all / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16",
            "data": "synthetic (seeded fBm ball, same generator as the GPU arm)",
            "config": bench_config(ws),
            "tris_per_s": tris_all / t_all,
            "cpu_baseline": {"value": value, "unit": "Gvoxels/s", "cores": threads, "kind": "port",
                             "sample": (f"1024x1024x{nz} middle z-slab (z={z0}..{z0 + nz}) per step, 3 isovalues, "
                                        "min/max + compaction + marching cubes with vertices and indices written")},
            "e2e": {"value": value, "unit": "Gvoxels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------- GPU side
def launches_per_extraction(grid, shape_zyx=None, esz=2, block=BLOCK):
    """Kernel launches of one plain extraction: leaf min/max (with the strip-column
    patch when the TMA leaf pass covers more than one 512-byte x-strip), octree,
    filter, count + scan, emit."""
    m = max(grid)
    levels = 1
    while m > 1:
        m >>= 1
        levels += 1
    patch = 0
    if shape_zyx is not None:
        X = shape_zyx[2]
        tma_leaf = esz >= 2 and (X * esz) % 16 == 0 and block in (4, 8, 16)
        patch = 1 if tma_leaf and X * esz > 512 else 0
    return 1 + patch + (1 if levels > 1 else 0) + 1 + 2 + 1


def read_traffic():
    """DRAM bytes per 1024^3 min/max launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "minmax_leaf_u16_b8.txt")
    try:
        for line in open(p):
            if line.startswith("dram_bytes_per_launch_1024^3:"):
                return float(line.split(":")[1])
    except Exception:
        pass
    return None


def run_mtx(args):
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from meshtrex_b200 import api, synth

    vol = load_or_make_volume(args.cache)
    torch.cuda.synchronize()
    ctx = api.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream)

    # size the outputs from one drop-in extraction per isovalue
    caps = []
    for iso in ISOS:
        m = api.extract(vol, BLOCK, iso, ctx=ctx)
        caps.append((m.vertices.shape[0], m.indices.shape[0], m.active_ids.shape[0]))
        del m
    exts = [api.AsyncExtractor(ctx, vol, BLOCK, iso, v + 1024, t + 1024, max_active_blocks=a + 1024)
            for iso, (v, t, a) in zip(ISOS, caps)]
    # the timed step: the three extractions are independent, so each runs on its
    # own stream with its own context, and one's emit overlaps the next one's
    # min/max streaming
    xstreams = [torch.cuda.Stream() for _ in ISOS]
    xctxs = [api.Context(local, stream=s_) for s_ in xstreams]
    pexts = [api.AsyncExtractor(c_, vol, BLOCK, iso, v + 1024, t + 1024, max_active_blocks=a + 1024)
             for c_, iso, (v, t, a) in zip(xctxs, ISOS, caps)]

    def serial_step():
        for e in exts:
            e.run()

    def step():
        start = torch.cuda.Event()
        start.record(stream)
        for s_, e in zip(xstreams, pexts):
            s_.wait_event(start)
            e.run()
        for s_ in xstreams:
            done = torch.cuda.Event()
            done.record(s_)
            stream.wait_event(done)

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    for _ in range(max(3, args.warmup)):
        step()
        serial_step()
    ctx.synchronize()

    # per-stage times (and the dominant kernel's roofline) from serial steps,
    # where the stages do not overlap
    prof = api.Profiler(ctx)
    ctx.set_profiler(prof)
    prof.begin_frame()
    pstats = max(3, min(10, args.steps))
    for _ in range(pstats):
        serial_step()
    prof.end_frame()
    ctx.set_profiler(None)
    regions = prof.regions()
    prof.close()
    ctx.synchronize()

    clocks = Clocks(local)
    clocks.start()
    # keep the GPU busy for >= 1 s before the timed steps so the clock samples see load
    t_soak = time.perf_counter()
    while time.perf_counter() - t_soak < 1.0:
        step()
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    ctx.synchronize()  # raises on any device-side error
    for c_ in xctxs:
        c_.synchronize()
    ms = e0.elapsed_time(e1)
    t_local = ms / 1000.0
    t_max = max_over_ranks(t_local, ws)
    counters = [e.counters.cpu().numpy().view(np.uint32) for e in pexts]
    for c, e, pe in zip(counters, exts, pexts):
        assert c[4] == 0, f"device status {c[4]}"
        ref = e.counters.cpu().numpy().view(np.uint32)
        V_, I_ = int(c[0]), int(c[1])
        assert (V_, I_) == (int(ref[0]), int(ref[1]))
        assert torch.equal(pe.vertices[:V_].view(torch.int32), e.vertices[:V_].view(torch.int32))
        assert torch.equal(pe.indices[: I_ // 3], e.indices[: I_ // 3])
    V = [int(c[0]) for c in counters]
    T = [int(c[1]) // 3 for c in counters]
    pexts = None
    for c_ in xctxs:
        c_.close()
    xctxs = xstreams = None
    nvox = N ** 3
    steps = args.steps
    value = job_throughput(3 * nvox * steps, ws, t_max) / 1e9
    tris_s = job_throughput(sum(T) * steps, ws, t_max)

    # one profiler frame covers the serial steps: per-extraction stage times
    per_stage = {k: regions[k][0] / (3 * pstats) for k in regions}
    peak, peak_kind = peak_hbm()
    leaf_ms = per_stage.get("MinMax_Leaf_Pass")
    grid = ((N + BLOCK - 1) // BLOCK,) * 3
    nblocks = grid[0] * grid[1] * grid[2]
    leaf_bytes = nvox * 2 + nblocks * 8
    achieved = leaf_bytes / (leaf_ms / 1000.0) / 1e9 if leaf_ms else None
    traffic = read_traffic()
    step_bytes = 3 * nvox * 2 + sum(v * 12 + t * 12 for v, t in zip(V, T))
    pipe_gbs = step_bytes * steps / t_local / 1e9

    line = {"metric": METRIC, "value": value, "unit": "Gvoxels/s", "n_gpus": ws, "steps": steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * t_max / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u16",
            "data": "synthetic (seeded fBm ball generated on the device; no dataset)",
            "config": bench_config(ws),
            "streams": "the step's 3 extractions on 3 streams (one context each)",
            "tris_per_s": tris_s, "vertices_per_step": sum(V), "triangles_per_step": sum(T),
            "stages_ms_per_extraction": per_stage,
            "roofline": {"bound": "hbm", "kernel": "minmax_leaf_tma_kernel<uint16_t,8>",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None,
                         "traffic": traffic, "algorithmic_bytes": leaf_bytes, "peak_kind": f"{peak_kind} (burst copy)"},
            "pipeline_roofline": {"achieved": pipe_gbs, "peak": peak, "unit": "GB/s", "frac": pipe_gbs / peak,
                                  "bytes_per_step": step_bytes,
                                  "what": "volume read once per extraction + mesh written (12 B/vertex, 12 B/triangle)"},
            "gpu_launches": launches_per_extraction(grid, (N, N, N), 2, BLOCK) * 3 * steps,
            "clocks": clk}

    if rank == 0 and not args.no_cpu:
        host = vol.cpu().view(torch.int16).numpy().view(np.uint16)
        line["parity"] = oracle_parity(host, exts, nproc())
        if ws == 1:
            allcore, one = cpu_baselines(host, "cuda")
            line["cpu_baseline"] = allcore
            line["cpu_baseline_1thread"] = one
        del host

    if not args.no_e2e:
        line["e2e"] = run_e2e(ctx, vol, ws, steps=max(1, min(3, steps)))

    if not args.no_batch:
        del exts
        line["batched"] = run_batched(ctx, stream, steps=max(3, min(20, steps)), scale_down=args.batch_scale,
                                      fixed=args.batch_fixed, with_cpu=not args.no_cpu)

    if not args.no_backward:
        line["backward"] = run_backward(ctx, stream, steps=max(3, min(20, steps)))

    if not args.no_cpu and rank == 0:
        line["blobs"] = run_blobs(ctx, stream, steps=max(3, min(20, steps)))

    if not args.no_gyroid:
        exts = vol = None  # release the 1024^3 volume and its outputs first
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        line["gyroid"] = run_gyroid(ctx, stream, steps=max(3, min(10, steps)), n=args.gyroid_size,
                                    fixed=args.gyroid_fixed, with_cpu=not args.no_cpu and rank == 0)

    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


def load_or_make_volume(cache):
    """The fBm ball on the device; with --cache, read from / saved to a raw file."""
    from meshtrex_b200 import synth
    if cache and os.path.exists(cache) and os.path.getsize(cache) == 2 * N ** 3:
        a = np.fromfile(cache, dtype=np.int16).reshape(N, N, N)
        return torch.from_numpy(a).cuda().view(torch.uint16)
    vol = synth.fbm_ball(N, seed=1, device="cuda")
    if cache:
        vol.cpu().view(torch.int16).numpy().tofile(cache)
    return vol


def run_e2e(ctx, vol_dev, ws, steps):
    """The drop-in C-ABI path from pinned host memory.  Each step takes its
    input volume from pinned host memory once, with
    mtx_upload_compute_min_max_mip (z-slabs on a copy stream, the first
    extraction's leaf min/max consuming each slab as it lands), then runs the
    three extractions through computeMinMaxMip (the second and third, on the
    resident volume), filterActiveBlocks, readActiveBlockCount and
    extractMeshletDescriptors, and copies every mesh to pinned host memory.
    Two contexts alternate between steps: step k + 1's upload is enqueued when
    step k begins, so that it crosses PCIe while step k is extracted and read
    back.  One untimed step warms the allocations."""
    from meshtrex_b200 import api
    t = torch.empty(vol_dev.numel() * vol_dev.element_size(), dtype=torch.uint8, pin_memory=True)
    t.copy_(vol_dev.view(torch.uint8).reshape(-1))
    host = t.numpy().view(np.uint16).reshape(N, N, N)
    local = torch.cuda.current_device()
    streams = [torch.cuda.Stream() for _ in range(2)]
    ctxs = [api.Context(local, stream=s_) for s_ in streams]
    out_v = [torch.empty(1, dtype=torch.float32, pin_memory=True) for _ in ISOS]
    out_i = [torch.empty(1, dtype=torch.int32, pin_memory=True) for _ in ISOS]
    pcs = [api.push_constants((N, N, N), BLOCK, iso) for iso in ISOS]

    def upload(k):
        c_ = ctxs[k % 2]
        return api.upload_compute_min_max_mip(c_, host, pcs[0])

    def extract_step(k, v, mm0, prefetch):
        c_, s_ = ctxs[k % 2], streams[k % 2]
        nxt = upload(k + 1) if prefetch else None
        h2d, d2h, live = v.data.size, 0, []
        for j, pc in enumerate(pcs):
            mm = mm0 if j == 0 else api.compute_min_max_mip(c_, v, pc)
            f = api.filter_active_blocks(c_, mm, pc)
            api.read_active_block_count(c_, f)
            x = api.extract_meshlet_descriptors(c_, mm, f, pc)
            nv, ni = x.out.vertexBuffer.size, x.out.indexBuffer.size
            if out_v[j].numel() * 4 < nv:
                out_v[j] = torch.empty(nv // 4 + 1, dtype=torch.float32, pin_memory=True)
            if out_i[j].numel() * 4 < ni:
                out_i[j] = torch.empty(ni // 4 + 1, dtype=torch.int32, pin_memory=True)
            with torch.cuda.stream(s_):  # device -> pinned host copies of the mesh, on the extraction's stream
                if nv:
                    out_v[j][: nv // 4].copy_(api.device_view(x.out.vertexBuffer.ptr, (nv // 4,), torch.float32),
                                              non_blocking=True)
                if ni:
                    out_i[j][: ni // 4].copy_(api.device_view(x.out.indexBuffer.ptr, (ni // 4,), torch.int32),
                                              non_blocking=True)
            d2h += nv + ni
            live.append((mm, f, x))
        s_.synchronize()  # the step's meshes are on the host
        for mm, f, x in live:
            x.free()
            f.free()
            mm.free()
        api.free_volume(c_, v)
        return nxt, h2d, d2h

    nxt = upload(0)
    extract_step(0, *nxt, prefetch=False)  # untimed
    torch.cuda.synchronize()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    h2d = d2h = 0
    t0 = time.perf_counter()
    cur = upload(0)
    for k in range(steps):
        cur, a_, b_ = extract_step(k, *cur, prefetch=k + 1 < steps)
        h2d += a_
        d2h += b_
    torch.cuda.synchronize()
    t = max_over_ranks(time.perf_counter() - t0, ws)
    for c_ in ctxs:
        c_.close()
    return {"value": job_throughput(3 * N ** 3 * steps, ws, t) / 1e9, "unit": "Gvoxels/s",
            "h2d_bytes_per_step": h2d // steps, "d2h_bytes_per_step": d2h // steps, "steps": steps,
            "what": "per step: the volume from pinned host memory once (mtx_upload_compute_min_max_mip, z-slabs "
                    "with the first extraction's leaf min/max overlapped), then per isovalue computeMinMaxMip -> "
                    "filterActiveBlocks -> readActiveBlockCount -> extractMeshletDescriptors -> mesh copied to "
                    "pinned host memory; two contexts alternate so that the next step's upload overlaps this "
                    "step's extractions"}


def batch_cpu_baseline(vols, jobs, blocks, threads: int, target_s: float):
    """The oracle's full path (min/max, compaction, marching cubes with the mesh
    written) over the batch's jobs in job order on `threads` host cores, until
    about target_s: a bounded sample of the workload, in job voxels a second."""
    from oracle import oracle as O
    hosts, secs, vox, n = {}, 0.0, 0, 0
    for v, iso in jobs:
        if v not in hosts:
            hosts[v] = vols[v].cpu().numpy()
        t0 = time.perf_counter()
        O.extract(hosts[v], blocks[v], iso, nthreads=threads)
        secs += time.perf_counter() - t0
        vox += hosts[v].size
        n += 1
        if secs >= target_s:
            break
    return vox / secs / 1e9, n, secs


def run_batched(ctx, stream, steps, scale_down=1, fixed=False, with_cpu=False):
    """The 64-volume mix (anisotropic edges from {64..512}, uint8/uint16/float32,
    1-16 isovalues each, seed 3): one batched run per step (a CUDA graph of the
    batched min/max and the persistent extraction kernel) against the same
    jobs as plain per-job launches of the asynchronous whole-path call, eager
    and recorded into a CUDA graph.  Per-job outputs are compared bit for bit."""
    from meshtrex_b200 import api, synth
    t_gen = time.perf_counter()
    items = synth.batch(seed=3, n=64, device="cuda", scale_down=scale_down)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t_gen
    vols = [it.volume for it in items]
    jobs = [(v, iso) for v, it in enumerate(items) for iso in it.isovalues]
    # block edge of every volume and the batched kernel's block warps from the batch autotuner
    t_tune = time.perf_counter()
    if fixed:  # profiling runs: block 8, as many block warps as fit
        tune = {"blockEdges": [BLOCK] * len(vols), "blockWarps": 0, "candidates": 0}
    else:
        tune = api.autotune_batch(ctx, vols, jobs)
    t_tune = time.perf_counter() - t_tune
    blocks, block_warps = tune["blockEdges"], tune["blockWarps"]
    esz = {torch.uint8: 1, torch.uint16: 2, torch.float32: 4}
    vol_bytes = sum(v.numel() * esz[v.dtype] for v in vols)
    job_voxels = sum(vols[v].numel() for v, _ in jobs)

    # one run sized small reports the pooled sizes it needs; the timed batch is sized exactly
    probe = api.Batch(ctx, vols, blocks, jobs, vertex_capacity=1 << 20, triangle_capacity=1 << 20,
                      block_warps=block_warps)
    probe.run()
    _, need = probe.results(check=False)
    probe.close()
    b = api.Batch(ctx, vols, blocks, jobs, max_active_blocks=need["activeBlocks"],
                  vertex_capacity=need["vertexCount"], triangle_capacity=need["triangleCount"], use_graph=True,
                  block_warps=block_warps)
    for _ in range(3):
        b.run()
    res, tot = b.results()

    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        b.run()
    e1.record(stream)
    torch.cuda.synchronize()
    t_batch = e0.elapsed_time(e1) / 1000.0 / steps
    res, tot = b.results()

    # plain per-job launches on the same jobs, outputs sized from the batch's results
    exts = [api.AsyncExtractor(ctx, vols[v], blocks[v], iso, r["vertexCount"] + 1, r["indexCount"] // 3 + 1,
                               max_active_blocks=r["meshletCount"] + 1)
            for (v, iso), r in zip(jobs, res)]

    def plain_step():
        for e in exts:
            e.run()

    plain_step()
    torch.cuda.synchronize()
    identical = True
    for e, r in zip(exts, res):
        c = e.counters.cpu().numpy().view(np.uint32)
        gv, gi, _ = b.mesh(r)
        same = (int(c[4]) == 0 and int(c[0]) == r["vertexCount"] and int(c[1]) == r["indexCount"]
                and torch.equal(e.vertices[: r["vertexCount"]].view(torch.int32), gv.view(torch.int32))
                and torch.equal(e.indices[: r["indexCount"] // 3], gi))
        identical = identical and same
    psteps = max(1, min(steps, 5))
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(psteps):
        plain_step()
    e1.record(stream)
    torch.cuda.synchronize()
    t_plain = e0.elapsed_time(e1) / 1000.0 / psteps

    # the same plain launches recorded into one CUDA graph
    t_plain_graph = None
    try:
        g = torch.cuda.CUDAGraph()
        cs = torch.cuda.Stream()
        ctx.set_stream(cs)
        with torch.cuda.graph(g, stream=cs):
            plain_step()
        ctx.set_stream(stream)
        g.replay()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(psteps):
            g.replay()
        e1.record(stream)
        torch.cuda.synchronize()
        t_plain_graph = e0.elapsed_time(e1) / 1000.0 / psteps
        del g
    except Exception as ex:  # capture is reported, not required
        ctx.set_stream(stream)
        t_plain_graph = f"capture failed: {ex}"
    ctx.synchronize()

    V, T = tot["vertexCount"], tot["triangleCount"]
    alg_bytes = vol_bytes + 12 * V + 12 * T
    peak, peak_kind = peak_hbm()
    out = {
        "workload": "64 volumes (edges from {64,96,128,192,256,384,512} per axis, uint8/uint16/float32 Gaussian "
                    "blobs, seed 3), 1-16 isovalues each in the 10th-90th percentile; block edges and block warps "
                    "from mtx_autotune_batch"
                    + (f"; edges divided by {scale_down}" if scale_down > 1 else ""),
        "volumes": len(vols), "jobs": len(jobs), "volume_bytes": vol_bytes, "job_voxels": job_voxels,
        "active_blocks": tot["activeBlocks"], "vertices": V, "triangles": T,
        "ms_batched": 1000.0 * t_batch, "ms_plain_launches": 1000.0 * t_plain,
        "ms_plain_graph": (1000.0 * t_plain_graph) if isinstance(t_plain_graph, float) else t_plain_graph,
        "speedup_vs_plain_launches": t_plain / t_batch,
        "speedup_vs_plain_graph": (t_plain_graph / t_batch) if isinstance(t_plain_graph, float) else None,
        "identical_to_plain": identical,
        "gvoxels_per_s": job_voxels / t_batch / 1e9, "tris_per_s": T / t_batch,
        "plain_gvoxels_per_s": job_voxels / t_plain / 1e9,
        "roofline": {"bound": "hbm", "achieved": alg_bytes / t_batch / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg_bytes / t_batch / 1e9 / peak, "algorithmic_bytes": alg_bytes,
                     "what": "each volume read once + 12 B per vertex + 12 B per triangle written",
                     "peak_kind": peak_kind},
        "gpu_launches_per_step": 2,
        "plain_launches_per_step": sum(launches_per_extraction(tuple((n + blocks[v] - 1) // blocks[v]
                                                                     for n in vols[v].shape), tuple(vols[v].shape),
                                                               vols[v].element_size(), blocks[v]) for v, _ in jobs),
        "autotuned": {"block_edges": sorted(set(blocks)), "block_edge_per_dtype": {
            str(dt).replace("torch.", ""): sorted({blocks[v] for v in range(len(vols)) if vols[v].dtype == dt})
            for dt in (torch.uint8, torch.uint16, torch.float32)}, "block_warps": block_warps,
            "candidates": tune["candidates"], "tune_s": t_tune},
        "generate_s": t_gen, "steps": steps, "plain_steps": psteps,
    }
    for e in exts:
        del e
    b.close()
    if with_cpu:
        threads = nproc()
        g_all, n_all, s_all = batch_cpu_baseline(vols, jobs, blocks, threads, 10.0)
        g_one, n_one, s_one = batch_cpu_baseline(vols, jobs, blocks, 1, 10.0)
        out["cpu_baseline"] = {
            "allcore_gvoxels_per_s": g_all, "1thread_gvoxels_per_s": g_one, "cores": threads, "kind": "port",
            "sample": (f"the first {n_all} jobs in job order on all threads ({s_all:.1f} s) and the first {n_one} "
                       f"on one thread ({s_one:.1f} s), each job's full mesh at its block edge")}
    return out


def run_blobs(ctx, stream, steps):
    """The CPU-runnable plain workload: 256^3 uint8 Gaussian blobs + N(0, 4)
    (seed 0), block 8^3, isovalue 128.  The asynchronous whole-path call timed
    with CUDA events (the volume is 16 MiB, so L2 holds it: this leg is
    latency-bound and reported beside the CPU path, not as the headline), and
    the oracle's full mesh on the same host bytes on one thread and on all
    host threads, checked against the GPU's bit for bit."""
    from meshtrex_b200 import api, synth
    from oracle import oracle as O
    vol = synth.blobs(256, seed=0, device="cuda")
    torch.cuda.synchronize()
    host = vol.cpu().numpy()
    ref = O.extract(host, 8, 128.0, nthreads=nproc())
    ex = api.AsyncExtractor(ctx, vol, 8, 128.0, ref.n_vertices + 1, ref.n_triangles + 1,
                            max_active_blocks=len(ref.ids) + 1)
    for _ in range(3):
        ex.run()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        ex.run()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    c = ex.counters.cpu().numpy().view(np.uint32)
    V, T = int(c[0]), int(c[1]) // 3
    match = (int(c[4]) == 0 and V == ref.n_vertices and T == ref.n_triangles
             and np.array_equal(ex.vertices[:V].cpu().numpy().view(np.uint32), ref.xyz.view(np.uint32))
             and np.array_equal(ex.indices[:T].cpu().numpy().view(np.uint32), ref.indices))

    def cpu(threads):
        secs, reps = 0.0, 0
        while reps == 0 or (secs < 3.0 and reps < 50):
            t0 = time.perf_counter()
            O.extract(host, 8, 128.0, nthreads=threads)
            secs += time.perf_counter() - t0
            reps += 1
        return host.size * reps / secs / 1e9
    nvox = host.size
    return {"workload": "256^3 uint8 Gaussian blobs + N(0, 4) (seed 0), block 8^3, isovalue 128",
            "vertices": V, "triangles": T, "active_blocks": len(ref.ids), "ms": ms,
            "gvoxels_per_s": nvox / ms / 1e6, "tris_per_s": T / ms * 1e3,
            "pipeline_roofline_frac": (nvox + 12 * V + 12 * T) / ms / 1e6 / peak_hbm()[0],
            "oracle_match": bool(match),
            "cpu_1thread_gvoxels_per_s": cpu(1), "cpu_allcore_gvoxels_per_s": cpu(nproc()), "cpu_cores": nproc(),
            "steps": steps}


def run_backward(ctx, stream, steps):
    """The differentiation workload: 512^3 float32 torus SDF (R 0.3, r 0.1) +
    0.05 fBm (seed 4), isovalue 0, block 8^3.  Forward = the whole plain
    extraction (asynchronous call: min/max, octree, filter, count, emit);
    backward = mtx_extract_backward from dL/dvertex of the loss
    mean_v (|v - c| - 0.35)^2 (v in [0, 1] coordinates) to the dense
    dL/dfield and dL/diso, in both modes.  Device times with CUDA events."""
    import ctypes as C

    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api, synth
    n, block, iso = 512, 8, 0.0
    vol = synth.torus(n, seed=4, device="cuda")
    torch.cuda.synchronize()
    v = api.wrap_volume(vol)
    pc = api.push_constants((n, n, n), block, iso)
    mm = api.compute_min_max_mip(ctx, v, pc)
    f = api.filter_active_blocks(ctx, mm, pc)
    nact = api.read_active_block_count(ctx, f)
    x = api.extract_meshlet_descriptors(ctx, mm, f, pc)
    V, T = x.vertex_count, x.index_count // 3
    verts = x.vertices().requires_grad_(True)
    loss = ((verts / (n - 1) - 0.5).norm(dim=1) - 0.35).pow(2).mean()
    (gv,) = torch.autograd.grad(loss, [verts])
    gv = gv.contiguous()
    fwd = api.AsyncExtractor(ctx, vol, block, iso, V + 1024, T + 1024, max_active_blocks=nact + 1024)
    dfield = torch.empty((n, n, n), dtype=torch.float32, device="cuda")
    diso = torch.empty(1, dtype=torch.float32, device="cuda")

    def bwd(mode):
        L.check(L.lib().mtx_extract_backward(ctx.handle, C.byref(v), C.byref(pc), C.byref(f.out),
                                             C.c_void_p(x.out.meshletDescriptorBuffer.ptr), V,
                                             C.c_void_p(gv.data_ptr()), 3, L.FRAME_VOXEL,
                                             C.c_void_p(dfield.data_ptr()), C.c_void_p(diso.data_ptr()), mode),
                "mtx_extract_backward", ctx.handle)

    def timed(fn):
        for _ in range(3):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    t_fwd = timed(fwd.run)
    t_atomic = timed(lambda: bwd(L.ADJOINT_ATOMIC))
    t_det = timed(lambda: bwd(L.ADJOINT_DETERMINISTIC))
    ctx.synchronize()
    c = fwd.counters.cpu().numpy().view(np.uint32)
    assert int(c[4]) == 0 and int(c[0]) == V
    nvox = n ** 3
    bwd_bytes = 12 * V + 2 * 4 * V + 4 * nvox
    fwd_bytes = 4 * nvox + 12 * V + 12 * T
    peak, peak_kind = peak_hbm()
    out = {
        "workload": "512^3 float32 torus SDF (R 0.3, r 0.1) + 0.05 fBm (4 octaves, seed 4), isovalue 0, block 8^3; "
                    "loss mean_v (|v - c| - 0.35)^2",
        "vertices": V, "triangles": T, "active_blocks": nact,
        "ms_forward": t_fwd, "ms_backward_atomic": t_atomic, "ms_backward_deterministic": t_det,
        "bwd_fwd_ratio_atomic": t_atomic / t_fwd, "bwd_fwd_ratio_deterministic": t_det / t_fwd,
        "forward_gbs": fwd_bytes / (t_fwd / 1000.0) / 1e9,
        "roofline": {"bound": "hbm", "achieved": bwd_bytes / (t_atomic / 1000.0) / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": bwd_bytes / (t_atomic / 1000.0) / 1e9 / peak,
                     "algorithmic_bytes": bwd_bytes, "peak_kind": peak_kind,
                     "what": "atomic mode: 12 B/vertex dL/dvertex read + 2 x 4 B edge endpoints + 4 B/voxel dL/dfield"},
        "steps": steps,
    }
    x.free()
    f.free()
    mm.free()
    del fwd, dfield, vol
    return out


def run_gyroid(ctx, stream, steps, n=2048, fixed=False, with_cpu=False):
    """The large float32 workload: n^3 gyroid sin(kx)cos(ky) + sin(ky)cos(kz) +
    sin(kz)cos(kx), k = 2 pi 12, + N(0, 0.02) (seed 2), isovalue 0 (32 GiB at
    2048^3).  mtx_autotune picks the block edge, warps, staging and min/max
    slices; the chosen shape and the default one (block 8^3, default tuning)
    are then timed with the asynchronous whole-path call."""
    from meshtrex_b200 import _lib as L
    from meshtrex_b200 import api, synth
    t0 = time.perf_counter()
    vol = synth.gyroid(n, seed=2, device="cuda")
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t0
    t0 = time.perf_counter()
    default = {"minmaxZChunk": 0, "minmaxSlices": 0, "extractWarps": 0, "staging": 0, "extractCtasPerSm": 0}
    if fixed:  # profiling runs: block 8, default tuning
        tune = {"blockEdge": 8, "tuning": default, "candidates": 0}
    else:
        tune = api.autotune(ctx, vol, 0.0)  # best of three repetitions per candidate
    t_tune = time.perf_counter() - t0

    def timed(block, tuning):
        ctx.set_tuning(tuning["minmaxZChunk"], tuning["minmaxSlices"], tuning["extractWarps"], tuning["staging"])
        m = api.extract(vol, block, 0.0, ctx=ctx)
        V, T, A = m.vertices.shape[0], m.indices.shape[0], m.active_ids.shape[0]
        del m
        ex = api.AsyncExtractor(ctx, vol, block, 0.0, V + 1024, T + 1024, max_active_blocks=A + 1024)
        for _ in range(2):
            ex.run()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            ex.run()
        e1.record(stream)
        torch.cuda.synchronize()
        ctx.synchronize()
        c = ex.counters.cpu().numpy().view(np.uint32)
        assert int(c[4]) == 0 and int(c[0]) == V and int(c[1]) == 3 * T
        # per-stage split of the same call (profiler events between the stages)
        prof = api.Profiler(ctx)
        ctx.set_profiler(prof)
        prof.begin_frame()
        for _ in range(3):
            ex.run()
        prof.end_frame()
        ctx.set_profiler(None)
        stages = {k: v[0] / 3 for k, v in prof.regions().items()}
        prof.close()
        del ex
        return e0.elapsed_time(e1) / steps, V, T, A, stages

    ms_tuned, V, T, A, stages = timed(tune["blockEdge"], tune["tuning"])
    ms_default, V8, T8, _, _ = (ms_tuned, V, T, A, stages) if fixed else timed(8, default)
    cpu = None
    if with_cpu:  # the oracle on z-slabs of the same field, all host threads and one thread
        from oracle import oracle as O
        res = {}
        for threads, nz in ((nproc(), 64), (1, 8)):
            z0 = n // 2
            slab = vol[z0:z0 + nz + 1].contiguous().cpu().numpy()
            t0 = time.perf_counter()
            O.extract(slab, tune["blockEdge"], 0.0, nthreads=threads)
            res[threads] = slab.size / (time.perf_counter() - t0) / 1e9
        cpu = {"allcore_gvoxels_per_s": res[nproc()], "1thread_gvoxels_per_s": res[1], "cores": nproc(),
               "sample": f"z-slabs of {n}x{n}x65 (all threads) and {n}x{n}x9 (one thread) at the middle, the "
                         "autotuned block edge, full mesh"}
    ctx.set_tuning(0, 0, 0, 0)
    nvox = n ** 3
    peak, peak_kind = peak_hbm()
    alg = 4 * nvox + 12 * V + 12 * T
    out = {
        "workload": f"{n}^3 float32 gyroid (k = 2 pi 12) + N(0, 0.02), seed 2, isovalue 0",
        "autotuned": {"block": tune["blockEdge"], "tuning": tune["tuning"], "candidates": tune["candidates"],
                      "tune_s": t_tune},
        "ms_tuned": ms_tuned, "ms_default_b8": ms_default, "speedup_vs_default": ms_default / ms_tuned,
        "gvoxels_per_s": nvox / ms_tuned / 1e6, "tris_per_s": T / ms_tuned * 1e3,
        "vertices": V, "triangles": T, "active_blocks": A, "triangles_b8": T8,
        "stages_ms": stages, "cpu_baseline": cpu,
        "pipeline_roofline": {"achieved": alg / ms_tuned / 1e6, "peak": peak, "unit": "GB/s",
                              "frac": alg / ms_tuned / 1e6 / peak, "algorithmic_bytes": alg, "peak_kind": peak_kind,
                              "what": "volume read once + 12 B per vertex + 12 B per triangle written"},
        "generate_s": t_gen, "steps": steps,
    }
    del vol
    torch.cuda.empty_cache()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="mtx", choices=["mtx", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline and oracle parity legs")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched 64-volume leg")
    ap.add_argument("--no-backward", action="store_true", help="skip the backward (adjoint) leg")
    ap.add_argument("--batch-scale", type=int, default=1, help="divide the batch's volume edges (profiling runs only)")
    ap.add_argument("--no-gyroid", action="store_true", help="skip the autotuned 2048^3 float32 gyroid leg")
    ap.add_argument("--gyroid-size", type=int, default=2048, help="gyroid edge (profiling runs only)")
    ap.add_argument("--gyroid-fixed", action="store_true", help="gyroid at block 8, no autotuner (profiling runs only)")
    ap.add_argument("--batch-fixed", action="store_true", help="batch at block 8, no autotuner (profiling runs only)")
    ap.add_argument("--size", type=int, default=1024, help="volume edge (profiling runs only)")
    ap.add_argument("--cache", default="", help="raw file to read/write the generated volume")
    args = ap.parse_args()
    rc = relaunch_ranks(args.gpus, sys.argv[1:])
    if rc is not None:
        return rc
    global N
    N = args.size
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_mtx(args)


if __name__ == "__main__":
    sys.exit(main())
