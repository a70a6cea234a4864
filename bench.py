"""Benchmark: Mtri/s and frames/s of Piko's binned raster pipeline on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl piko|reference]

A step is one frame of the scene-scale raster workload: the 174,000-triangle
procedural forest at 1920x1080 with textured Lambert shading (seeded synthetic
stand-in for the reference's forest scene, whose mesh is not shipped).  The
frame is the plain form: one scene per launch sequence (setup, tile scan,
scatter, tile raster), replayed as a CUDA graph.

value    Mtri/s over all ranks = input triangles (before culling) / device
         time per frame, inputs resident in HBM.  L2 is flushed (a 512 MiB
         write) between timed frames; the flush is outside each frame's events.
e2e      the same metric through the C ABI with host buffers: every step
         uploads the frame's vertex attributes from pinned memory, renders and
         reads the colour and depth buffers back.
roofline the dominant kernel (by device time) against the measured HBM copy
         bandwidth, with the algorithmic bytes of that kernel per launch.
cpu_baseline  the reference's own CPU pipeline (oracle/_ref, built from the
         reference's stage code) on the same geometry, timed on this host.
batched  the 64-scene mix in one launch sequence vs 64 plain launches.

Multi-GPU: replicas only (every rank renders its own copy of the frame; the
only cross-rank traffic is the timing barrier and the max-over-ranks
reduction).  --impl reference runs the reference's CPU pipeline instead.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mtri/s and frames/s plain vs batched on 1 B200; served p50/p99 latency"
UNIT = "Mtri/s"
L2_FLUSH_BYTES = 512 << 20
# setup, large-triangle count, scan, scatter (list and large-triangle walks), tile raster
LAUNCHES_PER_FRAME = 5
PROFILE_SUMMARY = os.path.join(ROOT, "profiles", "raster_frag8_forest1080p.md")


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="piko", choices=["piko", "reference"])
    p.add_argument("--tile", type=int, default=8)
    p.add_argument("--no-batched", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-served", action="store_true")
    p.add_argument("--no-reyes", action="store_true")
    p.add_argument("--e2e-lanes", type=int, default=2,
                   help="frames in flight in the end-to-end measurement (one context, stream and host thread each;"
                        " 2 measured fastest: 3 and 4 add copy-engine contention)")
    p.add_argument("--batched-only", action="store_true",
                   help="only the 64-scene batched leg (tuning, then the timed replays); prints its JSON")
    p.add_argument("--reyes-only", action="store_true",
                   help="only the Reyes workload (4 jittered samples, Phong) and its reference-sampling variant")
    p.add_argument("--untuned", action="store_true",
                   help="with --batched-only: the single-configuration batch (--tile), no tuning")
    p.add_argument("--serve-seconds", type=float, default=10.0,
                   help="served form: length of the request stream (the workload's 10 s)")
    p.add_argument("--serve-rate", type=float, default=2000.0,
                   help="served form: Poisson request rate (1/s), the workload's 2,000/s")
    p.add_argument("--stress-rate", type=float, default=8000.0,
                   help="served form, second (stress) line: a rate above what one request per launch sustains"
                        " (0 = no stress line)")
    p.add_argument("--stress-seconds", type=float, default=3.0)
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(x, dist=None, device="cpu"):
    """The largest value of x over all ranks (times are reported as the max
    over ranks); identity without a process group."""
    if dist is None or not dist.is_initialized():
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, units_per_rank, ms):
    """Units per second over all ranks, in millions (replicas: each rank
    processes its own copy of the units in ms)."""
    return world * units_per_rank / (ms / 1e3) / 1e6


def workload_config(sc, tile):
    return {"workload": "forest174k_1920x1080_textured", "triangles": sc.n, "width": sc.W, "height": sc.H,
            "form": "plain (one scene per launch sequence, CUDA graph replay)", "tile_px": tile,
            "texture": "512x512 RGBA8 seeded noise", "parallelism": "replicas",
            "l2": "flushed between timed frames (512 MiB write), flush outside the frame events"}


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", f"piko_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.device), "-lms", "100"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


REYES_PROFILE = os.path.join(ROOT, "profiles", "reyes_dice_sphere720p.md")


def profile_value(path, key):
    """A figure from a committed ncu summary (a line "key: value")."""
    try:
        for line in open(path):
            if line.startswith(key + ":"):
                return float(line.split(":")[1].split()[0])
    except Exception:
        pass
    return None


def profile_traffic():
    """dram bytes per launch of the dominant kernel, from the committed ncu summary."""
    try:
        for line in open(PROFILE_SUMMARY):
            if line.startswith("dram_bytes_per_launch_full:"):
                return float(line.split(":")[1].split()[0])
    except Exception:
        pass
    return None


# ---------------------------------------------------------------- reference arm
def run_reference(args, sc_builder):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle
    sc = sc_builder()
    cfg = workload_config(sc, args.tile)
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference source tree absent)"}))
        return
    threads = max(64, os.cpu_count() or 1)
    xyz, icol = oracle.r1_setup(sc)
    r = oracle.RefRaster(sc.W, sc.H, xyz, icol)
    try:
        for _ in range(args.warmup):
            r.frame(threads)
        ns = [r.frame(threads) for _ in range(args.steps)]
        fb_mt, _ = r.read()
        r.frame(1)
        fb_1, _ = r.read()
    finally:
        r.close()
    ms = float(np.mean(ns)) / 1e6
    v = sc.n / (ms / 1e3) / 1e6
    sample = (f"{args.steps} full frames of the {sc.n}-triangle forest at {sc.W}x{sc.H}, Gouraud colour "
              f"(the reference has no texturing); {threads}-thread Process runner; "
              f"image equals the 1-thread image: {bool(np.array_equal(fb_mt, fb_1))}")
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "int32 28.4 fixed point + f32", "data": "synthetic",
           "config": cfg,
           "cpu_baseline": dict({"value": v, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
                                **host_info()),
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def cpu_model():
    """The host CPU's model name (first entry of /proc/cpuinfo)."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def host_info():
    return {"host_cpus": os.cpu_count(), "cpu_model": cpu_model()}


def _ref_frames(r, threads, budget_s, max_frames):
    """Median wall time (ms) of the reference's frames (prepare + run_single,
    as its doPerfTest times them) after one warm-up frame, within budget_s."""
    r.frame(threads)
    ns = []
    t0 = time.time()
    while (time.time() - t0 < budget_s and len(ns) < max_frames) or len(ns) < 3:
        ns.append(r.frame(threads))
    return float(np.median(ns)) / 1e6, len(ns)


def cpu_baseline(sc, budget_s=6.0):
    """The reference's own CPU raster pipeline (oracle/_ref) on the forest's
    geometry: its generated 64-thread Process runner (the headline) and the
    deterministic one-thread run beside it; the oracle port when the reference
    build is absent."""
    import oracle
    xyz, icol = oracle.r1_setup(sc)
    if oracle.ref_available():
        r = oracle.RefRaster(sc.W, sc.H, xyz, icol)
        try:
            ms, k = _ref_frames(r, 64, budget_s, 200)
            ms1, k1 = _ref_frames(r, 1, budget_s / 3, 20)
        finally:
            r.close()
        return dict({"value": sc.n / (ms / 1e3) / 1e6, "unit": UNIT, "cores": 64, "kind": "reference",
                     "sample": f"{k} frames (median) of the {sc.n}-triangle forest, {sc.W}x{sc.H}, Gouraud colour "
                               f"(no texturing in the reference); the reference's 64-thread Process runner",
                     "ms_per_frame": ms,
                     "one_thread": {"value": sc.n / (ms1 / 1e3) / 1e6, "ms_per_frame": ms1, "frames": k1}},
                    **host_info())
    t0 = time.time()
    oracle.raster_frame(sc.W, sc.H, xyz, icol)
    ms = (time.time() - t0) * 1e3
    return dict({"value": sc.n / (ms / 1e3) / 1e6, "unit": UNIT, "cores": 1, "kind": "port",
                 "sample": "1 frame of the forest through the oracle restatement", "ms_per_frame": ms}, **host_info())


def cpu_baseline_reyes(sc, budget_s=3.0):
    """The reference's Reyes pipeline on the sphere workload, built with the
    workload's constants (split below 16 px, at most 10 splits, 16x16 dice;
    oracle/_ref/libpiko_ref_reyes_c2.so) and its own sampling (one centre sample
    per pixel, corner-lit colour: the reference has no multisampling or Phong),
    at 64 threads and at one thread; frames/s."""
    import oracle
    if not (oracle.ref_available() and oracle.ref_c2_available()):
        return None
    r = oracle.RefReyes(sc, workload_constants=True)
    try:
        ms, k = _ref_frames(r, 64, budget_s, 20)
        ms1, k1 = _ref_frames(r, 1, budget_s, 20)
    finally:
        r.close()
    return dict({"value": 1e3 / ms, "unit": "frames/s", "cores": 64, "kind": "reference",
                 "sample": f"{k} frames (median) of the 32-patch sphere at {sc.W}x{sc.H}, the reference's sampling "
                           f"and shading, its 64-thread runner (Split loop included)",
                 "ms_per_frame": ms, "one_thread": {"value": 1e3 / ms1, "ms_per_frame": ms1, "frames": k1}},
                **host_info())


def cpu_baseline_c0(sc, budget_s=2.0):
    """The reference's raster pipeline on the plain 4,096-triangle scene at
    512x512, at 64 threads and one thread."""
    import oracle
    if not oracle.ref_available():
        return None
    xyz, icol = oracle.r1_setup(sc)
    r = oracle.RefRaster(sc.W, sc.H, xyz, icol)
    try:
        ms, k = _ref_frames(r, 64, budget_s, 200)
        ms1, k1 = _ref_frames(r, 1, budget_s, 200)
    finally:
        r.close()
    return dict({"value": sc.n / (ms / 1e3) / 1e6, "unit": UNIT, "cores": 64, "kind": "reference",
                 "sample": f"{k} frames (median) of the {sc.n}-triangle plain scene at {sc.W}x{sc.H}",
                 "ms_per_frame": ms, "one_thread": {"value": sc.n / (ms1 / 1e3) / 1e6, "ms_per_frame": ms1,
                                                    "frames": k1}}, **host_info())


def cpu_baseline_mix(mix):
    """The reference's raster pipeline over the 64-scene mix, one frame per
    scene in turn at 64 threads (its generated runner): frames/s = 64 / the sum
    of the frame times (inputs set up outside the timed frames)."""
    import oracle
    if not oracle.ref_available():
        return None
    tot = 0.0
    for sc in mix:
        xyz, icol = oracle.r1_setup(sc)
        r = oracle.RefRaster(sc.W, sc.H, xyz, icol)
        try:
            tot += r.frame(64) / 1e6
        finally:
            r.close()
    tris = sum(sc.n for sc in mix)
    return dict({"value": len(mix) / (tot / 1e3), "unit": "frames/s", "cores": 64, "kind": "reference",
                 "sample": f"one frame of each of the {len(mix)} mix scenes, 64-thread runner",
                 "ms_total": tot, "Mtri_per_s": tris / (tot / 1e3) / 1e6}, **host_info())


# ---------------------------------------------------------------- our arm
def main():
    args = parse_args()
    rank, world, local = dist_env()
    import piko_loader
    pk = piko_loader.load()

    def build_scene():
        return pk.scenes.forest_scene()

    if args.impl == "reference":
        run_reference(args, build_scene)
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    if args.reyes_only:
        ctx = pk.Context(device=local)
        stream = torch.cuda.Stream()
        flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
        out = run_reyes(pk, ctx, stream, flush, args)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "reyes": out}))
        ctx.close()
        if dist is not None:
            dist.destroy_process_group()
        return

    if args.batched_only:
        ctx = pk.Context(device=local)
        stream = torch.cuda.Stream()
        flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
        out = run_batched_only(pk, ctx, stream, flush, args)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "batched": out}))
        ctx.close()
        if dist is not None:
            dist.destroy_process_group()
        return

    sc = build_scene()
    ctx = pk.Context(device=local)
    pipe = pk.Pipe(ctx, "raster", tile_px=args.tile)
    scene = pk.Scene(pipe, sc)
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    clocks = ClockSampler(local)
    clocks.start()

    # first frame: sizes the bin queues (an overflow re-renders) and checks status
    scene.run(sptr)
    scene.finish()
    one = pk.Batch(ctx, [scene])

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            flush.fill_(1.0)
            one.run(sptr, graph=True)
        one.finish()
        barrier()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        for i in range(args.steps):
            flush.fill_(float(i))
            starts[i].record(stream)
            one.run(sptr, graph=True)
            ends[i].record(stream)
        barrier()
        st = one.finish()
    frame_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    ms = max_over_ranks(float(np.mean(frame_ms)), dist, "cuda")
    value = whole_job_rate(world, sc.n, ms)
    # the same frame with the workload's stated 16x16-pixel bins (coverage and
    # the image are bin-size invariant; 8x8 tiles are the headline's tuning)
    t16_ms = max_over_ranks(time_plain_frames(pk, ctx, sc, 16, stream, flush, args), dist, "cuda")
    tile16 = {"tile_px": 16, "ms_per_frame": t16_ms, "value": whole_job_rate(world, sc.n, t16_ms), "unit": UNIT}

    # per-kernel device times (events between the kernels of a frame)
    kctx = pk.Context(device=local, time_kernels=True)
    kpipe = pk.Pipe(kctx, "raster", tile_px=args.tile)
    kscene = pk.Scene(kpipe, sc)
    # event spans of a frame: setup + large-triangle count, scan, scatter (list
    # and large-triangle walks), tile raster (raster_frag8 for 8x8 tiles)
    tile_kernel = "raster_frag8" if args.tile == 8 else "raster_tiles"
    names = ["raster_setup", "scan_tiles", "raster_scatter", tile_kernel]
    kms = np.zeros(4)
    reps = max(5, min(args.steps, 20))
    with torch.cuda.stream(stream):
        kscene.run(sptr)
        kscene.finish()
        for _ in range(reps):
            flush.fill_(2.0)
            kscene.run(sptr)
            kst = kscene.stats()
            kms += np.array(kst["kernel_ms"][:4])
    kms /= reps
    kscene.close(); kpipe.close(); kctx.close()
    dom = int(np.argmax(kms))
    W, H = sc.W, sc.H
    tex_bytes = int(sc.texture.nbytes) if sc.texture is not None else 0
    alg = {"raster_setup": sc.n * 120, "scan_tiles": 0, "raster_scatter": 0,
           tile_kernel: W * H * 8 + tex_bytes}
    peak, peak_kind = measured_peak_gbs()
    ach = alg[names[dom]] / (kms[dom] / 1e3) / 1e9
    frame_alg = sc.n * 120 + W * H * 8 + tex_bytes
    roofline = {"bound": "hbm", "kernel": names[dom], "achieved": ach, "peak": peak, "unit": "GB/s",
                "frac": ach / peak, "peak_kind": peak_kind, "traffic": profile_traffic(),
                "algorithmic_bytes_per_launch": alg[names[dom]],
                "kernel_ms": {n: float(v) for n, v in zip(names, kms)},
                "frame": {"algorithmic_bytes": frame_alg, "achieved": frame_alg / (ms / 1e3) / 1e9,
                          "frac": frame_alg / (ms / 1e3) / 1e9 / peak}}

    # e2e through the C ABI with pinned host buffers; positions and normals in
    # the packed float3 layout (piko_scene_desc.packed: their w components
    # carry nothing, and the upload is the step's bottleneck)
    keep = {}
    pin = {}
    for k in ("pos", "nrm", "col", "uv"):
        a = getattr(sc, k)
        if a is None:        # the forest has no colour array: the fixed material colour
            continue
        if k in ("pos", "nrm"):
            a = np.asarray(a)[..., :3]
        t = torch.from_numpy(np.ascontiguousarray(a, np.float32)).pin_memory()
        pin[k] = t
        keep[k] = t.numpy()
    import copy
    psc = copy.copy(sc)
    psc.pos, psc.nrm, psc.col, psc.uv = keep["pos"], keep["nrm"], keep.get("col"), keep.get("uv")
    from piko_b200 import runtime as rt
    desc, _ = rt.scene_desc(psc, packed=True)
    escene = pk.Scene(pipe, psc, packed=True)
    fb_pin = torch.empty((H, W), dtype=torch.int32).pin_memory()
    z_pin = torch.empty((H, W), dtype=torch.float32).pin_memory()
    fb_np, z_np = fb_pin.numpy().view(np.uint32), z_pin.numpy()
    h2d = sum(v.nbytes for v in keep.values())
    d2h = W * H * 8
    e2e_steps = max(3, min(args.steps, 20))
    with torch.cuda.stream(stream):
        for _ in range(2):
            escene.upload(desc, sptr)
            escene.run(sptr)
            escene.read(fb_np, z_np)
        barrier()
        e_ms = []
        for i in range(e2e_steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            escene.upload(desc, sptr)
            escene.run(sptr)
            escene.read(fb_np, z_np)
            b.record(stream)
            b.synchronize()
            e_ms.append(a.elapsed_time(b))
        barrier()
    escene.close()
    serial_ms = max_over_ranks(float(np.mean(e_ms)), dist, "cuda")
    # Several frames in flight: one context per host thread (as the C ABI
    # asks), each with its own copy of the scene, stream and pinned output
    # buffers; of n lanes, thread k renders steps k, k + n, ...  Every step
    # still uploads its inputs and reads its image and depth back; the copy
    # engines overlap one frame's upload with another's readback.
    pipe_ms = run_e2e_pipelined(pk, psc, desc, args, e2e_steps, H, W, local)
    e2e_ms = max_over_ranks(pipe_ms, dist, "cuda")
    e2e = {"value": whole_job_rate(world, sc.n, e2e_ms), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms,
           "pipeline": f"{args.e2e_lanes} frames in flight ({args.e2e_lanes} contexts, streams and host threads); "
                       "per step: upload from pinned host memory (positions and normals as float3), render, "
                       "read colour + depth back",
           "serial": {"value": whole_job_rate(world, sc.n, serial_ms), "ms_per_step": serial_ms,
                      "pipeline": "one frame at a time on one stream"}}

    batched = None
    if not args.no_batched:
        batched = run_batched(pk, ctx, stream, flush, args, dist, world)
    reyes = None if args.no_reyes else run_reyes(pk, ctx, stream, flush, args)
    served = None
    if not args.no_served:
        served = run_served(pk, ctx, args)
    clk = clocks.stop()

    c0 = run_c0(pk, ctx, stream, flush, args, dist, world)

    # the reference's CPU paths, on rank 0 at N=1 only, after the GPU legs
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(sc)
        c0["cpu_baseline"] = cpu_baseline_c0(pk.scenes.plain_scene())
        if reyes is not None:
            reyes["cpu_baseline"] = cpu_baseline_reyes(pk.scenes.sphere_patches())
        if batched is not None:
            batched["cpu_baseline"] = cpu_baseline_mix(pk.scenes.batch_mix(64))

    one.close()
    scene.close()
    pipe.close()
    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms, "frames_per_s": 1e3 / ms * world,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
               "dtype": "int32 28.4 fixed point + f32", "data": "synthetic", "config": workload_config(sc, args.tile),
               "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
               "gpu_launches": LAUNCHES_PER_FRAME * args.steps, "status": int(st["status"]),
               "frame": {"kept": int(st["prims_kept"]), "fragments": int(st["covered"]),
                         "bin_entries": int(st["bin_entries"])}}
        out["tile16"] = tile16
        out["c0"] = c0
        if batched is not None:
            out["batched"] = batched
        if reyes is not None:
            out["reyes"] = reyes
        if served is not None:
            out["served"] = served
        print(json.dumps(out))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    ctx.close()


def time_plain_frames(pk, ctx, sc, tile, stream, flush, args):
    """Mean device time (ms) of graph-replayed plain frames of `sc` with
    `tile`-pixel tiles, L2 flushed between frames (outside the events)."""
    import torch
    pipe = pk.Pipe(ctx, "raster", tile_px=tile)
    scene = pk.Scene(pipe, sc)
    sptr = stream.cuda_stream
    one = pk.Batch(ctx, [scene])
    with torch.cuda.stream(stream):
        scene.run(sptr)
        scene.finish()
        for _ in range(max(args.warmup, 3)):
            flush.fill_(1.0)
            one.run(sptr, graph=True)
        one.finish()
        torch.cuda.synchronize()
        ms = []
        for i in range(max(args.steps, 10)):
            flush.fill_(float(i))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            one.run(sptr, graph=True)
            b.record(stream)
            b.synchronize()
            ms.append(a.elapsed_time(b))
        st = one.finish()
    assert st["status"] == 0
    one.close()
    scene.close()
    pipe.close()
    return float(np.mean(ms))


def run_c0(pk, ctx, stream, flush, args, dist, world):
    """The plain CPU-sized case: 4,096 triangles at 512x512, seed 0 (graph
    replays, device time per frame)."""
    sc = pk.scenes.plain_scene()
    ms = max_over_ranks(time_plain_frames(pk, ctx, sc, args.tile, stream, flush, args), dist, "cuda")
    return {"workload": "plain4096_512x512 (seed 0)", "triangles": sc.n, "tile_px": args.tile, "ms_per_frame": ms,
            "value": whole_job_rate(world, sc.n, ms), "unit": UNIT, "frames_per_s": 1e3 / ms * world}


def run_e2e_pipelined(pk, psc, desc, args, steps, H, W, device):
    """Device time (ms per step, CUDA events over both streams) of `steps`
    end-to-end frames through the C ABI with args.e2e_lanes frames in flight."""
    import threading
    import torch
    lanes = []
    nl = max(1, args.e2e_lanes)
    for k in range(nl):
        c = pk.Context(device=device)
        p = pk.Pipe(c, "raster")
        s = pk.Scene(p, psc, packed=True)
        st = torch.cuda.Stream()
        fb = torch.empty((H, W), dtype=torch.int32).pin_memory()
        z = torch.empty((H, W), dtype=torch.float32).pin_memory()
        lanes.append({"ctx": c, "pipe": p, "scene": s, "stream": st, "fb": fb, "z": z,
                      "fb_np": fb.numpy().view(np.uint32), "z_np": z.numpy()})
    errors = []

    def work(k, n):
        L = lanes[k]
        sp = L["stream"].cuda_stream
        try:
            for _ in range(n):
                L["scene"].upload(desc, sp)
                L["scene"].run(sp)
                L["scene"].read(L["fb_np"], L["z_np"])
        except Exception as e:  # reported after the join
            errors.append(e)

    # warm-up: both lanes, concurrently
    ts = [threading.Thread(target=work, args=(k, 2)) for k in range(nl)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(nl)]
    start.record(lanes[0]["stream"])
    for k in range(1, nl):
        lanes[k]["stream"].wait_event(start)
    ts = [threading.Thread(target=work, args=(k, (steps + nl - 1 - k) // nl)) for k in range(nl)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    for k in range(nl):
        ends[k].record(lanes[k]["stream"])
    torch.cuda.synchronize()
    if errors:
        raise errors[0]
    ms = max(start.elapsed_time(e) for e in ends) / steps
    for L in lanes:
        L["scene"].close()
        L["pipe"].close()
        L["ctx"].close()
    return ms


def run_batched(pk, ctx, stream, flush, args, dist, world):
    """The 64-scene mix: the tuned batch (one launch sequence per tuned
    configuration group, parallel branches of one replayed graph) and the
    single-configuration batch vs the same 64 scenes rendered as 64 plain
    launch sequences."""
    import torch
    mix = pk.scenes.batch_mix(64)
    pipe = pk.Pipe(ctx, "raster", tile_px=args.tile)
    scenes = [pk.Scene(pipe, s) for s in mix]
    sptr = stream.cuda_stream
    # the autotuner picks tile size, CTAs per SM and chunk size per scene-size
    # bucket on this mix (untimed); the batch groups scenes by configuration
    t0 = time.perf_counter()
    tuner = pk.Tuner().tune(ctx, scenes, reps=5)
    tune_s = time.perf_counter() - t0
    batch = pk.Batch(ctx, scenes, tuner=tuner)
    untuned = pk.Batch(ctx, scenes)
    singles = [pk.Batch(ctx, [s]) for s in scenes]
    reps = max(3, min(args.steps, 10))
    with torch.cuda.stream(stream):
        for _ in range(2):
            batch.run(sptr, graph=True)
            batch.finish()
            untuned.run(sptr, graph=True)
            untuned.finish()
            for b in singles:
                b.run(sptr, graph=True)
            for b in singles:
                b.finish()
        torch.cuda.synchronize()
        tb, tu, tp = [], [], []
        for i in range(reps):
            flush.fill_(3.0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            batch.run(sptr, graph=True)
            b.record(stream)
            flush.fill_(3.5)
            e, f = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e.record(stream)
            untuned.run(sptr, graph=True)
            f.record(stream)
            flush.fill_(4.0)
            c, d = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            c.record(stream)
            for s in singles:
                s.run(sptr, graph=True)
            d.record(stream)
            torch.cuda.synchronize()
            tb.append(a.elapsed_time(b))
            tu.append(e.elapsed_time(f))
            tp.append(c.elapsed_time(d))
        st = batch.finish()
        untuned.finish()
        # the drop-in loop: each scene rendered and finished in turn, like the
        # reference's synchronous run_single
        td = []
        for i in range(reps):
            flush.fill_(5.0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for s in scenes:
                s.run(sptr)
                s.finish()
            td.append((time.perf_counter() - t0) * 1e3)
    ms_b, ms_u, ms_p, ms_d = float(np.mean(tb)), float(np.mean(tu)), float(np.mean(tp)), float(np.mean(td))
    tris = sum(s.n for s in mix)
    table = {str(k): {"tile_px": v["tile_px"], "ctas_per_sm": v["ctas_per_sm"], "chunk_entries": v["chunk_entries"],
                      "ms": round(v["ms"], 4), "scenes": sum(1 for s in mix if pk.tune_bucket(s.W, s.H, s.n) == k)}
             for k, v in tuner.table().items()}
    for s in singles:
        s.close()
    batch.close()
    untuned.close()
    tuner.close()
    for s in scenes:
        s.close()
    pipe.close()
    return {"workload": "64-scene mix (1K-200K triangles, 256^2..1920x1080, seeds 0..63)",
            "triangles": tris, "ms_batched": ms_b, "ms_batched_untuned": ms_u, "ms_64_plain": ms_p,
            "ms_64_dropin": ms_d, "tuner": {"buckets": table, "tune_seconds": round(tune_s, 2),
                                            "bucket": "resolution class (<=256^2, <=512^2, <=1280x720, larger) * 4 + "
                                                      "triangle class (<4K, <16K, <64K, more)"},
            "frames_per_s_batched": 64 * 1e3 / ms_b * world, "frames_per_s_plain": 64 * 1e3 / ms_p * world,
            "frames_per_s_dropin": 64 * 1e3 / ms_d * world,
            "Mtri_per_s_batched": tris / (ms_b / 1e3) / 1e6 * world,
            "speedup_batched_vs_plain": ms_p / ms_b, "speedup_batched_vs_dropin": ms_d / ms_b,
            "speedup_tuned_vs_untuned": ms_u / ms_b,
            "plain": "64 single-scene graph replays queued back to back on one stream (device time)",
            "dropin": "run + finish per scene, host wall clock (the reference's synchronous run_single loop)",
            "status": int(st["status"])}


def run_batched_only(pk, ctx, stream, flush, args):
    """Tuning on the 64-scene mix, then --steps replays of the tuned batch
    (device time each); nothing else is launched, so a profiler's launch list
    after the tuning is the batched form alone."""
    import torch
    mix = pk.scenes.batch_mix(64)
    pipe = pk.Pipe(ctx, "raster", tile_px=args.tile)
    scenes = [pk.Scene(pipe, s) for s in mix]
    sptr = stream.cuda_stream
    tuner = None if args.untuned else pk.Tuner().tune(ctx, scenes, reps=5)
    batch = pk.Batch(ctx, scenes, tuner=tuner)
    ms = []
    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            batch.run(sptr, graph=True)
            batch.finish()
        for _ in range(args.steps):
            flush.fill_(6.0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.nvtx.range_push("batched")
            a.record(stream)
            batch.run(sptr, graph=True)
            b.record(stream)
            torch.cuda.nvtx.range_pop()
            batch.finish()
            ms.append(a.elapsed_time(b))
    groups = ([(args.tile, 0, 0)] if tuner is None else
              sorted({(v["tile_px"], v["ctas_per_sm"], v["chunk_entries"]) for v in tuner.table().values()}))
    batch.close()
    if tuner is not None:
        tuner.close()
    for s in scenes:
        s.close()
    pipe.close()
    return {"workload": "64-scene mix, tuned batch only", "ms_batched": float(np.mean(ms)), "groups": groups}


REYES_WORKLOAD = dict(split_threshold_px=16.0, max_splits=10, dice_grid=16, samples_per_pixel=4, sample_seed=1,
                      phong=True)


def run_reyes(pk, ctx, stream, flush, args):
    """The Reyes workload: 32 sphere patches at 1280x720, split below 16 px,
    at most 10 splits, 16x16 dice grids, 4 jittered samples per pixel (seed 1),
    Phong shading; device time per frame.  The reference's own sampling (one
    centre sample, corner-lit colour) is timed beside it."""
    import torch
    sc = pk.scenes.sphere_patches()
    sptr = stream.cuda_stream
    reps = max(3, min(args.steps, 20))
    out = {}
    variants = (("c2", REYES_WORKLOAD),
                ("reference_sampling", dict(REYES_WORKLOAD, samples_per_pixel=1, phong=False)))
    for name, kw in variants:
        pipe = pk.Pipe(ctx, "reyes", **kw)
        scene = pk.Scene(pipe, sc)
        with torch.cuda.stream(stream):
            scene.run(sptr)
            scene.finish()
            ms = []
            for _ in range(reps):
                flush.fill_(5.0)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                scene.run(sptr)
                b.record(stream)
                scene.finish()
                ms.append(a.elapsed_time(b))
            st = scene.stats()
        scene.close()
        pipe.close()
        m = float(np.mean(ms))
        out[name] = {"ms_per_frame": m, "frames_per_s": 1e3 / m, "leaves": int(st["prims_kept"]),
                     "micropolygons": int(st["upolys"]), "covered_samples": int(st["covered"]),
                     "status": int(st["status"])}
    out["e2e"] = reyes_e2e(pk, ctx, stream, sc, reps)
    c2 = out["c2"]
    # algorithmic bytes per frame: the patches once (16 float4 control points)
    # and RGBA8 + f32 depth once per pixel
    alg = sc.n * 256 + sc.W * sc.H * 8
    peak, kind = measured_peak_gbs()
    gbs = alg / (c2["ms_per_frame"] * 1e-3) / 1e9
    roof = {"bound": "issue", "hbm_achieved_gbs": gbs, "hbm_peak_gbs": peak, "hbm_frac": gbs / peak,
            "peak_kind": kind, "algorithmic_bytes": alg,
            "fp32_issue_frac_dice": profile_value(REYES_PROFILE, "fp32_issue_frac_dice"),
            "fp32_source": "ncu, profiles/reyes_dice_sphere720p.md"}
    return {"workload": "sphere32_1280x720 (split < 16 px, <= 10 splits, 16x16 dice, 4 jittered spp, Phong)",
            "ms_per_frame": c2["ms_per_frame"], "frames_per_s": c2["frames_per_s"], "leaves": c2["leaves"],
            "micropolygons": c2["micropolygons"], "covered_samples": c2["covered_samples"], "status": c2["status"],
            "roofline": roof, "e2e": out["e2e"], "reference_sampling": out["reference_sampling"]}


def reyes_e2e(pk, ctx, stream, sc, steps):
    """The Reyes workload end to end through the C ABI: every step uploads the
    patches from pinned host memory, renders and reads colour and depth back
    into pinned host memory; frames/s over the device time of the steps."""
    import copy
    import torch
    from piko_b200 import runtime as rt
    pipe = pk.Pipe(ctx, "reyes", **REYES_WORKLOAD)
    scene = pk.Scene(pipe, sc)
    pin = torch.from_numpy(np.ascontiguousarray(sc.patches)).pin_memory()
    psc = copy.copy(sc)
    psc.patches = pin.numpy()
    desc, _ = rt.scene_desc(psc)
    fb = torch.empty((sc.H, sc.W), dtype=torch.int32).pin_memory()
    z = torch.empty((sc.H, sc.W), dtype=torch.float32).pin_memory()
    fb_np, z_np = fb.numpy().view(np.uint32), z.numpy()
    sptr = stream.cuda_stream
    with torch.cuda.stream(stream):
        for _ in range(2):
            scene.upload(desc, sptr)
            scene.run(sptr)
            scene.read(fb_np, z_np)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(steps):
            scene.upload(desc, sptr)
            scene.run(sptr)
            scene.read(fb_np, z_np)
        b.record(stream)
        b.synchronize()
    ms = a.elapsed_time(b) / steps
    scene.close()
    pipe.close()
    return {"value": 1e3 / ms, "unit": "frames/s", "ms_per_step": ms, "h2d_bytes_per_step": int(sc.patches.nbytes),
            "d2h_bytes_per_step": int(sc.W * sc.H * 8),
            "pipeline": "one frame at a time on one stream: upload patches, render, read colour + depth back"}


def serve_stream(pk, ctx, rs, ys, rate, seconds, seed):
    """One Poisson request stream at `rate` requests/s for `seconds`, replayed
    through continuous batching and through one request per launch sequence."""
    from piko_b200 import serve
    stream = serve.make_stream(seed=seed, n_raster_scenes=len(rs), rate_hz=rate, seconds=seconds)
    warm = serve.make_stream(seed=seed + 1, n_raster_scenes=len(rs), rate_hz=rate, seconds=0.25)
    out = {"requests": len(stream), "rate_hz": rate, "seconds": seconds, "reyes_fraction": 0.2,
           "hbm_budget_bytes": 120 << 30}
    for name, opts in (("continuous", dict(lanes=3, max_batch=64)), ("plain_loop", dict(lanes=1, max_batch=1))):
        server = pk.Server(ctx, hbm_budget_bytes=120 << 30, max_slots=256, max_pixels=1920 * 1080, **opts)
        serve.replay(server, warm, rs, ys)
        server.drain(600000)
        server.reset_stats()
        serve.replay(server, stream, rs, ys)
        server.drain(600000)
        st = server.stats()
        server.close()
        out[name] = {"p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"], "max_ms": st["max_ms"],
                     "completed": int(st["completed"]), "throughput_rps": st["completed"] / max(st["span_s"], 1e-9),
                     "mean_batch": st["mean_batch"], "hbm_bytes": int(st["hbm_bytes"])}
    return out


def run_served(pk, ctx, args):
    """The served workload: a Poisson request stream at --serve-rate requests/s
    (2,000/s) for --serve-seconds (10 s); 80% raster requests on the 64
    resident mix scenes with a re-seeded camera each, 20% Reyes requests (the
    sphere workload, orbiting camera); admission against a 120 GiB HBM budget.
    Continuous batching (3 streams in flight, up to 64 requests per launch
    sequence) vs one request per launch sequence; latency = submit to
    completion on the host clock.  A second, labelled stress line replays a
    shorter stream at --stress-rate, above what one request per launch
    sustains, where batching has queued requests to merge."""
    mix = pk.scenes.batch_mix(64)
    rpipe = pk.Pipe(ctx, "raster", tile_px=args.tile)
    ypipe = pk.Pipe(ctx, "reyes", **REYES_WORKLOAD)
    rs = [pk.Scene(rpipe, s) for s in mix]
    ys = [pk.Scene(ypipe, pk.scenes.sphere_patches())]
    out = serve_stream(pk, ctx, rs, ys, args.serve_rate, args.serve_seconds, seed=7)
    if args.stress_rate > 0:
        out["stress"] = serve_stream(pk, ctx, rs, ys, args.stress_rate, args.stress_seconds, seed=17)
    for s in rs + ys:
        s.close()
    rpipe.close()
    ypipe.close()
    return out


if __name__ == "__main__":
    main()
