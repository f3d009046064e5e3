"""Benchmarks of the hot path on B200. Prints one JSON line (rank 0).

--workload serve (default): the served request stream (configuration 4): 64 resident scenes, jobs of
{256^2, 720p, 1080p} x {4, 16, 64} spp arriving as Poisson streams at 50, 200 and 800 jobs/s, served
in waves by lrc_server (continuous batching under an HBM budget) and, in the same run, one at a time
through lrc_trace; Mrays/s of the served streams, p50/p99 latency of both, the offered load, a
stream below capacity and an end-to-end pass with images read back to the host.

--workload builder: a BVH build (LBVH or PLOC over N triangles) plus one pass of
closest-hit rays through it. N = 4M triangles with centroids uniform in the unit cube, Gaussian
edges (sigma = 0.002 N^-1/3), 2 % of them scaled x50; 16M rays from a sphere of radius 2 toward
uniform points of the cube. One step = triangle boxes, Morton codes, radix sort, hierarchy (PLOC
by default: the reference's builder for meshes), then 16M closest-hit queries. Mrays/s of the step.

--workload batch: the multi-scene launch. 256 box scenes (icospheres and bevelled boxes in the
open box with its lamp) with triangle counts log-uniform in [1k, 200k], resolutions from {128^2,
256^2, 512^2}, spp from {8, 32, 128}, depth 8. One step = every scene built (LBVH, then PLOC) and
every image traced, all in one CUDA graph of the batch engine (persistent path-regenerating trace
kernel, launch shape picked by the autotuner). The plain path - per scene two builds and one
lrc_trace launch, one scene after another - is timed in the same run on the same jobs; its images
equal the batched ones to the bit (checked every run), so the RMSE is equal by construction.
Mrays/s (closest-hit + shadow rays, counted on the device) of the step.

--workload caustics: light-traced caustics of the plain render (the box, its lamp and 64
icospheres, 256^2) with the reference render's default of one light path per camera path (256^2
x 16 spp = 1M light paths per step, lrc_caustics_sums into device sums, fast mode). Mrays/s
(closest-hit + shadow rays) of the step; the reference's light_trace_caustics on this host's cores
is the baseline.

--workload media: the plain render's box with 16 icospheres and a 40x32x40-voxel cloud of
participating medium (foggy_cornell), 256x256, 16 spp: the plain path and the megakernel batch
(the wavefront does not take media); the reference's trace_image with the same Volume as the
baseline.

--workload textures: the plain render's box with 16 icospheres and textured materials (a colour
checker, a metal-rough map and a bump normal map, 64x64 RGBA8; textured_cornell), 256x256, 16 spp;
the reference's trace_image with the same TexMaps as the baseline.

--workload denoise: the denoiser (prep + 5 a-trous passes) on a 1920x1080 image of the plain
render's scene at 4 spp (guide + guided samples made once, outside the timed region). Mpixels/s;
roofline against HBM with 232 algorithmic bytes per pixel (prep reads the 4 planes, 64 B, and
writes 16; each pass reads its 8 + 8 B and writes 8; the last reads the albedo, 16, and writes
the image, 16). The baseline is the numpy restatement of the filter (the reference's own runs only
as WGSL) on a 480x270 crop.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload serve|builder|batch|...] ...
  python bench.py --impl reference ...   the reference's own CPU path on this host's cores

Multi-GPU: replicas (each rank builds and traces its own copy of the workload; no collective on the
data path), timed as the max over ranks.
"""
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

METRIC = "Mrays/s (build + closest-hit pass over the builder workload)"
METRIC_BATCH = "Mrays/s (256-scene batched launch: builds + path tracing, closest-hit + shadow rays)"
METRIC_SERVE = "Mrays/s and p50/p99 job latency (served request stream, Poisson arrivals)"
METRIC_RENDER = "Mrays/s (one image: closest-hit + shadow rays)"
METRIC_DENOISE = "Mpixels/s (denoiser: prep + 5 a-trous passes, 1920x1080)"
METRIC_CAUSTICS = "Mrays/s (light-traced caustics: closest-hit + shadow rays of the light paths)"
METRIC_REALTIME = "frames/s (moving camera: guide + temporal gradients + reprojection + 1-spp guided trace + denoise)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=4 * 1024 * 1024)
    ap.add_argument("--rays", type=int, default=16 * 1024 * 1024)
    ap.add_argument("--builder", default="ploc", choices=["ploc", "lbvh"])
    ap.add_argument("--bits", type=int, default=30, choices=[30, 63])
    ap.add_argument("--walk", type=int, default=1, choices=[0, 1, 2],
                    help="builder: the ray queries' walk (lrc_scene_set_walk): 0 the tree as built, 1 tight boxes, "
                         "2 tight 8-wide quantised nodes")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="builder: the soup and its rays scaled by this (555: the reference's scene units, where the "
                         "triangles' 1e-3 box padding has its intended relative size)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--workload", default="serve", choices=["builder", "batch", "serve", "render", "instanced",
                                                                     "caustics", "denoise", "media", "textures",
                                                                     "realtime"])
    ap.add_argument("--rates", default="50,200,800", help="serve: Poisson arrival rates (jobs/s)")
    ap.add_argument("--budget-gb", type=float, default=24.0, help="serve: the server's HBM budget for jobs")
    ap.add_argument("--wave-paths", type=int, default=32 << 20, help="serve: paths per wave")
    ap.add_argument("--wave-slots", type=int, default=1 << 23, help="serve: the waves' paths in flight")
    ap.add_argument("--wave-variant", type=int, default=None,
                    help="serve: the waves' wavefront launch shape (lrc_server_set_wavefront's variant; default "
                         "LRC_WAVEFRONT_DEFAULT_VARIANT)")
    ap.add_argument("--serve-policy", type=int, default=2, choices=[0, 1, 2],
                    help="serve: how a wave is made (lrc_server_set_policy: 0 even shares, 1 oldest first, "
                         "2 fewest paths left first)")
    ap.add_argument("--denoise-low-spp", action="store_true",
                    help="serve: jobs of 4 spp are denoised (LRC_SERVE_DENOISE; the plain path: guide, guided "
                         "trace, lrc_denoise)")
    ap.add_argument("--scenes", type=int, default=256, help="batch: scenes (jobs)")
    ap.add_argument("--plain-steps", type=int, default=1, help="batch: timed passes of the plain path")
    ap.add_argument("--cpu-scenes", type=int, default=8, help="batch: scenes the CPU baseline samples")
    ap.add_argument("--engine", default="wavefront", choices=["wavefront", "megakernel"], help="batch: the engine")
    ap.add_argument("--split-samples", action="store_true",
                    help="render: one image traced by all ranks, each a share of every pixel's samples, then one "
                         "sum all-reduce (strong scaling)")
    ap.add_argument("--stepped", action="store_true",
                    help="batch, render, instanced: the wavefront engine's passes launched from the host (for ncu, "
                         "which cannot see into graph loops)")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)      # (at least 3 untimed steps before the timed ones)
    return a


# DRAM bytes read + written by one launch of the builder line's closest-hit kernel at the default
# configuration (4M soup triangles, 16M rays, PLOC 30-bit, the walk's tree) and that launch's
# duration under the profiler: one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum,
# gpu__time_duration.sum) of the 4th closest_kernel launch in
# `python bench.py --workload builder --steps 1 --warmup 3 --no-cpu --e2e-steps 1`
BUILDER_CLOSEST_DRAM = {"bytes_per_launch": 216.0e9, "ms_per_launch": 127.97}


def config(a, world):
    scaled = f", scaled x{a.scale:g}" if a.scale != 1.0 else ""
    c = {"workload": f"builder+closest-hit: {a.n} triangles (soup{scaled}), {a.rays} rays, {a.builder.upper()} "
                     f"{a.bits}-bit Morton", "triangles": a.n, "rays": a.rays, "builder": a.builder,
         "key_bits": a.bits, "walk": ("tree as built", "tight boxes", "8-wide quantised nodes")[a.walk],
         "parallelism": f"replicas x{world}",
         "l2": "inputs larger than L2 (triangles 48 B x N + rays 24 B x R > 126 MB)"}
    if a.scale != 1.0:
        c["scale"] = a.scale
    return c


def max_over_ranks(ms, dist, device):
    """The step time of the job: the slowest rank's (all ranks take part; one rank: as is)."""
    if not dist:
        return ms
    import torch
    t = torch.tensor([float(ms)], device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def library_sort_ms(n, bits, stream, device, reps=10):
    """A library radix sort of as many keys, for comparison with the build's sort: torch.sort
    (stable, CUB's radix sort underneath) of n uniform keys of the build's width, returning the
    sorted keys and the permutation (int64 indices: 4 bytes a key more per pass than the build's
    32-bit items), timed by CUDA events on the build's stream after 3 warm-up calls."""
    import torch
    g = torch.Generator(device=device).manual_seed(5)
    if bits == 63:
        keys = torch.randint(0, 1 << 62, (n,), dtype=torch.int64, device=device, generator=g)
    else:
        keys = torch.randint(0, 1 << bits, (n,), dtype=torch.int32, device=device, generator=g)
    for _ in range(3):
        torch.sort(keys, stable=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        torch.sort(keys, stable=True)
    e1.record(stream)
    torch.cuda.synchronize()
    return {"what": "torch.sort(stable=True) of the same number of uniform %d-bit keys, with int64 indices" % bits,
            "ms_per_sort": e0.elapsed_time(e1) / reps}


def whole_job_rate(units_per_rank, world, ms):
    """Replicas: every rank processed units_per_rank units in the job's ms; the whole job's rate
    in millions of units per second (weak scaling: the work grows with the ranks)."""
    return world * units_per_rank / (ms / 1e3) / 1e6


class Clocks:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={self.Q}", "--format=csv,noheader",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except subprocess.TimeoutExpired:
                self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        mhz = [float(r[1].split()[0]) for r in rows if r[1].strip().split()[0].replace(".", "").isdigit()]
        mx = [float(r[2].split()[0]) for r in rows if r[2].strip().split()[0].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_baseline(a, cor, orig, dirs, sample_rays):
    """The reference's own CPU path on this host's cores: 4-wide SAH build (scene_set_accel) +
    scene_intersect over a bounded sample of the rays; Mrays/s of the whole workload estimated as
    rays / (build + sample time x rays / sample)."""
    from oracle import oracle as O
    lib = O.ref_lib()
    cores = lib.rb_max_threads()
    ref = O.RefScene()
    ref.material(0, (0.5, 0.5, 0.5))
    ref.triangles(cor, np.zeros(cor.shape[0], np.int32))
    t0 = time.perf_counter()
    ref.set_accel()
    t_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    ref.intersect(orig[:sample_rays], dirs[:sample_rays])
    t_trace = time.perf_counter() - t0
    ref.close()
    total = t_build + t_trace * (a.rays / sample_rays)
    return {"value": a.rays / total / 1e6, "unit": "Mrays/s", "cores": cores, "kind": "reference",
            "sample": f"scene_set_accel (4-wide SAH) over all {a.n} triangles ({t_build:.2f} s) + scene_intersect "
                      f"of {sample_rays} of the {a.rays} rays ({t_trace:.2f} s), scaled to all rays"}


def run_reference(a):
    """--impl reference --workload builder: the reference's own CPU implementation of the path (SAH
    BVH build + scene_intersect of every ray) on this host's cores, each step the whole workload
    (about 25 s on 16 cores: no sample is scaled up)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from little_renderer_b200 import workloads as W
    cor = W.soup(a.n, 1) * np.float32(a.scale)
    sample = a.rays
    o, d = W.rays_at_cube(sample, 2, scale=a.scale)
    from oracle import oracle as O
    lib = O.ref_lib()
    cores = lib.rb_max_threads()
    times = []
    for step in range(a.warmup + a.steps):
        ref = O.RefScene()
        ref.material(0, (0.5, 0.5, 0.5))
        ref.triangles(cor, np.zeros(a.n, np.int32))
        t0 = time.perf_counter()
        ref.set_accel()
        tb = time.perf_counter() - t0
        t0 = time.perf_counter()
        ref.intersect(o, d)
        tt = time.perf_counter() - t0
        ref.close()
        if step >= a.warmup:
            times.append(tb + tt * (a.rays / sample))
    ms = 1e3 * statistics.median(times)
    v = a.rays / (ms / 1e3) / 1e6
    line = {"metric": METRIC, "value": v, "unit": "Mrays/s", "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference", "config": config(a, 1),
            "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": cores, "kind": "reference",
                             "sample": f"per step: scene_set_accel (4-wide SAH) over {a.n} triangles + "
                                       f"scene_intersect of all {a.rays} rays"},
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def batch_config(a, world, jobs):
    px = sum(sc["width"] * sc["height"] for sc in jobs)
    paths = sum(sc["width"] * sc["height"] * sc["spp"] for sc in jobs)
    tris = sum(sc["corners"].shape[0] for sc in jobs)
    return {"workload": f"batched multi-scene launch: {len(jobs)} box scenes, triangles log-uniform in [1k, 200k] "
                        f"({tris} in all), resolutions {{128^2, 256^2, 512^2}}, spp {{8, 32, 128}}, depth 8; builds "
                        "LBVH then PLOC per scene; one CUDA graph", "scenes": len(jobs), "triangles": tris,
            "pixels": px, "paths": paths, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (all scenes' triangles and trees, images and per-task sums > 126 MB)"}


def ref_box_scene(O, sc):
    ref = O.RefScene()
    for m in sc["materials"]:
        ref.material(m["type"], m["albedo"], m["emission"], m["ior"], m["metallic"], m["roughness"], m["transmission"])
    ref.triangles(sc["corners"], sc["tri_mats"])
    lamp = sc["lamp"]
    ref.quad(lamp["q"], lamp["u"], lamp["v"], lamp["material"], light=True)
    return ref


def batch_cpu_sample(a, jobs, seconds=20.0):
    """The reference's CPU path tracer (scene_set_accel + trace_image, all host cores) on a fixed
    seeded subset of the jobs: the first cpu_scenes scenes, each built and a band of its rows traced
    at the job's spp (about 300k paths per scene, fewer once `seconds` are spent). Returns
    (Mrays/s, cores, sample text)."""
    from oracle import oracle as O
    lib = O.ref_lib()
    cores = lib.rb_max_threads()
    rays = 0
    t_all = 0.0
    done = []
    for i, sc in enumerate(jobs[:a.cpu_scenes]):
        if t_all > seconds:
            break
        ref = ref_box_scene(O, sc)
        c = sc["camera"]
        fau = np.array([*c["from"], *c["at"], *c["up"]], np.float32)
        w, h, spp = sc["width"], sc["height"], sc["spp"]
        rows = max(1, min(h, 300_000 // (w * spp)))
        t0 = time.perf_counter()
        ref.set_accel()
        _, (closest, shadow) = ref.trace_image(fau, c["vfov"], w, h, spp, i, sc["max_depth"], y0=h // 2 - rows // 2,
                                               rows=rows)
        t_all += time.perf_counter() - t0
        rays += closest + shadow
        done.append(f"{sc['corners'].shape[0]} tris {w}x{rows} rows x {spp} spp")
        ref.close()
    return rays / t_all / 1e6, cores, (f"the first {len(done)} scenes of the batch (scene_set_accel, 4-wide SAH, + "
                                       f"trace_image of a central band): " + "; ".join(done) +
                                       f"; {rays} rays in {t_all:.1f} s; the whole batch extrapolated at that rate")


def run_reference_batch(a):
    """--impl reference --workload batch: the reference's CPU path tracer on this host's cores, each
    step the bounded sample of batch_cpu_sample (the whole batch would take hours)."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    from little_renderer_b200 import workloads as W
    jobs = W.batch_scenes(a.scenes, seed=11)
    vals = []
    for step in range(a.warmup + a.steps):
        v, cores, sample = batch_cpu_sample(a, jobs, seconds=4.0)
        if step >= a.warmup:
            vals.append(v)
    v = statistics.median(vals)
    line = {"metric": METRIC_BATCH, "value": v, "unit": "Mrays/s", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "impl": "reference", "config": batch_config(a, 1, jobs),
            "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": cores, "kind": "reference", "sample": sample},
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_batch(a):
    import torch
    import little_renderer_b200 as L
    from little_renderer_b200 import render as R, workloads as W

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    jobs = W.batch_scenes(a.scenes, seed=11 + rank)
    ctx = L.Context(local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    scenes = [R.world_scene(ctx, sc, 0) for sc in jobs]
    params = [L.native.trace_params(R.camera12(sc), sc["width"], sc["height"], sc["max_depth"], 1, 1, 0, 1000 + i)
              for i, sc in enumerate(jobs)]
    imgs = [torch.zeros(sc["height"], sc["width"], 4, device=dev) for sc in jobs]
    torch.cuda.synchronize()

    def plain_step():
        for s, p, img, sc in zip(scenes, params, imgs, jobs):
            s.build(0, 30)
            s.build(1, 30)
            s.trace_device(p, sc["spp"], img.data_ptr())

    def timed(fn, n):
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ctx.sync()
        return max_over_ranks(e0.elapsed_time(e1), dist, dev)

    # the plain path: one pass for its images (and its warm-up), then the timed passes
    for img in imgs:
        img.zero_()
    plain_step()
    ctx.sync()
    torch.cuda.synchronize()
    plain_imgs = [img.cpu() for img in imgs]
    plain_ms = timed(plain_step, a.plain_steps) / a.plain_steps

    def builds_step():
        for s in scenes:
            s.build(0, 30)
            s.build(1, 30)

    build_ms = timed(builds_step, 1)

    # the batch: every job with LBVH-then-PLOC builds; the autotuner's shape; one graph per step
    b = L.native.Batch(ctx)
    b.set_engine(1 if a.engine == "wavefront" else 0)
    for s, p, img, sc in zip(scenes, params, imgs, jobs):
        b.add(s, p, sc["spp"], img.data_ptr(), builder=2, key_bits=30)
    b.run(build=True, zero=True)
    variant, grid, ns_task = b.tune()
    shapes = L.native.wavefront_shapes() if a.engine == "wavefront" else L.native.batch_shapes()
    def batch_step():
        if a.stepped:
            b.run(build=True, zero=True, stepped=True)
        else:
            b.run(build=True, graph=True, zero=True)

    for _ in range(a.warmup):
        batch_step()
    ctx.sync()
    torch.cuda.synchronize()
    batch_imgs = [img.cpu() for img in imgs]
    same = all(torch.equal(x, y) for x, y in zip(plain_imgs, batch_imgs))
    _, rays = b.rays()
    clk = Clocks(local)
    ms = timed(batch_step, a.steps)
    clocks = clk.stop()
    info = b.info()
    ms_step = ms / a.steps
    value = world * rays * a.steps / (ms / 1e3) / 1e6
    plain_value = world * rays / (plain_ms / 1e3) / 1e6

    # end to end through the public API with host buffers: every scene's triangles copied in from
    # pinned memory, the batch run (builds + trace), every image copied out, inside each step
    pins = [torch.from_numpy(L.pack_tris(W.corners_to_quv(sc["corners"]), sc["tri_mats"]).view(np.int32)).pin_memory()
            for sc in jobs]
    host_tris = [p.numpy().view(np.uint32) for p in pins]
    outs = [torch.empty(sc["height"], sc["width"], 4).pin_memory() for sc in jobs]

    def e2e_step():
        for t, s in zip(host_tris, scenes):
            s.set_triangles(t)
        b.run(build=True, graph=True, zero=True)
        for o, img in zip(outs, imgs):
            o.copy_(img, non_blocking=True)

    e2e_step()
    e2e_steps = max(1, min(a.steps, 3))
    e_ms = timed(e2e_step, e2e_steps) / e2e_steps
    _, e2e_rays = b.rays()
    e2e = {"value": world * rays / (e_ms / 1e3) / 1e6, "unit": "Mrays/s",
           "h2d_bytes_per_step": int(sum(p.numel() * 4 for p in pins)),
           "d2h_bytes_per_step": int(sum(o.numel() * 4 for o in outs)), "ms_per_step": e_ms,
           "images_equal_plain": all(torch.equal(x, y) for x, y in zip(plain_imgs, outs)),
           "rays_equal": bool(e2e_rays == rays)}

    peak, peak_kind = peaks()
    line = {"metric": METRIC_BATCH, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": batch_config(a, world, jobs),
            "clocks": clocks, "e2e": e2e,
            "gpu_launches": a.steps * (len(jobs) * (5 + 4 + 6) + 2),
            "plain": {"value": plain_value, "unit": "Mrays/s", "ms_per_step": plain_ms, "builds_ms": build_ms,
                      "what": "per scene: LBVH build, PLOC build, one lrc_trace launch; scenes one after another"},
            "speedup_vs_plain": value / plain_value, "images_equal_plain": bool(same),
            "rays_per_step": int(rays), "paths_per_step": int(sum(sc["width"] * sc["height"] * sc["spp"] for sc in jobs)),
            "batch": {"engine": a.engine, "tasks": info["tasks"],
                      "shape": dict(zip(("block", "minb", "per_sm"), shapes[variant])),
                      ("paths_in_flight" if a.engine == "wavefront" else "grid"): grid,
                      "ns_per_task_tuned": ns_task, "graph_replayed": info["graph_used"]},
            "roofline": {"bound": "hbm", "kernel": "batch_kernel", "achieved": None, "peak": peak, "unit": "GB/s",
                         "peak_kind": peak_kind, "frac": None, "traffic": None,
                         "note": "latency-bound traversal over L2-resident scenes; DRAM traffic from the ncu summary"}}
    if rank == 0 and world == 1 and not a.no_cpu:
        v, cores, sample = batch_cpu_sample(a, jobs)
        line["cpu_baseline"] = {"value": v, "unit": "Mrays/s", "cores": cores, "kind": "reference", "sample": sample}
    b.close()
    for s in scenes:
        s.close()
    ctx.close()
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


SERVE_JOBS_PER_STEP = 5      # a serve step: 5 jobs of each rate's stream
# DRAM bytes read + written by one launch of the served line's closest-hit kernel, and that
# launch's duration under the profiler: one ncu capture (dram__bytes_read.sum +
# dram__bytes_write.sum, gpu__time_duration.sum) of launches 81-83 of wf_intersect_kernel in
# `python bench.py --steps 2 --warmup 3 --rates 200` (the timed stepped run's full-queue passes)
SERVE_ISECT_DRAM = {"bytes_per_launch": 474.4e6, "ms_per_launch": 3.74}


def serve_jobs(n, rate, seed, nscenes, inst_ids):
    """n jobs with Poisson arrivals at `rate`/s: (arrival s, scene index, width, height, spp, motion
    frame or None); a tenth of them move the instances of an instanced scene."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    res = [(256, 256), (1280, 720), (1920, 1080)]
    out = []
    for i in range(n):
        w, h = res[rng.integers(0, 3)]
        spp = int(rng.choice([4, 16, 64]))
        if rng.random() < 0.1:
            out.append((float(t[i]), int(rng.choice(inst_ids)), w, h, spp, float(rng.uniform(1, 30))))
        else:
            out.append((float(t[i]), int(rng.integers(0, nscenes)), w, h, spp, None))
    return out


def serve_world_counts():
    """The triangle counts of the stream's 56 box scenes (log-uniform in [1k, 2M], seeded)."""
    rng = np.random.default_rng(17)
    lo, hi = np.log(1_000), np.log(2_000_000)
    return [int(np.exp(rng.uniform(lo, hi))) for _ in range(56)]


class ServeWorlds:
    """The stream's box scenes made on first use (scene k is box_scene(5000 + k, counts[k]))."""

    def __init__(self):
        self.counts = serve_world_counts()
        self.made = {}

    def __getitem__(self, k):
        from little_renderer_b200 import workloads as W
        if k not in self.made:
            self.made[k] = W.box_scene(5000 + k, self.counts[k], 256, 256, 16)
        return self.made[k]


def serve_scene_dicts():
    """The 64 resident scenes of the served stream: 56 box scenes (triangles log-uniform in [1k, 2M])
    and 8 instanced boxes of 2000 instances; (dicts, indices of the instanced ones, triangles)."""
    from little_renderer_b200 import workloads as W
    worlds = ServeWorlds()
    dicts = [worlds[k] for k in range(56)]
    inst_ids = []
    for i in range(8):
        dicts.append(W.instanced_box(6000 + i, n_instances=2000))
        inst_ids.append(len(dicts) - 1)
    tris = sum(worlds.counts) + sum(len(dicts[k]["corners"]) for k in inst_ids)
    return dicts, inst_ids, tris


def serve_cpu_jobs(nscenes_world, seed, count):
    """A seeded sample of the stream's jobs the reference's CPU path tracer traces whole: world
    scenes only (no moved instances), jobs of at most 4M paths (256^2 at any spp, 720p at 4 spp)."""
    rng = np.random.default_rng(seed)
    out = []
    res = [(256, 256), (1280, 720)]
    while len(out) < count:
        w, h = res[rng.integers(0, 2)]
        spp = int(rng.choice([4, 16, 64]))
        if w * h * spp > 4 << 20:
            continue
        out.append((int(rng.integers(0, nscenes_world)), w, h, spp, int(rng.integers(0, 1 << 30))))
    return out


def serve_cpu_sample(dicts, seconds, seed=23):
    """The reference's trace_image (scene_set_accel, 4-wide SAH, all host cores) on whole sampled
    jobs of the stream until `seconds` are spent: (Mrays/s, cores, rays, seconds, description)."""
    from oracle import oracle as O
    from little_renderer_b200 import workloads as W
    lib = O.ref_lib()
    cores = lib.rb_max_threads()
    rays, t_all, done, built = 0, 0.0, [], {}
    for k, w, h, spp, jseed in serve_cpu_jobs(56, seed, 64):
        if t_all > seconds:
            break
        sc = dicts[k]
        if k not in built:
            ref = ref_box_scene(O, sc)
            ref.set_accel()                          # (the scene's tree is resident, as the served scenes')
            built[k] = ref
        ref = built[k]
        c = sc["camera"]
        fau = np.array([*c["from"], *c["at"], *c["up"]], np.float32)
        t0 = time.perf_counter()
        _, (closest, shadow) = ref.trace_image(fau, c["vfov"], w, h, spp, jseed, sc["max_depth"])
        t_all += time.perf_counter() - t0
        rays += closest + shadow
        done.append(f"{sc['corners'].shape[0]} tris {w}x{h} x {spp} spp")
    for ref in built.values():
        ref.close()
    text = (f"trace_image of {len(done)} whole jobs of the stream (world scenes, jobs of at most 4M paths; "
            f"trees built beforehand as the served scenes' are resident): " + "; ".join(done) +
            f"; {rays} rays in {t_all:.1f} s")
    return rays / t_all / 1e6, cores, rays, t_all, text


def run_reference_serve(a):
    """--impl reference --workload serve: the reference has no server; its own CPU path tracer
    (trace_image on this host's cores) on whole sampled jobs of the same stream, each step about
    3 s of them; Mrays/s."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    dicts = ServeWorlds()                             # (only the sampled scenes are made)
    tris = None
    vals, rays_all, secs_all, text = [], 0, 0.0, ""
    for step in range(a.warmup + a.steps):
        v, cores, rays, secs, text = serve_cpu_sample(dicts, 3.0, seed=100 + step)
        if step >= a.warmup:
            vals.append(v)
            rays_all += rays
            secs_all += secs
    v = rays_all / secs_all / 1e6
    line = {"metric": METRIC_SERVE, "value": v, "unit": "Mrays/s", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1e3 * secs_all / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": serve_config(a, tris),
            "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": cores, "kind": "reference",
                             "sample": "per step about 3 s of " + text.split(":")[0] + " (seeded, one sample a step)"},
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "step_values": vals}
    print(json.dumps(line), flush=True)


def serve_config(a, tris):
    tris = f"{tris} triangles: " if tris else ""
    return {"workload": f"served request stream: 64 resident scenes ({tris}56 box scenes of 1k-2M "
                        "triangles, 8 instanced boxes of 2000 instances), jobs {256^2, 720p, 1080p} x spp "
                        "{4, 16, 64}, depth 8, a tenth moving their scene's 2000 instances (top level refit), "
                        "Poisson arrivals", "rates": a.rates, "jobs_per_step": SERVE_JOBS_PER_STEP,
            "jobs_per_rate": SERVE_JOBS_PER_STEP * a.steps, "budget_gb": a.budget_gb, "wave_paths": a.wave_paths,
            "wave_slots": a.wave_slots, "wave_variant": a.wave_variant, "serve_policy": a.serve_policy,
            "parallelism": "one GPU",
            "denoise_low_spp": bool(a.denoise_low_spp),
            "l2": "inputs larger than L2 (resident scenes' triangles and trees, images, wavefront state > 126 MB)"}


def run_serve(a):
    """--workload serve (the default): the served request stream (configuration 4). 64 resident
    scenes; jobs (scene, resolution in {256^2, 720p, 1080p}, spp in {4, 16, 64}; a tenth move their
    scene's 2000 instances: the top level refit first) arriving as a Poisson stream at each rate,
    served in waves by lrc_server under an HBM budget; then the same stream through the plain path
    one job at a time (lrc_trace per job, in arrival order). A step is SERVE_JOBS_PER_STEP jobs of
    every rate's stream: --steps K times K x 5 jobs at each rate, after --warmup W x 5 untimed jobs.
    Latency = end - arrival (host clock). A stream at 0.8 x the measured served capacity follows
    (below capacity, where a latency is a latency and not a backlog), then the middle rate's stream
    served again end to end (each image read back to pinned host memory inside the span)."""
    import torch
    import little_renderer_b200 as L
    if a.wave_variant is None:
        a.wave_variant = L.native.LRC_WAVEFRONT_DEFAULT_VARIANT
    from little_renderer_b200 import render as R, workloads as W

    if int(os.environ.get("RANK", "0")) != 0:
        return
    dev = torch.device("cuda", 0)
    ctx = L.Context(0)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    dicts, inst_ids, tris = serve_scene_dicts()
    scenes = [R.instanced_box_scene(ctx, sc, 1) if k in inst_ids else R.world_scene(ctx, sc, 1)
              for k, sc in enumerate(dicts)]
    motions = {k: W.rigid_motion(2000, 7000 + k) for k in inst_ids}
    originals = {k: W.instance_records(dicts[k]) for k in inst_ids}
    ctx.sync()
    jps = SERVE_JOBS_PER_STEP

    def records(job):
        k, frame = job[1], job[5]
        return W.instance_records(dict(dicts[k], xf=W.moved_xf(dicts[k]["xf"], motions[k], frame)))

    def params(job, idx):
        sc = dicts[job[1]]
        return L.native.trace_params(W.camera(sc["camera"], job[2] / job[3]), job[2], job[3], 8, 1, 1, 0, 9000 + idx)

    def pct(x, q):
        return float(np.percentile(np.asarray(x), q)) if len(x) else None

    def denoised(job):
        return bool(a.denoise_low_spp and job[4] == 4)

    def served(jobs, recs, keep=0, readback=False):
        """lrc_server over the stream: submit each job at its arrival, step waves while any is held.
        keep: images of the first jobs kept (host); readback: every image read to pinned host memory."""
        sv = L.native.Server(ctx, int(a.budget_gb * 2**30), a.wave_paths)
        sv.set_wavefront(a.wave_slots, a.wave_variant)
        sv.set_policy(a.serve_policy)
        pinned = torch.empty(1920 * 1080 * 4, dtype=torch.float32).pin_memory() if readback else None
        lat, rays, ids, kept, d2h = [], 0, {}, {}, 0
        nxt, done = 0, 0
        t0 = L.native.clock_ms()
        while done < len(jobs):
            now = (L.native.clock_ms() - t0) / 1e3
            while nxt < len(jobs) and jobs[nxt][0] <= now:
                j = jobs[nxt]
                ids[sv.submit(scenes[j[1]], params(j, nxt), j[4], recs[nxt], 0, denoise=denoised(j))] = nxt
                nxt += 1
            st = sv.state()
            if st["queued"] + st["active"] == 0:
                if nxt < len(jobs):
                    time.sleep(max(0.0, min(0.002, jobs[nxt][0] - now)))
                continue
            if sv.step():
                for jid, k in list(ids.items()):
                    r = sv.result(jid)
                    if r is None:
                        continue
                    if readback:
                        nb = jobs[k][2] * jobs[k][3] * 16
                        ctx.check(ctx.L.lrc_server_read(sv.h, jid, L.native.C.c_void_p(pinned.data_ptr())))
                        d2h += nb
                        t_end = L.native.clock_ms()
                    else:
                        t_end = r[4]
                    lat.append(t_end - (t0 + jobs[k][0] * 1e3))
                    rays += r[1]
                    if k < keep:
                        kept[k] = sv.image(jid)
                    sv.release(jid)
                    del ids[jid]
                    done += 1
        span = (L.native.clock_ms() - t0) / 1e3
        waves, kernels, gpu_ms = sv.stats()
        sv.close()
        return {"lat": lat, "rays": rays, "span": span, "kept": kept, "d2h": d2h, "waves": waves, "kernels": kernels,
                "gpu_s": gpu_ms / 1e3}

    def plain(jobs, recs, keep=0, flags=0):
        """One job at a time in arrival order, each traced alone through lrc_trace (large ones on the
        wavefront engine, as lrc_trace runs them; flags LRC_TRACE_MEGAKERNEL: all on the one-kernel
        path); the scene put back after a moved-instance job."""
        lat, rays, kept = [], 0, {}
        t0 = L.native.clock_ms()
        for k, j in enumerate(jobs):
            now = (L.native.clock_ms() - t0) / 1e3
            if j[0] > now:
                time.sleep(j[0] - now)
            s = scenes[j[1]]
            if recs[k] is not None:
                s.move_instances(recs[k], 0)
            img = torch.zeros(j[3], j[2], 4, device=dev)
            p = params(j, k)
            nr = L.native.C.c_uint64()
            if denoised(j):
                planes = torch.zeros(4, j[3], j[2], 4, device=dev)
                s.guide_device(p, planes.data_ptr())
                ctx.check(ctx.L.lrc_trace(s.h, L.native.C.byref(p), 0, j[3], 0, j[4],
                                          L.native.C.c_void_p(planes.data_ptr()), L.native.C.byref(nr),
                                          L.native.LRC_TRACE_GUIDED | L.native.LRC_DEVICE | flags))
                ctx.denoise_device(j[2], j[3], planes.data_ptr(), img.data_ptr())
            else:
                ctx.check(ctx.L.lrc_trace(s.h, L.native.C.byref(p), 0, j[3], 0, j[4],
                                          L.native.C.c_void_p(img.data_ptr()), L.native.C.byref(nr),
                                          L.native.LRC_DEVICE | flags))
            if recs[k] is not None:
                s.move_instances(originals[j[1]], 0)
            ctx.sync()
            rays += nr.value
            lat.append(L.native.clock_ms() - (t0 + j[0] * 1e3))
            if k < keep:
                kept[k] = img.cpu().numpy()
        span = (L.native.clock_ms() - t0) / 1e3
        for k in inst_ids:
            scenes[k].move_instances(originals[k], 1)
        return {"lat": lat, "rays": rays, "span": span, "kept": kept}

    def stream_of(rate, n, seed):
        jobs = serve_jobs(n, rate, seed, 56, inst_ids)
        return jobs, [records(j) if j[5] is not None else None for j in jobs]

    rates = [float(r) for r in a.rates.split(",")]
    # warm-up (untimed): W steps' jobs of the first rate, served and plain
    wj, wr = stream_of(rates[0], jps * a.warmup, 999)
    served(wj, wr)
    plain(wj[: max(2, jps)], wr[: max(2, jps)])
    clk = Clocks(0)
    results = {}
    served_rays, served_span, jobs_done, paths_all, check_all, launches, waves = 0, 0.0, 0, 0, True, 0, 0
    n_per_rate = jps * a.steps
    for rate in rates:
        jobs, recs = stream_of(rate, n_per_rate, int(rate))
        sv = served(jobs, recs, keep=4)
        pl = plain(jobs, recs, keep=4)
        equal = all(np.array_equal(sv["kept"][k], pl["kept"][k]) for k in sv["kept"])
        check_all = check_all and equal and sv["rays"] == pl["rays"]
        mean_job_s = sv["span"] / len(jobs)              # (the served stream's time per job at capacity)
        results[str(int(rate))] = {
            "served": {"p50_ms": pct(sv["lat"], 50), "p99_ms": pct(sv["lat"], 99), "mrays_s": sv["rays"] / sv["span"] / 1e6,
                       "span_s": sv["span"], "latency_samples": len(sv["lat"]), "waves": sv["waves"],
                       "device_busy": sv["gpu_s"] / sv["span"]},
            "plain": {"p50_ms": pct(pl["lat"], 50), "p99_ms": pct(pl["lat"], 99), "mrays_s": pl["rays"] / pl["span"] / 1e6,
                      "span_s": pl["span"], "latency_samples": len(pl["lat"])},
            "served_vs_plain": (sv["rays"] / sv["span"]) / (pl["rays"] / pl["span"]),
            "offered_load_rho": rate * mean_job_s,
            "jobs": len(jobs), "motion_jobs": sum(1 for j in jobs if j[5] is not None),
            "paths": int(sum(j[2] * j[3] * j[4] for j in jobs)), "rays": int(sv["rays"]),
            "images_equal_plain": bool(equal), "rays_equal_plain": bool(sv["rays"] == pl["rays"])}
        served_rays += sv["rays"]
        served_span += sv["span"]
        launches += sv["kernels"]
        waves += sv["waves"]
        print(f"serve rate {rate:g}/s: served {sv['span']:.1f} s ({sv['rays'] / sv['span'] / 1e6:.0f} Mrays/s, "
              f"{sv['waves']} waves, device busy {sv['gpu_s'] / sv['span']:.2f}), plain {pl['span']:.1f} s ({pl['rays'] / pl['span'] / 1e6:.0f} Mrays/s); "
              f"images equal {equal}", file=sys.stderr, flush=True)
        jobs_done += len(jobs)
        paths_all += results[str(int(rate))]["paths"]
    # the middle rate's stream once more through the one-kernel path alone (LRC_TRACE_MEGAKERNEL: the
    # plain path before large images went to the wavefront engine)
    mid = rates[len(rates) // 2]
    jobs, recs = stream_of(mid, n_per_rate, int(mid))
    mk = plain(jobs, recs, keep=4, flags=L.native.LRC_TRACE_MEGAKERNEL)
    r_mid = results[str(int(mid))]
    r_mid["plain_megakernel"] = {"p50_ms": pct(mk["lat"], 50), "p99_ms": pct(mk["lat"], 99),
                                 "mrays_s": mk["rays"] / mk["span"] / 1e6, "span_s": mk["span"],
                                 "latency_samples": len(mk["lat"])}
    r_mid["served_vs_plain_megakernel"] = r_mid["served"]["mrays_s"] / r_mid["plain_megakernel"]["mrays_s"]
    print(f"serve rate {mid:g}/s: plain on the one-kernel path {mk['span']:.1f} s "
          f"({mk['rays'] / mk['span'] / 1e6:.0f} Mrays/s)", file=sys.stderr, flush=True)
    clocks = clk.stop()
    # below capacity: 0.8 x the served jobs/s just measured, the same number of jobs
    capacity = jobs_done / served_span
    sub_rate = 0.8 * capacity
    jobs, recs = stream_of(sub_rate, n_per_rate, 4242)
    sv = served(jobs, recs)
    pl = plain(jobs, recs)
    results["sub_capacity"] = {
        "rate_jobs_s": sub_rate, "capacity_jobs_s": capacity,
        "served": {"p50_ms": pct(sv["lat"], 50), "p99_ms": pct(sv["lat"], 99), "mrays_s": sv["rays"] / sv["span"] / 1e6,
                   "span_s": sv["span"], "latency_samples": len(sv["lat"])},
        "plain": {"p50_ms": pct(pl["lat"], 50), "p99_ms": pct(pl["lat"], 99), "mrays_s": pl["rays"] / pl["span"] / 1e6,
                  "span_s": pl["span"], "latency_samples": len(pl["lat"])},
        "jobs": len(jobs)}
    # end to end: the middle rate's stream again, every finished image read back to pinned host
    # memory inside the span; the host sends each job's parameters (and moved instances' records)
    jobs, recs = stream_of(mid, n_per_rate, int(mid))
    e = served(jobs, recs, readback=True)
    h2d = sum(96 + (r.nbytes if r is not None else 0) for r in recs)
    e2e = {"value": e["rays"] / e["span"] / 1e6, "unit": "Mrays/s", "rate_jobs_s": mid,
           "h2d_bytes_per_step": int(h2d / a.steps), "d2h_bytes_per_step": int(e["d2h"] / a.steps),
           "ms_per_step": 1e3 * e["span"] / a.steps, "p50_ms": pct(e["lat"], 50), "p99_ms": pct(e["lat"], 99)}
    # the dominant kernel (the wavefront's closest hit) measured live on a sample of the middle rate's
    # stream: its first jobs without moved instances (about 1G paths) as one batch, run pass by pass (STEPPED: CUDA
    # events around every closest-hit launch), first with the counting build of the kernel (the
    # walks' box and triangle tests: the algorithmic bytes), then with the plain one (its time)
    peak, peak_kind = peaks()
    sample, sample_paths = [], 0
    for k, j in enumerate(jobs):                     # (the first jobs without moved instances, ~1G paths)
        if j[5] is None and sample_paths < 1_000_000_000:
            sample.append((k, j))
            sample_paths += j[2] * j[3] * j[4]
    imgs = [torch.zeros(j[3], j[2], 4, device=dev) for _, j in sample]
    bb = L.native.Batch(ctx)
    bb.set_wavefront(a.wave_slots, a.wave_variant)
    for (k, j), t in zip(sample, imgs):
        bb.add(scenes[j[1]], params(j, k), j[4], t.data_ptr())
    bb.run(zero=True, stepped=True, count=True)
    counted = bb.step_stats()
    bb.run(zero=True, stepped=True)
    timed = bb.step_stats()
    bb.close()
    bytes_per_ray = (counted["box_tests"] * 32 + counted["tri_tests"] * 48) / max(counted["intersect_rays"], 1)
    alg_bytes = bytes_per_ray * timed["intersect_rays"]
    achieved = alg_bytes / (timed["intersect_ms"] / 1e3) / 1e9
    dram_gbs = SERVE_ISECT_DRAM["bytes_per_launch"] / (SERVE_ISECT_DRAM["ms_per_launch"] / 1e3) / 1e9
    roofline = {"kernel": "wf_intersect_kernel (the wavefront's closest hit)", "bound": "hbm", "achieved": achieved,
                "peak": peak, "unit": "GB/s", "peak_kind": peak_kind, "frac": achieved / peak,
                "traffic": SERVE_ISECT_DRAM["bytes_per_launch"],
                "traffic_from": "ncu dram__bytes_read.sum + dram__bytes_write.sum, launches 81-83 of the kernel in "
                                "`python bench.py --steps 2 --warmup 3 --rates 200` (full queues)",
                "dram_gbs": dram_gbs, "frac_dram": dram_gbs / peak,
                "bytes_per_ray": bytes_per_ray, "box_tests_per_ray": counted["box_tests"] / max(counted["intersect_rays"], 1),
                "tri_tests_per_ray": counted["tri_tests"] / max(counted["intersect_rays"], 1),
                "algorithmic_bytes_per_launch": alg_bytes / max((timed["kernels"] - 1) // 4, 1),
                "ms_per_launch": timed["intersect_ms"] / max((timed["kernels"] - 1) // 4, 1),
                "measured_on": f"{len(sample)} jobs of the {mid:g}/s stream as one batch, run pass by pass "
                               f"({timed['intersect_rays']} closest-hit rays, {timed['intersect_ms']:.1f} ms in the "
                               "kernel); bytes per ray = box tests x 32 + triangle tests x 48 from the counting "
                               "build of the kernel on the same run"}
    value = served_rays / served_span / 1e6
    cpu_v, cores, _, _, text = serve_cpu_sample(dicts, 15.0)
    line = {"metric": METRIC_SERVE, "value": value, "unit": "Mrays/s", "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1e3 * served_span / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": serve_config(a, tris), "clocks": clocks, "e2e": e2e, "roofline": roofline,
            "gpu_launches": int(launches), "waves": int(waves),
            "gpu_launches_counted": "the served streams' trace kernels: per wave the wavefront's clear and resolve "
                                    "and 4 kernels a pass (advance, closest hit, shade, shadow), passes read from "
                                    "the device; admission copies, refits and the denoiser not counted",
            "cpu_baseline": {"value": cpu_v, "unit": "Mrays/s", "cores": cores, "kind": "reference", "sample": text},
            "plain_mrays_s": sum(r["plain"]["mrays_s"] * r["plain"]["span_s"] for k, r in results.items()
                                 if k != "sub_capacity") / sum(r["plain"]["span_s"] for k, r in results.items()
                                                               if k != "sub_capacity"),
            "served_vs_plain": None, "equal_rmse": {"images_equal_plain": check_all,
                                                    "how": "the first 4 jobs of each rate: served image = plain "
                                                           "image to the bit, and served rays = plain rays"},
            "rates": results, "jobs_timed": jobs_done, "paths_timed": paths_all}
    plain_rays = sum(r["rays"] for k, r in results.items() if k != "sub_capacity")
    plain_span = sum(r["plain"]["span_s"] for k, r in results.items() if k != "sub_capacity")
    line["plain_mrays_s"] = plain_rays / plain_span / 1e6
    line["served_vs_plain"] = value / line["plain_mrays_s"]
    line["served_vs_plain_megakernel"] = r_mid["served_vs_plain_megakernel"]
    # (the two one-job-at-a-time denominators by name: each job alone through lrc_trace as shipped,
    # which puts large images on the wavefront engine - the best plain path - and, at the middle
    # rate, each job alone on the one-kernel path)
    line["plain_best_mrays_s"] = line["plain_mrays_s"]
    line["plain_megakernel_mrays_s"] = r_mid["plain_megakernel"]["mrays_s"]
    line["denominators"] = ("plain_mrays_s: each job alone through lrc_trace as shipped (jobs of 2^20 paths and "
                            "more on the wavefront engine); served_vs_plain_megakernel: at the middle rate, each "
                            "job alone on the one-kernel path (LRC_TRACE_MEGAKERNEL)")
    for s_ in scenes:
        s_.close()
    ctx.close()
    print(json.dumps(line), flush=True)


def ref_field_scene(O, sc):
    ref = O.RefScene()
    for m in sc["materials"]:
        ref.material(m["type"], m["albedo"], m["emission"], m["ior"], m["metallic"], m["roughness"], m["transmission"])
    g = sc["ground"]
    ref.quad(g["q"], g["u"], g["v"], g["material"])
    for tri, mm in zip(sc["meshes"], sc["mesh_mats"]):
        ref.mesh(tri, np.full(tri.shape[0], mm, np.int32))
    for i in range(sc["xf"].shape[0]):
        ref.instance(int(sc["mesh_of"][i]), sc["xf"][i].reshape(-1), -1)
    ref.env(sc["sky"])
    return ref


def run_render(a):
    """--workload render (configuration 0: the box, its lamp and 64 icospheres, 256^2, 16 spp,
    depth 8) or --workload instanced (configuration 2: 5000 instances of 14 meshes of 10k-100k
    triangles, a 2048 x 1024 sky, 1280 x 720, 64 spp, depth 12). One step = one image. The plain
    path (one lrc_trace launch) is the line's value; the same image through the batch's wavefront
    and its persistent megakernel (one job each, tuned) is timed in the same run; the images are
    compared bit for bit. cpu_baseline: the reference's trace_image (16 cores) on a band of rows."""
    import torch
    import little_renderer_b200 as L
    from little_renderer_b200 import render as R, workloads as W

    if int(os.environ.get("RANK", "0")) != 0:
        return
    inst = a.workload == "instanced"
    media = a.workload == "media"
    tex = a.workload == "textures"
    dev = torch.device("cuda", 0)
    sc = (W.instanced_field() if inst else W.foggy_cornell(width=256, height=256) if media else
          W.textured_cornell(width=256, height=256) if tex else W.cornell_spheres())
    if media or tex:
        sc["spp"] = 16
    ctx = L.Context(0)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    s = R.instanced_scene(ctx, sc, 1) if inst else R.world_scene(ctx, sc, 1)
    w, h, spp = sc["width"], sc["height"], sc["spp"]
    p = L.native.trace_params(W.camera(sc["camera"], w / h), w, h, sc["max_depth"], 1, 1, 0, 1)
    img = torch.zeros(h, w, 4, device=dev)
    torch.cuda.synchronize()
    _, rays = s.trace(p, spp)                             # (one image on the host: its ray count)

    def timed(fn, n):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ctx.sync()
        return e0.elapsed_time(e1) / n

    def plain():
        s.trace_device(p, spp, img.data_ptr())

    for _ in range(a.warmup):
        plain()
    clk = Clocks(0)
    ms = timed(plain, a.steps)
    clocks = clk.stop()
    img.zero_()
    plain()
    ctx.sync()
    torch.cuda.synchronize()
    want = img.cpu()
    engines = {}
    for name, eng in ((("megakernel", 0),) if media else (("wavefront", 1), ("megakernel", 0))):
        b = L.native.Batch(ctx)
        b.set_engine(eng)
        b.add(s, p, spp, img.data_ptr())
        b.run(zero=True, stepped=a.stepped and eng == 1)
        v, g, _ = b.tune()

        def run_engine():
            if a.stepped and eng == 1:
                b.run(zero=True, stepped=True)
            else:
                b.run(graph=True, zero=True)

        for _ in range(a.warmup):
            run_engine()
        bms = timed(run_engine, a.steps)
        ctx.sync()
        torch.cuda.synchronize()
        engines[name] = {"value": rays / (bms / 1e3) / 1e6, "ms_per_step": bms, "variant": v,
                         ("paths_in_flight" if eng else "grid"): g, "images_equal_plain": bool(torch.equal(img.cpu(), want))}
        b.close()
    # end to end: the host image copied in and out around the launch (lrc_trace with a host array)
    acc = np.zeros((h, w, 4), np.float32)
    t0 = time.perf_counter()
    for _ in range(max(1, min(a.steps, 3))):
        s.trace(p, spp, accum=acc)
    e_ms = (time.perf_counter() - t0) * 1e3 / max(1, min(a.steps, 3))
    # the reference's CPU path tracer on a central band of rows
    cpu = None
    if not a.no_cpu:
        from oracle import oracle as O
        ref = ref_field_scene(O, sc) if inst else None
        if ref is None:
            ref = O.RefScene()
            for m in sc["materials"]:
                ref.material(m["type"], m["albedo"], m["emission"], m["ior"], m["metallic"], m["roughness"],
                             m["transmission"])
            ref.triangles(sc["corners"], sc["tri_mats"])
            lamp = sc["lamp"]
            ref.quad(lamp["q"], lamp["u"], lamp["v"], lamp["material"], light=True)
            for v in sc.get("volumes", []):
                ref.volume(*v)
            for px, srgb, wu, wv in sc.get("texmaps", []):
                ref.texmap(px, srgb, wu, wv)
            for i, m in enumerate(sc["materials"]):
                t = m.get("tex")
                if t:
                    ref.material_textures(i, t.get("base", 0), t.get("mr", 0), t.get("normal", 0), t.get("emissive", 0),
                                          t.get("occlusion", 0), t.get("uv_scale", 0.0), t.get("normal_scale", 0.0))
            if sc.get("texcoords"):
                ref.texcoords(*sc["texcoords"])
        t0 = time.perf_counter()
        ref.set_accel()
        rows = max(1, min(h, (4 if inst else 64)))
        c = sc["camera"]
        fau = np.array([*c["from"], *c["at"], *c["up"]], np.float32)
        _, (cl, sh) = ref.trace_image(fau, c["vfov"], w, h, spp, 1, sc["max_depth"], y0=h // 2 - rows // 2, rows=rows)
        t_cpu = time.perf_counter() - t0
        cores = O.ref_lib().rb_max_threads()
        ref.close()
        cpu = {"value": (cl + sh) / t_cpu / 1e6, "unit": "Mrays/s", "cores": cores, "kind": "reference",
               "sample": f"scene_set_accel + trace_image of {rows} central rows at {spp} spp "
                         f"({cl + sh} rays in {t_cpu:.1f} s)"}
    value = rays / (ms / 1e3) / 1e6
    line = {"metric": METRIC_RENDER, "value": value, "unit": "Mrays/s", "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": ("instanced scene: 5000 instances of 14 meshes (10k-100k triangles), 2048x1024 sky, "
                                    "1280x720, 64 spp, depth 12" if inst else
                                    "the box, its lamp, 16 icospheres and a 40x32x40-voxel cloud (optical depth up to "
                                    "~7), 256x256, 16 spp, depth 8" if media else
                                    "the box, its lamp and 16 icospheres with colour, metal-rough and normal maps "
                                    "(64x64 RGBA8), 256x256, 16 spp, depth 8" if tex else
                                    "the box, its lamp and 64 icospheres (20.5k triangles), 256x256, 16 spp, depth 8"),
                       "rays_per_image": int(rays), "paths_per_image": w * h * spp,
                       "l2": "one image's scene and image held in HBM; successive images reuse L2 (the workload's own)"},
            "clocks": clocks, "engines": engines,
            "e2e": {"value": rays / (e_ms / 1e3) / 1e6, "unit": "Mrays/s", "h2d_bytes_per_step": w * h * 16,
                    "d2h_bytes_per_step": w * h * 16, "ms_per_step": e_ms},
            "gpu_launches": a.steps}
    if cpu:
        line["cpu_baseline"] = cpu
    s.close()
    ctx.close()
    print(json.dumps(line), flush=True)


def run_render_split(a):
    """--workload render --split-samples: configuration 0's image (the box, its lamp and 64
    icospheres, 256x256, 16 spp, depth 8, fast mode) traced by all N ranks together: each rank its
    share of every pixel's samples, then one sum all-reduce of the 1 MB accumulation buffer over
    NCCL (render.trace_split). Strong scaling: the image's work is fixed. At N = 1 the plain path.
    Rank 0 compares the split image with one rank's whole image (the same samples summed in
    another order). e2e: the same with the image read back to pinned host memory each step."""
    import datetime
    import torch
    import little_renderer_b200 as L
    from little_renderer_b200 import render as R, workloads as W

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    sc = W.cornell_spheres()
    w, h, spp = sc["width"], sc["height"], sc["spp"]
    ctx = L.Context(local)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    s = R.world_scene(ctx, sc, 1)
    p = L.native.trace_params(W.camera(sc["camera"], w / h), w, h, sc["max_depth"], 1, 1, 0, 1)
    acc = torch.zeros(h, w, 4, device=dev)
    host = torch.zeros(h, w, 4).pin_memory()
    torch.cuda.synchronize()
    whole, rays = s.trace(p, spp)                    # (the image's rays, and one rank's whole image)

    def step():
        acc.zero_()
        R.trace_split(s, p, spp, acc, dist)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    ctx.sync()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = Clocks(local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ctx.sync()
    ms = max_over_ranks(e0.elapsed_time(e1), dist, dev) / a.steps
    split = acc.cpu().numpy()
    err = float(np.sqrt(((split - whole) ** 2).sum() / (whole ** 2).sum()))
    counts_equal = bool(np.array_equal(split[..., 3], whole[..., 3]))
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(max(3, min(a.steps, 10))):
        step()
        host.copy_(acc, non_blocking=True)
        stream.synchronize()
    e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3, dist, dev) / max(3, min(a.steps, 10))
    s.close()
    ctx.close()
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({"metric": METRIC_RENDER, "value": rays / (ms / 1e3) / 1e6, "unit": "Mrays/s",
                          "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms,
                          "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
                          "data": "synthetic",
                          "config": {"workload": "the box, its lamp and 64 icospheres (20.5k triangles), 256x256, "
                                                 "16 spp, depth 8, one image split by samples over the ranks",
                                     "parallelism": f"sample split x{world}", "rays_per_image": int(rays),
                                     "relRMSE_to_one_rank": err, "sample_counts_equal": counts_equal,
                                     "l2": "one image's scene and image held in HBM; successive images reuse L2 "
                                           "(the workload's own)"},
                          "clocks": clocks,
                          "e2e": {"value": rays / (e_ms / 1e3) / 1e6, "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": w * h * 16, "ms_per_step": e_ms},
                          "gpu_launches": a.steps, "cpu_baseline": None}), flush=True)


def caustics_setup():
    from little_renderer_b200 import workloads as W
    sc = W.cornell_spheres()
    w, h, spp = sc["width"], sc["height"], sc["spp"]
    c = sc["camera"]
    fau = np.array([*c["from"], *c["at"], *c["up"]], np.float32)
    return sc, w, h, w * h * spp, fau


def caustics_config(sc, photons):
    return {"workload": f"light-traced caustics of the box, its lamp and 64 icospheres (20.5k triangles), "
                        f"{sc['width']}x{sc['height']}, {photons} light paths (1 per camera path at {sc['spp']} spp), "
                        f"depth {sc['max_depth']}",
            "light_paths": photons,
            "l2": "the scene and the 1.5 MB of sums stay in L2 (the workload's own)"}


def ref_cornell(O, sc):
    ref = O.RefScene()
    for m in sc["materials"]:
        ref.material(m["type"], m["albedo"], m["emission"], m["ior"], m["metallic"], m["roughness"], m["transmission"])
    ref.triangles(sc["corners"], sc["tri_mats"])
    lamp = sc["lamp"]
    ref.quad(lamp["q"], lamp["u"], lamp["v"], lamp["material"], light=True)
    ref.set_accel()
    return ref


def caustics_cpu(sc, photons, fau, seconds=15.0):
    """The reference's light_trace_caustics on this host's cores: whole runs of the workload's light
    paths until about `seconds` have passed. Returns (Mrays/s, cores, sample text)."""
    from oracle import oracle as O
    ref = ref_cornell(O, sc)
    t0 = time.perf_counter()
    rays = runs = 0
    while True:
        _, (cl, sh) = ref.light_trace_caustics(fau, sc["camera"]["vfov"], sc["width"], sc["height"], photons,
                                               sc["max_depth"], 0x5EED0F11A57 + runs)
        rays += cl + sh
        runs += 1
        if time.perf_counter() - t0 > seconds:
            break
    t = time.perf_counter() - t0
    cores = O.ref_lib().rb_max_threads()
    ref.close()
    return rays / t / 1e6, cores, f"{runs} runs of light_trace_caustics, {photons} light paths each ({rays} rays in {t:.1f} s)"


def run_reference_caustics(a):
    """--impl reference --workload caustics: the reference's light_trace_caustics on this host's cores."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    sc, w, h, photons, fau = caustics_setup()
    from oracle import oracle as O
    ref = ref_cornell(O, sc)
    for i in range(a.warmup):
        ref.light_trace_caustics(fau, sc["camera"]["vfov"], w, h, photons, sc["max_depth"], 100 + i)
    t0 = time.perf_counter()
    rays = 0
    for i in range(a.steps):
        _, (cl, sh) = ref.light_trace_caustics(fau, sc["camera"]["vfov"], w, h, photons, sc["max_depth"], i)
        rays += cl + sh
    t = time.perf_counter() - t0
    cores = O.ref_lib().rb_max_threads()
    ref.close()
    v = rays / t / 1e6
    print(json.dumps({"impl": "reference", "metric": METRIC_CAUSTICS, "value": v, "unit": "Mrays/s", "n_gpus": 0,
                      "steps": a.steps, "warmup": a.warmup, "ms_per_step": t * 1e3 / a.steps, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                      "config": caustics_config(sc, photons),
                      "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": cores, "kind": "reference",
                                       "sample": f"{a.steps} runs of light_trace_caustics ({rays} rays)"},
                      "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
          flush=True)


def run_caustics(a):
    """--workload caustics: lrc_caustics_sums of the workload's light paths into device sums, fast
    mode; e2e: lrc_caustics with a host image (copied in and out)."""
    import torch
    import little_renderer_b200 as L
    from little_renderer_b200 import render as R, workloads as W

    if int(os.environ.get("RANK", "0")) != 0:
        return
    sc, w, h, photons, fau = caustics_setup()
    dev = torch.device("cuda", 0)
    ctx = L.Context(0)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    s = R.world_scene(ctx, sc, 1)
    p = L.native.trace_params(W.camera(sc["camera"], w / h), w, h, sc["max_depth"], 1, 1, 0, 1)
    sums = torch.zeros(h * w * 3, dtype=torch.int64, device=dev)
    torch.cuda.synchronize()
    _, rays = s.caustics(p, photons, 7)

    def step(i):
        s.caustics_sums_device(p, photons, 7 + i, sums.data_ptr())

    def timed(n):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(n):
            step(i)
        e1.record(stream)
        torch.cuda.synchronize()
        ctx.sync()
        return e0.elapsed_time(e1) / n

    # the launch variants (register caps), each timed briefly; the fastest is the timed one
    variants = {}
    for v in range(ctx.caustics_variant(-1)):
        ctx.caustics_variant(v)
        timed(2)
        variants[v] = rays / (timed(5) / 1e3) / 1e6
    best = max(variants, key=variants.get)
    ctx.caustics_variant(best)
    for i in range(a.warmup):
        step(i)
    torch.cuda.synchronize()
    ctx.sync()
    clk = Clocks(0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(a.steps):
        step(i)
    e1.record(stream)
    torch.cuda.synchronize()
    ctx.sync()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1) / a.steps
    img = np.zeros((h, w, 3), np.float32)
    n_e2e = max(1, min(a.steps, 5))
    t0 = time.perf_counter()
    for i in range(n_e2e):
        s.caustics(p, photons, 7, img)
    e_ms = (time.perf_counter() - t0) * 1e3 / n_e2e
    cpu = None
    if not a.no_cpu:
        v, cores, sample = caustics_cpu(sc, photons, fau)
        cpu = {"value": v, "unit": "Mrays/s", "cores": cores, "kind": "reference", "sample": sample}
    s.close()
    ctx.close()
    print(json.dumps({"metric": METRIC_CAUSTICS, "value": rays / (ms / 1e3) / 1e6, "unit": "Mrays/s", "n_gpus": 1,
                      "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                      "config": dict(caustics_config(sc, photons), rays_per_step=int(rays),
                                     mpaths_per_s=photons / (ms / 1e3) / 1e6, variant=best,
                                     variants_mrays={str(k): round(x, 1) for k, x in variants.items()}),
                      "clocks": clocks,
                      "e2e": {"value": rays / (e_ms / 1e3) / 1e6, "unit": "Mrays/s", "h2d_bytes_per_step": w * h * 12,
                              "d2h_bytes_per_step": w * h * 12, "ms_per_step": e_ms},
                      "gpu_launches": a.steps, "cpu_baseline": cpu}), flush=True)


DENOISE_BYTES_PER_PIXEL = 80 + 5 * 24 + 16 + 16


def run_denoise(a):
    """--workload denoise: lrc_denoise (device arrays) on a 1080p image's planes; e2e: lrc_denoise
    with host planes and image (copied in and out)."""
    import torch
    import little_renderer_b200 as L
    from little_renderer_b200 import render as R, workloads as W

    if int(os.environ.get("RANK", "0")) != 0:
        return
    w, h, spp = 1920, 1080, 4
    sc = W.cornell_spheres(width=w, height=h)
    dev = torch.device("cuda", 0)
    ctx = L.Context(0)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    s = R.world_scene(ctx, sc, 1)
    p = L.native.trace_params(W.camera(sc["camera"], w / h), w, h, sc["max_depth"], 1, 1, 0, 1)
    planes = torch.zeros(4, h, w, 4, device=dev)
    out = torch.zeros(h, w, 4, device=dev)
    torch.cuda.synchronize()
    s.guide_device(p, planes.data_ptr())
    s.trace_guided_device(p, spp, planes.data_ptr())
    ctx.sync()

    def step():
        ctx.denoise_device(w, h, planes.data_ptr(), out.data_ptr())

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    ctx.sync()
    clk = Clocks(0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ctx.sync()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1) / a.steps
    # end to end: planes in and the image out through pinned host memory, copies timed
    host_planes = planes.cpu().pin_memory().numpy()
    img = torch.zeros(h, w, 4).pin_memory().numpy()
    n_e2e = max(3, min(a.steps, 20))
    ctx.denoise(host_planes, out=img)
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        ctx.denoise(host_planes, out=img)
    e_ms = (time.perf_counter() - t0) * 1e3 / n_e2e
    assert np.array_equal(img, out.cpu().numpy())
    cpu = None
    if not a.no_cpu:
        from oracle import denoise_oracle as D
        crop = np.ascontiguousarray(host_planes[:, h // 2 - 135:h // 2 + 135, w // 2 - 240:w // 2 + 240])
        t0 = time.perf_counter()
        runs = 0
        while True:
            D.denoise(crop)
            runs += 1
            if time.perf_counter() - t0 > 10.0:
                break
        t = time.perf_counter() - t0
        cpu = {"value": runs * crop.shape[1] * crop.shape[2] / t / 1e6, "unit": "Mpixels/s", "cores": 1, "kind": "port",
               "sample": f"{runs} runs of the numpy restatement on a 480x270 crop in {t:.1f} s"}
    peak_gbs, peak_src = peaks()
    gbs = DENOISE_BYTES_PER_PIXEL * w * h / (ms / 1e3) / 1e9
    s.close()
    ctx.close()
    print(json.dumps({"metric": METRIC_DENOISE, "value": w * h / (ms / 1e3) / 1e6, "unit": "Mpixels/s", "n_gpus": 1,
                      "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f16 between passes)", "data": "synthetic",
                      "config": {"workload": f"denoiser on the plain render's scene at {w}x{h}, {spp} spp (planes "
                                             "made once), prep + 5 a-trous passes",
                                 "l2": "the 33 MB of packed passes stay in L2 between passes (the workload's own)"},
                      "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak_gbs, "unit": "GB/s",
                                   "frac": gbs / peak_gbs, "traffic": None,
                                   "algorithmic_bytes_per_pixel": DENOISE_BYTES_PER_PIXEL,
                                   "peak_source": peak_src},
                      "clocks": clocks,
                      "e2e": {"value": w * h / (e_ms / 1e3) / 1e6, "unit": "Mpixels/s", "h2d_bytes_per_step": w * h * 64,
                              "d2h_bytes_per_step": w * h * 16, "ms_per_step": e_ms},
                      "gpu_launches": 6 * a.steps, "cpu_baseline": cpu}), flush=True)


REALTIME_LAUNCHES = 14   # guide 1, gmatch 1, gradient samples 1, gfilter 3, reprojection 1, trace 1, denoiser 6


def run_realtime(a):
    """--workload realtime: the viewer's loop with temporal gradients on the plain render's scene
    at 1280x720, the camera sliding 2 units a frame (back and forth): each step (frame) makes the
    new guide, the tiles' gradient samples and filtered lambda, the previous frame's samples
    reprojected with each pixel's history (at most 32, 8 without a lambda), 1 guided sample a
    pixel (lrc_trace_frame: all of it in one call), and the denoised image. The same frames as
    separate calls (lrc_guide, lrc_reproject_gradients, lrc_trace, lrc_denoise) are timed beside
    it, stage by stage, and give the same planes. e2e: the frames
    with the denoised image read back to pinned host memory each frame (the scene stays resident,
    as in a viewer). cpu_baseline: the reference's trace_image at 1 spp on a band of rows, scaled
    to the frame (the reference has no CPU reprojection or denoiser)."""
    import torch
    import little_renderer_b200 as L
    from little_renderer_b200 import render as R, workloads as W
    from oracle import oracle as O

    if int(os.environ.get("RANK", "0")) != 0:
        return
    w, h = 1280, 720
    sc = W.cornell_spheres(width=w, height=h)
    dev = torch.device("cuda", 0)
    ctx = L.Context(0)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    s = R.world_scene(ctx, sc, 1)
    c0 = sc["camera"]

    def params(f):                   # (back and forth: 2 units a frame, 80 frames a period)
        cam = dict(c0)
        dx = 2.0 * (abs(f % 80 - 40) - 20)
        cam["from"] = (c0["from"][0] + dx, c0["from"][1], c0["from"][2])
        cam["at"] = (c0["at"][0] + dx, c0["at"][1], c0["at"][2])
        return L.native.trace_params(W.camera(cam, w / h), w, h, sc["max_depth"], 1, 1, 0, 7)

    planes = [torch.zeros(4, h, w, 4, device=dev), torch.zeros(4, h, w, 4, device=dev)]
    out = torch.zeros(h, w, 4, device=dev)
    host_img = torch.zeros(h, w, 4).pin_memory()
    state = {"f": 0}
    stage_ms = np.zeros(4)

    def frame_one():                 # lrc_trace_frame + lrc_denoise
        f = state["f"]
        cur, prev = planes[f % 2], planes[(f + 1) % 2]
        if f > 0:
            s.trace_frame_device(params(f - 1), params(f), f, 1, prev.data_ptr(), cur.data_ptr(), 32, 8)
        else:
            s.trace_frame_device(None, params(f), f, 1, 0, cur.data_ptr(), 32, 8)
        ctx.denoise_device(w, h, cur.data_ptr(), out.data_ptr())
        state["f"] = f + 1

    def frame(events=None):          # the same as separate calls, timed stage by stage
        f = state["f"]
        cur, prev = planes[f % 2], planes[(f + 1) % 2]
        p = params(f)
        if events:
            events[0].record(stream)
        s.guide_device(p, cur.data_ptr())
        if events:
            events[1].record(stream)
        if f > 0:
            s.reproject_gradients_device(params(f - 1), p, f, prev.data_ptr(), cur.data_ptr(), 32, 8)
        else:
            cur[:2].zero_()
        if events:
            events[2].record(stream)
        s.trace_guided_device(p, 1, cur.data_ptr(), spp0=f)
        if events:
            events[3].record(stream)
        ctx.denoise_device(w, h, cur.data_ptr(), out.data_ptr())
        if events:
            events[4].record(stream)
        state["f"] = f + 1

    def warm(fn):                    # frames 0 .. warmup - 1: both ways time the same frames after
        state["f"] = 0
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize()
        ctx.sync()

    # the separate calls, stage by stage
    warm(frame)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(5)] for _ in range(a.steps)]
    for i in range(a.steps):
        frame(evs[i])
    torch.cuda.synchronize()
    ctx.sync()
    sep_ms = evs[0][0].elapsed_time(evs[-1][4]) / a.steps
    for e in evs:
        for k in range(4):
            stage_ms[k] += e[k].elapsed_time(e[k + 1]) / a.steps
    # the same next frame both ways: equal planes
    f_chk = state["f"]
    frame()
    sep_planes = planes[f_chk % 2].clone()
    state["f"] = f_chk
    frame_one()
    torch.cuda.synchronize()
    ctx.sync()
    same_planes = bool(torch.equal(sep_planes, planes[f_chk % 2]))
    # lrc_trace_frame: the line's value
    warm(frame_one)
    clk = Clocks(0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        frame_one()
    e1.record(stream)
    torch.cuda.synchronize()
    ctx.sync()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1) / a.steps
    cur = planes[(state["f"] - 1) % 2]
    hist = cur[0][..., 3].float()
    history_mean = float(hist.mean())
    finite = bool(torch.isfinite(out).all())
    # a frame's rays (closest-hit + shadow) of its 1-spp trace, counted on one host call
    pr = params(state["f"] - 1)
    host_planes = cur.cpu().numpy().copy()
    _, rays = s.trace_guided(pr, 1, host_planes, spp0=state["f"])
    # end to end: each frame's denoised image read back to pinned host memory
    n_e2e = max(3, min(a.steps, 20))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        frame_one()
        host_img.copy_(out, non_blocking=True)
        stream.synchronize()
    e_ms = (time.perf_counter() - t0) * 1e3 / n_e2e
    # the reference's CPU path tracer: 1 spp on a central band of rows
    cpu = None
    if not a.no_cpu:
        ref = ref_cornell(O, sc)
        rows = 64
        c = c0
        fau = np.array([*c["from"], *c["at"], *c["up"]], np.float32)
        t0 = time.perf_counter()
        _, (cl, sh) = ref.trace_image(fau, c["vfov"], w, h, 1, 1, sc["max_depth"], y0=h // 2 - rows // 2, rows=rows)
        t_cpu = time.perf_counter() - t0
        cores = O.ref_lib().rb_max_threads()
        ref.close()
        cpu = {"value": 1e3 / (t_cpu * 1e3 * h / rows), "unit": "frames/s", "cores": cores, "kind": "reference",
               "sample": f"scene_set_accel + trace_image of {rows} central rows at 1 spp ({cl + sh} rays in "
                         f"{t_cpu:.2f} s), scaled to the {h}-row frame; the reference has no CPU reprojection or "
                         "denoiser"}
    peak_gbs, peak_src = peaks()
    dn_gbs = DENOISE_BYTES_PER_PIXEL * w * h / (stage_ms[3] / 1e3) / 1e9
    s.close()
    ctx.close()
    print(json.dumps({"metric": METRIC_REALTIME, "value": 1e3 / ms, "unit": "frames/s", "n_gpus": 1,
                      "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f16 between denoiser passes)",
                      "data": "synthetic",
                      "config": {"workload": f"the box, its lamp and 64 icospheres (20.5k triangles), {w}x{h}, depth "
                                             f"{sc['max_depth']}, the camera sliding 2 units a frame; history at most "
                                             "32 samples (8 without a gradient), 1 new sample a pixel a frame",
                                 "separate_calls": {"ms_per_frame": sep_ms, "frames_per_s": 1e3 / sep_ms,
                                                    "stage_ms": {"guide": stage_ms[0],
                                                                 "gradients+reprojection": stage_ms[1],
                                                                 "trace_1spp": stage_ms[2], "denoise": stage_ms[3]},
                                                    "planes_equal_trace_frame": same_planes},
                                 "rays_per_frame_trace": int(rays),
                                 "trace_Mrays_per_s": rays / (stage_ms[2] / 1e3) / 1e6,
                                 "mean_samples_a_pixel_after_trace": history_mean, "image_finite": finite,
                                 "l2": "the frame's 59 MB of planes and the scene stay in HBM; L2 not flushed (the "
                                       "workload's own: a viewer's frames follow one another)"},
                      "roofline": {"kernel": "denoiser passes (the frame's HBM-bound stage; the trace is "
                                             "traversal-latency-bound)", "bound": "hbm", "achieved": dn_gbs,
                                   "peak": peak_gbs, "unit": "GB/s", "frac": dn_gbs / peak_gbs, "traffic": None,
                                   "algorithmic_bytes_per_pixel": DENOISE_BYTES_PER_PIXEL, "peak_source": peak_src},
                      "clocks": clocks,
                      "e2e": {"value": 1e3 / e_ms, "unit": "frames/s", "h2d_bytes_per_step": 0,
                              "d2h_bytes_per_step": w * h * 16, "ms_per_step": e_ms},
                      "gpu_launches": REALTIME_LAUNCHES * a.steps, "cpu_baseline": cpu}), flush=True)


def main():
    a = parse()
    if a.impl == "reference":
        if a.workload == "serve":
            run_reference_serve(a)
        elif a.workload == "batch":
            run_reference_batch(a)
        elif a.workload == "caustics":
            run_reference_caustics(a)
        elif a.workload == "realtime":
            print(json.dumps({"impl": "reference", "metric": METRIC_REALTIME, "unavailable":
                              "the reference's reprojection, temporal gradients and denoiser exist only as WGSL, "
                              "which cannot run on this box; its CPU path tracer is the cpu_baseline leg of the ours "
                              "line"}), flush=True)
        elif a.workload == "denoise":
            print(json.dumps({"impl": "reference", "metric": METRIC_DENOISE, "unavailable":
                              "the reference's denoiser exists only as WGSL (denoise.wgsl), which cannot run on this "
                              "box; its numpy restatement is the cpu_baseline leg of the ours line"}), flush=True)
        elif a.workload in ("render", "instanced", "media", "textures"):
            print(json.dumps({"impl": "reference", "metric": METRIC_RENDER, "unavailable":
                              "this workload's CPU baseline is the cpu_baseline leg of the ours line"}), flush=True)
        else:
            run_reference(a)
        return
    if a.workload == "batch":
        run_batch(a)
        return
    if a.workload == "serve":
        run_serve(a)
        return
    if a.workload == "render" and a.split_samples:
        run_render_split(a)
        return
    if a.workload in ("render", "instanced", "media", "textures"):
        run_render(a)
        return
    if a.workload == "caustics":
        run_caustics(a)
        return
    if a.workload == "denoise":
        run_denoise(a)
        return
    if a.workload == "realtime":
        run_realtime(a)
        return
    import torch
    import little_renderer_b200 as L
    from little_renderer_b200 import workloads as W

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    builder = 1 if a.builder == "ploc" else 0

    cor = W.soup(a.n, 1 + rank) * np.float32(a.scale)
    quv = W.corners_to_quv(cor)
    tris = L.pack_tris(quv)
    orig, dirs = W.rays_at_cube(a.rays, 2 + rank, scale=a.scale)

    ctx = L.Context(local)
    # a stream of our own (the default stream's handle is 0, which lrc_set_stream reads as "the
    # context's own"): the kernels and the timing events then share it
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    scene = L.Scene(ctx)
    d_tris = torch.from_numpy(tris.view(np.int32)).to(dev)
    d_o = torch.from_numpy(orig).to(dev)
    d_d = torch.from_numpy(dirs).to(dev)
    d_p = torch.empty(a.rays, dtype=torch.int32, device=dev)
    d_t = torch.empty(a.rays, dtype=torch.float32, device=dev)

    scene.set_triangles(None, device_ptr=d_tris.data_ptr(), n=a.n)
    scene.set_walk(a.walk)

    def step():
        scene.build(builder, a.bits)
        scene.intersect_device(d_o.data_ptr(), d_d.data_ptr(), a.rays, d_p.data_ptr(), d_t.data_ptr())

    for _ in range(a.warmup):
        step()
    ctx.sync()
    # traversal statistics (the algorithmic bytes per ray), outside the timed region
    sample = min(a.rays, 1 << 20)
    boxes_tested, tris_tested = scene.trace_stats((sample, d_o.data_ptr(), d_d.data_ptr()))

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = Clocks(local)
    # stage times by CUDA events on the launching stream, live over the timed region
    ctx.set_timing(True)
    ctx.timings()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(a.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ctx.sync()
    stages = ctx.timings()
    ctx.set_timing(False)
    ms = max_over_ranks(ev0.elapsed_time(ev1), dist, dev)
    if dist:
        dist.barrier()
    ms_step = ms / a.steps
    value = whole_job_rate(a.rays * a.steps, world, ms)

    # end to end through the C ABI with host (pinned) buffers: copies in and out inside each step
    pin_tris = torch.from_numpy(tris.view(np.int32)).pin_memory()
    pin_o = torch.from_numpy(orig).pin_memory()
    pin_d = torch.from_numpy(dirs).pin_memory()
    pin_p = torch.empty(a.rays, dtype=torch.int32).pin_memory()
    pin_t = torch.empty(a.rays, dtype=torch.float32).pin_memory()
    np_tris = pin_tris.numpy().view(np.uint32)
    np_o, np_d, np_p, np_t = pin_o.numpy(), pin_d.numpy(), pin_p.numpy(), pin_t.numpy()

    def e2e_step():
        scene.set_triangles(np_tris)
        scene.build(builder, a.bits)
        ctx.check(ctx.L.lrc_scene_intersect(scene.h, L.native._ptr(np_o), L.native._ptr(np_d), a.rays, 0.0, 1e30,
                                            L.native._ptr(np_p), L.native._ptr(np_t), 0))

    e2e_step()
    scene.set_triangles(None, device_ptr=d_tris.data_ptr(), n=a.n)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.e2e_steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e_ms = max_over_ranks(e0.elapsed_time(e1), dist, dev)
    e2e = {"value": whole_job_rate(a.rays * a.e2e_steps, world, e_ms), "unit": "Mrays/s",
           "h2d_bytes_per_step": int(tris.nbytes + orig.nbytes + dirs.nbytes),
           "d2h_bytes_per_step": int(a.rays * 8), "ms_per_step": e_ms / a.e2e_steps}

    # roofline of the dominant kernel (from the stage times): traversal or the build's sort
    peak, peak_kind = peaks()
    per = a.steps  # the stage timer ran over the timed steps
    trace_ms = stages["trace"][0] / per
    sort_ms = stages["sort"][0] / per
    bytes_per_ray = (boxes_tested * 32 + tris_tested * 48) / sample
    trace_bytes = bytes_per_ray * a.rays
    kb = 8 if a.bits == 63 else 4
    sort_bytes = a.n * (kb + (a.bits + 7) // 8 * 2 * (kb + 4))
    rl_trace = {"kernel": "closest_kernel", "bound": "hbm", "achieved": trace_bytes / (trace_ms / 1e3) / 1e9,
                "peak": peak, "unit": "GB/s", "peak_kind": peak_kind, "traffic": None,
                "algorithmic_bytes_per_launch": trace_bytes, "bytes_per_ray": bytes_per_ray,
                "ms_per_launch": trace_ms}
    if (a.n, a.rays, a.builder, a.bits, a.scale, a.walk) == (4 << 20, 16 << 20, "ploc", 30, 1.0, 1):
        dram_gbs = BUILDER_CLOSEST_DRAM["bytes_per_launch"] / (BUILDER_CLOSEST_DRAM["ms_per_launch"] / 1e3) / 1e9
        rl_trace.update({"traffic": BUILDER_CLOSEST_DRAM["bytes_per_launch"],
                         "traffic_from": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the 4th closest_kernel "
                                         "launch of `python bench.py --workload builder --steps 1 --warmup 3 --no-cpu "
                                         "--e2e-steps 1`", "dram_gbs": dram_gbs, "frac_dram": dram_gbs / peak})
    rl_trace["frac"] = rl_trace["achieved"] / peak
    rl_sort = {"kernel": "onesweep (all passes)", "bound": "hbm", "achieved": sort_bytes / (sort_ms / 1e3) / 1e9,
               "peak": peak, "unit": "GB/s", "peak_kind": peak_kind, "traffic": None,
               "algorithmic_bytes_per_launch": sort_bytes, "ms_per_launch": sort_ms}
    rl_sort["frac"] = rl_sort["achieved"] / peak
    rl_sort["library_sort"] = library_sort_ms(a.n, a.bits, stream, dev)
    dominant = rl_trace if trace_ms >= sum(v[0] for k, v in stages.items() if k != "trace") / per else rl_sort

    passes = 8 if a.bits == 63 else 4
    launches_per_step = 3 + 1 + passes + (2 if builder else 1) + 1
    line = {"metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config(a, world),
            "clocks": clocks, "e2e": e2e, "gpu_launches": launches_per_step * a.steps,
            "roofline": dominant, "roofline_sort": rl_sort, "roofline_trace": rl_trace,
            "stage_ms_per_step": {k: v[0] / per for k, v in stages.items()},
            "traversal": {"box_tests_per_ray": boxes_tested / sample, "tri_tests_per_ray": tris_tested / sample}}
    if rank == 0 and world == 1 and not a.no_cpu:
        line["cpu_baseline"] = cpu_baseline(a, cor, orig, dirs, sample_rays=1 << 21)
    scene.close()
    ctx.close()
    if dist:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
