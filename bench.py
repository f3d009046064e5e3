"""Benchmark of the hot path: a BVH build (LBVH or PLOC over N triangles) plus one pass of
closest-hit rays through it, on B200. Prints one JSON line (rank 0).

Workload (the builder + closest-hit configuration, synthetic and seeded): N = 4M triangles with
centroids uniform in the unit cube, Gaussian edges (sigma = 0.002 N^-1/3), 2 % of them scaled x50;
16M rays from a sphere of radius 2 toward uniform points of the cube. One step = triangle boxes,
Morton codes, radix sort, hierarchy (PLOC by default: the reference's builder for meshes), then
16M closest-hit queries. metric: Mrays/s of the whole step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--builder ploc|lbvh] [--bits 30|63]
  python bench.py --impl reference ...   the reference's own CPU path (SAH build + scene_intersect)

Multi-GPU: replicas (each rank builds and traces its own scene; no collective on the data path),
timed as the max over ranks.
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
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--e2e-steps", type=int, default=5)
    return ap.parse_args()


def config(a, world):
    return {"workload": f"builder+closest-hit: {a.n} triangles (soup), {a.rays} rays, {a.builder.upper()} "
                        f"{a.bits}-bit Morton", "triangles": a.n, "rays": a.rays, "builder": a.builder,
            "key_bits": a.bits, "parallelism": f"replicas x{world}",
            "l2": "inputs larger than L2 (triangles 48 B x N + rays 24 B x R > 126 MB)"}


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
    """--impl reference: the reference's own CPU implementation of the path (SAH BVH build +
    scene_intersect) on this host's cores, each step a bounded sample of the workload."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from little_renderer_b200 import workloads as W
    cor = W.soup(a.n, 1)
    sample = 1 << 20
    o, d = W.rays_at_cube(sample, 2)
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
                                       f"scene_intersect of {sample} rays, scaled to {a.rays} rays"},
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
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

    cor = W.soup(a.n, 1 + rank)
    quv = W.corners_to_quv(cor)
    tris = L.pack_tris(quv)
    orig, dirs = W.rays_at_cube(a.rays, 2 + rank)

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
    ms = ev0.elapsed_time(ev1)
    if dist:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    ms_step = ms / a.steps
    value = world * a.rays * a.steps / (ms / 1e3) / 1e6

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
    e_ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e_ms = float(t.item())
    e2e = {"value": world * a.rays * a.e2e_steps / (e_ms / 1e3) / 1e6, "unit": "Mrays/s",
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
    rl_trace["frac"] = rl_trace["achieved"] / peak
    rl_sort = {"kernel": "onesweep (all passes)", "bound": "hbm", "achieved": sort_bytes / (sort_ms / 1e3) / 1e9,
               "peak": peak, "unit": "GB/s", "peak_kind": peak_kind, "traffic": None,
               "algorithmic_bytes_per_launch": sort_bytes, "ms_per_launch": sort_ms}
    rl_sort["frac"] = rl_sort["achieved"] / peak
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
