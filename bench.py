"""Benchmark: Nova path tracing on B200, plain wavefront, heightfield workload.

Workload (one step = one full render): a 1024 x 1024 quad heightfield (2,097,152 triangles) from
seeded 6-octave fBm (amplitude 0.3), per-quad material 50/50 Lambert / GGX conductor, a
2048 x 1024 log-normal(0, 1.5) float environment map, 1920 x 1080 pixels, 64 spp, max depth 8,
Russian roulette from bounce 3.  Synthetic seeded data (no dataset exists for this path).

Metric: Mrays/s = closest-hit rays traced on the device / device render time (CUDA events on the
render stream), whole job over all ranks.  `e2e` is the same metric through the C ABI starting
from pinned host buffers each step: scene upload + device BVH build + render + film readback.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun, one rank per GPU) every rank renders its own 64-sample range of a 64N-spp
image and the films are summed with one NCCL all-reduce (weak scaling).  --impl reference times
the CPU implementation of the path (the oracle restatement of the reference's CPU Nova path; the
reference itself cannot be built here) on the host cores on a bounded pixel sample.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CFG = dict(n=1024, width=1920, height=1080, spp=64, depth=8, rr_start=3, env_w=2048, env_h=1024, seed=0)
WORKLOAD = "heightfield 1024^2 quads (2,097,152 tris), env 2048x1024, 1920x1080, 64 spp, depth 8, RR from 3"
METRIC = "Mrays/s (plain wavefront path tracing, heightfield workload)"


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


class ClockSampler:
    """Samples SM clocks / throttle reasons with nvidia-smi during the timed region."""

    def __init__(self, gpu_index=0):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_scene():
    from axomae_b200 import scenes
    return scenes.heightfield_scene(n=CFG["n"], width=CFG["width"], height=CFG["height"], env_w=CFG["env_w"],
                                    env_h=CFG["env_h"], seed=CFG["seed"])


def scene_bytes(scene):
    b = 0
    for m in scene["meshes"]:
        b += sum(np.asarray(m[k]).nbytes for k in ("vertices", "normals", "tangents", "bitangents", "uv", "indices"))
    for t in scene["textures"]:
        b += np.asarray(t["pixels"]).nbytes
    return b


def cpu_sample(scene, frac_stride=64, threads=0):
    """Oracle render of every `frac_stride`-th pixel (all samples): Mrays/s on the host cores."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_binding as ob
    ob.build()
    t0 = time.perf_counter()
    osc = ob.OracleScene(scene)
    build_s = time.perf_counter() - t0
    W, H = CFG["width"], CFG["height"]
    ids = np.arange(0, W * H, frac_stride, dtype=np.int32)
    opt = ob.options(W, H, CFG["spp"], CFG["depth"], seed=CFG["seed"], rr_start=CFG["rr_start"], threads=threads)
    _, st = osc.render(opt, pixel_ids=ids)
    cores = threads if threads > 0 else os.cpu_count()
    return {"mrays": st.traced / st.seconds / 1e6, "seconds": st.seconds, "traced": st.traced,
            "node_visits_per_ray": st.node_visits / max(1, st.traced), "tri_tests_per_ray": st.tri_tests / max(1, st.traced),
            "segments": st.segments, "pixels": int(ids.size), "cores": cores, "build_s": build_s}


def run_reference(args, rank, world):
    if rank != 0:
        return
    scene = make_scene()
    stride = int(os.environ.get("NOVA_BENCH_CPU_STRIDE", "64"))
    for _ in range(args.warmup if args.warmup < 1 else 1):
        pass
    vals = []
    last = None
    for _ in range(args.steps):
        last = cpu_sample(scene, stride)
        vals.append(last["mrays"])
    v = float(np.median(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": last["seconds"] * 1000.0, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": WORKLOAD, "pixel_sample": "every %dth pixel, all 64 spp" % stride},
            "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": last["cores"], "kind": "port",
                             "sample": "oracle (CPU restatement of the reference Nova path) on every %dth pixel of "
                                       "the 1920x1080 frame, 64 spp, %d pixels" % (stride, last["pixels"])},
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import torch
    from axomae_b200 import native
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    scene = make_scene()
    W, H, spp, depth = CFG["width"], CFG["height"], CFG["spp"], CFG["depth"]
    ctx = native.Context(local_rank)
    t0 = time.perf_counter()
    ctx.upload(scene)
    upload_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    ctx.build(width=args.bvh_width)
    build_s = time.perf_counter() - t0
    info = ctx.info()
    spp_total = spp * world
    film = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    frame = native.make_frame(scene, W, H, spp_total, depth, seed=CFG["seed"], sample_begin=rank * spp,
                              sample_count=spp, rr_start=CFG["rr_start"], reset=1)

    def step():
        st = ctx.render(frame, film_device_ptr=film.data_ptr())
        if world > 1:
            dist.all_reduce(film)
            film.div_(world)
        return st

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    traced = 0
    dev_ms = 0.0
    trace_ms = 0.0
    shade_ms = 0.0
    kernels = 0
    waves = 0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        ev0.record()
        for _ in range(args.steps):
            st = step()
            traced += st.traced
            dev_ms += st.device_ms
            trace_ms += st.trace_ms
            shade_ms += st.shade_ms
            kernels += st.kernels
            waves += st.waves
        ev1.record()
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    wall_ms = ev0.elapsed_time(ev1)
    step_ms = max(dev_ms, wall_ms) / args.steps  # the render stream's events; the torch-stream bracket
    if dist:
        t = torch.tensor([step_ms, float(traced)], dtype=torch.float64, device="cuda")
        mx = t.clone()
        dist.all_reduce(mx[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        step_ms, traced_all = float(mx[0]), float(t[1])
    else:
        traced_all = float(traced)
    value = traced_all / args.steps / (step_ms / 1e3) / 1e6

    # end to end through the C ABI from pinned host buffers: upload + build + render + readback
    e2e = None
    if rank == 0 and not args.no_e2e:
        pinned = pin_scene(scene)
        host_film = torch.empty((H, W, 4), dtype=torch.float32).pin_memory()
        e_steps = max(1, min(args.steps, 3))
        ectx = native.Context(local_rank)
        eframe = native.make_frame(scene, W, H, spp, depth, seed=CFG["seed"], rr_start=CFG["rr_start"])

        def e2e_step():
            t0 = time.perf_counter()
            ectx.upload(pinned)
            t1 = time.perf_counter()
            ectx.build(width=args.bvh_width)
            t2 = time.perf_counter()
            st = ectx.render(eframe, film_host=host_film.numpy())
            t3 = time.perf_counter()
            return st.traced, (t1 - t0, t2 - t1, t3 - t2)

        e2e_step()  # untimed: the context's first render allocates its path queues and film
        e_traced = 0
        stages = np.zeros(3)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e_steps):
            tr, st3 = e2e_step()
            e_traced += tr
            stages += st3
        ectx.synchronize()
        e_s = time.perf_counter() - t0
        ectx.close()
        e2e = {"value": e_traced / e_s / 1e6, "unit": "Mrays/s", "h2d_bytes_per_step": scene_bytes(scene),
               "d2h_bytes_per_step": W * H * 16, "steps": e_steps, "warmup": 1,
               "upload_ms": 1e3 * stages[0] / e_steps, "build_ms": 1e3 * stages[1] / e_steps,
               "render_ms": 1e3 * stages[2] / e_steps,
               "timing": "host wall clock around upload (pinned H2D) + BVH build + render + film D2H"}

    if rank != 0:
        ctx.close()
        if dist:
            dist.destroy_process_group()
        return
    cpu = None
    if not args.no_cpu:
        cpu = cpu_sample(scene, int(os.environ.get("NOVA_BENCH_CPU_STRIDE", "64")))
    pk = peaks()
    hbm = pk.get("hbm_gbs")
    peak_src = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    # Algorithmic bytes per traced ray (reference binary BVH node/triangle counts measured by the
    # oracle on this workload's rays): 32 B ray + 16 B hit + 64 B per inner-node visit + 36 B per
    # triangle test.
    if cpu:
        b_ray = 32 + 16 + 64 * cpu["node_visits_per_ray"] + 36 * cpu["tri_tests_per_ray"]
    else:
        b_ray = None
    trace_rate = traced / (trace_ms / 1e3) if trace_ms > 0 else None
    roof = None
    if b_ray and trace_rate:
        achieved = trace_rate * b_ray / 1e9
        roof = {"bound": "hbm", "kernel": "k_trace", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_source": peak_src, "traffic": None,
                "bytes_per_ray": b_ray, "trace_ms_per_step": trace_ms / args.steps}
    line = {"metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded heightfield + log-normal env map)",
            "config": {"workload": WORKLOAD, "spp_per_gpu": spp, "bvh_width": args.bvh_width or 2, "parallelism": "sample-range partition + NCCL film "
                       "all-reduce" if world > 1 else "single GPU", "l2": "working set larger than L2 (BVH %d nodes "
                       "x 64 B + %d tris x 48 B)" % (info["nodes"], info["triangles"])},
            "e2e": e2e, "roofline": roof,
            "cpu_baseline": None if not cpu else {
                "value": cpu["mrays"], "unit": "Mrays/s", "cores": cpu["cores"], "kind": "port",
                "sample": "oracle on every %sth pixel of the frame, 64 spp (%d pixels, %.1f s)" % (
                    os.environ.get("NOVA_BENCH_CPU_STRIDE", "64"), cpu["pixels"], cpu["seconds"])},
            "clocks": clk.summary(), "gpu_launches": kernels,
            "extra": {"waves_per_step": waves / args.steps, "traced_per_step": traced / args.steps,
                      "trace_ms_per_step": trace_ms / args.steps, "shade_ms_per_step": shade_ms / args.steps,
                      "bvh_build_s": build_s, "upload_s": upload_s, "bvh_nodes": info["nodes"],
                      "device_bytes": info["device_bytes"]}}
    print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()


def pin_scene(scene):
    import torch

    def pin(a):
        a = np.ascontiguousarray(a)
        raw = a.view(np.int32) if a.dtype == np.uint32 else a
        t = torch.from_numpy(raw).pin_memory()
        keep.append(t)
        return t.numpy().view(a.dtype)

    keep = []

    out = dict(scene)
    out["meshes"] = [{k: pin(v) for k, v in m.items()} for m in scene["meshes"]]
    out["textures"] = [dict(t, pixels=pin(t["pixels"])) for t in scene["textures"]]
    out["_pinned"] = keep
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--frame", type=int, nargs=2, metavar=("W", "H"), help="override the frame size (profiling)")
    ap.add_argument("--spp", type=int, help="override samples per pixel (profiling)")
    ap.add_argument("--bvh-width", type=int, default=0, choices=[0, 2, 8], help="BVH layout (0 = library default)")
    args = ap.parse_args()
    if args.frame:
        CFG["width"], CFG["height"] = args.frame
    if args.spp:
        CFG["spp"] = args.spp
    if args.frame or args.spp:
        global WORKLOAD
        WORKLOAD = WORKLOAD.replace("1920x1080, 64 spp", "%dx%d, %d spp" % (CFG["width"], CFG["height"], CFG["spp"]))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus if args.gpus else 1)))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if "RANK" not in os.environ:
        world = 1
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
