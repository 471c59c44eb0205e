"""Benchmark: Nova path tracing on B200 — batched vs plain wavefront.

Default workload ("batched", one step = one render of all jobs): 32 seeded jobs, each a scene of
50k-500k triangles (random UV spheres + boxes; 1/3 Lambert, 1/3 GGX conductor, 1/3 GGX dielectric
IOR 1.5; 256x128 log-normal float environment), a square frame whose pixel count is log-uniform in
[256^2, 2048^2], spp drawn from {1, 4, 16, 64}, max depth from {3, 6, 12}, Sobol seed 0.  The
batched arm renders all 32 frames with one nova_b200_render_batch call (one device-driven
wavefront); the plain arm renders the same frames with one nova_b200_render call each.  Both run the
same estimator on the same sample indices, so their images are equal (checked bit for bit every
run) and so is their RMSE against the CPU oracle (reported on a pixel sample).

Second workload ("heightfield", --workload heightfield): a 1024 x 1024 quad heightfield
(2,097,152 triangles), 50/50 Lambert / GGX conductor, 2048 x 1024 log-normal(0, 1.5) environment,
1920 x 1080, 64 spp, depth 8, Russian roulette from bounce 3; plain wavefront only.

Metric: Mrays/s = closest-hit rays traced on the device / device render time (CUDA events on the
render stream), whole job over all ranks.  `e2e` is the same metric through the C ABI from pinned
host buffers each step: scene upload + device BVH build + render + film readback.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload batched|heightfield|instanced]

With N > 1 (torchrun, one rank per GPU) every rank renders its own sample range of every frame
(frame spp x N in total) and the films are summed with one NCCL all-reduce (weak scaling).
--impl reference times the CPU implementation of the path (the oracle restatement of the
reference's CPU Nova path; the reference itself cannot be built as a whole) on the host cores: whole
frames of one sample per pixel, the reference's tiles and worker pool, each job's frame time
extrapolated to its spp (8 jobs per step, rotating); the instanced workload on a pixel subset.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time
import traceback

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HF = dict(n=1024, width=1920, height=1080, spp=64, depth=8, rr_start=3, env_w=2048, env_h=1024, seed=0)
HF_WORKLOAD = "heightfield 1024^2 quads (2,097,152 tris), env 2048x1024, 1920x1080, 64 spp, depth 8, RR from 3"
HF_METRIC = "Mrays/s (plain wavefront path tracing, heightfield workload)"
IN = dict(width=3840, height=2160, spp=16, depth=12)
IN_WORKLOAD = ("instanced: 1000 rigid instances of 10 seeded 10k-tri meshes (10,000,000 instanced tris, "
               "Lambert / GGX conductor / GGX dielectric / Burley) in a 100^3 box, env 4096x2048, 3840x2160, "
               "16 spp, depth 12")
IN_METRIC = "Mrays/s (plain wavefront path tracing, instanced workload)"
BATCH_WORKLOAD = ("32 jobs: mixed spheres+boxes scenes of 50k-500k tris (Lambert / GGX conductor / GGX "
                  "dielectric IOR 1.5), square frames log-uniform 256^2-2048^2, spp in {1,4,16,64}, "
                  "depth in {3,6,12}, seed 0")
BATCH_METRIC = ("Mrays/s batched wavefront (32-job batch; plain wavefront on the same jobs in extra.plain; "
                "adjoint/forward time ratio in extra.adjoint)")


# DRAM bytes per traced ray that ncu measured for k_trace (dram__bytes_read.sum +
# dram__bytes_write.sum over full waves of 8,388,608 rays): batched workload waves 1-2, and the
# heightfield's first wave (camera rays only).
K_TRACE_DRAM_BYTES_PER_RAY = {"batched": 72.0, "heightfield": 238.4, "instanced": None}
# L2 bytes per traced ray (lts__t_bytes.sum) ncu measured for the binary-BVH k_trace on the
# batched workload's full waves 6-8: L1 serves ~2/3 of the requests, L2 ~90 % of the rest.
K_TRACE_L2_BYTES_PER_RAY = {"batched": 521.0, "heightfield": None, "instanced": None}


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


# ----------------------------------------------------------------------------------------------
# workloads: a list of jobs {scene, width, height, spp, depth, rr_start}


def make_jobs(workload):
    from axomae_b200 import scenes
    if workload == "heightfield":
        s = scenes.heightfield_scene(n=HF["n"], width=HF["width"], height=HF["height"], env_w=HF["env_w"],
                                     env_h=HF["env_h"], seed=HF["seed"])
        return [{"scene": s, "width": HF["width"], "height": HF["height"], "spp": HF["spp"], "depth": HF["depth"],
                 "rr_start": HF["rr_start"]}]
    if workload == "instanced":
        s = scenes.instanced_scene(n_meshes=10, n_instances=1000, tris_per_mesh=10000, width=IN["width"],
                                   height=IN["height"], seed=0, env_w=4096, env_h=2048)
        return [{"scene": s, "width": IN["width"], "height": IN["height"], "spp": IN["spp"], "depth": IN["depth"],
                 "rr_start": -1}]
    jobs = scenes.batch_jobs(32, seed=0)
    for j in jobs:
        j["rr_start"] = -1
    return jobs


def scene_bytes(scene):
    b = 0
    for m in scene["meshes"]:
        b += sum(np.asarray(m[k]).nbytes for k in ("vertices", "normals", "tangents", "bitangents", "uv", "indices"))
    for t in scene["textures"]:
        b += np.asarray(t["pixels"]).nbytes
    return b


def oracle_module():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_binding as ob
    ob.build()
    return ob


def oracle_scenes(jobs):
    """Oracle scenes (reference BVH builds) of all jobs, built on a thread pool (the builds run in
    C with the GIL released)."""
    from concurrent.futures import ThreadPoolExecutor
    ob = oracle_module()
    with ThreadPoolExecutor(max_workers=min(len(jobs), usable_cores())) as ex:
        return list(ex.map(lambda j: ob.OracleScene(j["scene"]), jobs))


def usable_cores():
    """Host cores this process may run on (its CPU affinity, which a container can narrow)."""
    try:
        return len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def cpu_sample(jobs, stride, threads=0, oscs=None, films=None):
    """Oracle render of every `stride`-th pixel of every job (all samples): Mrays/s on the host
    cores (threads=0: every usable core), the reference-BVH node visits / triangle tests per ray,
    and, when GPU films are given, the relative RMSE of those films against the oracle on the
    sampled pixels."""
    if threads <= 0:
        threads = usable_cores()
    t0 = time.perf_counter()
    ob = oracle_module()
    if oscs is None:
        oscs = oracle_scenes(jobs)
    build_s = time.perf_counter() - t0
    traced = seconds = nodes = tris = 0
    pixels = 0
    sq, cnt = 0.0, 0
    for k, (j, osc) in enumerate(zip(jobs, oscs)):
        W, H = j["width"], j["height"]
        ids = np.arange(k % stride, W * H, stride, dtype=np.int32)
        opt = ob.options(W, H, j["spp"], j["depth"], seed=0, rr_start=j["rr_start"], threads=threads)
        ref, st = osc.render(opt, pixel_ids=ids)
        traced += st.traced
        seconds += st.seconds
        nodes += st.node_visits
        tris += st.tri_tests
        pixels += ids.size
        if films is not None:
            r = ref.reshape(-1, 4)[ids, :3].astype(np.float64)
            g = films[k].reshape(-1, 4)[ids, :3].astype(np.float64)
            d = (g - r) / np.maximum(r, 1e-3)
            sq += float((d * d).sum())
            cnt += d.size
    cores = threads
    return {"mrays": traced / seconds / 1e6, "seconds": seconds, "traced": traced, "pixels": pixels,
            "node_visits_per_ray": nodes / max(1, traced), "tri_tests_per_ray": tris / max(1, traced),
            "cores": cores, "build_s": build_s, "oscs": oscs,
            "rel_rmse": float(np.sqrt(sq / cnt)) if cnt else None}


def cpu_frames(jobs, subset=None, threads=0, oscs=None):
    """The reference's own frame loop on whole frames: one frame of one sample per pixel of each job in
    `subset` (all jobs by default), every pixel in the reference's 20x20 tiles on a worker pool of
    every usable core, the running-mean film.  Every frame of a job costs the same in expectation
    (only the sample index differs), so each job's frame is extrapolated to its spp: Mrays/s =
    sum(rays_j * spp_j) / sum(seconds_j * spp_j), the full workload's rate.  Returns per-job
    (rays, seconds, node visits, triangle tests, pixels), so that rotating subsets (the reference
    arm's steps) add up to the same estimate."""
    if threads <= 0:
        threads = usable_cores()
    ob = oracle_module()
    if oscs is None:
        oscs = oracle_scenes(jobs)
    subset = range(len(jobs)) if subset is None else subset
    per_job = {}
    for k in subset:
        j = jobs[k]
        W, H = j["width"], j["height"]
        opt = ob.options(W, H, 1, j["depth"], seed=0, rr_start=j["rr_start"], threads=threads)
        _, st = oscs[k].render(opt)
        per_job[k] = (st.traced, st.seconds, st.node_visits, st.tri_tests, W * H)
    return per_job


def frames_rate(jobs, per_job, threads):
    """Full-workload estimate from per-job whole-frame timings (see cpu_frames)."""
    rays = sum(v[0] * jobs[k]["spp"] for k, v in per_job.items())
    secs = sum(v[1] * jobs[k]["spp"] for k, v in per_job.items())
    nodes = sum(v[2] * jobs[k]["spp"] for k, v in per_job.items())
    tris = sum(v[3] * jobs[k]["spp"] for k, v in per_job.items())
    return {"mrays": rays / secs / 1e6, "seconds": sum(v[1] for v in per_job.values()),
            "traced": sum(v[0] for v in per_job.values()), "pixels": sum(v[4] for v in per_job.values()),
            "node_visits_per_ray": nodes / max(1, rays), "tri_tests_per_ray": tris / max(1, rays),
            "cores": threads, "jobs_timed": len(per_job)}


def cpu_sampling(workload):
    """How the CPU legs sample the workload: whole frames, except the instanced scene, whose
    reference BVH leaves one 5.25 M-triangle leaf (a CPU ray costs ~5 M triangle tests), where a
    pixel subset is all that fits in a bounded sample."""
    return "pixels" if workload == "instanced" else "frames"


def frames_sample_text(jobs, threads):
    return ("oracle (CPU restatement of the reference Nova path) rendering whole frames the way the reference does: "
            "one frame of 1 sample per pixel per job, 20x20 tiles on a pool of %d workers, running-mean film; each "
            "job's frame time extrapolated to its spp (sum rays*spp / sum seconds*spp over %d jobs)" % (threads, len(jobs)))


def cpu_stride(workload):
    """Pixel stride of the pixel-subset sample (the instanced workload's CPU timing and, for the
    others, the untimed film-vs-oracle check)."""
    env = os.environ.get("NOVA_BENCH_CPU_STRIDE")
    if env:
        return int(env)
    if workload == "instanced":
        # the reference builder leaves this scene in one 5.25 M-triangle leaf (its SAH starts from
        # (float)INT_MAX and no split of a node this large scores below it), so a CPU ray costs
        # ~5 M triangle tests
        return 49152
    if workload == "heightfield":
        return 16
    return 64


CONFIG_L2 = "inputs larger than L2 (no flush): the scenes' triangles and BVHs exceed the 126 MB L2"


def bench_config(workload, nj):
    """The config both arms print (identical, so the two lines describe the same workload)."""
    return {"workload": workload, "jobs": nj, "l2": CONFIG_L2}


def run_reference(args, rank, world):
    if rank != 0:
        return
    jobs = make_jobs(args.workload)
    oscs = oracle_scenes(jobs)
    threads = usable_cores()
    metric = {"heightfield": HF_METRIC, "instanced": IN_METRIC}.get(args.workload, BATCH_METRIC)
    workload = {"heightfield": HF_WORKLOAD, "instanced": IN_WORKLOAD}.get(args.workload, BATCH_WORKLOAD)
    secs = []
    if cpu_sampling(args.workload) == "frames":
        # each step: one whole frame of each of 8 jobs, rotating through all of them
        per_step = min(8, len(jobs))
        for _ in range(min(args.warmup, 1)):
            cpu_frames(jobs, subset=[0], oscs=oscs)
        per_job = {}
        for step in range(args.steps):
            sub = [(step * per_step + q) % len(jobs) for q in range(per_step)]
            t0 = time.perf_counter()
            got = cpu_frames(jobs, subset=sub, oscs=oscs)
            secs.append(time.perf_counter() - t0)
            for k, v in got.items():  # a job timed again adds its frame to the job's totals
                if k in per_job:
                    a = per_job[k]
                    per_job[k] = tuple(x + y for x, y in zip(a[:4], v[:4])) + (a[4],)
                else:
                    per_job[k] = v
        v = frames_rate(jobs, per_job, threads)["mrays"]
        sample = frames_sample_text(jobs, threads) + "; 8 jobs per step, rotating"
    else:
        stride = cpu_stride(args.workload)
        for _ in range(min(args.warmup, 1)):
            cpu_sample(jobs, stride * 4, oscs=oscs)
        vals = []
        last = None
        for _ in range(args.steps):
            t0 = time.perf_counter()
            last = cpu_sample(jobs, stride, oscs=oscs)
            secs.append(time.perf_counter() - t0)
            vals.append(last["mrays"])
        v = float(np.median(vals))
        sample = ("oracle (CPU restatement of the reference Nova path, thread pool of %d workers) on every %dth pixel "
                  "of the frame, all samples: %d pixels" % (last["cores"], stride, last["pixels"]))
    line = {"impl": "reference", "metric": metric, "value": v, "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(secs)) * 1000.0,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scenes and env maps)", "config": bench_config(workload, len(jobs)),
            "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------------------------


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


class Acc:
    """Sums render stats over steps."""

    def __init__(self):
        self.traced = self.paths = self.kernels = self.waves = 0
        self.dev_ms = self.trace_ms = self.shade_ms = 0.0

    def add(self, st):
        self.traced += st.traced
        self.paths += st.paths
        self.kernels += st.kernels
        self.waves += st.waves
        self.dev_ms += st.device_ms
        self.trace_ms += st.trace_ms
        self.shade_ms += st.shade_ms


def timed(step, steps, torch, dist, clock=None):
    """Runs `steps` steps between barriers + synchronizes; returns (Acc, ms per step over the
    render stream and the torch stream, max over ranks, traced rays summed over ranks)."""
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    acc = Acc()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(steps):
        for st in step():
            acc.add(st)
    ev1.record()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms = max(acc.dev_ms, ev0.elapsed_time(ev1)) / steps
    traced = float(acc.traced)
    if dist:
        t = torch.tensor([step_ms, traced], dtype=torch.float64, device="cuda")
        mx = t.clone()
        dist.all_reduce(mx[:1], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[1:], op=dist.ReduceOp.SUM)
        step_ms, traced = float(mx[0]), float(t[1])
    return acc, step_ms, traced


ADJ_CFG = dict(width=256, height=256, spp=64, depth=4)


def film_io_timing(local_rank, cpu_baseline=True, reps=10):
    """The film outputs and the .hdr path at 3840 x 2160 RGBA float (133 MB per film): device time
    of each kernel or kernel chain (CUDA events, median of `reps` calls) against its algorithmic
    bytes and the HBM copy peak; the whole nova_b200_hdr_write / nova_b200_hdr_read between host
    pixels and a file by wall clock; and the oracle writing and reading the same file on one host
    core (the reference's stb path restated)."""
    import tempfile
    import torch
    from axomae_b200 import native
    W, H = 3840, 2160
    n = W * H * 4
    px_bytes = W * H * 16
    hbm = peaks().get("hbm_gbs") or 6650.0
    rng = np.random.default_rng(1)
    host = rng.lognormal(0, 1, (H, W, 4)).astype(np.float32)
    c = native.Context(local_rank)
    part = torch.from_numpy(host).cuda()
    acc = torch.rand((H, W, 4), device="cuda")
    fin = torch.empty_like(acc)
    disp = torch.empty_like(acc)
    snap = torch.zeros((1080, 1920, 4), device="cuda")
    back = torch.empty_like(acc)
    out = {}

    def timed(name, fn, algo_bytes):
        ms = []
        for _ in range(reps + 1):
            fn()
            ms.append(c.last_call_ms())
        t = float(np.median(ms[1:]))
        gbs = algo_bytes / (t / 1e3) / 1e9
        out[name] = {"device_ms": t, "algorithmic_bytes": algo_bytes, "achieved_gbs": gbs, "frac_of_hbm": gbs / hbm}

    timed("k_accumulate", lambda: c.film_accumulate(part.data_ptr(), acc.data_ptr(), fin.data_ptr(), n, 3),
          4 * px_bytes)
    timed("k_display_blend", lambda: c.display_blend(part.data_ptr(), acc.data_ptr(), disp.data_ptr(), n, 3),
          3 * px_bytes)
    # the resample reads four texels (12 B each) per output pixel and writes 12 B
    timed("k_snapshot", lambda: c.snapshot(fin.data_ptr(), W, H, 4, snap.data_ptr(), 1920, 1080),
          1920 * 1080 * (4 * 12 + 12))
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "film")
        # device work of a write (encode, run-length packing, offsets, gather) and of a read
        # (expansion, decode): algorithmic bytes = float pixels + RGBE pixels, once each
        timed("hdr_write_device", lambda: c.hdr_write(path, W, H, 4, pixels_device_ptr=fin.data_ptr()),
              W * H * (16 + 4))
        timed("hdr_read_device", lambda: c.hdr_read(path + ".hdr", rgba_device_ptr=back.data_ptr()), W * H * (4 + 16))
        walls, reads = [], []
        for _ in range(3):
            t0 = time.perf_counter()
            c.hdr_write(path, W, H, 4, pixels_host=host)
            walls.append(time.perf_counter() - t0)
        back_host = np.empty((H, W, 4), np.float32)
        for _ in range(3):
            t0 = time.perf_counter()
            c.hdr_read(path + ".hdr", rgba_host=back_host)
            reads.append(time.perf_counter() - t0)
        file_mb = os.path.getsize(path + ".hdr") / 1e6
        out["hdr_write_e2e"] = {"seconds": float(np.median(walls)), "mpix_per_s": W * H / float(np.median(walls)) / 1e6,
                                "file_mb": file_mb, "h2d_bytes": px_bytes, "d2h_bytes": int(file_mb * 1e6),
                                "note": "nova_b200_hdr_write from host pixels, wall clock: H2D, device encode and "
                                        "packing, D2H of the packed bytes, file write"}
        out["hdr_read_e2e"] = {"seconds": float(np.median(reads)), "mpix_per_s": W * H / float(np.median(reads)) / 1e6,
                               "h2d_bytes": int(file_mb * 1e6), "d2h_bytes": px_bytes,
                               "note": "nova_b200_hdr_read to host pixels, wall clock: file read, packet-header scan "
                                       "on the host, H2D of the file, device expansion and decode, D2H"}
        if cpu_baseline:
            ob = oracle_module()
            t0 = time.perf_counter()
            ob.hdr_write(os.path.join(d, "cpu"), host, W, H, 4)
            cw = time.perf_counter() - t0
            t0 = time.perf_counter()
            data = open(os.path.join(d, "cpu.hdr"), "rb").read()
            _, _, _, q = ob.hdr_parse(data)
            ob.rgbe_decode(q.reshape(-1, 4))
            cr = time.perf_counter() - t0
            out["cpu_baseline"] = {"hdr_write_mpix_per_s": W * H / cw / 1e6, "hdr_read_mpix_per_s": W * H / cr / 1e6,
                                   "cores": 1, "kind": "port",
                                   "sample": "the same 3840x2160 film written and read back by the oracle "
                                             "(stbi_write_hdr / stbi_loadf restated, one thread)"}
    c.close()
    out["workload"] = "3840x2160 RGBA float film; snapshot to 1920x1080; .hdr file in a temporary directory"
    return out


BAKE_SAMPLES = 128


def bake_timing(local_rank, cpu_baseline=True, reps=5):
    """The irradiance bake on the heightfield workload's 2048 x 1024 log-normal(0, 1.5) environment
    map: 64 x 64 (the editor's size) and 512 x 256 outputs, BAKE_SAMPLES samples per texel.  Device
    side: nova_b200_bake_irradiance on device buffers, wall clock around the call (it synchronises),
    median of `reps`; CPU side: the oracle's restatement of the reference's CPU bake with its 8
    worker threads (TextureProcessing.cpp:10-64).  Unit: output texels x samples per second."""
    import torch
    from axomae_b200 import native, scenes
    s = scenes.heightfield_scene(n=8, width=16, height=16, env_w=HF["env_w"], env_h=HF["env_h"], seed=HF["seed"])
    env = next(t for t in s["textures"] if t["format"] == "f32")
    src = np.asarray(env["pixels"], np.float32).reshape(env["height"], env["width"], 4)
    c = native.Context(local_rank)
    out = {"env": "%dx%d float RGBA" % (env["width"], env["height"]), "samples": BAKE_SAMPLES}
    try:
        ts = torch.from_numpy(np.ascontiguousarray(src)).cuda()
        for ow, oh in ((64, 64), (512, 256)):
            dst = torch.zeros((oh, ow, 4), device="cuda")
            walls = []
            for _ in range(reps + 1):
                t0 = time.perf_counter()
                c.bake_irradiance(ts.data_ptr(), env["width"], env["height"], 4, ow, oh, BAKE_SAMPLES, dst.data_ptr())
                walls.append(time.perf_counter() - t0)
            w = float(np.median(walls[1:]))
            rec = {"seconds": w, "gtexel_samples_per_s": ow * oh * BAKE_SAMPLES / w / 1e9}
            if cpu_baseline:
                ob = oracle_module()
                t0 = time.perf_counter()
                ob.bake_irradiance(src, ow, oh, BAKE_SAMPLES, threads=8)
                cw = time.perf_counter() - t0
                rec["cpu"] = {"seconds": cw, "gtexel_samples_per_s": ow * oh * BAKE_SAMPLES / cw / 1e9, "cores": 8,
                              "kind": "port"}
            out["%dx%d" % (ow, oh)] = rec
    finally:
        c.close()
    return out


def adjoint_timing(local_rank, reps=3):
    """The differentiable configuration: the 64-sphere scene at 256 x 256, 64 spp, depth 4, with
    per-triangle albedo (init 0.5) and per-material roughness (init 0.3) as parameters and an L2
    loss against a target rendered with seeded albedo U[0.2, 0.8] and roughness U[0.1, 0.6].
    Returns the device times of one forward render and one replay-adjoint backward."""
    import torch
    from axomae_b200 import native, scenes
    W, H, spp, depth = ADJ_CFG["width"], ADJ_CFG["height"], ADJ_CFG["spp"], ADJ_CFG["depth"]
    s = scenes.spheres_scene(W, H)
    c = native.Context(local_rank)
    c.upload(s)
    c.build()
    ntri, nmat = c.info()["triangles"], len(s["materials"])
    rng = np.random.default_rng(0)
    alb_t = torch.tensor(rng.uniform(0.2, 0.8, (ntri, 3)), dtype=torch.float32, device="cuda")
    rough_t = torch.tensor(rng.uniform(0.1, 0.6, nmat), dtype=torch.float32, device="cuda")
    alb = torch.full((ntri, 3), 0.5, device="cuda")
    rough = torch.full((nmat,), 0.3, device="cuda")
    fr = native.make_frame(s, W, H, spp, depth)
    T = torch.zeros((H, W, 4), device="cuda")
    c.set_diff_params(alb_t.data_ptr(), rough_t.data_ptr())
    c.render(fr, film_device_ptr=T.data_ptr())
    c.set_diff_params(alb.data_ptr(), rough.data_ptr())
    img = torch.zeros((H, W, 4), device="cuda")
    ga = torch.zeros_like(alb)
    gr = torch.zeros_like(rough)
    fwd, bwd, bwd_reuse = [], [], []
    for _ in range(reps + 1):
        st = c.render(fr, film_device_ptr=img.data_ptr())
        dI = torch.zeros_like(img)
        dI[..., :3] = 2.0 * (img[..., :3] - T[..., :3])
        torch.cuda.synchronize()  # dI is written on torch's stream, the backward runs on the context's
        rst = c.backward(fr, dI.data_ptr(), ga.data_ptr(), gr.data_ptr(), reuse_primal=True)
        bst = c.backward(fr, dI.data_ptr(), ga.data_ptr(), gr.data_ptr())
        fwd.append(st.device_ms)
        bwd.append(bst.device_ms)
        bwd_reuse.append(rst.device_ms)
    c.close()
    f, b, br = float(np.median(fwd[1:])), float(np.median(bwd[1:])), float(np.median(bwd_reuse[1:]))
    return {"workload": "64 spheres (65,538 tris) 256x256, 64 spp, depth 4; params: %d x 3 albedo + %d roughness"
                        % (ntri, nmat), "forward_ms": f, "backward_ms": b, "backward_over_forward": b / f,
            "backward_reusing_forward_ms": br, "backward_reusing_forward_over_forward": br / f,
            "forward_mrays": st.traced / f / 1e3,
            "note": "device time (CUDA events); backward = radiance replay + adjoint replay (no stored tape); the "
                    "reusing variant takes the per-path radiance the forward render left in the radiance buffer"}


def instanced_bvh_forms(ctx, job, frame, reps=2):
    """The instanced scene (1000 instances of 10 meshes) with each BVH form: the flat binary BVH over
    every instanced triangle's world box (width 2) and the two-level one, a BVH per mesh under a
    BVH over the instances (width 1, as the reference's Embree scene keeps them).  Per form: the
    build's wall clock (one synchronous call), the device memory, and the render's Mrays/s (device
    time, median of `reps` after one warm-up)."""
    import torch
    out = {}
    for name, width in (("flat", 2), ("two_level", 1)):
        t0 = time.perf_counter()
        ctx.build(width=width)
        build_s = time.perf_counter() - t0
        info = ctx.info()
        film = torch.zeros((job["height"], job["width"], 4), device="cuda")
        vals = []
        for _ in range(reps + 1):
            st = ctx.render(frame, film_device_ptr=film.data_ptr())
            vals.append(st.traced / st.device_ms / 1e3)
        out[name] = {"width": width, "build_ms": build_s * 1e3, "nodes": info["nodes"],
                     "device_bytes": info["device_bytes"], "mrays": float(np.median(vals[1:])),
                     "trace_ms": st.trace_ms}
    return out


def instanced_gradients(local_rank, width, reps=2):
    """Roughness gradients of the instanced scene at 512 x 512 (16 spp, depth 12): per-material
    roughness (8 materials, init 0.3) against a target rendered with seeded roughness U[0.1, 0.6];
    the loss is the L2 distance of log(1 + radiance), so the environment's brightest texels (the
    log-normal map reaches ~1e3) do not swamp it; device times of one forward render and one
    replay-adjoint backward (roughness only)."""
    import torch
    from axomae_b200 import native, scenes
    W = H = 512
    spp, depth = IN["spp"], IN["depth"]
    s = scenes.instanced_scene(n_meshes=10, n_instances=1000, tris_per_mesh=10000, width=W, height=H, seed=0,
                               env_w=4096, env_h=2048)
    c = native.Context(local_rank)
    try:
        c.upload(s)
        c.build(width=width)
        nmat = len(s["materials"])
        rng = np.random.default_rng(1)
        rough_t = torch.tensor(rng.uniform(0.1, 0.6, nmat), dtype=torch.float32, device="cuda")
        rough = torch.full((nmat,), 0.3, device="cuda")
        fr = native.make_frame(s, W, H, spp, depth)
        T = torch.zeros((H, W, 4), device="cuda")
        c.set_diff_params(None, rough_t.data_ptr())
        c.render(fr, film_device_ptr=T.data_ptr())
        c.set_diff_params(None, rough.data_ptr())
        img = torch.zeros((H, W, 4), device="cuda")
        gr = torch.zeros_like(rough)
        fwd, bwd = [], []
        loss = None
        for _ in range(reps + 1):
            st = c.render(fr, film_device_ptr=img.data_ptr())
            dI = torch.zeros_like(img)
            li, lt = torch.log1p(img[..., :3]), torch.log1p(T[..., :3])
            dI[..., :3] = 2.0 * (li - lt) / (1.0 + img[..., :3])
            loss = float(((li - lt) ** 2).sum())
            gr.zero_()
            torch.cuda.synchronize()  # dI and the zeroed gradient are written on torch's stream
            bst = c.backward(fr, dI.data_ptr(), None, gr.data_ptr())
            fwd.append(st.device_ms)
            bwd.append(bst.device_ms)
        f, b = float(np.median(fwd[1:])), float(np.median(bwd[1:]))
        return {"workload": "instanced scene at 512x512, 16 spp, depth 12; params: %d material roughnesses" % nmat,
                "bvh_width": width, "forward_ms": f, "backward_ms": b, "backward_over_forward": b / f,
                "loss": loss, "image_max": float(img[..., :3].max()), "target_max": float(T[..., :3].max()),
                "grad_roughness": [float(x) for x in gr.cpu().numpy()],
                "note": "device time (CUDA events); backward = radiance replay + adjoint replay"}
    finally:
        c.close()


def run_ours(args, rank, world, local_rank):
    import torch
    from axomae_b200 import native
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    batched = args.workload == "batched"
    jobs = make_jobs(args.workload)
    nj = len(jobs)
    ctxs = [native.Context(local_rank) for _ in jobs]
    t0 = time.perf_counter()
    for c, j in zip(ctxs, jobs):
        c.upload(j["scene"])
    upload_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    for c in ctxs:
        c.build(width=args.bvh_width)
    build_s = time.perf_counter() - t0
    infos = [c.info() for c in ctxs]
    from axomae_b200 import multigpu
    frames = []
    for j in jobs:
        spp_total, begin, count = multigpu.weak_range(j["spp"], rank, world)
        frames.append(native.make_frame(j["scene"], j["width"], j["height"], spp_total, j["depth"], seed=0,
                                        sample_begin=begin, sample_count=count, rr_start=j["rr_start"], reset=1))
    sizes = [j["width"] * j["height"] * 4 for j in jobs]
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    flat = torch.zeros(int(offs[-1]), dtype=torch.float32, device="cuda")
    films = [flat[int(offs[k]):int(offs[k + 1])] for k in range(nj)]
    plain_flat = torch.zeros_like(flat)
    plain_films = [plain_flat[int(offs[k]):int(offs[k + 1])] for k in range(nj)]

    def render_and_reduce(buf, render):
        """This rank's renders, then (several ranks) the film reduction.  A rank whose render fails
        reports it in the reduction, so every rank raises RankFailure there instead of waiting."""
        if not dist:
            return render()
        try:
            out, failed = render(), False
        except RuntimeError:
            traceback.print_exc()
            out, failed = [], True
        multigpu.reduce_films(buf, 1, failed=failed)  # every rank rendered the same sample count
        return out

    def plain_step():
        return render_and_reduce(plain_flat, lambda: [c.render(f, film_device_ptr=p.data_ptr())
                                                      for c, f, p in zip(ctxs, frames, plain_films)])

    def batch_step():
        return render_and_reduce(flat, lambda: [native.render_batch(ctxs, frames,
                                                                    films_device=[p.data_ptr() for p in films])])

    arms = {"plain": plain_step}
    if batched:
        arms["batched"] = batch_step
    res = {}
    clk_summary = None
    tuning = None
    tune_s = None
    if args.trace_mode is not None:  # a fixed trace mode for both arms (no autotuning)
        for c in ctxs:
            c.set_tuning(trace_mode=args.trace_mode)
    for name, step in arms.items():
        if name == "batched" and not args.no_autotune and args.trace_mode is None:
            # the batched system picks its launch tuning (queue capacity, block sizes, pixel tiles)
            # with the library's autotuner; the plain arm above ran with the library defaults
            t0 = time.perf_counter()
            tuning = native.autotune(ctxs, frames, None).as_dict()
            tune_s = time.perf_counter() - t0
        for _ in range(args.warmup):
            step()
        if name == ("batched" if batched else "plain"):
            with ClockSampler(local_rank) as clk:
                res[name] = timed(step, args.steps, torch, dist)
            clk_summary = clk.summary()
        else:
            res[name] = timed(step, args.steps, torch, dist)
    head = "batched" if batched else "plain"
    acc, step_ms, traced_all = res[head]
    value = traced_all / args.steps / (step_ms / 1e3) / 1e6
    films_identical = None
    if batched:
        films_identical = bool(torch.equal(flat, plain_flat))

    # untimed: the same step once more in the counting trace mode (tuning.trace_mode 2), for the
    # closest-hit kernel's own work per ray (node visits, triangle tests) on this workload's rays
    counted = None
    saved = [c.get_tuning() for c in ctxs]
    try:
        for c, t in zip(ctxs, saved):
            tc = native.Tuning.from_buffer_copy(t)
            tc.trace_mode = 2
            tc.bvh_width = 0
            c.set_tuning(tc)
        sts = batch_step() if batched else plain_step()
        nodes = sum(s.node_visits for s in sts)
        tris = sum(s.tri_tests for s in sts)
        traced = sum(s.traced for s in sts)
        counted = {"node_visits_per_ray": nodes / max(1, traced), "tri_tests_per_ray": tris / max(1, traced)}
    finally:
        for c, t in zip(ctxs, saved):
            t2 = native.Tuning.from_buffer_copy(t)
            t2.bvh_width = 0
            c.set_tuning(t2)

    # end to end through the C ABI from pinned host buffers: upload + build + render + readback
    e2e = None
    if rank == 0 and not args.no_e2e:
        # pinned host copies of the scenes and their C descriptors, made once like a C++ caller's
        # buffers and structs; every step still copies all of the scene data to the device
        pinned = [native.prepare_scene(pin_scene(j["scene"])) for j in jobs]
        host_films = [torch.empty(s, dtype=torch.float32).pin_memory() for s in sizes]
        e_frames = [native.make_frame(j["scene"], j["width"], j["height"], j["spp"], j["depth"], seed=0,
                                      rr_start=j["rr_start"]) for j in jobs]
        e_steps = args.steps

        def e2e_step():
            hf = [h.numpy() for h in host_films]
            t0 = time.perf_counter()
            if batched:  # one pipelined call: uploads and builds on host threads while the chunks
                # whose scenes are ready render (the phases overlap, so only the total is timed)
                traced = native.upload_build_render_batch(ctxs, pinned, e_frames, films_host=hf,
                                                          width=args.bvh_width).traced
                t3 = time.perf_counter()
                return traced, (0.0, 0.0, t3 - t0)
            for c, p in zip(ctxs, pinned):
                c.upload(p)
            t1 = time.perf_counter()
            for c in ctxs:
                c.build(width=args.bvh_width)
            t2 = time.perf_counter()
            traced = sum(c.render(f, film_host=h).traced for c, f, h in zip(ctxs, e_frames, hf))
            t3 = time.perf_counter()
            return traced, (t1 - t0, t2 - t1, t3 - t2)

        e2e_step()  # untimed: first upload of pinned buffers
        e_traced = 0
        stages = np.zeros(3)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e_steps):
            tr, st3 = e2e_step()
            e_traced += tr
            stages += st3
        for c in ctxs:
            c.synchronize()
        e_s = time.perf_counter() - t0
        e2e = {"value": e_traced / e_s / 1e6, "unit": "Mrays/s",
               "h2d_bytes_per_step": int(sum(scene_bytes(j["scene"]) for j in jobs)),
               "d2h_bytes_per_step": int(sum(sizes) * 4), "steps": e_steps, "warmup": 1,
               "upload_ms": 1e3 * stages[0] / e_steps, "build_ms": 1e3 * stages[1] / e_steps,
               "render_ms": 1e3 * stages[2] / e_steps,
               "timing": "host wall clock around scene upload (pinned H2D) + BVH build + render + film D2H: %s" % (
                   "one nova_b200_upload_build_render_batch (upload, build and render overlap: render_ms is "
                   "the whole step)"
                   if batched else "nova_b200_upload_scene, nova_b200_build_bvh, nova_b200_render")}

    if rank != 0:
        for c in ctxs:
            c.close()
        if dist:
            dist.destroy_process_group()
        return

    cpu = None
    check = None
    if not args.no_cpu:
        host = [f.cpu().numpy() for f in films] if batched else [f.cpu().numpy() for f in plain_films]
        threads = usable_cores()
        if cpu_sampling(args.workload) == "frames":
            oscs = oracle_scenes(jobs)
            cpu = frames_rate(jobs, cpu_frames(jobs, oscs=oscs, threads=threads), threads)
            cpu["sample"] = frames_sample_text(jobs, threads)
            # untimed: the device films against the oracle on a pixel subset with all samples
            check = cpu_sample(jobs, cpu_stride(args.workload), oscs=oscs, films=host if world == 1 else None)
        else:
            cpu = cpu_sample(jobs, cpu_stride(args.workload), films=host if world == 1 else None)
            check = cpu
            cpu["sample"] = ("oracle on every %dth pixel of the frame, all samples (%d pixels, %.1f s)"
                             % (cpu_stride(args.workload), cpu["pixels"], cpu["seconds"]))
    pk = peaks()
    hbm = pk.get("hbm_gbs")
    peak_src = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    # Algorithmic bytes per traced ray (reference binary BVH node/triangle counts measured by the
    # oracle on this workload's rays): 32 B ray + 16 B hit + 64 B per inner-node visit + 36 B per
    # triangle test.
    # reference-BVH model: 32 B ray + 16 B hit + 64 B per inner-node visit + 36 B per triangle test,
    # with the visit counts the oracle measured on the reference's binary SAH BVH
    b_ref = 32 + 16 + 64 * cpu["node_visits_per_ray"] + 36 * cpu["tri_tests_per_ray"] if cpu else None
    if args.workload == "instanced":
        b_ref = None  # reference-BVH visit counts of a degenerate tree say nothing about k_trace
    # this kernel's own work: 32 B ray in, 16 B hit + 4 B queue slot out, one node record per visit
    # (binary 64 B, 8-wide 80 B) and 48 B per triangle tested, counted by the kernel itself
    node_bytes = 80 if (args.bvh_width or 2) == 8 else 64
    b_dev = (32 + 20 + node_bytes * counted["node_visits_per_ray"] + 48 * counted["tri_tests_per_ray"]
             if counted else None)
    trace_rate = acc.traced / (acc.trace_ms / 1e3) if acc.trace_ms > 0 else None
    roof = None
    if b_dev and trace_rate:
        achieved = trace_rate * b_dev / 1e9
        rays_per_wave = acc.traced / max(1, acc.waves)
        binary = (args.bvh_width or 2) == 2  # the ncu figures are the binary layout's
        dram_ray = (K_TRACE_DRAM_BYTES_PER_RAY[args.workload] or 0.0) if binary else 0.0
        l2_ray = K_TRACE_L2_BYTES_PER_RAY[args.workload] if binary else None
        roof = {"bound": "hbm", "kernel": "k_trace", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_source": peak_src,
                "traffic": dram_ray * rays_per_wave if dram_ray else None,
                "traffic_note": "DRAM bytes of one full wave (%.0f rays) at %.0f B/ray measured by ncu "
                                "(dram__bytes_read.sum + dram__bytes_write.sum) on this workload's k_trace waves; "
                                "achieved uses this kernel's algorithmic bytes: its own node visits and triangle "
                                "tests per ray, counted on this workload (trace_mode 2)" % (rays_per_wave, dram_ray),
                "dram_gbs_from_traffic": trace_rate * dram_ray / 1e9 if dram_ray else None,
                "l2_bytes_per_ray": l2_ray, "l2_gbs_from_traffic": trace_rate * l2_ray / 1e9 if l2_ray else None,
                "bytes_per_ray": b_dev, "node_visits_per_ray": counted["node_visits_per_ray"],
                "tri_tests_per_ray": counted["tri_tests_per_ray"], "trace_ms_per_step": acc.trace_ms / args.steps,
                "reference_bvh_model": None if not b_ref else {
                    "bytes_per_ray": b_ref, "node_visits_per_ray": cpu["node_visits_per_ray"],
                    "tri_tests_per_ray": cpu["tri_tests_per_ray"], "achieved": trace_rate * b_ref / 1e9,
                    "frac": trace_rate * b_ref / 1e9 / hbm}}
    extra = {"waves_per_step": acc.waves / args.steps, "traced_per_step": acc.traced / args.steps,
             "paths_per_step": acc.paths / args.steps, "trace_ms_per_step": acc.trace_ms / args.steps,
             "shade_ms_per_step": acc.shade_ms / args.steps, "bvh_build_s": build_s, "upload_s": upload_s,
             "bvh_nodes": sum(i["nodes"] for i in infos), "triangles": sum(i["triangles"] for i in infos),
             "device_bytes": sum(i["device_bytes"] for i in infos), "bvh_width": args.bvh_width or 2,
             "parallelism": "sample-range partition + NCCL film all-reduce" if world > 1 else "single GPU",
             "films_mb": int(sum(sizes) * 4 / 1e6)}
    if batched:
        pacc, pms, ptraced = res["plain"]
        pval = ptraced / args.steps / (pms / 1e3) / 1e6
        extra["plain"] = {"value": pval, "unit": "Mrays/s", "ms_per_step": pms, "gpu_launches": pacc.kernels,
                          "waves_per_step": pacc.waves / args.steps, "trace_ms_per_step": pacc.trace_ms / args.steps,
                          "shade_ms_per_step": pacc.shade_ms / args.steps}
        extra["batched_over_plain"] = value / pval
        extra["autotune"] = {"tuning": tuning, "seconds": tune_s,
                             "note": "batched arm only; the plain arm uses the default tuning"}
        extra["films_identical"] = films_identical
        extra["equal_rmse"] = ("batched and plain films compared bit for bit after the timed steps; "
                               "rel_rmse_vs_cpu is the per-pixel relative RMSE of the film against the oracle "
                               "on the CPU sample's pixels")
    if args.trace_mode is not None:
        extra["trace_mode"] = args.trace_mode
    if check:
        extra["rel_rmse_vs_cpu"] = check["rel_rmse"]
        extra["rel_rmse_pixels"] = "every %dth pixel of every frame, all samples" % cpu_stride(args.workload)
    if batched and not args.no_adjoint:
        extra["adjoint"] = adjoint_timing(local_rank)
    if args.workload == "instanced":
        extra["bvh_forms"] = instanced_bvh_forms(ctxs[0], jobs[0], frames[0])
        if not args.no_adjoint:
            extra["gradients_512"] = instanced_gradients(local_rank, args.bvh_width or 2)
    if batched and not args.no_film_io:
        extra["film_io"] = film_io_timing(local_rank, cpu_baseline=not args.no_cpu and local_rank == 0)
    if batched and not args.no_bake:
        try:  # the bake is a side measurement: a failure here is reported, never loses the bench line
            extra["bake"] = bake_timing(local_rank, cpu_baseline=not args.no_cpu and local_rank == 0)
        except Exception as e:  # noqa: BLE001
            extra["bake"] = {"error": repr(e)}
    metric = {"heightfield": HF_METRIC, "instanced": IN_METRIC}.get(args.workload, BATCH_METRIC)
    workload = {"heightfield": HF_WORKLOAD, "instanced": IN_WORKLOAD}.get(args.workload, BATCH_WORKLOAD)
    if args.frame or args.spp:
        workload += " (overridden: frame %s, spp %s)" % (args.frame, args.spp)
    line = {"metric": metric, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scenes and env maps)",
            "config": bench_config(workload, nj),
            "e2e": e2e, "roofline": roof,
            "cpu_baseline": None if not cpu else {
                "value": cpu["mrays"], "unit": "Mrays/s", "cores": cpu["cores"], "kind": "port",
                "sample": cpu["sample"]},
            "clocks": clk_summary, "gpu_launches": acc.kernels, "extra": extra}
    print(json.dumps(line), flush=True)
    for c in ctxs:
        c.close()
    if dist:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched", choices=["batched", "heightfield", "instanced"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="batched arm: keep the default launch tuning")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint/forward timing")
    ap.add_argument("--no-film-io", action="store_true", help="skip the film output / .hdr timing")
    ap.add_argument("--no-bake", action="store_true", help="skip the irradiance bake timing")
    ap.add_argument("--frame", type=int, nargs=2, metavar=("W", "H"), help="heightfield: override the frame size")
    ap.add_argument("--spp", type=int, help="heightfield: override samples per pixel")
    ap.add_argument("--trace-mode", type=int, choices=[0, 1, 3],
                    help="launch tuning's trace mode for both arms: 0 per-wave kernels, 1 persistent trace warps, "
                         "3 the persistent wavefront (one cooperative launch per chunk); default: autotuned")
    ap.add_argument("--bvh-width", type=int, default=0, choices=[0, 1, 2, 8],
                    help="BVH layout: 2 binary, 8 compressed 8-wide, 1 two-level (0 = library default)")
    args = ap.parse_args()
    if args.frame:
        HF["width"], HF["height"] = args.frame
    if args.spp:
        HF["spp"] = args.spp
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if "RANK" not in os.environ:
        world = 1
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
