#!/usr/bin/env python
"""Benchmark of the wavefront path tracer: Mrays/s at 1080p / 1.31M triangles (plain), the
equal-time relMSE of the learned-guided renderer against the plain one (the "guided" object), and
batched serving of 64 uneven requests in one CUDA-graph launch (the "batched" object).

Workload (one GPU): seeded displaced-icosphere field, 64 instances x 20,480 triangles (1.31M f32
triangles), 16-layer 1024^2 value-noise textures, 1920x1080, Medium shader, depth 12, no guiding,
ReSTIR off.  One step = one lam_render of 16 samples per pixel; 16 steps make the 256-spp image.

  python bench.py [--gpus N --steps K --warmup W]            this implementation (CUDA, sm_100a)
  python bench.py --impl reference [...]                     the reference path on the host cores
                                                             (CPU restatement of its shaders)
Multi-GPU (torchrun, one rank per GPU): every rank renders its own samples of the full frame with
a distinct seed (sample sharding, weak scaling); the images are summed with one NCCL all-reduce at
the end of the timed region.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mrays/s at 1080p/1.3M tris"
SEG_BYTES_EXTEND = 48   # ray (o, d, tmax) 28 B read + hit 20 B write per segment
SEG_BYTES_TOTAL = 280   # extend 48 + shade 232 (compulsory wavefront traffic per segment)
# DRAM bytes (read + write) per segment of the extend kernel: ncu's dram__bytes_read.sum +
# dram__bytes_write.sum over the 12 extend launches of one 960x540, 4-spp step of the same scene
# (7.20M segments; the full 1080p step is too large for a multi-metric capture), in the default
# material-ordered shading, from
#   ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum,gpu__time_duration.sum,lts__t_sector_hit_rate.pct
#       --clock-control none -k regex:extend_kernel -s 36 -c 12 python bench.py --width 960 --height 540 --spp 4
#       --steps 1 --warmup 3 --no-cpu-baseline --no-guided --no-batched --no-restir
# Traffic grows with the segments a launch processes, so a full launch's traffic is this times its segments.
EXTEND_DRAM_BYTES_PER_SEGMENT = 132.4
# What does bound the traversal kernel, from an ncu capture of two extend launches of the same
# 960x540 case (sections SpeedOfLight, ComputeWorkloadAnalysis, MemoryWorkloadAnalysis,
# WarpStateStats; command beside the figures in the extend-kernel profile summary): instruction issue.
EXTEND_MEASURED_BOUND = {"kind": "instruction issue (BVH and triangles stay in L2)", "issue_slots_busy": 0.750,
                         "alu_pipe": 0.588, "fma_pipe": 0.254, "dram_throughput": 0.010, "l2_throughput": 0.109,
                         "l2_hit_rate": 0.797, "threads_per_instruction": 18.9, "warps_active": 0.363,
                         "stalls_per_issue": {"wait": 1.95, "not_selected": 1.38, "long_scoreboard": 1.22},
                         "note": "mean of two launches of the 960x540, 4-spp case"}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=16)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--spp", type=int, default=16, help="samples per pixel per step")
    p.add_argument("--depth", type=int, default=12)
    p.add_argument("--width", type=int, default=1920)
    p.add_argument("--height", type=int, default=1080)
    p.add_argument("--instances", type=int, default=64)
    p.add_argument("--subdiv", type=int, default=5)
    p.add_argument("--tex", type=int, default=1024)
    p.add_argument("--cpu-seconds", type=float, default=15.0, help="budget of the CPU baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--out", default=None, help="also write the JSON line to this file")
    p.add_argument("--shade-order", default="auto", choices=["auto", "queue", "material"],
                   help="shade each bounce's hits in traversal order, sorted by shading class, or the "
                        "library's default (sorted except under Markov guiding)")
    p.add_argument("--no-guided", action="store_true", help="skip the guided-vs-plain equal-time measurement")
    p.add_argument("--guided-only", action="store_true", help="run only the guided-vs-plain measurement")
    p.add_argument("--guided-width", type=int, default=1920)
    p.add_argument("--guided-height", type=int, default=1080)
    p.add_argument("--guided-ref-spp", type=int, default=65536, help="spp of the plain reference image")
    p.add_argument("--guided-depth", type=int, default=8)
    p.add_argument("--guided-frac", type=float, default=0.5)
    p.add_argument("--guided-train-spp", type=int, default=32)
    p.add_argument("--guided-steps-per-wave", type=int, default=25)
    p.add_argument("--no-batched", action="store_true", help="skip the batched-serving measurement")
    p.add_argument("--no-restir", action="store_true", help="skip the ReSTIR GI frame-loop measurement")
    p.add_argument("--restir-only", action="store_true", help="run only the ReSTIR GI frame-loop measurement")
    p.add_argument("--restir-frames", type=int, default=120)
    p.add_argument("--restir-ref-spp", type=int, default=4096,
                   help="spp of the plain reference of each compared ReSTIR frame (two independent halves)")
    p.add_argument("--restir-compare", default="29,59,89,119",
                   help="orbit frames whose ReSTIR output is compared with plain path tracing at equal time")
    p.add_argument("--batched-only", action="store_true", help="run only the batched-serving measurement")
    p.add_argument("--batched-requests", type=int, default=64)
    p.add_argument("--batched-scenes", type=int, default=8, help="distinct scenes shared by the requests")
    return p.parse_args()


def workload_config(a):
    return {
        "workload": f"icosphere field {a.instances}x{20 * 4 ** a.subdiv} tris, {a.width}x{a.height}, "
                    f"{a.spp} spp/step, depth {a.depth}, Medium, plain (no guiding, ReSTIR off)",
        "triangles": a.instances * 20 * 4 ** a.subdiv,
        "resolution": [a.width, a.height],
        "spp_per_step": a.spp,
        "max_depth": a.depth,
        "textures": f"3 x 16 layers {a.tex}^2 RGBA8 value noise",
        "cache": "inputs larger than L2: path state + textures + triangles exceed 126 MB",
        "shade_order": a.shade_order,
    }


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons while the timed region runs."""

    def __init__(self, index):
        self.index, self.samples, self.stop_flag = index, [], threading.Event()
        self.t = threading.Thread(target=self.run, daemon=True)

    def run(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        while not self.stop_flag.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                vals = [v.strip() for v in out.stdout.strip().split(",")]
                if len(vals) == 6:
                    self.samples.append(vals)
            except Exception:
                pass
            self.stop_flag.wait(0.2)

    def __enter__(self):
        self.t.start()
        return self

    def __exit__(self, *exc):
        self.stop_flag.set()
        self.t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = sorted(float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit())
        mx = max((float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[2 + i].strip() == "Active"})
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(self.samples)}


def build_scene(a, packer=None):
    from lambent_b200 import scenes
    return scenes.icosphere_field(a.width, a.height, instances=a.instances, subdiv=a.subdiv, tex_size=a.tex,
                                  packer=packer)


def oracle_scene(a):
    """The workload's scene with its material records and camera packed by the oracle's own
    restatements of Material::new and Camera::from_proj_view: the CPU legs load no product code."""
    from oracle import oracle_py as O
    return build_scene(a, packer=O.OraclePacker)


def cpu_reference(a, seconds, scene=None):
    """The reference path on the host cores: the CPU restatement of its shaders, a crop of the
    same frame (full-frame rays and seeds) sized to about `seconds` of work."""
    from oracle import oracle_py as O
    from lambent_b200 import _abi
    cores = os.cpu_count() or 1
    if scene is None:
        scene = oracle_scene(a)
    osc = O.OracleScene(scene)
    w = h = min(128, min(a.width, a.height)) // 32 * 32  # calibration crop
    x0, y0 = a.width // 2 - w // 2, a.height // 2 - h // 2
    spp = 2
    t0 = time.perf_counter()
    r = osc.render(scene.camera, a.width, a.height, samples=spp, max_depth=a.depth, restir=_abi.RESTIR_DISABLED,
                   crop=(x0, y0, w, h), threads=cores)
    dt = time.perf_counter() - t0
    # fill the time budget: the largest centre crop up to 1024^2, then as many samples as fit
    side = min(1024, min(a.width, a.height)) // 32 * 32
    per_px = dt / (w * h * spp)  # seconds per pixel-sample at the calibration size
    spp = int(max(1, min(64, round(seconds / max(per_px * side * side, 1e-9)))))
    x0, y0 = a.width // 2 - side // 2, a.height // 2 - side // 2
    t0 = time.perf_counter()
    r = osc.render(scene.camera, a.width, a.height, samples=spp, max_depth=a.depth, restir=_abi.RESTIR_DISABLED,
                   crop=(x0, y0, side, side), threads=cores)
    dt = time.perf_counter() - t0
    w = h = side
    mrays = r["segments"] / dt / 1e6
    return {"value": round(mrays, 3), "unit": "Mrays/s", "cores": cores, "kind": "port",
            "sample": f"centre crop {w}x{h} of the {a.width}x{a.height} frame, {spp} spp, depth {a.depth}, "
                      f"{r['segments']} segments in {dt:.2f} s",
            "samples_per_s": round(r["samples"] / dt, 1)}


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    scene = oracle_scene(a)
    base = cpu_reference(a, a.cpu_seconds, scene)
    steps_ms = []
    # each step is a bounded sample of the workload; value = Mrays/s over the steps
    from oracle import oracle_py as O
    from lambent_b200 import _abi
    osc = O.OracleScene(scene)
    cores = os.cpu_count() or 1
    side = min(256, a.width, a.height)  # large enough that the host threads' start-up does not dominate a step
    segs = 0
    tot = 0.0
    for k in range(a.warmup + a.steps):
        x0, y0 = a.width // 2 - side // 2, a.height // 2 - side // 2
        t0 = time.perf_counter()
        r = osc.render(scene.camera, a.width, a.height, samples=2, max_depth=a.depth, restir=_abi.RESTIR_DISABLED,
                       crop=(x0, y0, side, side), threads=cores, seed_offset=k)
        dt = time.perf_counter() - t0
        if k >= a.warmup:
            segs += r["segments"]
            tot += dt
            steps_ms.append(dt * 1e3)
    v = segs / tot / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "Mrays/s", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(sum(steps_ms) / len(steps_ms), 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(a),
            "cpu_baseline": {"value": round(v, 3), "unit": "Mrays/s", "cores": cores, "kind": "port",
                             "sample": f"per step: centre crop {side}x{side}, 2 spp, depth {a.depth} "
                                       "(the reference's wgpu shaders need a graphics stack, unavailable on this box; "
                                       "this is the CPU restatement of those shaders)"},
            "e2e": {"value": round(v, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "calibration": base}
    emit(line, a)


def ordered(pipe, a):
    """Applies --shade-order to a new pipeline."""
    import lambent_b200 as lb
    from lambent_b200 import _abi
    pipe.set_shade_order({"auto": _abi.SHADE_ORDER_AUTO, "queue": _abi.SHADE_ORDER_QUEUE,
                          "material": _abi.SHADE_ORDER_MATERIAL}[a.shade_order])
    return pipe


def emit(line, a):
    s = json.dumps(line)
    print(s, flush=True)
    if a.out:
        with open(a.out, "w") as f:
            f.write(s + "\n")


def guided_equal_time(a, dev):
    """Equal-time relMSE of the learned-guided renderer against the plain one.

    Scene: the procedural Cornell box with a single 0.2 x 0.2 emitter above an occluding plate
    (indirect-heavy lighting), Medium shader, ReSTIR off.  The plain form renders 1024 spp in time T.
    The guided form (a fresh network, trained online on its first `train_spp` samples) renders
    32-spp chunks; its running mean is compared with the reference after each chunk, outside the
    timed region.  Each pipeline's first call, which allocates its wave buffers, is not timed.  relMSE = mean((x - ref)^2 / (ref^2 + 1e-2)) against a plain reference of
    `ref_spp` samples; the reference's own noise, estimated from its two halves, is subtracted.
    """
    import torch
    import lambent_b200 as lb
    from lambent_b200 import _abi, scenes
    W, H = a.guided_width, a.guided_height
    s = scenes.occluded_cornell(W, H)
    gs = lb.GpuScene(s)
    bufs = lb.DataBuffers(W, H, 1, 0)
    col = torch.zeros((H, W, 4), dtype=torch.float32, device=dev)
    tg = lb.targets_from(col)
    stream = torch.cuda.current_stream()

    def pipe(samples, mode=_abi.GUIDE_NONE, guide=None):
        p = ordered(lb.RayTracer(lb.path_tracing.Medium).create_pipeline(*s.layout_counts(), lb.PathTracerOpts(
            samples=samples, restir_temporal=_abi.RESTIR_DISABLED, max_depth=a.guided_depth, guide_mode=mode)), a)
        if guide is not None:
            p.set_guide(guide)
        return p

    def timed(p, seed):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        p.render(gs, bufs, s.camera, tg, seed, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3

    # reference: two independent halves
    pr = pipe(1024)
    halves = []
    t_ref = time.perf_counter()
    for h in range(2):
        acc = torch.zeros((H, W, 3), dtype=torch.float64, device=dev)
        n = max(1, a.guided_ref_spp // 2048)
        for k in range(n):
            pr.render(gs, bufs, s.camera, tg, 1_000_000 + (h * n + k) * 1024, stream)
            acc += col[..., :3].double()
        halves.append(acc / n)
    torch.cuda.synchronize()
    t_ref = time.perf_counter() - t_ref
    ref = (halves[0] + halves[1]) / 2
    den = ref ** 2 + 1e-2
    ref_noise = float((((halves[0] - halves[1]) ** 2) / den).mean()) / 4.0

    def relmse(img):
        return float((((img.double() - ref) ** 2) / den).mean()) - ref_noise

    # plain: 1024 spp in one call (after a warm-up call)
    p1 = pipe(1024)
    timed(p1, 5)
    T = min(timed(p1, 77 + 8191 * r) for r in range(2))
    e_plain = relmse(col[..., :3])
    segs_plain = p1.stats().ray_segments
    # guided: fresh network, 32-spp chunks until 1024 spp or 1.1 T.  As for plain, the pipeline's
    # first call (which allocates its wave buffers) is made outside the timed region, here with a
    # throwaway network; the fresh one is attached afterwards and trains inside the timed region.
    def guide_opts(seed):
        return lb.GuideOptions(train_spp=a.guided_train_spp, steps_per_wave=a.guided_steps_per_wave,
                               guide_fraction=a.guided_frac, learning_rate=5e-3, seed=seed)
    g_warm = lb.Guide(guide_opts(2))
    pg = pipe(32, _abi.GUIDE_LEARNED, g_warm)
    pg.render(gs, bufs, s.camera, tg, 31337, stream)
    torch.cuda.synchronize()
    g = lb.Guide(guide_opts(1))
    pg.set_guide(g)
    acc = torch.zeros((H, W, 3), dtype=torch.float64, device=dev)
    t, curve, k = 0.0, [], 0
    while k < 32 and (t < 1.1 * T or k < 2):
        t += timed(pg, 424242 + 32 * k)
        acc += col[..., :3].double()
        k += 1
        curve.append([32 * k, round(t, 5), relmse(acc / k)])
    assert pg.stats().error_flags == 0, "guided render reported an error"

    def time_to(target):
        prev = None
        for spp, tt, e in curve:
            if e <= target:
                if prev is None:
                    return tt
                (t0, e0) = prev
                # interpolate in log relMSE (relMSE ~ 1/time)
                import math
                f = (math.log(e0) - math.log(target)) / max(1e-12, math.log(e0) - math.log(e))
                return t0 + f * (tt - t0)
            prev = (tt, e)
        return None

    def at_time(T_):
        import math
        prev = None
        for spp, tt, e in curve:
            if tt >= T_:
                if prev is None:
                    return e
                t0, e0 = prev
                f = (T_ - t0) / max(1e-12, tt - t0)
                return math.exp(math.log(e0) + f * (math.log(e) - math.log(e0)))
            prev = (tt, e)
        return None

    t_hit = time_to(e_plain)
    e_eq = at_time(T)
    steps, trained = g.progress()
    return {
        "config": {"workload": f"occluded-light Cornell box (0.2x0.2 emitter above a plate), {W}x{H}, depth "
                               f"{a.guided_depth}, Medium, ReSTIR off",
                   "plain_spp": 1024, "reference_spp": 2 * max(1, a.guided_ref_spp // 2048) * 1024,
                   "network": "4 x 64 MLP, BF16 tcgen05, 8 vMF lobes, one-sample MIS with the cosine lobe at diffuse "
                              "vertices",
                   "guide_fraction": a.guided_frac, "train_spp": a.guided_train_spp,
                   "adam_steps": steps},
        "plain": {"time_s": round(T, 5), "relmse": round(e_plain, 6), "mrays_per_s": round(segs_plain / T / 1e6, 1)},
        "time_to_plain_quality_ratio": None if t_hit is None else round(t_hit / T, 4),
        "relmse_ratio_at_equal_time": None if e_eq is None else round(e_eq / e_plain, 4),
        "ref_noise_relmse": round(ref_noise, 7), "reference_seconds": round(t_ref, 2),
        "guided_curve": [[spp, tt, round(e, 6)] for spp, tt, e in curve],
        "target": "time_to_plain_quality_ratio <= 0.5 (relMSE of 1024-spp plain reached in half its time)",
    }


def restir_frames(a, dev):
    """ReSTIR GI frame loop: the Cornell box at 1920x1080, a 120-frame camera orbit at 1 spp per frame,
    per-pixel reservoirs, Markov-chain guiding, then temporal resampling, spatial resampling (5
    samples in a 61-pixel window) and the end-of-frame advance with M capped at 20, as the reference
    example drives them.  CUDA events around each pass give the split; 5 untimed frames first."""
    import math
    import torch
    import lambent_b200 as lb
    from lambent_b200 import _abi, scenes
    W, H = 1920, 1080
    s = scenes.cornell_box(W, H)
    gs = lb.GpuScene(s)
    world = 1_500_000
    bufs = lb.DataBuffers(W, H, world, _abi.BUFFER_ALL)
    pipe = ordered(lb.RayTracer(lb.path_tracing.Medium).create_pipeline(*s.layout_counts(), lb.PathTracerOpts(
        samples=1, restir_temporal=_abi.RESTIR_PER_PIXEL, max_depth=8, guide_mode=_abi.GUIDE_MARKOV)), a)
    col = torch.zeros((H, W, 4), dtype=torch.float32, device=dev)
    tg = lb.targets_from(col)
    stream = torch.cuda.current_stream()
    cams = []
    for f in range(a.restir_frames):
        th = math.radians(12.0) * math.sin(2.0 * math.pi * f / a.restir_frames)
        cams.append(scenes.make_camera((3.4 * math.sin(th), 1.0, 3.4 * math.cos(th)), (0.0, 1.0, 0.0), 40.0, W / H))
    adv = lb.AdvanceOptions(20)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    split = [0.0, 0.0, 0.0, 0.0]

    def frame(f, timed):
        if timed:
            ev[0].record(stream)
        pipe.render(gs, bufs, cams[f % len(cams)], tg, f, stream)
        if timed:
            ev[1].record(stream)
        bufs.temporal_resampling(f, stream)
        if timed:
            ev[2].record(stream)
        bufs.spatial_resampling(tg, 5, 61, f, stream)
        if timed:
            ev[3].record(stream)
        bufs.advance_frame(_abi.BUFFER_ALL, adv, stream)
        if timed:
            ev[4].record(stream)
            torch.cuda.synchronize()
            for k in range(4):
                split[k] += ev[k].elapsed_time(ev[k + 1])

    for f in range(5):
        frame(f, False)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for f in range(a.restir_frames):
        frame(f, False)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    pipe.set_profiling(True)  # segment count of the split frames
    pipe.profile_reset()
    for f in range(8):  # the split, from separately timed frames (events synchronise each frame)
        frame(f, True)
    segs_per_frame = pipe.profile().ray_segments / 8
    pipe.set_profiling(False)
    assert pipe.stats().error_flags == 0, "ReSTIR frame loop reported an error"
    n = a.restir_frames
    equal_time = restir_equal_time(a, dev, s, gs, pipe, col, tg, cams, ms / n)
    return {"config": {"workload": f"Cornell box (36 tris), {W}x{H}, {n}-frame orbit, 1 spp/frame, depth 8, "
                                   "Medium, per-pixel reservoirs, Markov chains (1.5M world cells), temporal + "
                                   "spatial (5 samples, 61-px window), M cap 20", "shade_order": a.shade_order},
            "equal_time": equal_time,
            "frames": n, "ms_per_frame": round(ms / n, 3), "frames_per_s": round(n / (ms / 1e3), 2),
            "render_mrays_per_s": round(segs_per_frame / (split[0] / 8 / 1e3) / 1e6, 1),
            "split_ms_per_frame": {"render": round(split[0] / 8, 3), "temporal": round(split[1] / 8, 3),
                                   "spatial": round(split[2] / 8, 3), "advance": round(split[3] / 8, 3)}}


def restir_equal_time(a, dev, s, gs, pipe, col, tg, cams, frame_ms):
    """Per-frame error of the ReSTIR GI loop against plain path tracing given the same time per frame.

    The orbit loop is replayed from fresh buffers; at each compared frame its output (the spatial
    pass's image) is kept.  Each kept frame's camera then gets a plain reference of `restir_ref_spp`
    samples in two independent halves (its own noise, relMSE(A, B) / 4, is subtracted) and a plain
    render of as many samples as the plain path traces in one ReSTIR frame's time.  relMSE =
    mean((x - ref)^2 / (ref^2 + 1e-2)) over pixels and colour channels."""
    import torch
    import lambent_b200 as lb
    from lambent_b200 import _abi
    W, H = s.width, s.height
    stream = torch.cuda.current_stream()
    compare = [int(x) for x in a.restir_compare.split(",") if x.strip() and int(x) < len(cams)]
    fresh = lb.DataBuffers(W, H, 1_500_000, _abi.BUFFER_ALL)
    kept = {}
    adv = lb.AdvanceOptions(20)
    for f in range(len(cams)):
        pipe.render(gs, fresh, cams[f], tg, f, stream)
        fresh.temporal_resampling(f, stream)
        fresh.spatial_resampling(tg, 5, 61, f, stream)
        fresh.advance_frame(_abi.BUFFER_ALL, adv, stream)
        if f in compare:
            kept[f] = col[..., :3].double().clone()
    del fresh
    plain_bufs = lb.DataBuffers(W, H, 1, 0)

    def plain_pipe(spp):
        return ordered(lb.RayTracer(lb.path_tracing.Medium).create_pipeline(*s.layout_counts(), lb.PathTracerOpts(
            samples=spp, restir_temporal=_abi.RESTIR_DISABLED, max_depth=8, guide_mode=_abi.GUIDE_NONE)), a)

    # plain time per sample at this resolution (after a warm-up call)
    p16 = plain_pipe(16)
    p16.render(gs, plain_bufs, cams[0], tg, 1, stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(4):
        p16.render(gs, plain_bufs, cams[0], tg, 2 + k, stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_per_spp = e0.elapsed_time(e1) / 64.0
    spp_eq = max(1, int(round(frame_ms / ms_per_spp)))
    p_eq = plain_pipe(spp_eq)
    chunk = min(1024, max(2, a.restir_ref_spp // 2))
    p_ref = plain_pipe(chunk)
    rows = []
    for f in compare:
        halves = []
        for h in range(2):
            acc = torch.zeros((H, W, 3), dtype=torch.float64, device=dev)
            reps = max(1, a.restir_ref_spp // (2 * chunk))
            for k in range(reps):
                p_ref.render(gs, plain_bufs, cams[f], tg, 5_000_000 + 100_000 * f + (h * reps + k) * chunk, stream)
                acc += col[..., :3].double()
            halves.append(acc / reps)
        ref = (halves[0] + halves[1]) / 2
        den = ref ** 2 + 1e-2
        noise = float((((halves[0] - halves[1]) ** 2) / den).mean()) / 4.0
        p_eq.render(gs, plain_bufs, cams[f], tg, 9_000_000 + f, stream)
        plain = col[..., :3].double()
        e_plain = float((((plain - ref) ** 2) / den).mean()) - noise
        e_restir = float((((kept[f] - ref) ** 2) / den).mean()) - noise
        # relMSE is a mean of squares: a few firefly pixels can dominate it, so the share of pixels whose
        # squared relative error exceeds 100 (error > 10x the reference) is reported beside it
        # (and the part of the relMSE sum that those pixels carry)
        # and the median pixel's squared relative error, which the few fireflies do not move
        def fireflies(img):
            sq = ((img - ref) ** 2) / den
            hot = sq.max(-1)[0] > 100.0
            return (float(hot.double().mean()), float(sq[hot].sum() / sq.sum().clamp_min(1e-30)),
                    float(sq.mean(-1).median()))
        fire_r, carried_r, med_r = fireflies(kept[f])
        fire_p, carried_p, med_p = fireflies(plain)
        rows.append({"frame": f, "restir_relmse": round(e_restir, 6), "plain_relmse": round(e_plain, 6),
                     "ratio": round(e_restir / e_plain, 4) if e_plain > 0 else None,
                     "ref_noise_relmse": round(noise, 7),
                     "firefly_pixel_share": {"restir": round(fire_r, 7), "plain": round(fire_p, 7)},
                     "firefly_relmse_share": {"restir": round(carried_r, 4), "plain": round(carried_p, 4)},
                     "median_pixel_relse": {"restir": round(med_r, 6), "plain": round(med_p, 6)}})
    torch.cuda.synchronize()
    ratios = sorted(r["ratio"] for r in rows if r["ratio"] is not None)
    return {"plain_spp_at_equal_time": spp_eq, "plain_ms_per_spp": round(ms_per_spp, 4),
            "median_ratio": ratios[len(ratios) // 2] if ratios else None,
            "restir_ms_per_frame": round(frame_ms, 3), "reference_spp": 2 * max(1, a.restir_ref_spp // (2 * chunk)) * chunk,
            "frames": rows,
            "note": "relMSE of the ReSTIR GI + Markov output of each frame and of a plain render of spp_at_equal_time "
                    "samples (the plain path's samples in one ReSTIR frame's time), both against a plain reference of "
                    "the same camera; ratio < 1 means ReSTIR wins at equal time"}


def batched_serving(a, dev):
    """Batched serving-style render: independent requests in one lam_batch_render, replayed as a
    CUDA graph with the autotuner's queue and launch sizes.

    Requests: resolutions uniform over {256^2, 512^2, 768x432, 1024^2}, spp uniform over {4, 16, 64},
    scenes from the Cornell-box generator filled with subdivided boxes up to 10k-500k triangles
    (log-uniform; `batched_scenes` distinct scenes shared by the requests), Medium, depth 8, seeded.
    Reports aggregate samples/s over the batch, per-request latency from the batch start to the
    request's completion (p50 / p99), and the same requests rendered one lam_render at a time.
    """
    import math
    import numpy as np
    import torch
    import lambent_b200 as lb
    from lambent_b200 import _abi, scenes
    rng = np.random.default_rng(2024)
    tri_counts = [int(round(math.exp(rng.uniform(math.log(10_000), math.log(500_000)))))
                  for _ in range(a.batched_scenes)]
    t0 = time.perf_counter()
    geo = [scenes.box_field(n, 256, 256, seed=k) for k, n in enumerate(tri_counts)]
    gsc = [lb.GpuScene(s) for s in geo]
    build_s = time.perf_counter() - t0
    sizes = [(256, 256), (512, 512), (768, 432), (1024, 1024)]
    reqs, keep = [], []
    for k in range(a.batched_requests):
        w, h = sizes[rng.integers(0, 4)]
        spp = int([4, 16, 64][rng.integers(0, 3)])
        sc = int(rng.integers(0, len(geo)))
        cam = scenes.make_camera((0.0, 1.0, 3.4), (0.0, 1.0, 0.0), 40.0, w / h)
        col = torch.zeros((h, w, 4), dtype=torch.float32, device=dev)
        keep.append(col)
        reqs.append((gsc[sc], cam, lb.targets_from(col), spp, 1000 * k))
    samples = sum(r[2].width * r[2].height * r[3] for r in reqs)
    opts = lb.PathTracerOpts(samples=1, restir_temporal=_abi.RESTIR_DISABLED, max_depth=8)
    pipe = lb.RayTracer(lb.path_tracing.Medium).create_pipeline(8, 8, 8, 8, opts)
    m = _batch_vs_sequential(lb, _abi, np, torch, pipe, reqs)
    T, lat, tuning, tune_s, segs = m["T"], m["lat"], m["tuning"], m["tune_s"], m["segs"]
    seq, seq_done, seq_b2b = m["seq"], m["seq_done"], m["seq_b2b"]
    # many small requests (128^2, 4 spp): where one render at a time cannot fill the GPU
    small = []
    for k in range(256):
        col = torch.zeros((128, 128, 4), dtype=torch.float32, device=dev)
        keep.append(col)
        small.append((gsc[k % len(gsc)], scenes.make_camera((0.0, 1.0, 3.4), (0.0, 1.0, 0.0), 40.0, 1.0),
                      lb.targets_from(col), 4, 7 * k))
    pipe_s = lb.RayTracer(lb.path_tracing.Medium).create_pipeline(8, 8, 8, 8, opts)
    ms_ = _batch_vs_sequential(lb, _abi, np, torch, pipe_s, small)
    small_samples = 256 * 128 * 128 * 4
    return {
        "config": {"workload": f"{len(reqs)} requests, resolutions {{256^2, 512^2, 768x432, 1024^2}}, spp {{4, 16, 64}}, "
                               f"{len(geo)} box-field Cornell scenes of {min(tri_counts)}-{max(tri_counts)} triangles "
                               "(log-uniform 10k-500k), Medium, depth 8",
                   "triangles": tri_counts, "samples": int(samples),
                   "tuning": {"wave_paths": tuning.wave_paths, "extend_blocks_per_sm": tuning.extend_blocks_per_sm,
                              "shade_blocks_per_sm": tuning.shade_blocks_per_sm, "cuda_graph": bool(tuning.use_graph)},
                   "autotune_s": round(tune_s, 2), "scene_build_s": round(build_s, 2)},
        "batch_s": round(T, 4), "samples_per_s": round(samples / T, 1), "mrays_per_s": round(segs / T / 1e6, 1),
        "latency_ms": {"p50": round(float(np.percentile(lat, 50)), 2), "p99": round(float(np.percentile(lat, 99)), 2),
                       "max": round(float(lat.max()), 2)},
        "sequential_s": round(seq, 4), "speedup_vs_sequential": round(seq / T, 3),
        "sequential_back_to_back_s": round(seq_b2b, 4),
        "sequential_latency_ms": {"p50": round(float(np.percentile(seq_done, 50)), 2),
                                  "p99": round(float(np.percentile(seq_done, 99)), 2)},
        "note": "sequential_s sums each request's own device time (no host gaps); sequential_back_to_back_s "
                "times the same lam_render calls issued back to back, host work included",
        "small_requests": {"workload": "256 requests of 128x128 at 4 spp on the same scenes, depth 8",
                           "samples": small_samples, "batch_s": round(ms_["T"], 4),
                           "samples_per_s": round(small_samples / ms_["T"], 1),
                           "sequential_s": round(ms_["seq"], 4),
                           "sequential_back_to_back_s": round(ms_["seq_b2b"], 4),
                           "speedup_vs_sequential_back_to_back": round(ms_["seq_b2b"] / ms_["T"], 3),
                           "latency_ms": {"p50": round(float(np.percentile(ms_["lat"], 50)), 2),
                                          "p99": round(float(np.percentile(ms_["lat"], 99)), 2)}},
    }


def _batch_vs_sequential(lb, _abi, np, torch, pipe, reqs):
    """The requests as one tuned lam_batch_render (CUDA graph; best of 3 timed replays) and as one
    lam_render each: per-request device time summed, and all of them issued back to back."""
    stream = torch.cuda.current_stream()
    t0 = time.perf_counter()
    tuning = pipe.batch_autotune(reqs, spp_divisor=4)
    tune_s = time.perf_counter() - t0
    pipe.batch_render(reqs, tuning, stream)  # graph capture + first replay
    torch.cuda.synchronize()
    times, lats = [], []
    for rep in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        pipe.batch_render(reqs, tuning, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
        lats.append(pipe.batch_latencies(len(reqs)))
    best = int(np.argmin(times))
    assert pipe.stats().error_flags == 0
    segs = pipe.stats().ray_segments
    singles, bufs_of = {}, {}
    seq, seq_done = 0.0, []
    for (g, cam, tg, spp, seed) in reqs:
        key = (spp, tg.width, tg.height)
        if key not in singles:
            singles[key] = lb.RayTracer(lb.path_tracing.Medium).create_pipeline(8, 8, 8, 8, lb.PathTracerOpts(
                samples=spp, restir_temporal=_abi.RESTIR_DISABLED, max_depth=8))
            bufs_of[key] = lb.DataBuffers(tg.width, tg.height, 1, 0)
        p1, bufs = singles[key], bufs_of[key]
        p1.render(g, bufs, cam, tg, seed, stream)  # warm-up (buffer allocation)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        p1.render(g, bufs, cam, tg, seed, stream)
        e1.record(stream)
        torch.cuda.synchronize()
        seq += e0.elapsed_time(e1) / 1e3
        seq_done.append(seq * 1e3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for (g, cam, tg, spp, seed) in reqs:
        key = (spp, tg.width, tg.height)
        singles[key].render(g, bufs_of[key], cam, tg, seed, stream)
    e1.record(stream)
    torch.cuda.synchronize()
    return {"T": times[best], "lat": np.asarray(lats[best]), "tuning": tuning, "tune_s": tune_s, "segs": segs,
            "seq": seq, "seq_done": seq_done, "seq_b2b": e0.elapsed_time(e1) / 1e3}


def run_ours(a):
    import numpy as np
    import torch
    import torch.distributed as dist
    import lambent_b200 as lb
    from lambent_b200 import _abi

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream()

    scene = build_scene(a)
    gscene = lb.GpuScene(scene)
    st = gscene.stats()
    tracer = lb.RayTracer(lb.path_tracing.Medium)
    opts = lb.PathTracerOpts(samples=a.spp, restir_temporal=lb.RestirTemporalMode.Disabled, max_depth=a.depth,
                             guide_mode=lb.GuideMode.NONE)
    pipe = ordered(tracer.create_pipeline(*scene.layout_counts(), opts), a)
    bufs = lb.DataBuffers(a.width, a.height, 1, 0)
    H, W = a.height, a.width
    color = torch.zeros((H, W, 4), dtype=torch.float32, device=dev)
    normal = torch.zeros_like(color)
    albedo = torch.zeros_like(color)
    tg = lb.targets_from(color, normal, albedo)
    from lambent_b200 import distributed as D

    # seeds: step k of this rank renders with D.rank_seed(0, rank, k), disjoint from every other rank
    for k in range(a.warmup):
        pipe.render(gscene, bufs, scene.camera, tg, D.rank_seed(0, rank, k), stream)
    torch.cuda.synchronize()
    pipe.set_profiling(True)
    pipe.profile_reset()

    def frame(seed):
        pipe.render(gscene, bufs, scene.camera, tg, seed, stream)
        return color

    def barrier():
        if world > 1:
            dist.barrier()

    barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clocks:
        start.record(stream)
        # sample sharding: the per-rank sum of the steps' frames, one all-reduce at the end
        D.render_sharded(frame, a.steps, first_step=a.warmup)
        end.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = start.elapsed_time(end)
    prof = pipe.profile()
    pipe.set_profiling(False)
    launches = pipe.stats().kernel_launches * a.steps
    segs = prof.ray_segments
    t = torch.tensor([ms, float(segs), float(prof.extend_ms), float(prof.shade_ms)], dtype=torch.float64, device=dev)
    if world > 1:
        tmax = t.clone()
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
        tsum = t.clone()
        dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
        ms_max, segs_total = tmax[0].item(), tsum[1].item()
    else:
        ms_max, segs_total = ms, float(segs)
    value = segs_total / (ms_max / 1e3) / 1e6

    # e2e through the public API with host buffers: render + colour D2H per step.  The step's input is
    # the 128-byte camera, a host record that lam_render passes by value to its launches.  Two target
    # sets: frame k's readback (on a copy stream) overlaps frame k+1's render, and a target is rendered
    # into again only after its previous readback has finished.
    colors = [color, torch.zeros_like(color)]
    tgs = [tg, lb.targets_from(colors[1], torch.zeros_like(color), torch.zeros_like(color))]
    host_imgs = [torch.empty((H, W, 4), dtype=torch.float32).pin_memory() for _ in range(2)]
    copy_stream = torch.cuda.Stream(device=dev)
    rendered = [torch.cuda.Event() for _ in range(2)]
    copied = [torch.cuda.Event() for _ in range(2)]
    pipe.profile_reset()
    pipe.set_profiling(True)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for k in range(a.steps):
        b = k % 2
        if k >= 2:
            stream.wait_event(copied[b])
        pipe.render(gscene, bufs, scene.camera, tgs[b], D.rank_seed(0, rank, a.warmup + a.steps + k), stream)
        rendered[b].record(stream)
        copy_stream.wait_event(rendered[b])
        with torch.cuda.stream(copy_stream):
            host_imgs[b].copy_(colors[b], non_blocking=True)
        copied[b].record(copy_stream)
    for b in range(min(2, a.steps)):
        stream.wait_event(copied[b])
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = e0.elapsed_time(e1)
    e2e_prof = pipe.profile()
    pipe.set_profiling(False)
    tt = torch.tensor([e2e_ms, float(e2e_prof.ray_segments)], dtype=torch.float64, device=dev)
    if world > 1:
        m = tt.clone()
        dist.all_reduce(m, op=dist.ReduceOp.MAX)
        s_ = tt.clone()
        dist.all_reduce(s_, op=dist.ReduceOp.SUM)
        e2e_ms_max, e2e_segs = m[0].item(), s_[1].item()
    else:
        e2e_ms_max, e2e_segs = e2e_ms, float(e2e_prof.ray_segments)
    e2e_value = e2e_segs / (e2e_ms_max / 1e3) / 1e6

    if rank == 0:
        hbm, peak_kind = peaks()
        ext_s = prof.extend_ms / 1e3
        achieved = segs * SEG_BYTES_EXTEND / ext_s / 1e9 if ext_s > 0 else 0.0
        shade_s = prof.shade_ms / 1e3
        shade_gbs = segs * (SEG_BYTES_TOTAL - SEG_BYTES_EXTEND) / shade_s / 1e9 if shade_s > 0 else 0.0
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(ms_max / a.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(a),
            "samples_per_s": round(W * H * a.spp * a.steps * world / (ms_max / 1e3), 1),
            "roofline": {"bound": "hbm", "kernel": "extend_kernel (BVH8 traversal)",
                         "achieved": round(achieved, 2), "peak": hbm, "unit": "GB/s",
                         "frac": round(achieved / hbm, 5), "peak_kind": f"{peak_kind} hbm_gbs",
                         "bytes_per_segment": SEG_BYTES_EXTEND,
                         "traffic": round(EXTEND_DRAM_BYTES_PER_SEGMENT * segs / max(1, prof.extend_launches)),
                         "traffic_note": "DRAM bytes per extend launch: ncu bytes/segment of a 960x540 capture x this "
                                         "run's segments per launch (BVH and triangle fetches that miss L2)",
                         "extend_ms": round(prof.extend_ms, 3), "shade_ms": round(prof.shade_ms, 3),
                         "generate_ms": round(prof.generate_ms, 3), "accumulate_ms": round(prof.accumulate_ms, 3),
                         "shade_gbs": round(shade_gbs, 2),
                         "measured_bound": EXTEND_MEASURED_BOUND,
                         # the whole wavefront against one GPU's HBM: compulsory bytes per segment
                         # (extend 48 + shade 232) at the achieved segment rate per GPU
                         "pipeline": {"bytes_per_segment": SEG_BYTES_TOTAL,
                                      "achieved": round(value / world * 1e6 * SEG_BYTES_TOTAL / 1e9, 2),
                                      "frac": round(value / world * 1e6 * SEG_BYTES_TOTAL / 1e9 / hbm, 5)}},
            "e2e": {"value": round(e2e_value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 128,
                    "d2h_bytes_per_step": H * W * 16,
                    "note": "per step: the 128-B host camera record passed by value into lam_render's launches, "
                            "and the rgba32f colour image read back to pinned host memory"},
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
            "scene": {"triangles": st.triangle_count, "blas_nodes": st.blas_node_count,
                      "tlas_nodes": st.tlas_node_count, "device_bytes": st.device_bytes,
                      "build_s": round(st.build_seconds, 3)},
        }
        if not a.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_reference(a, a.cpu_seconds)
        if world == 1 and not (a.no_guided and a.no_batched and a.no_restir):
            del gscene, pipe, bufs
            torch.cuda.empty_cache()
        if not a.no_guided and world == 1:
            line["guided"] = guided_equal_time(a, dev)
        if not a.no_batched and world == 1:
            line["batched"] = batched_serving(a, dev)
        if not a.no_restir and world == 1:
            line["restir"] = restir_frames(a, dev)
        emit(line, a)
    if world > 1:
        dist.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.batched_only:
        import torch
        torch.cuda.set_device(0)
        emit({"metric": "batched serving samples/s", "batched": batched_serving(a, torch.device("cuda", 0))}, a)
    elif a.restir_only:
        import torch
        torch.cuda.set_device(0)
        emit({"metric": "ReSTIR GI frame loop", "restir": restir_frames(a, torch.device("cuda", 0))}, a)
    elif a.guided_only:
        import torch
        torch.cuda.set_device(0)
        emit({"metric": "equal-time relMSE guided vs plain", "guided": guided_equal_time(a, torch.device("cuda", 0))}, a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
