"""Benchmark: Msamples/s of the B200 wavefront integrator on the mesh + glossy workload.

One step = one full frame of the workload (1920x1080, 64 spp, max depth 12 on a
1,310,720-triangle displaced icosphere + ground quad, rough dielectric and GGX
metal, 1024x512 environment with a sun lobe, f/2.8 thin lens). Synthetic,
seeded scene data (no assets). `value` is device-timed with the scene resident
on the GPU; `e2e` is the same metric through the C ABI call a host makes
(luz_gpu_render with a host film, device->host copy included).

Multi-GPU (torchrun, one process per GPU): every rank renders the full frame
with its own sample range (luz_b200.shard: rank r renders samples
[r * spp, (r + 1) * spp) of a world * spp frame), and one NCCL all-reduce per
step sums the films, normalised to the frame's mean: weak scaling over samples.

--impl reference times the Luz reference renderer (built from its own sources
into oracle/_ref/libluzref_fast.so) on the host cores on a bounded sample of
the same workload (the frame at 4 spp per step, Renderer::render).

Other workloads: --workload cornell300 (config 0: Cornell box 300x300, 50 spp,
depth 8), --workload instancing (config 2: 1e5 instances in an HG medium,
1280x720, 32 spp, depth 16) print the same line for those scenes.
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

METRIC = "Msamples/s"
UNIT = "Msamples/s"
REFERENCE_DIR = os.path.join(ROOT, "oracle")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mesh_glossy")
    ap.add_argument("--spp", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cache-min-rough", type=float, default=None,
                    help="cache workloads: LuzCacheParams.min_roughness (default per workload)")
    ap.add_argument("--cache-batch", type=int, default=16384, help="cache workloads: training rows per step")
    ap.add_argument("--cache-train-every", type=int, default=32, help="cache workloads: one training path in this many")
    ap.add_argument("--cache-warm-steps", type=int, default=0,
                    help="cache workloads: LuzCacheParams.warm_steps (0: the library's 64)")
    ap.add_argument("--cache-prefix", type=int, default=1,
                    help="cache workloads: first bounce whose vertex queries the cache")
    ap.add_argument("--cache-wave", type=int, default=0,
                    help="cache workloads: paths per wave of the cached render (0: its default, 4 Mi)")
    return ap.parse_args()


WORKLOAD_ALIASES = {"cornell300": "cornell", "instancing": "instancing_volumes"}


def workload(name, spp=None):
    from luz_b200 import scenes
    w = scenes.WORKLOADS[WORKLOAD_ALIASES.get(name, name)]()
    if spp:
        w.spp = spp
    return w


def config_of(w, n_gpus):
    return {"workload": f"{w.name} {w.width}x{w.height} {w.spp}spp depth{w.max_bounces}",
            "width": w.width, "height": w.height, "spp": w.spp, "max_bounces": w.max_bounces,
            "triangles": int(sum(m["positions"].shape[0] for m in w.scene.meshes)),
            "shards": f"sample ranges x{n_gpus}", "l2": "path state and scene > 126 MB L2; L2 flushed between steps",
            "seed": w.seed}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ["clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.hw_slowdown",
              "clocks_event_reasons.hw_thermal_slowdown", "clocks_event_reasons.sw_thermal_slowdown",
              "clocks_event_reasons.sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + ",".join(self.FIELDS),
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


PROFILE_SUMMARY = os.path.join(ROOT, "profiles", "k_extend_counters_mesh_glossy.md")


def profile_counters():
    """Per-extension-ray ncu figures of k_extend from the committed summary: DRAM bytes,
    L2 bytes (lts__t_bytes), L2 throughput as a fraction of its peak
    (lts__throughput.avg.pct_of_peak_sustained_elapsed / 100) and active lanes per
    warp instruction (smsp__thread_inst_executed_per_inst_executed)."""
    import re
    out = {}
    if os.path.exists(PROFILE_SUMMARY):
        txt = open(PROFILE_SUMMARY).read()
        for key, pat in (("dram", r"DRAM bytes per extension ray: ([0-9.]+)"),
                         ("l2", r"L2 bytes per extension ray: ([0-9.]+)"),
                         ("l2_frac", r"L2 throughput, fraction of peak: ([0-9.]+)"),
                         ("lanes", r"active lanes per warp instruction: ([0-9.]+)")):
            m = re.search(pat, txt)
            if m:
                out[key] = float(m.group(1))
    return out


def cpu_baseline(w, threads):
    """The reference renderer (oracle/_ref/libluzref_fast.so) on a bounded sample: the frame at 1 spp."""
    sys.path.insert(0, REFERENCE_DIR)
    from luz_b200 import native
    import oracle as O
    if not O.reference_available(fast=True):
        return None, "reference library oracle/_ref/libluzref_fast.so not built"
    ro = O.RefOracle(fast=True)
    rs = ro.scene(w.scene.build())
    p = native.params(w.width, w.height, 1, w.max_bounces, w.seed)
    _, ms, ns = rs.render(p, threads)
    spp = 1
    if ms < 8000.0:   # grow to about 10 s of CPU work
        spp = max(1, min(w.spp, int(10000.0 / max(ms, 1.0))))
        if spp > 1:
            p = native.params(w.width, w.height, spp, w.max_bounces, w.seed)
            _, ms, ns = rs.render(p, threads)
    rs.close()
    return {"value": ns / ms / 1e3, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"{w.width}x{w.height} at {spp} spp ({int(ns)} samples), render_ms {ms:.0f}"}, None


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = workload(args.workload, args.spp)
    threads = os.cpu_count() or 1
    sys.path.insert(0, REFERENCE_DIR)
    import oracle as O
    from luz_b200 import native
    if not O.reference_available(fast=True):
        print(json.dumps({"impl": "reference", "unavailable": "reference library oracle/_ref/libluzref_fast.so not built"}))
        return
    ro = O.RefOracle(fast=True)
    rs = ro.scene(w.scene.build())
    spp_step = min(w.spp, 4)
    p = native.params(w.width, w.height, spp_step, w.max_bounces, w.seed)
    for _ in range(args.warmup):
        rs.render(p, threads)
    times, samples = [], 0.0
    for _ in range(args.steps):
        _, ms, ns = rs.render(p, threads)
        times.append(ms)
        samples = ns
    ms = float(np.mean(times))
    value = samples / ms / 1e3
    cfg = config_of(w, 1)
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded scene generator)", "config": cfg,
           "impl": "reference",
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                            "sample": f"{w.width}x{w.height} at {spp_step} spp per step ({int(samples)} samples)"},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_ours(args):
    import torch
    from luz_b200 import native
    from luz_b200.desc import RENDER_COUNT, RENDER_PROFILE

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    w = workload(args.workload, args.spp)
    built = w.scene.build()
    g = native.GpuScene(built, device=local)
    npix = w.width * w.height
    film = torch.zeros(npix * 3, dtype=torch.float32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed, 0, rank * w.spp)
    from luz_b200.shard import render_sharded

    reduce_ev = []

    def all_reduce(t):   # the film exchange, timed with events on the launching stream
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        dist.all_reduce(t)
        a1.record(stream)
        reduce_ev.append((a0, a1))

    def step():
        if dist is None:
            return g.render_device(p, film.data_ptr(), stream.cuda_stream)
        out = {}

        def render_mean(offset, count):   # this rank's samples of the world * spp frame
            pr = native.params(w.width, w.height, count, w.max_bounces, w.seed, 0, offset)
            out["st"] = g.render_device(pr, film.data_ptr(), stream.cuda_stream)
            return film
        render_sharded(render_mean, w.spp * world, rank, world, all_reduce)
        return out["st"]

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    # A step's device time is the render's own CUDA events on the launching stream (recorded
    # before its first and after its last GPU operation: LuzRenderStats.render_ms) plus the
    # film all-reduce's events under torchrun (the two elementwise scalings of the 25 MB film
    # around it are left out). The events around the whole call (outer) also
    # hold the host's set-up before the first launch and its return after the last.
    times, outer, launches = [], [], 0
    clocks.start()
    for _ in range(args.steps):
        flush.zero_()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        reduce_ev.clear()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = step()
        e1.record(stream)
        torch.cuda.synchronize()
        launches += st.kernel_launches
        outer.append(e0.elapsed_time(e1))
        times.append(st.render_ms + sum(a0.elapsed_time(a1) for a0, a1 in reduce_ev))
    clk = clocks.stop()
    ms = float(np.mean(times))
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    samples_all = float(npix) * w.spp * world
    value = samples_all / ms / 1e3

    # end to end through the C ABI with a host film (device -> host copy in the timed region)
    e2e_ms = []
    host = torch.empty((w.height, w.width, 3), dtype=torch.float32, pin_memory=True).numpy()
    for i in range(max(1, min(args.steps, 3))):
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        host, _ = g.render(p, out=host)
        if dist is not None:
            ht = torch.from_numpy(host).cuda()
            dist.all_reduce(ht)
            host = (ht / world).cpu().numpy()
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2 = float(np.mean(e2e_ms))
    if dist is not None:
        t = torch.tensor([e2], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2 = float(t.item())

    # roofline of the dominant kernel (closest-hit traversal), from an instrumented extra frame
    pp = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed, 0, rank * w.spp)
    pp.flags = RENDER_PROFILE | RENDER_COUNT
    prof = g.render_device(pp, film.data_ptr(), stream.cuda_stream)
    pt = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed, 0, rank * w.spp)
    pt.flags = RENDER_PROFILE
    timed = g.render_device(pt, film.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    ext_rays = prof.extension_rays
    # algorithmic bytes of the closest-hit walk: 32 B per child box of every binary-node
    # visit the collapsed walk stands for (two per visit), 48 B per triangle test, 32 B
    # per top-level record, 32 B ray read + 20 B hit write per ray
    alg_bytes = 64.0 * prof.ext_bnodes + 48.0 * prof.ext_tris + 32.0 * prof.ext_top + 52.0 * ext_rays
    launch_ms = timed.extend_ms / max(1, timed.extend_launches)
    rays_per_launch = ext_rays / max(1, prof.extend_launches)
    bytes_per_launch = alg_bytes / max(1, prof.extend_launches)
    achieved = bytes_per_launch / (launch_ms * 1e-3) / 1e9 if launch_ms > 0 else None
    peak, peak_kind = measured_peak()
    pc = profile_counters()
    traffic = pc["dram"] * rays_per_launch if "dram" in pc else None
    l2_gbs = pc["l2"] * rays_per_launch / (launch_ms * 1e-3) / 1e9 if ("l2" in pc and launch_ms > 0) else None

    # the drop-in per frame as a host glue would run it: scene description, luz_gpu_scene_create
    # (host BVH build + upload), one render with a host film, destroy
    glue = None
    if rank == 0:
        t0 = time.perf_counter()
        b2 = w.scene.build()
        t1 = time.perf_counter()
        g2 = native.GpuScene(b2, device=local)
        t2 = time.perf_counter()
        _, st2 = g2.render(p)
        t3 = time.perf_counter()
        g2.close()
        t4 = time.perf_counter()
        glue = {"describe_ms": (t1 - t0) * 1e3, "scene_create_ms": (t2 - t1) * 1e3,
                "render_ms": (t3 - t2) * 1e3, "destroy_ms": (t4 - t3) * 1e3, "total_ms": (t4 - t0) * 1e3,
                "msamples_per_s": float(npix) * w.spp / ((t4 - t0) * 1e3) / 1e3,
                "what": "scene handle created and destroyed around one render (host wall clock)"}

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
               "config": config_of(w, world),
               "step_ms": [round(x, 2) for x in times],
               "step_ms_outer": [round(x, 2) for x in outer],
               "e2e": {"value": samples_all / e2 / 1e3, "unit": UNIT, "h2d_bytes_per_step": 32,
                       "d2h_bytes_per_step": npix * 3 * 4, "ms_per_step": [round(x, 2) for x in e2e_ms],
                       "host_film": "pinned"},
               "gpu_launches": int(launches),
               "clocks": clk,
               "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                            "kernel": "k_extend (closest-hit traversal)", "peak_kind": peak_kind,
                            "algorithmic_bytes_per_ray": alg_bytes / max(1.0, ext_rays),
                            "bytes_formula": "64 x binary node visits + 48 x triangle tests + 32 x top-level "
                                             "records + 52 per ray",
                            "rays_per_launch": rays_per_launch,
                            "launch_ms": launch_ms,
                            "traffic_source": "ncu dram bytes per extension ray x rays per launch "
                                              "(profiles/k_extend_counters_mesh_glossy.md)",
                            "l2_gbs": l2_gbs, "l2_frac": pc.get("l2_frac"),
                            "l2_source": "ncu lts__t_bytes per extension ray x rays per launch / live launch "
                                         "time; l2_frac = lts__throughput pct of peak (same summary)",
                            "simt_lanes": pc.get("lanes")},
               "stages_ms": {"extend": timed.extend_ms, "shade": timed.shade_ms, "shadow": timed.shadow_ms,
                             "total": timed.render_ms},
               "mrays_per_s": (timed.extension_rays + timed.shadow_rays) / timed.render_ms / 1e3 * world,
               "dropin_frame": glue}
        if world == 1 and not args.no_cpu_baseline:
            cb, why = cpu_baseline(w, os.cpu_count() or 1)
            out["cpu_baseline"] = cb if cb else {"value": None, "unavailable": why}
        print(json.dumps(out), flush=True)
    g.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_batch(args):
    """--workload batch48: 48 independent scenes (scenes.batch_workloads: 1e3-1e6 triangles,
    128^2-1024^2, 4-256 spp, depth 4-16) rendered one luz_gpu_render after another, then as
    one luz_gpu_batch_render call (multi-scene waves over one geometry arena, each wave a
    replayed CUDA graph, wave size autotuned on the first call). --workload batch48_small:
    the same mix at 64^2-256^2 and 1-16 spp, where a single render's fixed costs (launches,
    per-bounce tails) dominate. Host wall clock around the calls (host films, device->host
    copies included): an end-to-end figure."""
    from luz_b200 import native, scenes
    small = args.workload == "batch48_small"
    ws = scenes.batch_workloads(48, side_range=(64, 256), spp_range=(1, 16)) if small else scenes.batch_workloads(48)
    gs = [native.GpuScene(w.scene.build()) for w in ws]
    ps = [native.params(w.width, w.height, w.spp, w.max_bounces, w.seed) for w in ws]
    samples = float(sum(w.width * w.height * w.spp for w in ws))
    _, _, first = native.batch_render(gs, ps, report=True)      # autotunes the wave size
    for _ in range(max(1, args.warmup)):
        native.batch_render(gs, ps)
        for g, p in zip(gs, ps):
            g.render(p)
    t_seq, t_bat, dev_ms = [], [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        for g, p in zip(gs, ps):
            g.render(p)
        t_seq.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        _, _, rep = native.batch_render(gs, ps, report=True)
        t_bat.append(time.perf_counter() - t0)
        dev_ms.append(rep["render_ms"])
    tb, ts = statistics.median(t_bat), statistics.median(t_seq)
    out = {"metric": METRIC, "value": samples / tb / 1e6, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": tb * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
           "timing": "host wall clock around the C ABI calls (e2e, host films)",
           "config": {"workload": ("batch48_small: 48 scenes, 1e3-1e6 triangles, 64^2-256^2, 1-16 spp, depth 4-16"
                                   if small else
                                   "batch48: 48 scenes, 1e3-1e6 triangles, 128^2-1024^2, 4-256 spp, depth 4-16"),
                      "samples_per_step": samples,
                      "triangles": int(sum(g.info().mesh_triangles for g in gs))},
           "sequential": {"value": samples / ts / 1e6, "unit": UNIT, "ms_per_step": ts * 1e3},
           "batch_speedup": ts / tb,
           "batch_device_ms": float(np.median(dev_ms)),
           "autotuner": {"chosen_wave_paths": first["wave_paths"], "trials": first["trials"]},
           "waves": rep["waves"], "kernel_launches": rep["kernel_launches"]}
    print(json.dumps(out), flush=True)
    for g in gs:
        g.close()


def run_adjoint(args):
    """--workload adjoint_c3: albedo-texture gradient of the textured Cornell box (256x256,
    64 spp, depth 8, 32x32 back-wall texture): Madjoint paths/s = W*H*spp paths replayed per
    second of luz_gpu_adjoint_backward (both passes), device time from the call's CUDA events;
    beside it the same figure for the 64x64 roughness map of a Metal panel in the box and for
    the light-emission gradient (luz_gpu_adjoint_emission)."""
    from luz_b200 import native, scenes
    w = scenes.cornell_textured(256, 256, 64, 8)
    g = native.GpuScene(w.scene.build())
    p = native.params(w.width, w.height, w.spp, w.max_bounces, w.seed)
    tex = np.array(w.scene.textures[0])
    target = scenes.checker_texture()
    tg = native.GpuScene(scenes.cornell_textured(256, 256, 64, 8, texture=target).scene.build())
    goal, _ = tg.render(native.params(w.width, w.height, 1024, w.max_bounces, w.seed))
    for _ in range(max(1, args.warmup)):
        img, _ = g.adjoint_forward(p, 0, tex)
        g.adjoint_backward(p, 0, 2.0 * (img - goal) / img.size, tex.shape)
    fw, bw = [], []
    for _ in range(args.steps):
        img, sf = g.adjoint_forward(p, 0, tex)
        grad, sb = g.adjoint_backward(p, 0, 2.0 * (img - goal) / img.size, tex.shape)
        fw.append(sf.render_ms)
        bw.append(sb.render_ms)
    paths = float(w.width * w.height * w.spp)
    ms = float(np.mean(bw))
    # the other C3 parameters on the same box with a roughness-mapped Metal panel: the 64x64
    # roughness map (texture 1) and the light's emission, for the same kind of loss
    wr = scenes.cornell_rough_panel(256, 256, 64, 8)
    gr = native.GpuScene(wr.scene.build())
    pr = native.params(wr.width, wr.height, wr.spp, wr.max_bounces, wr.seed)
    rough = np.array(wr.scene.textures[1])
    img, _ = gr.render(pr)
    adj = (2.0 * (img - goal) / img.size).astype(np.float32)
    for _ in range(max(1, args.warmup)):
        gr.adjoint_backward(pr, 1, adj, rough.shape)
        gr.adjoint_emission(pr, adj)
    rw, ew = [], []
    for _ in range(args.steps):
        _, sr = gr.adjoint_backward(pr, 1, adj, rough.shape)
        _, se = gr.adjoint_emission(pr, adj)
        rw.append(sr.render_ms)
        ew.append(se.render_ms)
    out = {"metric": "Madjoint paths/s", "value": paths / ms / 1e3, "unit": "Mpaths/s", "n_gpus": 1,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
           "config": {"workload": "adjoint_c3: textured Cornell 256x256 64spp depth8, 32x32 albedo texture",
                      "loss": "mean squared error to the 1024-spp checker render"},
           "forward_ms": float(np.mean(fw)), "grad_norm": float(np.linalg.norm(grad)),
           "roughness_map": {"value": paths / float(np.mean(rw)) / 1e3, "unit": "Mpaths/s",
                             "ms": float(np.mean(rw)), "what": "64x64 Metal roughness map, both passes"},
           "emission": {"value": paths / float(np.mean(ew)) / 1e3, "unit": "Mpaths/s", "ms": float(np.mean(ew)),
                        "what": "every light's emitted radiance, one replay"}}
    print(json.dumps(out), flush=True)
    g.close()
    tg.close()
    gr.close()


def run_nfor(args):
    """--workload nfor1080: NFOR buffers of a 1920x1080, 16-spp render of the mesh + glossy
    scene (luz_gpu_render_ex), denoised by luz_gpu_nfor_denoise (host buffers in and out, host
    wall clock) and, once, by the reference's Denoise::applyNFOR on all host threads."""
    from luz_b200 import native
    w = workload("mesh_glossy", 16)
    g = native.GpuScene(w.scene.build())
    _, _, bufs, _ = g.render_ex(native.params(w.width, w.height, w.spp, w.max_bounces, w.seed), None, True)
    g.close()
    for _ in range(max(1, args.warmup)):
        native.nfor_denoise(bufs)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        native.nfor_denoise(bufs)
        ts.append(time.perf_counter() - t0)
    t = statistics.median(ts)
    px = float(w.width * w.height)
    out = {"metric": "Mpixels/s denoised", "value": px / t / 1e6, "unit": "Mpixels/s", "n_gpus": 1,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded scene render)",
           "timing": "host wall clock around luz_gpu_nfor_denoise (host buffers in and out)",
           "config": {"workload": "nfor1080: NFOR buffers of mesh_glossy 1920x1080 16spp, default NFORSettings"}}
    sys.path.insert(0, REFERENCE_DIR)
    import oracle as O
    if O.reference_available(fast=True):
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        O.RefOracle(fast=True).nfor(bufs, threads=threads)
        tc = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": px / tc / 1e6, "unit": "Mpixels/s", "cores": threads, "kind": "reference",
                               "sample": f"the same buffers, Denoise::applyNFOR, {tc * 1e3:.0f} ms"}
    print(json.dumps(out), flush=True)


def run_cache(args):
    """--workload cache_cornell | cache_room | cache_glossy: time to equal error, learned
    radiance cache against the plain integrator. cache_cornell is config 0 (Cornell box
    300x300, depth 8) and its error is measured against the reference's own film at 65,536
    spp (tests/golden/oracle64k_cornell300.npz); cache_glossy is the 1080p mesh frame, its
    error measured on the seeded 4,096 pixels the reference rendered at 65,536 spp
    (tests/golden/oracle64k_glossy_full.npz); cache_room (the box closed with the camera
    inside, longer paths; no reference film) against a 4096-spp plain render with its own
    seed. Error = relative MSE, mean((x - ref)^2 / (ref^2 + 0.01)). Each curve is device
    time (CUDA events around the render call; the cached call includes all its training)
    against error over a range of spp (seed 202), every cached render starting from an
    untrained cache. The speedup at a target error is plain time / cached time to reach it
    (log-log interpolation); the targets are the plain image's errors at three spp, and
    value is the speedup at the highest (the quality of a finished frame). On cache_glossy
    the 1% largest per-pixel errors are dropped before the mean (environment-light fireflies
    otherwise decide the error of a 4,096-pixel sample)."""
    from luz_b200 import desc as D
    from luz_b200 import native, scenes
    golden = os.path.join(ROOT, "tests", "golden")
    sub = None
    if args.workload == "cache_glossy":
        w = scenes.mesh_glossy(spp=1)
        gd = np.load(os.path.join(golden, "oracle64k_glossy_full.npz"))
        sub = (gd["y"].astype(np.int64) * w.width + gd["x"]).astype(np.int64)
        ref = gd["rgb"].astype(np.float64)
        ref_kind = "reference film at 65,536 spp on 4,096 seeded pixels"
        spps = [1, 2, 4, 8, 16, 32, 64]
        targets = (4, 16, 64)
    else:
        w = scenes.cornell(300, 300, 1, 8, closed=args.workload == "cache_room")
        spps = [2, 4, 8, 16, 32, 64, 128, 256]
        targets = (16, 64, 256)
    g = native.GpuScene(w.scene.build())
    W, H, MB = w.width, w.height, w.max_bounces
    tuned = {"wave_paths": args.cache_wave} if args.cache_wave else {}
    if args.workload == "cache_cornell":
        ref = np.load(os.path.join(golden, "oracle64k_cornell300.npz"))["rgb"].astype(np.float64)
        ref_kind = "reference film at 65,536 spp (Renderer::render)"
    elif args.workload == "cache_room":
        ref, _ = g.render(native.params(W, H, 4096, MB, 101))
        ref = ref.astype(np.float64)
        ref_kind = "plain GPU render at 4096 spp, independent seed"

    min_rough = args.cache_min_rough if args.cache_min_rough is not None else 0.0

    def relmse(img):
        if sub is None:
            return float(np.mean((img.astype(np.float64) - ref) ** 2 / (ref ** 2 + 0.01)))
        x = img.reshape(-1, 3)[sub].astype(np.float64)
        e = np.sort(np.mean((x - ref) ** 2 / (ref ** 2 + 0.01), axis=1))
        return float(np.mean(e[:len(e) - len(e) // 100]))

    def cached_render(c, p):   # the handle's wave size applies to the cached render only
        g.set_tuning(**tuned)
        try:
            return c.render(g, p)
        finally:
            g.set_tuning()

    def new_cache():
        return native.RadianceCache(D.cache_params(seed=3, batch=args.cache_batch, train_every=args.cache_train_every,
                                                   prefix=args.cache_prefix, warm_steps=args.cache_warm_steps,
                                                   min_roughness=min_rough))

    for _ in range(max(1, args.warmup)):
        g.render(native.params(W, H, 2, MB, 7))
        c = new_cache()
        cached_render(c, native.params(W, H, 2, MB, 7))
        c.close()
    plain, cached = [], []
    for spp in spps:
        img, st = g.render(native.params(W, H, spp, MB, 202))
        plain.append((spp, st.render_ms, relmse(img)))
        c = new_cache()
        img, st = cached_render(c, native.params(W, H, spp, MB, 202))
        cached.append((spp, st.render_ms, relmse(img)))
        c.close()

    def time_to(curve, target):
        if curve[0][2] <= target:
            return curve[0][1]
        for (s0, t0, e0), (s1, t1, e1) in zip(curve, curve[1:]):
            if e0 >= target >= e1 and e0 > e1:
                a = (np.log(e0) - np.log(target)) / (np.log(e0) - np.log(e1))
                return float(np.exp(np.log(t0) + a * (np.log(t1) - np.log(t0))))
        return None

    at = {}
    for ts in targets:
        target = plain[spps.index(ts)][2]
        tp, tc = time_to(plain, target), time_to(cached, target)
        at[f"plain_{ts}spp"] = {"target_error": target, "plain_ms": tp, "cached_ms": tc,
                                "speedup": (tp / tc) if (tp and tc) else None}
    head = at[f"plain_{targets[-1]}spp"]
    out = {"metric": "time-to-equal-error speedup (cached vs plain)", "value": head["speedup"], "unit": "x",
           "n_gpus": 1, "steps": 1, "warmup": args.warmup, "ms_per_step": head["cached_ms"],
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 paths, f16 MLP",
           "data": "synthetic (seeded scene generator)",
           "config": {"workload": f"{args.workload}: {w.name} {W}x{H} depth {MB}",
                      "error": "relative MSE mean((x - ref)^2 / (ref^2 + 0.01))"
                               + (", 1% largest pixels dropped" if sub is not None else ""), "reference": ref_kind,
                      "target": f"error of the plain {targets[-1]}-spp image",
                      "cache": f"prefix {args.cache_prefix}, NEE explicit at the cache vertex, one training path in {args.cache_train_every} "
                               "(self-training: it ends in the cache at its next eligible vertex), "
                               f"batch {args.cache_batch} (up to 16 steps per wave), lr 1e-2, first sample plain with "
                               f"{args.cache_warm_steps or 64} warm-up steps, min roughness {min_rough:g}, "
                               f"waves of {args.cache_wave or 4194304} paths"},
           "speedup_at": at,
           "plain": {"curve": [{"spp": s, "ms": t, "relmse": e} for s, t, e in plain]},
           "cached": {"curve": [{"spp": s, "ms": t, "relmse": e} for s, t, e in cached]}}
    print(json.dumps(out), flush=True)
    g.close()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload in ("batch48", "batch48_small"):
        run_batch(args)
    elif args.workload == "adjoint_c3":
        run_adjoint(args)
    elif args.workload == "nfor1080":
        run_nfor(args)
    elif args.workload in ("cache_cornell", "cache_room", "cache_glossy"):
        run_cache(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
