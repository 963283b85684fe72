#!/usr/bin/env python
"""Throughput of the ray/scene hot path on B200.

Workload (one "step"): closest-hit queries for 2^24 incoherent rays (origins uniform in a cube of
side 3, directions uniform on the sphere) against a displaced icosphere of 1,310,720 triangles
(radius 1, value-noise displacement amplitude 0.05, 8 octaves), tree = the reference's SAH tree.
Metric: Mrays/s, whole job.  Each rank traces its own 2^24 rays (weak scaling, no collective on
the data path; ranks only meet for the barrier and the max-over-ranks of the device time).

Beside the headline it reports the 1920x1080 primary-ray modes (normal / depth / hit count) and,
on rank 0 with one GPU, the reference's own CPU traversal timed on this host's cores.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
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

METRIC = "Mrays/s & Mpaths/s at 1M tris; equal-time relMSE guided vs plain"
WORKLOAD = ("closest-hit ray queries: 2^24 incoherent rays vs a 1,310,720-triangle displaced icosphere "
            "(reference SAH tree), FP32")
HBM_FALLBACK_GBS = 6650.0


def args_():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--rays-log2", type=int, default=24)
    p.add_argument("--subdiv", type=int, default=8)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-extras", action="store_true", help="skip the primary-ray and path-tracing side metrics")
    p.add_argument("--c4-only", action="store_true",
                   help="only the guided-vs-plain measurement on the 64-scene batch set (one JSON line)")
    p.add_argument("--c4-spp", type=int, default=1024)
    p.add_argument("--c4-ref-spp", type=int, default=2048)
    p.add_argument("--c4-steps", type=int, default=256)
    p.add_argument("--c4-mix", type=float, default=0.5)
    p.add_argument("--c4-depth", type=int, default=0, help="guided_depth of the C4 guides (0: every vertex)")
    p.add_argument("--pt-only", action="store_true",
                   help="only the C0 and C2 path-tracing measurements (one JSON line)")
    p.add_argument("--pt-renders", type=int, default=7, help="timed renders per workload (the median is kept)")
    p.add_argument("--pt-workload", choices=["both", "box", "layered"], default="both")
    p.add_argument("--pt-host-loop", action="store_true",
                   help="path tracing with the host-driven loop (profilers cannot see into the device loop)")
    p.add_argument("--guide-train-only", action="store_true",
                   help="only the guide's training-step times on 2^18 device records (one JSON line)")
    return p.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.samples = []
        self.gpu = gpu_index
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.p = None

    def _read(self):
        for line in self.p.stdout:
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                self.samples.append(f)

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def build_scene(subdiv):
    from swpathtracer_b200 import scenes
    return scenes.displaced_mesh_scene(subdiv).build()


def cpu_baseline(packed, rays_np, budget_rays):
    """The reference's own SBVH::intersect (oracle/_ref) on this host's cores, over a bounded sample."""
    sample = rays_np[:budget_rays]
    cores = os.cpu_count() or 1
    try:
        from oracle.bindings import RefHarness
        h = RefHarness()
        kind = "reference"
        t0 = time.perf_counter()
        rs = h.scene(packed, n_threads=cores)
        ref_build_s = time.perf_counter() - t0
        r = rs.intersect(sample, n_threads=cores, want_normals=False)
        secs = r["seconds"]
    except FileNotFoundError:
        from oracle.bindings import Oracle
        kind = "port"
        osc = Oracle().scene(packed)
        t0 = time.perf_counter()
        osc.intersect(sample, n_threads=cores, want_normals=False)
        secs = time.perf_counter() - t0
    out = {"value": round(len(sample) / secs / 1e6, 4), "unit": "Mrays/s", "cores": cores, "kind": kind,
           "sample": "%d of the step's incoherent rays, SBVH::intersect per ray, OpenMP over rays" % len(sample)}
    if kind == "reference":
        out["sbvh_build_s"] = round(ref_build_s, 2)   # SBVH::build, single-threaded in the reference
    return out


def guided_vs_plain(spt, scenes, dev, torch, name, sb, spp, ref_spp, steps, seeds=(7, 8, 9, 10), mix=0.5,
                    cache_res=0):
    """Equal-time relMSE of guided vs plain path tracing (128^2, max length 5).  Plain and guided both
    render `spp` samples per seed; each image's relMSE mean((I - R)^2 / (R^2 + 1e-2)) against a
    `ref_spp` plain render is multiplied by its wall time (relMSE falls as 1/time), and the ratio
    plain / guided of the products, summed over the seeds, is the relMSE ratio at equal time
    (> 1: guiding wins).  The guided time includes the guide's online training (`steps` Adam steps of
    2^16 records) and its lobe-cache refreshes; each seed trains a fresh guide, which samples its
    mixture with probability `mix` from a lobe cache of `cache_res`^3 cells (0: the default)."""
    import numpy as np
    gs = spt.GpuScene(dev, sb.build())
    cam = scenes.box_camera(128, 128)
    img = torch.empty(128 * 128 * 3, dtype=torch.float32, device="cuda")

    def render(n, seed, guide=None):
        p = scenes.pt_params(spp=n, sampler="jittered", termination="max-length", path_length=5, seed=seed)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if guide is None:
            gs.pathtrace_device(cam, p, img.data_ptr())
        else:
            gs.pathtrace_guided_device(cam, p, guide, img.data_ptr())
        torch.cuda.synchronize()
        return img.cpu().numpy().reshape(128, 128, 3).copy(), time.perf_counter() - t0

    def relmse(a, b):
        return float(np.mean((a - b) ** 2 / (b ** 2 + 1e-2)))

    render(64, 1)
    ref, _ = render(ref_spp, 99)
    ep = eg = tp = tg = 0.0
    for seed in seeds:
        plain, t = render(spp, seed)
        g = spt.Guide(dev, spt.guide_config(batch=1 << 16, max_steps=steps, mix=mix, seed=seed,
                                                 cache_res=cache_res))
        guided, u = render(spp, seed, g)
        g.close()
        if t < 0.2:
            # renders of about 100 ms are timed three times per arm (the same work, a fresh guide each
            # time) and the median kept: the guided arm's training loop waits on the host, so one
            # stretch of host contention would otherwise decide the line
            ts, us = [t], [u]
            for _ in range(2):
                ts.append(render(spp, seed)[1])
                g = spt.Guide(dev, spt.guide_config(batch=1 << 16, max_steps=steps, mix=mix, seed=seed,
                                                         cache_res=cache_res))
                us.append(render(spp, seed, g)[1])
                g.close()
            t, u = sorted(ts)[1], sorted(us)[1]
        ep, tp = ep + relmse(plain, ref), tp + t
        eg, tg = eg + relmse(guided, ref), tg + u
    gs.close()
    k = len(seeds)
    return {name + "_spp": spp, name + "_relmse_plain": round(ep / k, 6), name + "_relmse_guided": round(eg / k, 6),
            name + "_wall_ms_plain": round(1e3 * tp / k, 2), name + "_wall_ms_guided": round(1e3 * tg / k, 2),
            name + "_equal_time_relmse_ratio_plain_over_guided": round((ep * tp) / (eg * tg), 4)}


def path_tracing(spt, scenes, dev, torch, subdiv, renders=7, workload="both", host_loop=False):
    """Path tracing of C0 (box, 256^2, 16 spp, max length 5) and C2 (the layered mesh in the box x3,
    800 x 600, RR after 3, cap 16; 16 spp: the throughput does not depend on spp), each the median of
    `renders` device-timed renders (spt_pathtrace_device: one launch of the render's graph).  With
    host_loop, the same render as a one-job batch whose loop the host drives (tune.host_loop: a graph
    of two iterations replayed from the host, which kernel profilers can see into)."""
    from swpathtracer_b200 import abi
    extras = {}
    tune = abi.Tune(capacity=1 << 21, extend_block=128, shade_block=128, traversal=-1, check_every=8, host_loop=1)
    for key, sb, cam, prm in (
            ("pt_box_256x256_16spp", scenes.box_scene(5), scenes.box_camera(256, 256),
             scenes.pt_params(spp=16, sampler="jittered", termination="max-length", path_length=5, seed=3)),
            ("pt_layered_800x600_rr3_max16", scenes.layered_box_scene(subdiv), scenes.layered_box_camera(800, 600),
             scenes.pt_params(spp=16, sampler="jittered", termination="russian-roulette", path_length=3,
                              max_depth=16, seed=4))):
        if workload != "both" and not key.startswith("pt_" + workload):
            continue
        pgs = spt.GpuScene(dev, sb.build())
        img = torch.empty(cam.width * cam.height * 3, dtype=torch.float32, device="cuda")
        if host_loop:
            one = lambda: spt.render_batch(dev, [(pgs, cam, prm)], [img.data_ptr()], tune=tune)[0]
        else:
            one = lambda: pgs.pathtrace_device(cam, prm, img.data_ptr())
        for _ in range(2):
            one()
        # renders of a few ms each; the median is robust to a transient on a shared machine
        runs = sorted((one() for _ in range(renders)), key=lambda r: r.gpu_ms)
        mid = runs[len(runs) // 2]
        paths, segs, ms = mid.paths, mid.segments, mid.gpu_ms
        extras[key + "_Mpaths_s"] = round(paths / (ms / 1e3) / 1e6, 3)
        extras[key + "_Mrays_s"] = round(segs / (ms / 1e3) / 1e6, 2)
        extras[key + "_segments_per_path"] = round(segs / paths, 3)
        pgs.close()
    return extras


def guided_c4(spt, scenes, dev, torch, spp=1024, ref_spp=2048, batch=1 << 18, steps=256, mix=0.5, depth=0, n=64):
    """Guided vs plain path tracing on the whole 64-scene batch set (each scene at its own resolution,
    128^2 to 1024^2, max path length 5), the guide configured as specified: batch 2^18 training records,
    Adam lr 1e-2, mix 0.5.  Per scene: a plain render and a guided render of `spp` samples (the guided
    one trains a fresh guide for `steps` optimiser steps during the render), each timed on the host with
    the device synchronised, and a plain reference of `ref_spp` samples made of two independent halves.

    relMSE = mean((I - R)^2 / (R^2 + 1e-2)).  A reference of finite spp adds its own noise to both
    arms' relMSE, which pulls the ratio towards 1; the two halves measure that noise: the variance of
    their mean R is (R1 - R2)^2 / 4 per pixel, and subtracting it from each arm's relMSE gives the
    debiased figures (`..._debiased`).  The equal-time ratio is sum(relMSE_plain * t_plain) /
    sum(relMSE_guided * t_guided) over the scenes (relMSE falls as 1 / time), > 1 when guiding wins;
    the geometric mean of the per-scene ratios is reported beside it.  `depth` > 0 guides only the
    first `depth` vertices of a path (guided_depth); `..._nonfinite_pixels` counts NaN or infinite
    values over all guided images (0 expected)."""
    import math

    def relmse(a, b):
        return float(torch.mean((a - b) ** 2 / (b * b + 1e-2)).item())

    rows = []
    nonfinite = 0
    for i, (sb, cam, _, desc) in enumerate(scenes.batched_scenes()[:n]):
        gs = spt.GpuScene(dev, sb.build())
        npx = cam.width * cam.height

        def render(k, seed, guide=None):
            img = torch.empty(npx * 3, dtype=torch.float32, device="cuda")
            p = scenes.pt_params(spp=k, sampler="jittered", termination="max-length", path_length=5, seed=seed)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            if guide is None:
                gs.pathtrace_device(cam, p, img.data_ptr())
            else:
                gs.pathtrace_guided_device(cam, p, guide, img.data_ptr())
            torch.cuda.synchronize()
            return img, time.perf_counter() - t0

        render(4, 1)
        r1, _ = render(ref_spp // 2, 100003 + i)
        r2, _ = render(ref_spp // 2, 200003 + i)
        ref = 0.5 * (r1 + r2)
        ref_noise = float(torch.mean(0.25 * (r1 - r2) ** 2 / (ref * ref + 1e-2)).item())
        plain, tp = render(spp, 7 + i)
        g = spt.Guide(dev, spt.guide_config(batch=batch, max_steps=steps, mix=mix, seed=7 + i, guided_depth=depth))
        guided, tg = render(spp, 7 + i, g)
        g.close()
        if tp < 0.5:
            # a render of tens of milliseconds is timed three times per arm (the same work: the same
            # seeds, a fresh guide each time) and the median kept, so that one host hiccup does not
            # decide the scene; the images of the first renders are the ones compared
            tps, tgs = [tp], [tg]
            for _ in range(2):
                tps.append(render(spp, 7 + i)[1])
                g = spt.Guide(dev, spt.guide_config(batch=batch, max_steps=steps, mix=mix, seed=7 + i,
                                                    guided_depth=depth))
                tgs.append(render(spp, 7 + i, g)[1])
                g.close()
            tp, tg = sorted(tps)[1], sorted(tgs)[1]
        gs.close()
        nonfinite += int((~torch.isfinite(guided)).sum().item())
        ep, eg = relmse(plain, ref), relmse(guided, ref)
        rows.append((desc, ep, eg, tp, tg, ref_noise))
        del r1, r2, ref, plain, guided
    sp = sum(r[1] * r[3] for r in rows)
    sg = sum(r[2] * r[4] for r in rows)
    spd = sum(max(r[1] - r[5], 0.0) * r[3] for r in rows)
    sgd = sum(max(r[2] - r[5], 0.0) * r[4] for r in rows)
    per = [(r[1] * r[3]) / max(r[2] * r[4], 1e-30) for r in rows]
    key = "guided_c4_64scenes_%dspp" % spp
    out = {key + "_equal_time_relmse_ratio_plain_over_guided": round(sp / sg, 4),
           key + "_equal_time_relmse_ratio_debiased": round(spd / max(sgd, 1e-30), 4),
           key + "_geomean_per_scene_ratio": round(math.exp(sum(math.log(x) for x in per) / len(per)), 4),
           key + "_per_scene_ratios": [round(x, 3) for x in per],
           key + "_per_scene_ms_plain_guided": [[round(1e3 * r[3], 1), round(1e3 * r[4], 1)] for r in rows],
           key + "_wall_s_plain": round(sum(r[3] for r in rows), 3),
           key + "_wall_s_guided": round(sum(r[4] for r in rows), 3),
           key + "_reference_spp": ref_spp, key + "_nonfinite_pixels": nonfinite,
           key + "_guide": {"batch": batch, "steps": steps, "mix": mix, "guided_depth": depth}}
    by_kind = {}
    for r, x in zip(rows, per):
        by_kind.setdefault(r[0].split(", ")[-1].split(" ")[0], []).append(x)
    out[key + "_geomean_ratio_by_material"] = {k: round(math.exp(sum(math.log(v) for v in vs) / len(vs)), 3)
                                               for k, vs in sorted(by_kind.items())}
    return out


def guide_train_steps(spt, abi, dev, torch, n=1 << 18, steps=10, warmup=3):
    """Device time of one optimiser step of the guide on n records already in device memory
    (spt_guide_train_device), for both training paths: tcgen05 tiles of 128 records with tensor-memory
    accumulators, and the warp-level mma.sync kernels.  Synthetic records: positions uniform in the
    unit box, directions uniform on the sphere, weights uniform in [0, 2)."""
    import numpy as np
    rng = np.random.default_rng(1)
    r = np.zeros(n, abi.GUIDE_RECORD_DTYPE)
    r["pos"] = rng.uniform(0.02, 0.98, (n, 3))
    for k in ("normal", "wo", "wi"):
        v = rng.normal(size=(n, 3))
        r[k] = v / np.linalg.norm(v, axis=1, keepdims=True)
    r["weight"] = rng.uniform(0.0, 2.0, n)
    d = torch.from_numpy(r.view(np.uint8).copy()).cuda()
    out = {}
    for name, path in (("tcgen05", abi.GUIDE_TRAIN_TCGEN05), ("mma_sync", abi.GUIDE_TRAIN_MMA_SYNC)):
        g = spt.Guide(dev, spt.guide_config(batch=n, train_path=path, seed=2))
        for _ in range(warmup):
            g.train_device(d.data_ptr(), n)
        ms = sorted(g.train_device(d.data_ptr(), n) for _ in range(steps))
        g.close()
        med = ms[len(ms) // 2]
        out["guide_train_step_2e18_%s_ms" % name] = round(med, 4)
        out["guide_train_step_2e18_%s_Mrecords_s" % name] = round(n / (med / 1e3) / 1e6, 1)
    return out


def cpu_pathtrace_baseline(subdiv):
    """The reference's own PathTracer::render (oracle/_ref) on this host's cores, on bounded samples of
    the two path-tracing workloads (4 spp of the box scene, 1 spp of the layered 1.3M-tri scene).
    The reference has no depth cap next to russian roulette: its layered run caps at 1000 bounces."""
    from swpathtracer_b200 import scenes
    try:
        from oracle.bindings import RefHarness
        h = RefHarness()
    except FileNotFoundError:
        return None
    cores = os.cpu_count() or 1
    out = {"cores": cores, "kind": "reference", "unit": "Mpaths/s"}
    for key, sb, cam, prm in (
            ("pt_box_256x256", scenes.box_scene(5), scenes.box_camera(256, 256),
             scenes.pt_params(spp=4, sampler="jittered", termination="max-length", path_length=5, seed=3)),
            ("pt_layered_800x600_rr3", scenes.layered_box_scene(subdiv), scenes.layered_box_camera(800, 600),
             scenes.pt_params(spp=1, sampler="jittered", termination="russian-roulette", path_length=3, seed=4))):
        rs = h.scene(sb.build(), n_threads=cores)
        _, secs = rs.pathtrace(cam, prm, n_threads=cores)
        out[key + "_Mpaths_s"] = round(cam.width * cam.height * prm.spp / secs / 1e6, 4)
    out["sample"] = "PathTracer::render, box 256x256 at 4 spp, layered 800x600 at 1 spp, OpenMP over rows"
    return out


def run_reference(a):
    """--impl reference: the reference's CPU path on the same workload (rank 0 only)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from swpathtracer_b200 import scenes
    packed = build_scene(a.subdiv)
    n_step = 1 << 20
    rays = scenes.incoherent_rays(1 << a.rays_log2, seed=1)
    cores = os.cpu_count() or 1
    try:
        from oracle.bindings import RefHarness
        rs = RefHarness().scene(packed, n_threads=cores)
        kind = "reference"
        run = lambda s: rs.intersect(s, n_threads=cores, want_normals=False)["seconds"]
    except FileNotFoundError:
        from oracle.bindings import Oracle
        osc = Oracle().scene(packed)
        kind = "port"

        def run(s):
            t0 = time.perf_counter()
            osc.intersect(s, n_threads=cores, want_normals=False)
            return time.perf_counter() - t0
    for w in range(a.warmup):
        run(rays[(w * n_step) % len(rays):][:n_step])
    total = 0.0
    for k in range(a.steps):
        total += run(rays[(k * n_step) % len(rays):][:n_step])
    value = a.steps * n_step / total / 1e6
    out = {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "Mrays/s", "n_gpus": a.gpus,
           "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(1000 * total / a.steps, 3),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": WORKLOAD, "rays_per_step": n_step, "tris": int(packed.n_prims)},
           "cpu_baseline": {"value": round(value, 4), "unit": "Mrays/s", "cores": cores, "kind": kind,
                            "sample": "%d rays per step of the 2^24-ray set, SBVH::intersect per ray" % n_step},
           "e2e": {"value": round(value, 4), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    a = args_()
    if a.impl == "reference":
        run_reference(a)
        return
    import torch
    import torch.distributed as dist

    import swpathtracer_b200 as spt
    from swpathtracer_b200 import abi, scenes

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if a.guide_train_only:
        dev = spt.Device(local)
        print(json.dumps(guide_train_steps(spt, abi, dev, torch)), flush=True)
        dev.close()
        return
    if a.pt_only:
        dev = spt.Device(local)
        print(json.dumps(path_tracing(spt, scenes, dev, torch, a.subdiv, renders=a.pt_renders, workload=a.pt_workload,
                                      host_loop=a.pt_host_loop)), flush=True)
        dev.close()
        return
    if a.c4_only:
        dev = spt.Device(local)
        print(json.dumps(guided_c4(spt, scenes, dev, torch, spp=a.c4_spp, ref_spp=a.c4_ref_spp, steps=a.c4_steps,
                                   mix=a.c4_mix, depth=a.c4_depth)), flush=True)
        dev.close()
        return
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    packed = build_scene(a.subdiv)
    t_build = time.perf_counter()
    bvh = spt.Bvh(packed)
    build_ms = (time.perf_counter() - t_build) * 1e3
    dev = spt.Device(local)
    gs = spt.GpuScene(dev, packed, bvh)
    n = 1 << a.rays_log2
    rays_np = scenes.incoherent_rays(n, seed=1 + rank)
    d_rays = torch.from_numpy(rays_np).to("cuda")
    d_hits = torch.empty((n, 4), dtype=torch.int32, device="cuda")

    # reference traversal counts on a sample of the same rays: the per-ray algorithmic work
    ns = 1 << 20
    t_tests = torch.empty(ns, dtype=torch.int32, device="cuda")
    t_prim = torch.empty(ns, dtype=torch.int32, device="cuda")
    gs.count_device(d_rays.data_ptr(), ns, None, t_tests.data_ptr(), None, t_prim.data_ptr())
    torch.cuda.synchronize()
    t_tri = float(t_prim.double().mean())
    t_box = float(t_tests.double().mean()) - t_tri
    bytes_per_ray = 24.0 * t_box + 36.0 * t_tri + 32.0 + 16.0

    # A step is spt_intersect_device's three stages called one by one, so that the traversal kernel's
    # own time can be bracketed by events inside the timed region: the coherence order of the batch
    # (three kernels: per-block key histograms, their per-key offsets, the scan of the key totals
    # with the scatter), the persistent closest-hit kernel in that order (after a one-thread kernel
    # that holds the order's traced count to the batch), and the gather of the hits back to the rays'
    # own indices.  All of it runs on the legacy default stream, torch's current stream here, so the
    # events see the kernels.
    d_order = torch.empty(2 * n + 1, dtype=torch.int32, device="cuda")
    d_hits_ordered = torch.empty((n, 4), dtype=torch.int32, device="cuda")
    kernels_per_step = 6

    def step(mid=None):
        gs.ray_order_device(d_rays.data_ptr(), n, d_order.data_ptr(), 0)
        if mid:
            mid[0].record()
        gs.intersect_ordered_device(d_rays.data_ptr(), d_order.data_ptr(), n, d_hits_ordered.data_ptr(), 0)
        if mid:
            mid[1].record()
        gs.hits_unorder_device(d_order.data_ptr(), n, d_hits_ordered.data_ptr(), d_hits.data_ptr(), 0)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = Clocks(local)
    # The traversal kernel is bracketed by a pair of timing events on every tenth step: an event pair
    # costs about 50 us of a 5 ms step (the stream drains at each timing event), so every step would
    # take 1 % off the measured value; the sampled launches give the kernel's average duration.
    every = 10
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    mids = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
            for _ in range((a.steps + every - 1) // every)]
    torch.cuda.synchronize()
    ev0.record()
    for k in range(a.steps):
        step(mids[k // every] if k % every == 0 else None)
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    ms_trace = sum(b.elapsed_time(c) for b, c in mids) / len(mids)
    clk = clocks.stop()
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    ms_step = ms / a.steps
    value = world * n * a.steps / (ms / 1000.0) / 1e6

    # end to end through the public C-ABI entry point with pinned host buffers, the rays laid out as
    # the reference's Ray (origin then direction, 24 bytes: spt_intersect_packed)
    rays6 = np.ascontiguousarray(np.concatenate([rays_np[:, 0:3], rays_np[:, 4:7]], axis=1))
    h_rays = torch.from_numpy(rays6).pin_memory()
    h_rays_np = h_rays.numpy()
    h_hits = torch.empty((n, 4), dtype=torch.int32).pin_memory().numpy().view(abi.HIT_DTYPE).reshape(n)
    gs.intersect(h_rays_np, out=h_hits)
    t0 = time.perf_counter()
    e2e_steps = max(1, min(a.steps, 5))
    for _ in range(e2e_steps):
        gs.intersect(h_rays_np, out=h_hits)
    e2e = n * e2e_steps / (time.perf_counter() - t0) / 1e6
    if world > 1:
        t = torch.tensor([e2e], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        e2e = float(t.item()) * world

    hbm, peak_kind = peaks()
    achieved = bytes_per_ray * n / (ms_trace / 1000.0) / 1e9
    traffic = None
    prof = {}
    tpath = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            prof = json.load(f).get("k_intersect_df_ordered") or {}
        if prof:
            traffic = prof["bytes_per_ray"] * n
    # the kernel's own work on a sample of the same rays (an extra, untimed launch with counters)
    work_nodes, work_prims = gs.traversal_work_device(d_rays.data_ptr(), ns, d_hits.data_ptr())

    out = {"metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": WORKLOAD, "rays_per_step_per_gpu": n, "tris": int(packed.n_prims),
                      "l2": "inputs larger than L2: 512 MB of rays streamed per step (scene 97 MB stays in L2)",
                      "parallelism": "replicas" if world > 1 else "single GPU"},
           # The fraction is the reference's algorithmic bytes per ray (its unpruned node and triangle
           # payloads) over the measured HBM copy bandwidth.  The kernel is not HBM-bound: it reads
           # most of those bytes from L1/L2, and the ncu capture behind profiles/dram_traffic.json
           # shows it issue- and latency-bound (issue_active, lanes per instruction, dram_frac).
           "roofline": {"bound": "issue", "denominator": "hbm", "achieved": round(achieved, 1), "peak": hbm,
                        "unit": "GB/s", "frac": round(achieved / hbm, 4), "traffic": traffic,
                        "peak_source": peak_kind,
                        "algorithmic_bytes_per_ray": round(bytes_per_ray, 2),
                        "ref_box_tests_per_ray": round(t_box, 3), "ref_tri_tests_per_ray": round(t_tri, 3),
                        "kernel_node_visits_per_ray": round(work_nodes / ns, 3),
                        "kernel_box_tests_per_ray": round(8.0 * work_nodes / ns, 3),
                        "kernel_prim_tests_per_ray": round(work_prims / ns, 3),
                        "kernel_ms": round(ms_trace, 4), "kernel": "k_intersect_df_ordered",
                        "ordering_and_gather_ms": round(ms_step - ms_trace, 4),
                        "dram_frac": (round(traffic / (ms_trace / 1000.0) / 1e9 / hbm, 4) if traffic else None),
                        "issue_active_frac": prof.get("issue_active"),
                        "lanes_per_instruction": prof.get("lanes_per_instruction"),
                        "profile": prof.get("source")},
           "e2e": {"value": round(e2e, 3), "unit": "Mrays/s", "h2d_bytes_per_step": n * 24,
                   "d2h_bytes_per_step": n * 16},
           "gpu_launches": kernels_per_step * a.steps,
           "bvh_build_ms": round(build_ms, 1),
           "clocks": clk}

    # the submetrics are single-GPU measurements: under torchrun (N > 1) they would hold every rank's
    # GPU for minutes while only rank 0 works, so they run at N = 1 only
    if rank == 0 and world == 1 and not a.no_extras:
        extras = {}
        for name, mode in (("normal", abi.RAYCAST_NORMAL), ("depth", abi.RAYCAST_DEPTH), ("count", abi.RAYCAST_COUNT)):
            cam = scenes.displaced_mesh_camera(1920, 1080)
            elem = {abi.RAYCAST_NORMAL: 12, abi.RAYCAST_DEPTH: 4, abi.RAYCAST_COUNT: 8}[mode]
            buf = torch.empty(1920 * 1080 * elem, dtype=torch.uint8, device="cuda")
            for _ in range(3):
                gs.raycast_device(cam, mode, buf.data_ptr())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(10):
                gs.raycast_device(cam, mode, buf.data_ptr())
            e1.record()
            torch.cuda.synchronize()
            extras["primary_1920x1080_" + name + "_Mrays_s"] = round(1920 * 1080 * 10 / (e0.elapsed_time(e1) / 1e3) / 1e6, 2)
        # the device-built tree (spt_bvh_build_device) of the same mesh: build time, and the headline
        # queries over it (same closest hits except equal-t ties)
        spt.Bvh(packed, device=dev).close()   # first call: module loading
        t_dev = time.perf_counter()
        dbvh = spt.Bvh(packed, device=dev)
        extras["bvh_build_device_ms"] = round((time.perf_counter() - t_dev) * 1e3, 1)
        dgs = spt.GpuScene(dev, packed, dbvh)
        for _ in range(3):
            dgs.intersect_device(d_rays.data_ptr(), n, d_hits.data_ptr(), 0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(20):
            dgs.intersect_device(d_rays.data_ptr(), n, d_hits.data_ptr(), 0)
        e1.record()
        torch.cuda.synchronize()
        extras["device_tree_closest_hit_Mrays_s"] = round(n * 20 / (e0.elapsed_time(e1) / 1e3) / 1e6, 1)
        dgs.close()
        dbvh.close()
        # path tracing: the CPU-runnable box scene (20,492 tris, 256x256, 16 spp, max length 5) and the
        # 1.3M-tri layered scene (800x600, russian roulette after 3, max depth 16), Mpaths/s
        extras.update(path_tracing(spt, scenes, dev, torch, a.subdiv))
        # batched uneven scenes: 64 seeded scenes (1k-500k tris, 128^2-1024^2, 64 spp) in one wavefront,
        # settings from the autotuner (its trials are not timed)
        batch = scenes.batched_scenes()
        packs = [sb.build() for sb, _, _, _ in batch]
        # scene set-up of the 64 scenes (tree + device upload): the reference's tree built on the host,
        # and the device-built tree (spt_bvh_build_device)
        t_setup = time.perf_counter()
        for p_ in packs:
            spt.GpuScene(dev, p_, spt.Bvh(p_, device=dev)).close()
        extras["batch64_setup_device_tree_s"] = round(time.perf_counter() - t_setup, 3)
        t_setup = time.perf_counter()
        jobs = [(spt.GpuScene(dev, p_), cam, prm) for p_, (_, cam, prm, _) in zip(packs, batch)]
        extras["batch64_setup_host_tree_s"] = round(time.perf_counter() - t_setup, 3)
        bufs = [torch.empty(cam.width * cam.height * 3, dtype=torch.float32, device="cuda") for _, cam, _ in jobs]
        tune = spt.autotune(dev, jobs, None)
        st = spt.render_batch(dev, jobs, [b.data_ptr() for b in bufs], tune=tune)
        paths = sum(s_.paths for s_ in st)
        extras["batch64_Mpaths_s"] = round(paths / (st[0].gpu_ms / 1e3) / 1e6, 3)
        extras["batch64_Mrays_s"] = round(st[0].segments / (st[0].gpu_ms / 1e3) / 1e6, 2)
        extras["batch64_tune"] = {"capacity": tune.capacity, "shade_block": tune.shade_block,
                                  "traversal": tune.traversal, "stack": tune.stack,
                                  "sort_shading": tune.sort_shading}
        extras["batch64_paths"] = paths
        for g_, _, _ in jobs:
            g_.close()
        # guided rendering: a room lit through a 0.1 x 0.1 window (directional transport), and the
        # small-light box (light found mostly via a two-sided emitter's halo; guiding loses there)
        extras.update(guided_vs_plain(spt, scenes, dev, torch, "guided_window_room_128x128",
                                      scenes.window_room_scene(0.1), 16384, 262144, 32, seeds=tuple(range(7, 15))))
        extras.update(guided_vs_plain(spt, scenes, dev, torch, "guided_small_light_128x128",
                                      scenes.small_light_box_scene(), 4096, 16384, 32, seeds=(7,)))
        # guided rendering on the whole 64-scene batch set, equal-time relMSE against plain
        extras.update(guided_c4(spt, scenes, dev, torch))
        # the guide's optimiser step at the configured batch of 2^18 records
        extras.update(guide_train_steps(spt, abi, dev, torch))
        out["submetrics"] = extras
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(packed, rays_np, 1 << 22)
        if not a.no_extras:
            pt = cpu_pathtrace_baseline(a.subdiv)
            if pt:
                out["cpu_baseline"]["pathtrace"] = pt
    if rank == 0:
        print(json.dumps(out), flush=True)
    gs.close()
    dev.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
