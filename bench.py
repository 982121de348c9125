#!/usr/bin/env python
"""SPPM throughput of the B200-native pipeline (one JSON line on stdout).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config caustic]

Workload (default): the caustic Cornell box — 149,862 triangles (unit box, 256x256-vertex sine
water surface as a GGX dielectric, 20k-triangle GGX conductor sphere), 1024x1024 pixels, 2^20
photons per iteration, max depth 12, grid 50 (initial radius 1% of the scene diagonal), 16 direct
samples, alpha 0.7, fp32.  A step is one SPPM iteration (trace -> emit -> hash/scan/sort ->
gather), replayed from a captured CUDA graph, inputs resident in HBM.  Scene data is synthetic
(procedural generator, seeded), the reference's .glb assets being unavailable.

value    = photons emitted per second over all ranks (Mphotons/s), CUDA events on the library
           stream around K graph replays, max over ranks.
e2e      = the same metric through the public API with host traffic every step: the round seed
           is drawn on the host (renderer.cpp:65) and copied from pinned memory, one round is
           replayed, and the tonemapped 8-bit image is read back (output.cpp:52-83).
roofline = the dominant kernel's algorithmic bytes per launch / its CUDA-event duration, against
           the measured HBM copy bandwidth.
--impl reference times the reference algorithm on the host cores (the oracle port: the
reference's OpenCL kernels have no CPU runtime here) on a bounded sample of the same workload.
Multi-GPU: N ranks render independent replicas (weak scaling, no collective on this path); with
--shard they render one image together (strong scaling): pixel and photon-path ranges per rank and
one NCCL all-gather of the stored photons per round, results bit-identical to one GPU.
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
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

CONFIGS = {
    # name: kind, detail, width, height, photons, depth, grid_res, rounds(config), note
    "cornell": dict(kind=0, detail=0, width=512, height=512, photons=1 << 18, depth=8, grid=50, rounds=64,
                    desc="empty Cornell box, 12 triangles, 512x512, 2^18 photons/iter, depth 8"),
    "caustic": dict(kind=1, detail=0, width=1024, height=1024, photons=1 << 20, depth=12, grid=50, rounds=256,
                    desc="caustic Cornell box, 149,862 triangles, 1024x1024, 2^20 photons/iter, depth 12"),
    "atrium": dict(kind=2, detail=0, width=1920, height=1080, photons=1 << 22, depth=16, grid=64, rounds=256,
                   desc="procedural atrium, 262,898 triangles, 1920x1080, 2^22 photons/iter, depth 16"),
}
METRIC = "Mphotons/s"
# dram__bytes_read.sum + dram__bytes_write.sum of a reference stage's kernels per round, from an
# ncu capture of one whole round of the caustic workload at 1/2 resolution and 1/4 photons (512x512
# pixels, 2^18 photon paths, ~425k stored photons), scaled by 4 to the full workload (pixels for
# trace_rays, photon paths or stored photons for the others; the 125,001-cell scan does not scale).
# trace_rays = k_trace_persistent 220.3 MB + k_shadow 105.9 + k_nee_resolve 76.3 + k_spec_resolve
# 13.3; emit_photons = k_emit_persistent 103.5 + k_emit_start 0.05 + k_scan 1.1 + k_compact 29.4;
# scatter_photons = the two radix passes 9.5 + k_sorted_records 11.9; gather_flux = k_pixel_keys 8.3
# + the pixel radix sort 6.4 + k_gather 58.7.  The integer stages' arrays stay in the 126 MB L2
# between kernels, so their DRAM bytes fall below the compulsory bytes.
NCU_TRAFFIC: dict = {"caustic": {"trace_rays": 1663.3e6, "emit_photons": 536.2e6, "hash_photons": 28.2e6,
                                 "scan": 0.51e6, "scatter_photons": 85.6e6, "gather_flux": 293.8e6}}


def load_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        try:
            for line in Path(self.path).read_text().splitlines():
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9 and f[1].replace(".", "").isdigit():
                    rows.append(f)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        mx = float(rows[0][2])
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())
                if any(r[3].replace(".", "").isdigit() for r in rows) else None}


def make_args(cfg: dict, scale: int = 1):
    import phosphor_b200 as P
    return P.ArgsList(width=cfg["width"] // scale, height=cfg["height"] // scale,
                      photons_per_round=max(1, cfg["photons"] // (scale * scale)), max_photon_bounces=cfg["depth"],
                      grid_res=cfg["grid"], seed=1, sppm_alpha=0.7, direct_samples=16)


def cpu_oracle_sample(cfg: dict, threads: int, min_seconds: float = 10.0, max_rounds: int = 8) -> dict:
    """The reference algorithm (oracle port, fp32) on the host cores, on the workload itself: one
    untimed round, then whole rounds until `min_seconds` have passed (at most `max_rounds`)."""
    import oracle as O
    args = make_args(cfg, 1)
    scene = O.GeneratedScene(cfg["kind"], seed=1, width=args.width, height=args.height, detail=cfg["detail"])
    orc = O.Oracle(scene)
    state = orc.render(args.params(), 1, prec=0, threads=threads)  # warm-up round
    dt, rounds, stage = 0.0, 0, [0.0] * 4
    while rounds < max_rounds and (rounds < 1 or dt < min_seconds):
        t0 = time.perf_counter()
        state = orc.render(args.params(), 1, prec=0, threads=threads, state=state)
        dt += time.perf_counter() - t0
        stage = [s + float(x) for s, x in zip(stage, state["seconds"])]
        rounds += 1
    photons = args.photons_per_round * rounds
    return {"value": photons / dt / 1e6, "unit": METRIC, "cores": threads, "kind": "port",
            "seconds": dt, "stage_seconds": stage,
            "sample": f"{rounds} SPPM round(s) of the workload itself ({args.width}x{args.height} px, "
                      f"{args.photons_per_round} photons/round) after one untimed round, fp32 oracle port of the "
                      f"reference kernels, {threads} threads"}


def run_reference(a, cfg: dict) -> dict:
    threads = os.cpu_count() or 1
    # each step is one whole round of the workload (about 3 s on 16 cores) unless that would make
    # the run longer than a few minutes; then 1/scale of the resolution and 1/scale^2 of the photons
    scale = 1 if a.steps + a.warmup <= 40 else 2 if a.steps + a.warmup <= 160 else 4
    import oracle as O
    args = make_args(cfg, scale)
    # the scene comes from the oracle library's copy of the generators: this arm maps no CUDA library
    scene = O.GeneratedScene(cfg["kind"], seed=1, width=args.width, height=args.height, detail=cfg["detail"])
    orc = O.Oracle(scene)
    state = None
    for _ in range(a.warmup):
        state = orc.render(args.params(), 1, prec=0, threads=threads, state=state)
    times = []
    for _ in range(a.steps):
        t0 = time.perf_counter()
        state = orc.render(args.params(), 1, prec=0, threads=threads, state=state)
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = args.photons_per_round * a.steps / tot / 1e6
    part = "the workload itself" if scale == 1 else f"1/{scale * scale} of the workload's pixels and photons"
    sample = (f"each step: one SPPM round at {args.width}x{args.height} px, {args.photons_per_round} photons "
              f"({part}, same scene), fp32 oracle port of the reference kernels (no CPU OpenCL runtime exists "
              f"for the reference's .cl), {threads} threads")
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * tot / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (procedural scene)",
            "config": {"workload": a.config, "desc": cfg["desc"], "sample_scale": scale},
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# Compulsory bytes per round of each reference stage: the records the stage must read or write
# once (hit points, photons, cells, SPPM state) plus the scene geometry for the two traversal
# stages, in the reference's device layout (triangles 180 B: vertices, normals, tangents 48 B each,
# UVs 32 B, material 4 B; BVH 32 B per node, 2n-1 nodes).
SCENE_BYTES_PER_TRI = 180 + 64


def algorithmic_bytes(P: int, Ns: int, C: int, ntri: int) -> dict:
    scene = SCENE_BYTES_PER_TRI * ntri
    return {
        "trace_rays": 96 * P + scene,                      # 6 float4 hit point written per pixel
        "emit_photons": 24 * Ns + scene,                   # position + RGBE + octahedral per stored photon
        "hash_photons": 16 * Ns + 4 * Ns + 4 * C + 8 * Ns,  # positions read, keys written, counts zeroed + RMW
        "scan": 8 * C,                                     # counts read, starts written
        "scatter_photons": 28 * Ns + 24 * Ns,              # key + record read, record written
        "gather_flux": 168 * P + 24 * Ns + 8 * C,          # hit point, flux/weight/radiance RMW, photons, ranges
    }


# the library's stages (phx_stage_ms) that implement each reference stage
STAGE_MAP = {"trace_rays": ["trace", "shadow"], "emit_photons": ["emit", "emit_scan"], "hash_photons": ["hash"],
             "scan": ["cell_scan"], "scatter_photons": ["sort", "records"], "gather_flux": ["gather"]}


def run_ours(a, cfg: dict) -> dict | None:
    import numpy as np
    import torch

    import phosphor_b200 as P
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    args = make_args(cfg)
    if a.binary_bvh:
        args.flags = args.flags | 4  # PHX_F_BINARY_BVH
    if a.quant_bvh:
        args.flags = args.flags | 16  # PHX_F_QUANT_BVH
    if a.host_bvh:
        args.flags = args.flags | 32  # PHX_F_HOST_BVH
    if a.leaf_size:
        args.bvh_leaf_size = a.leaf_size
    scene = P.SceneData.generate(cfg["kind"], seed=1, width=args.width, height=args.height, detail=cfg["detail"])
    r = P.Renderer(args, device=local)
    r.set_scene(scene)
    if a.simple or a.persistent or a.concurrent_passes or a.pipeline_rounds is not None:
        t = r.tuning()
        if a.simple or a.persistent:
            t.persistent = 1 if a.persistent else 0
        if a.concurrent_passes:
            t.concurrent_passes = 1
        if a.pipeline_rounds is not None:
            t.pipeline_rounds = a.pipeline_rounds
        r.set_tuning(t)
    tuned = None
    if a.autotune:
        tt = r.autotune(4)
        tuned = {f: getattr(tt, f) for f, _ in tt._fields_ if f != "reserved"}
    ext = torch.cuda.ExternalStream(r.stream(), device=local)
    r.iterate(max(3, a.warmup))

    def barrier():
        torch.cuda.synchronize(local)
        if dist is not None:
            dist.barrier()

    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(ext)
        r.iterate(a.steps)
        ev1.record(ext)
        ev1.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    if dist is not None:
        t = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    info = r.info()
    value = world * args.photons_per_round * a.steps / (ms / 1e3) / 1e6

    # per-stage CUDA-event durations over K profiled replays (same graph plus event nodes)
    r.profile(True)
    r.iterate(a.steps)
    stages = r.stage_ms()
    r.profile(False)
    info = r.info()
    n_s = info.n_photons
    Pn = info.n_pixels
    C = info.bucket_count
    ntri = scene.n_triangles
    peak, peak_kind = load_peaks()
    algo = algorithmic_bytes(Pn, n_s, C, ntri)
    per_stage = {}
    for k, parts in STAGE_MAP.items():
        t = sum(stages[x] for x in parts)
        per_stage[k] = {"kernels": parts, "ms": round(t, 4), "algo_bytes": algo[k],
                        "gbs": round(algo[k] / (t * 1e-3) / 1e9, 1) if t > 0 else None,
                        "frac": round(algo[k] / (t * 1e-3) / 1e9 / peak, 5) if t > 0 else None,
                        "traffic": NCU_TRAFFIC.get(a.config, {}).get(k) if a.scale == 1 else None}
    dom = max(per_stage, key=lambda k: per_stage[k]["ms"])
    achieved = algo[dom] / (per_stage[dom]["ms"] * 1e-3) / 1e9
    traffic = NCU_TRAFFIC.get(a.config, {}).get(dom) if a.scale == 1 else None
    roofline = {"bound": "hbm", "kernel": dom, "kernels": STAGE_MAP[dom], "achieved": round(achieved, 2),
                "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 5), "traffic": traffic,
                "peak_source": peak_kind, "per_stage": per_stage}
    # the whole iteration against the same peak: all stages' compulsory bytes over the iteration
    it_bytes = sum(algo.values())
    roofline["iteration"] = {"algo_bytes": it_bytes, "ms": round(ms / a.steps, 4),
                             "gbs": round(it_bytes / (ms / a.steps * 1e-3) / 1e9, 1),
                             "frac": round(it_bytes / (ms / a.steps * 1e-3) / 1e9 / peak, 5)}
    # traversal rates of the dominant kernels (not HBM bound): camera paths, shadow rays (every
    # diffuse hit point's direct_samples rays plus the deferred specular samples), photon paths
    hit = int((r.read("HP_EMISSION")[:, 3] == 1.0).sum())
    shadow_rays = hit * args.direct_samples + info.spec_samples
    rays = {"camera_paths_per_s": Pn / (stages["trace"] * 1e-3), "photon_paths_per_s":
            args.photons_per_round / (stages["emit"] * 1e-3), "shadow_rays_per_round": shadow_rays,
            "shadow_rays_per_s": shadow_rays / (stages["shadow"] * 1e-3)}

    # end to end through the public API: host seed in (pinned H2D), one round, 8-bit image out
    host_rng = [0]

    def pcg_seed(seed):
        s = (2891336453 + seed) & 0xFFFFFFFF
        return (s * 747796405 + 2891336453) & 0xFFFFFFFF

    def random_u32():
        old = host_rng[0]
        host_rng[0] = (old * 747796405 + 2891336453) & 0xFFFFFFFF
        return (((old >> ((old >> 28) + 4)) ^ old) * 277803737) & 0xFFFFFFFF

    host_rng[0] = pcg_seed(args.seed + 1)
    for _ in range(2):
        r.round_seeded(random_u32())
        r.image_u8()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    for _ in range(a.steps):
        r.round_seeded(random_u32())
        img = r.image_u8()
    e1.record(ext)
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    if dist is not None:
        t = torch.tensor([e2e_ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e = {"value": world * args.photons_per_round * a.steps / (e2e_ms / 1e3) / 1e6, "unit": METRIC,
           "h2d_bytes_per_step": 4, "d2h_bytes_per_step": int(img.nbytes),
           "ms_per_step": e2e_ms / a.steps}
    kernels = info.kernels_per_round

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_oracle_sample(cfg, threads=os.cpu_count() or 1)
    r.close()
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return None
    return {"metric": METRIC, "value": round(value, 3), "unit": METRIC, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(ms / a.steps, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": {"workload": a.config, "desc": cfg["desc"], "form": "CUDA-graph replay, all stages on device",
                       "l2": "per-iteration working set (~0.4 GB) larger than L2; scene geometry L2-resident",
                       "parallelism": f"replicas x{world}", "stored_photons": n_s, "pixels": Pn,
                       "cells": C, "autotuned": tuned},
            "roofline": roofline, "rays": rays, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": kernels * a.steps, "kernels_per_round": kernels, "clocks": clk.summary()}


def run_batch16(a) -> dict:
    """The 16-scene batch workload: uneven scenes, all advanced per launch from one captured graph, against the
    plain per-pass form running the scenes one after another."""
    import torch

    import phosphor_b200 as P
    from phosphor_b200 import rmse as R
    specs = R.uneven_batch_specs()
    scenes = [s.scene() for s in specs]
    photons = sum(s.photons for s in specs)
    b = P.Batch(scenes, [s.args() for s in specs])
    ext = torch.cuda.ExternalStream(b.stream())
    b.iterate(max(3, a.warmup), graph=True)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        e0.record(ext)
        b.iterate(a.steps, graph=True)
        e1.record(ext)
        e1.synchronize()
    ms = e0.elapsed_time(e1) / a.steps
    b.profile(True)
    b.iterate(a.steps, graph=True)
    stages = b.stage_ms()
    b.close()
    plain = []
    for s, sc in zip(specs, scenes):
        r = P.Renderer(s.args())
        r.set_scene(sc)
        r.round()
        t0 = time.perf_counter()
        for _ in range(a.steps):
            r.round()
        plain.append((time.perf_counter() - t0) / a.steps)
        r.close()
    plain_ms = 1e3 * sum(plain)
    return {"metric": METRIC, "value": round(photons / (ms * 1e-3) / 1e6, 3), "unit": METRIC, "n_gpus": 1,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scenes)",
            "config": {"workload": "batch16",
                       "desc": "16 uneven scenes (12..291k triangles, 256^2..1024^2, 2^16..2^21 photons, alpha "
                               "U[0.6,0.8]) advanced together, one launch per stage, CUDA-graph replay",
                       "photons_per_round": photons, "triangles": [sc.n_triangles for sc in scenes]},
            "plain_sequential": {"value": round(photons / (plain_ms * 1e-3) / 1e6, 3), "unit": METRIC,
                                 "ms_per_round_all_scenes": round(plain_ms, 3),
                                 "ms_per_scene": [round(1e3 * t, 3) for t in plain]},
            "speedup_vs_plain": round(plain_ms / ms, 3), "stage_ms": stages, "clocks": clk.summary()}


# The time-to-RMSE study on the 16-scene uneven batch (target: graph + batched at least 3x faster
# than the plain per-pass form).  At these sizes two independent 1024-round renders still differ by
# RMSE 0.006-0.014, so the references take 8192 rounds; a second, independent 2048-round set
# measures their noise.  The whole study takes about 20 GPU-minutes: it runs as --config ttr16.
TTR_TARGET = 0.01
TTR_REF_ROUNDS = 8192
TTR_REF_CHECK_ROUNDS = 2048
TTR_CHECK = 32
TTR_MAX_ROUNDS = 2048
TTR_PIPELINE = 2               # rounds in flight per graph replay (8 sets of this batch's buffers exceed HBM)
TTR_CAL_SEED_OFFSET = 2000003  # the calibration renders' seeds: independent of the FP64 images' and the study's
TTR_CHECK_SEED_OFFSET = 3000017


def time_to_rmse_batch16(a) -> dict:
    """Time to RMSE <= 0.01 on the uneven batch: 16 scenes from the three generators (12..291k
    triangles, 256^2..1024^2 pixels, 2^16..2^21 photons per round, alpha U[0.6, 0.8]).

    * reference of each scene: TTR_REF_ROUNDS rounds of a long fp32 render with an independent seed
      (a converged CPU FP64 render at this size is out of reach).  Its noise is measured against a
      second independent render of TTR_REF_CHECK_ROUNDS rounds (RMSE^2 = s_ref^2 + s_check^2 with
      s_check^2 ~ 4 s_ref^2 for noise falling as rounds^-1/2), and its agreement with double
      precision on 1/8-scale copies of the same scenes rendered the same way and by the FP64 oracle
      (tests/golden/batch16_fp64_refs.npz);
    * rounds to target R*_s: the first multiple of TTR_CHECK at which the scene's display image
      (output.cpp:40-76, before quantisation) is within the target of its reference; both forms give
      bit-identical images round by round, so R*_s holds for both; a scene that misses by
      TTR_MAX_ROUNDS is charged TTR_MAX_ROUNDS in both;
    * plain form: every scene alone, R*_s rounds of per-pass launches with the reference's two host
      syncs per round, wall clock end to end (scene set-up excluded), its final RMSE checked;
    * graph + batched form: all scenes in one batch, rounds replayed from captured graphs with rounds
      in flight, each scene retired at its R*_s, wall clock end to end (graph capture included)."""
    import numpy as np

    from phosphor_b200 import rmse as R
    specs = R.uneven_batch_specs()
    t0 = time.perf_counter()
    refs = R.batch_images(specs, TTR_REF_ROUNDS, seed_offset=R.RMSE_REF_SEED_OFFSET, pipeline=TTR_PIPELINE)
    t_refs = time.perf_counter() - t0
    check = R.batch_images(specs, TTR_REF_CHECK_ROUNDS, seed_offset=TTR_CHECK_SEED_OFFSET, pipeline=TTR_PIPELINE)
    ref_vs_check = [R.rmse(x, y) for x, y in zip(refs, check)]
    del check
    cal = None
    fx = ROOT / "tests" / "golden" / "batch16_fp64_refs.npz"
    if fx.exists():
        z = np.load(fx)
        small = [R.scaled(s, int(z["scale"])) for s in specs]
        fp64 = [z[f"scene{i}"].astype(np.float64) / 65535.0 for i in range(len(small))]
        imgs = R.batch_images(small, TTR_REF_ROUNDS, seed_offset=TTR_CAL_SEED_OFFSET, pipeline=TTR_PIPELINE)
        cal_rmse = [R.rmse(img, ref) for img, ref in zip(imgs, fp64)]
        # the same photon and camera paths (the FP64 images' seeds and round count): what remains is
        # the arithmetic, fp32 on the GPU against double precision
        same = R.batch_images(small, int(z["rounds"]), seed_offset=R.RMSE_REF_SEED_OFFSET, pipeline=TTR_PIPELINE)
        same_rmse = [R.rmse(img, ref) for img, ref in zip(same, fp64)]
        cal = {"scale": int(z["scale"]), "fp64_rounds": int(z["rounds"]), "fp32_rounds": TTR_REF_ROUNDS,
               "rmse_fp32_ref_vs_fp64": [round(x, 5) for x in cal_rmse], "max": round(max(cal_rmse), 5),
               "rmse_fp32_vs_fp64_same_paths": [round(x, 6) for x in same_rmse],
               "max_same_paths": round(max(same_rmse), 6)}
    r_star, curve = R.rounds_to_target(specs, refs, TTR_TARGET, TTR_MAX_ROUNDS, TTR_CHECK)
    capped = [i for i, r in enumerate(r_star) if r is None]
    r_eff = [TTR_MAX_ROUNDS if r is None else r for r in r_star]
    plain = [R.time_plain_run(s, r) for s, r in zip(specs, r_eff)]
    t_plain = sum(dt for dt, _ in plain)
    plain_rmse = [R.rmse(img, ref) for (_, img), ref in zip(plain, refs)]
    t_batch = R.time_batched_schedule(specs, r_eff, pipeline=TTR_PIPELINE)
    # the scenes that reach the target, alone: the stalled ones (alpha near 0.6: the radius
    # re-initialisation of gather_flux.cl:50-56) never do, in any form
    conv = [i for i, r in enumerate(r_star) if r is not None]
    t_plain_conv = sum(plain[i][0] for i in conv)
    t_batch_conv = R.time_batched_schedule([specs[i] for i in conv], [r_star[i] for i in conv],
                                           pipeline=TTR_PIPELINE) if conv else None
    # the reference's kernel shapes in the plain form, end to end, on the converging scenes
    ref_conv = [R.time_plain_run(specs[i], r_star[i], reference_shaped=True) for i in conv]
    t_ref_conv = sum(dt for dt, _ in ref_conv)
    same_img = all(np.array_equal(img, plain[i][1]) for (_, img), i in zip(ref_conv, conv))
    # the reference's kernel shapes (one thread per item, its median-split tree, NEE inline), per
    # round on a 20-round sample of each scene: a secondary, extrapolated comparison
    t_ref_shape = sum(r * R.time_plain(s, 20, reference_shaped=True) for s, r in zip(specs, r_eff))
    return {"metric": "time to RMSE 0.01 (s), graph + batched vs plain", "target_rmse": TTR_TARGET,
            "workload": "batch16: 16 uneven scenes, 256^2..1024^2 px, 2^16..2^21 photons, alpha U[0.6, 0.8]",
            "reference": f"fp32 GPU render, {TTR_REF_ROUNDS} rounds, independent seed", "reference_s": round(t_refs, 1),
            "reference_vs_independent_check_rmse": [round(x, 5) for x in ref_vs_check],
            "reference_noise_estimate": [round(x / 5 ** 0.5, 5) for x in ref_vs_check],
            "calibration": cal, "scenes": len(specs), "check_every": TTR_CHECK, "round_cap": TTR_MAX_ROUNDS,
            "rounds_to_target": r_star, "capped_scenes": capped,
            "rmse_at_last_check": [round(x, 5) for x in curve[-1][1]] if curve else None,
            "plain_final_rmse": [round(x, 5) for x in plain_rmse],
            "plain_s": round(t_plain, 3), "plain_s_per_scene": [round(dt, 3) for dt, _ in plain],
            "graph_batched_s": round(t_batch, 3), "speedup": round(t_plain / t_batch, 3),
            "alpha": [round(sp.alpha, 4) for sp in specs], "converging_scenes": conv,
            "converging_plain_s": round(t_plain_conv, 3),
            "converging_graph_batched_s": round(t_batch_conv, 3) if t_batch_conv else None,
            "converging_speedup": round(t_plain_conv / t_batch_conv, 3) if t_batch_conv else None,
            "converging_plain_reference_shaped_s": round(t_ref_conv, 3),
            "converging_speedup_vs_reference_shaped": round(t_ref_conv / t_batch_conv, 3) if t_batch_conv else None,
            "reference_shaped_images_identical": same_img,
            "plain_reference_shaped_s_extrapolated": round(t_ref_shape, 2),
            "speedup_vs_reference_shaped": round(t_ref_shape / t_batch, 2)}


def time_to_rmse_full_size() -> dict:
    """The timing half of the full-size study, short enough for the default run: the scenes of the
    uneven batch that reach RMSE 0.01, each given its rounds to target as the full study measured
    them (rmse.UNEVEN_ROUNDS_TO_TARGET; `--config ttr16` re-derives them with its references), in the
    plain per-pass form one scene at a time and in the graph + batched form (autotuned first, each
    scene retired at its count), both end to end; the stalled scenes reach the target in no form."""
    from phosphor_b200 import rmse as R
    specs = R.uneven_batch_specs()
    conv = [i for i, r in enumerate(R.UNEVEN_ROUNDS_TO_TARGET) if r is not None]
    rounds = [R.UNEVEN_ROUNDS_TO_TARGET[i] for i in conv]
    plain = [R.time_plain_run(specs[i], r)[0] for i, r in zip(conv, rounds)]
    info: dict = {}
    t_batch = R.time_batched_schedule([specs[i] for i in conv], rounds, pipeline=TTR_PIPELINE, autotune=True,
                                      info=info)
    return {"workload": "the uneven batch's scenes that reach RMSE 0.01 (256^2..1024^2 px, 2^16..2^21 photons)",
            "scenes": conv, "rounds_to_target": rounds, "plain_s": round(sum(plain), 3),
            "plain_s_per_scene": [round(t, 3) for t in plain], "graph_batched_s": round(t_batch, 3),
            "speedup": round(sum(plain) / t_batch, 3), "autotune_s": round(info.get("autotune_s", 0.0), 2),
            "stalled_scenes": [i for i, r in enumerate(R.UNEVEN_ROUNDS_TO_TARGET) if r is None]}


def time_to_rmse_small(a) -> dict | None:
    """The small-scene study (16 uneven scenes of 32..64 px, 2^14..2^16 photons, converged FP64
    oracle references committed in tests/golden/rmse_refs.npz): rounds to RMSE <= 0.01, and the
    wall time of the graph + batched form (scenes retired at their own round counts) against the
    plain per-pass form, scenes one at a time, timed per round on 40 rounds."""
    import numpy as np

    from phosphor_b200 import rmse as R
    fx = ROOT / "tests" / "golden" / "rmse_refs.npz"
    if not fx.exists():
        return None
    z = np.load(fx)
    specs = R.rmse_batch()
    refs = [z[f"scene{i}"].astype(np.float64) / 65535.0 for i in range(len(specs))]
    max_rounds = 4096
    r_star, curve = R.rounds_to_target(specs, refs, 0.01, max_rounds=max_rounds, check_every=4)
    # a scene that has not reached the target by the cap is charged the cap in both forms
    capped = [i for i, r in enumerate(r_star) if r is None]
    r_eff = [max_rounds if r is None else r for r in r_star]
    t_plain = [R.time_plain(s, 40) for s in specs]
    t_ref = [R.time_plain(s, 40, reference_shaped=True) for s in specs]
    t_batch = R.time_batched(specs, 200)
    t_sched = R.time_batched_schedule(specs, r_eff)
    out = {"target_rmse": 0.01, "reference": f"FP64 oracle, {int(z['rounds'])} rounds, independent seed",
           "scenes": len(specs), "rounds_to_target": r_star, "round_cap": max_rounds, "capped_scenes": capped,
           "final_rmse": [round(x, 5) for x in curve[-1][1]]}
    tp = sum(r * t for r, t in zip(r_eff, t_plain))
    tb = t_sched  # wall time, each scene retired from the batch at its own round count
    tr = sum(r * t for r, t in zip(r_eff, t_ref))
    out.update({"plain_s": round(tp, 3), "graph_batched_s": round(tb, 3), "speedup": round(tp / tb, 2),
                "plain_reference_shaped_s": round(tr, 3), "speedup_vs_reference_shaped": round(tr / tb, 2),
                "plain_ms_per_round": [round(1e3 * t, 3) for t in t_plain],
                "plain_reference_shaped_ms_per_round": [round(1e3 * t, 3) for t in t_ref],
                "batched_ms_per_round": round(1e3 * t_batch, 3),
                "graph_batched_no_retire_s": round(max(r_eff) * t_batch, 3)})
    return out


def run_shard(a, cfg: dict) -> dict | None:
    """One image over N GPUs (strong scaling): rank r traces its pixel range and emits its range of
    photon paths; one NCCL all-gather of the stored photons per round; every rank gathers its own
    pixels (bit-identical to one GPU).  Rounds are host-synchronised (the exchange needs the
    per-rank photon counts)."""
    import datetime

    import torch

    import phosphor_b200 as P
    from phosphor_b200.renderer import nccl_unique_id
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    args = make_args(cfg)
    scene = P.SceneData.generate(cfg["kind"], seed=1, width=args.width, height=args.height, detail=cfg["detail"])
    r = P.Renderer(args, device=local)
    r.set_scene(scene)
    r.shard(rank, world)
    uid = [nccl_unique_id() if rank == 0 else None]
    if dist is not None:
        dist.broadcast_object_list(uid, src=0)
    r.shard_nccl(uid[0])
    ext = torch.cuda.ExternalStream(r.stream(), device=local)
    for _ in range(max(3, a.warmup)):
        r.shard_round()

    def barrier():
        torch.cuda.synchronize(local)
        if dist is not None:
            dist.barrier()

    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(ext)
        for _ in range(a.steps):
            r.shard_round()
        ev1.record(ext)
        ev1.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    if dist is not None:
        tt = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    info = r.info()
    r.close()
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return None
    value = args.photons_per_round * a.steps / (ms / 1e3) / 1e6
    return {"metric": METRIC, "value": round(value, 3), "unit": METRIC, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(ms / a.steps, 4), "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": {"workload": a.config, "desc": cfg["desc"], "form": "sharded rounds, host-synchronised",
                       "parallelism": f"pixel and photon-path shards x{world}, one NCCL photon all-gather per round",
                       "stored_photons": info.n_photons},
            "e2e": {"value": round(value, 3), "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 8 + 4 * world},
            "gpu_launches": info.kernels_per_round * a.steps, "clocks": clk.summary()}


def run_inverse(a) -> dict:
    """Differentiable SPPM: recover 32 materials' base colour and roughness and the sun's power of
    the atrium at 512x512 from target images, Adam 200 steps at lr 1e-2, 2^20 photons per forward
    pass, gradients from the library's adjoint."""
    from phosphor_b200 import inverse as INV
    cfg = INV.InverseConfig()
    if a.scale > 1:
        cfg.width //= a.scale
        cfg.height //= a.scale
        cfg.photons //= a.scale * a.scale
    with ClockSampler(0) as clk:
        res = INV.run(cfg)
    return {"metric": "Adam steps/s (forward + adjoint)", "value": round(1e3 / res["ms_per_step"], 3),
            "unit": "steps/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic (procedural atrium, seeded materials)",
            "config": {"workload": "inverse", "desc": f"atrium {cfg.width}x{cfg.height}, {cfg.photons} photons per "
                                                      f"forward pass, {res['n_params']} parameters, Adam lr {cfg.lr}"},
            "result": res, "clocks": clk.summary()}


def scene_setup_times() -> dict:
    """Scene setup of the caustic (149,862 triangles) and atrium (262,898) scenes: the traversal
    tree built on the host and on the GPU (triangles resident on the device), and the whole
    set_scene with either, as phx_info reports it (trees, uploads)."""
    import numpy as np

    import phosphor_b200 as P
    from phosphor_b200 import _capi as A
    res = {}
    for name, kind, w, h in (("caustic", A.PHX_SCENE_CAUSTIC, 1024, 1024), ("atrium", A.PHX_SCENE_ATRIUM, 1920, 1080)):
        scene = P.SceneData.generate(kind, seed=1, width=w, height=h)
        host = P.traversal_bvh(scene, 4, True, -1)
        P.traversal_bvh(scene, 4, True, 0)  # warm-up (module load, allocations)
        dev = P.traversal_bvh(scene, 4, True, 0)
        same = bool(np.array_equal(host.nodes.view(np.uint32), dev.nodes.view(np.uint32)) and
                    np.array_equal(host.trirec.view(np.uint32), dev.trirec.view(np.uint32)))
        row = {"triangles": scene.n_triangles, "traversal_tree_host_ms": round(host.build_ms, 2),
               "traversal_tree_gpu_ms": round(dev.build_ms, 2), "identical": same}
        for tag, flags in (("host", A.PHX_F_HOST_BVH), ("gpu", 0)):
            args = P.ArgsList(width=w, height=h, photons_per_round=1 << 16, flags=flags)
            with P.Renderer(args) as r:
                r.set_scene(scene)
                info = r.info()
            row[f"set_scene_{tag}_ms"] = round(info.setup_ms, 1)
            row[f"trees_{tag}_ms"] = round(info.bvh_build_ms, 1)
        res[name] = row
    return res


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=list(CONFIGS) + ["batch16", "inverse", "ttr16"], default="caustic")
    ap.add_argument("--no-rmse", action="store_true", help="skip the time-to-RMSE study (1 GPU only)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-inverse", action="store_true", help="skip the inverse-rendering block (1 GPU only)")
    ap.add_argument("--no-setup", action="store_true", help="skip the scene-setup (tree build) timings")
    ap.add_argument("--simple", action="store_true", help="one-thread-per-item kernels instead of lane refill")
    ap.add_argument("--persistent", action="store_true", help="lane-refill state-machine kernels")
    ap.add_argument("--binary-bvh", action="store_true", help="traverse child pairs instead of 4-wide nodes")
    ap.add_argument("--quant-bvh", action="store_true", help="4-wide nodes with 8-bit child boxes")
    ap.add_argument("--host-bvh", action="store_true", help="build the traversal tree on the host")
    ap.add_argument("--leaf-size", type=int, default=0, help="triangles per leaf of the traversal tree (0: library default)")
    ap.add_argument("--autotune", action="store_true", help="run the library autotuner before timing")
    ap.add_argument("--shard", action="store_true",
                    help="one image over all GPUs (strong scaling) instead of one replica per GPU")
    ap.add_argument("--pipeline-rounds", type=int, default=None,
                    help="rounds each graph replay captures and overlaps (1 = off; default: the library's)")
    ap.add_argument("--concurrent-passes", action="store_true",
                    help="camera and photon passes on two branches of the captured round")
    ap.add_argument("--scale", type=int, default=1,
                    help="divide the resolution by s and the photon count by s^2 (small profiling cases only)")
    a = ap.parse_args()
    a.warmup = max(3, a.warmup)
    if a.config == "batch16":
        if a.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "batch16 has no reference arm; use --config"
                              " caustic"}))
            return 0
        print(json.dumps(run_batch16(a)))
        return 0
    if a.config == "ttr16":
        if a.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the time-to-RMSE study compares two forms of "
                              "this library; use --config caustic"}))
            return 0
        print(json.dumps(time_to_rmse_batch16(a)))
        return 0
    if a.config == "inverse":
        if a.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no adjoint; use --config"
                              " caustic"}))
            return 0
        print(json.dumps(run_inverse(a)))
        return 0
    cfg = dict(CONFIGS[a.config])
    if a.scale > 1:
        cfg.update(width=cfg["width"] // a.scale, height=cfg["height"] // a.scale,
                   photons=max(1, cfg["photons"] // (a.scale * a.scale)),
                   desc=cfg["desc"] + f" (scaled 1/{a.scale} for profiling; not a bench value)")
    if a.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        print(json.dumps(run_reference(a, cfg)))
        return 0
    out = run_shard(a, cfg) if a.shard else run_ours(a, cfg)
    if out is not None:
        if not a.no_rmse and out["n_gpus"] == 1 and a.scale == 1:
            out["time_to_rmse"] = time_to_rmse_small(a)
        if not a.no_rmse and out["n_gpus"] == 1 and a.scale == 1:
            out["time_to_rmse_full_size"] = time_to_rmse_full_size()
        if not a.no_setup and out["n_gpus"] == 1 and a.scale == 1:
            out["scene_setup"] = scene_setup_times()
        if not a.no_inverse and out["n_gpus"] == 1 and a.scale == 1:
            # inverse rendering through the adjoint (atrium 512x512, 200 Adam steps)
            inv = run_inverse(a)
            out["inverse"] = {"steps_per_s": inv["value"], "desc": inv["config"]["desc"], **{
                k: inv["result"][k] for k in ("steps", "n_params", "common_random_numbers", "observed_materials_base",
                                              "observed_materials_roughness", "loss_first", "loss_last",
                                              "error_start", "error_end", "ms_per_step")}}
        print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
