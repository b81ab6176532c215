"""Benchmark of the plain wavefront path tracer on the terrain workload.

Workload (one step): heightfield terrain on a 1024x1024 grid (2,093,058 triangles, 6 octaves of
seeded value noise, amplitude 0.2) plus 64 instanced level-5 icospheres (20,480 triangles each)
under seeded transforms, GLTF metallic-roughness materials, a 512x256 procedural HDR sky with a 5e3
sun lobe over 0.5 degrees; 1920x1080 pixels, 64 samples per pixel, path length 3..12 with Russian
roulette.  The BVH and triangles (~200 MB) exceed the 126 MB L2, so no flush is needed between
steps.

Metric: Mrays/s = (extension + shadow rays traced) / GPU time, summed over all ranks.
Multi-GPU (torchrun): every rank renders the same view with its own frame seeds (weak scaling),
and the per-rank images are summed into rank 0 with one NCCL reduce per step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SPP = 64
MIN_LEN, MAX_LEN = 3, 12
WORKLOAD = ("terrain 1024^2 grid (2.09M tris) + 64 icospheres (1.31M tris), GLTF MR materials, 512x256 HDR sky "
            "with 5e3 sun; 1920x1080, 64 spp, path length 3..12, Russian roulette")
# Algorithmic bytes of one closest-hit query: ray read + hit write + one 128-byte node line per node
# fetch + one 48-byte record per triangle fetch, with the fetch counts of the sequential
# nearest-first BVH8 walk (the counting run).  NODE_PAYLOAD is the node's 80 bytes of content.
NODE_BYTES, NODE_PAYLOAD, TRI_BYTES, RAY_BYTES, HIT_BYTES = 128, 80, 48, 32, 16
SHADOW_RAY_BYTES = 64  # shadow-ray record read: origin + t_max, direction + slot, contribution
# Algorithmic bytes of shading: a path's 64-byte state read, the 64-byte material record, 3 x (4-byte
# index + 32 bytes of position/normal/uv), the 64-byte state written for a continuation ray, and a
# 48-byte shadow-ray record per NEE sample.
SHADE_IN_BYTES, SHADE_MAT_BYTES, SHADE_ATTR_BYTES, SHADE_OUT_BYTES, SHADOW_REC_BYTES = 64, 64, 3 * (4 + 32), 64, 48
GOLDEN_CFG5 = ROOT / "tests" / "golden" / "cfg5_1920x1080_subset30_fp64_262144spp.npz"
RELMSE_TARGET = 0.01
CACHE_WARMUP_FRAMES = 64      # radiance-cache forms: training frames before accumulation starts
CACHE_MIN_ROUGHNESS = 0.35    # path regularisation of the extra regularised 2-bounce line
# environment sampling of every estimator on the learned-cache scene: the bilinear-footprint pdf,
# whose expected image equals the texel pdf's (the sun of one texel otherwise leaves its bilinear
# halo to BSDF sampling)


def peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d.get("bf16_tflops", 1590.0)), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def bench_config(world: int, triangles: int) -> dict:
    """The `config` object of both arms' JSON lines (identical keys and values)."""
    return {"workload": WORKLOAD, "width": 1920, "height": 1080, "spp": SPP, "min_path_length": MIN_LEN,
            "max_path_length": MAX_LEN, "triangles": int(triangles), "l2": "inputs larger than L2 (no flush)",
            "parallelism": f"dp{world}: disjoint sample seeds per rank, images summed into rank 0"}


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        """Starts sampling and waits (up to 5 s) for the first sample, so that the samples cover the
        timed region that follows even when it lasts well under a second."""
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
            return
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < 5.0 and self.proc.poll() is None:
            if Path(self.file.name).stat().st_size > 0:
                break
            time.sleep(0.02)

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        rows = [r.split(",") for r in Path(self.file.name).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        if not sm:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows if len(r) >= 9 for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(rows[0][2]), "samples": len(sm), "reasons": reasons}


def cpu_oracle(wl):
    """FP32 build of the oracle (the CPU restatement of the same path), used as the CPU baseline."""
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle_lib import OracleScene  # noqa: E402 (checker code: CPU baseline leg only)
    return OracleScene(wl.scene, 2)


def cpu_stride(osc, wl, p, seconds: float, threads: int) -> int:
    """Pixel stride whose render takes about `seconds` on the host cores."""
    probe = 24
    t0 = time.perf_counter()
    osc.render(wl.view, p, wl.width, wl.height, precision=32, stride=probe, threads=threads)
    dt = time.perf_counter() - t0
    per_px = dt / (len(range(0, wl.height, probe)) * len(range(0, wl.width, probe)))
    return max(2, int(np.sqrt(wl.width * wl.height * per_px / max(seconds, 0.5))))


def cpu_sample(osc, wl, p, stride: int, threads: int) -> dict:
    """Times the oracle's FP32 build on every `stride`-th pixel of the workload."""
    t0 = time.perf_counter()
    r = osc.render(wl.view, p, wl.width, wl.height, precision=32, stride=stride, threads=threads)
    dt = time.perf_counter() - t0
    rays = r["extension_rays"] + r["shadow_rays"]
    npx = len(range(0, wl.height, stride)) * len(range(0, wl.width, stride))
    return {"rays": rays, "seconds": dt, "mrays_per_s": rays / dt / 1e6, "pixels": npx, "stride": stride}


def params(dev, spp: int, seed: int, flags: int = 0):
    p = dev.default_params() if dev is not None else None
    if p is None:
        from stratum2_b200 import _abi
        p = _abi.S2RenderParams()
        _abi.lib().s2_default_render_params(p)
    p.spp, p.frame_seed, p.min_path_length, p.max_path_length, p.flags = spp, seed, MIN_LEN, MAX_LEN, flags
    return p


def run_reference(args, rank: int, world: int):
    """Reference arm: the CPU restatement of the path on the host cores (the reference's own
    Vulkan/Slang implementation cannot be built or run here)."""
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle_lib import default_render_params  # noqa: E402 (the oracle's defaults: no product library)
    from stratum2_b200.scenegen import terrain_scene
    wl = terrain_scene()
    p = default_render_params()
    p.spp, p.min_path_length, p.max_path_length = SPP, MIN_LEN, MAX_LEN
    threads = os.cpu_count() or 1
    osc = cpu_oracle(wl)
    stride = cpu_stride(osc, wl, p, 5.0, threads)
    total_rays = 0.0
    total_s = 0.0
    for step in range(args.warmup + args.steps):
        p.frame_seed = 1000 * step
        r = cpu_sample(osc, wl, p, stride, threads)
        if step >= args.warmup:
            total_rays += r["rays"]
            total_s += r["seconds"]
    v = total_rays / total_s / 1e6
    line = {"metric": "Mrays/s", "value": v, "unit": "Mrays/s", "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene generator, no datasets)", "config": bench_config(world, wl.scene.triangle_count),
            "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": threads, "kind": "port",
                             "sample": f"pixel subset (stride {r['stride']}, {r['pixels']} pixels) x {SPP} spp per step"},
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank: int, world: int, local_rank: int):
    import torch
    import torch.distributed as dist

    from stratum2_b200 import Device, _abi
    from stratum2_b200.scenegen import terrain_scene

    torch.cuda.set_device(local_rank)
    dev = Device(local_rank)
    stream = torch.cuda.current_stream()
    dev.set_stream(stream.cuda_stream)
    wl = terrain_scene()
    dev.upload_scene(wl.scene)
    W, H = wl.width, wl.height
    rad = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    aovs = _abi.S2Aovs(rad.data_ptr(), None, None, None, None, None)

    from stratum2_b200.multi import combine_images, frame_seed, job_time_and_totals

    def seed(step: int) -> int:
        return frame_seed(step, rank, world, SPP)  # disjoint frame seeds per rank and step

    # autotuning (untimed set-up): wave size and traversal knobs for this workload
    tuning = None
    if not args.no_autotune:
        from stratum2_b200 import autotune
        tuning = autotune.autotune(dev, wl.view, params(dev, SPP, 7777), path=Path(tempfile.gettempdir()) / "s2_bench_tuning.json",
                                   force=True)
    # fetch counts for the algorithmic-byte model (untimed run, same seeds as timed step 0)
    cnt = dev.render_device(wl.view, params(dev, SPP, seed(0), _abi.FLAG_COUNT_FETCHES), aovs)
    for w in range(args.warmup):
        dev.render_device(wl.view, params(dev, SPP, seed(w + 1000)), aovs)
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    e0.record(stream)
    for step in range(args.steps):
        stats.append(dev.render_device(wl.view, params(dev, SPP, seed(step), _abi.FLAG_PROFILE_KERNELS), aovs))
        combine_images(rad, world, dist)  # sum the ranks' sample partitions of the frame into rank 0
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    rays = float(sum(s.extension_rays + s.shadow_rays for s in stats))
    paths = float(sum(s.paths for s in stats))
    ms, (rays, paths) = job_time_and_totals(ms, [rays, paths], world, dist, device="cuda")
    value = rays / ms / 1e3

    # end to end through the public API with host buffers (view/params in, all AOVs out into
    # page-locked frame buffers reused from frame to frame, as a viewer or encoder holds them)
    dev.set_stream(None)
    host_out = dev.host_result(W, H, pinned=True)
    for w in range(1):
        dev.render(wl.view, W, H, params=params(dev, SPP, seed(w + 2000)), out=host_out)
    t0 = time.perf_counter()
    e2e_rays = 0
    for step in range(args.steps):
        r = dev.render(wl.view, W, H, params=params(dev, SPP, seed(step + 3000)), out=host_out)
        e2e_rays += r.stats.extension_rays + r.stats.shadow_rays
    e2e_s = time.perf_counter() - t0
    e2e_s, (e2e_rays,) = job_time_and_totals(e2e_s, [float(e2e_rays)], world, dist, device="cuda")
    if rank != 0:
        return

    # roofline of the dominant kernel
    ext_ms = sum(s.extend_ms for s in stats); sh_ms = sum(s.shade_ms for s in stats); oc_ms = sum(s.occlude_ms for s in stats)
    ext_launches = sum(s.extend_launches for s in stats)
    ext_rays = sum(s.extension_rays for s in stats)
    n_node = cnt.extend_node_fetches / max(cnt.extension_rays, 1)
    n_tri = cnt.extend_tri_fetches / max(cnt.extension_rays, 1)
    bytes_per_ray = RAY_BYTES + HIT_BYTES + NODE_BYTES * n_node + TRI_BYTES * n_tri
    payload_per_ray = RAY_BYTES + HIT_BYTES + NODE_PAYLOAD * n_node + TRI_BYTES * n_tri
    rays_per_launch = ext_rays / max(ext_launches, 1)
    avg_launch_s = ext_ms / 1e3 / max(ext_launches, 1)
    # with shadow merging (the default) the timed traversal launches also trace the previous
    # bounce's shadow rays (the last bounce casts none: NEE needs a vertex below the maximum length)
    merged = dev.get_tuning().shadow_merge == _abi.SHADOW_MERGE_ON
    n_sh_node = cnt.shadow_node_fetches / max(cnt.shadow_rays, 1)
    n_sh_tri = cnt.shadow_tri_fetches / max(cnt.shadow_rays, 1)
    sh_bytes_per_ray = SHADOW_RAY_BYTES + NODE_BYTES * n_sh_node + TRI_BYTES * n_sh_tri
    sh_rays = sum(s.shadow_rays for s in stats) if merged else 0
    launch_bytes = (bytes_per_ray * ext_rays + sh_bytes_per_ray * sh_rays) / max(ext_launches, 1)
    achieved = launch_bytes / avg_launch_s / 1e9
    pk = peaks()
    trace_name = "k_trace (closest hits + the previous bounce's shadow rays)" if merged else "k_extend"
    dominant = max([(trace_name, ext_ms), ("k_shade", sh_ms), ("k_occlude", oc_ms)], key=lambda x: x[1])[0]
    roof = {"kernel": trace_name, "dominant_kernel": dominant, "bound": "hbm", "achieved": achieved,
            "peak": pk["hbm_gbs"], "peak_source": pk["source"] + " copy bandwidth", "unit": "GB/s",
            "frac": achieved / pk["hbm_gbs"],
            "traffic": None,
            "traffic_note": "DRAM bytes are not measurable inside the timed run; the ncu figures per launch are "
                            "in profiles/k_extend_terrain.md",
            "algorithmic_bytes_per_launch": launch_bytes,
            "bytes_per_ray": bytes_per_ray,
            "shadow_bytes_per_ray": sh_bytes_per_ray if merged else None,
            "byte_model": "extension ray: 32 ray + 16 hit + 128 per node fetch + 48 per triangle fetch; shadow ray "
                          "(merged launches): 64 record + 128 per node + 48 per triangle fetch; fetch counts of the "
                          "sequential nearest-first BVH8 walk (equal to the CPU BVH8 walker's)",
            "frac_node_payload_80B": (achieved * payload_per_ray / bytes_per_ray / pk["hbm_gbs"]) if not merged else None,
            "node_fetches_per_ray": n_node,
            "tri_fetches_per_ray": n_tri,
            "shadow_node_fetches_per_ray": n_sh_node,
            "avg_launch_ms": avg_launch_s * 1e3,
            "reading": "the byte model counts every node and triangle fetch as a line from HBM; a fraction near "
                       "or above 1 means most fetches are served from L1/L2 (the camera rays of one pixel's "
                       "samples traverse together), and the kernel's measured limit is instruction issue "
                       "(profiles/k_extend_terrain.md)"}
    # shading: the measurement plan's byte model per shaded path vertex (state in, hit, material
    # record, three indices + attributes), per continuation (state out) and per shadow ray record
    sh_launches = sum(s.shade_launches for s in stats)
    shade_bytes = ext_rays * (SHADE_IN_BYTES + HIT_BYTES + SHADE_MAT_BYTES + SHADE_ATTR_BYTES) + \
        (ext_rays - sum(s.paths for s in stats)) * SHADE_OUT_BYTES + sum(s.shadow_rays for s in stats) * SHADOW_REC_BYTES
    sh_achieved = shade_bytes / max(sh_ms, 1e-9) / 1e6
    roof_shade = {"kernel": "k_shade", "bound": "hbm", "achieved": sh_achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                  "frac": sh_achieved / pk["hbm_gbs"], "traffic": None,
                  "algorithmic_bytes_per_launch": shade_bytes / max(sh_launches, 1),
                  "avg_launch_ms": sh_ms / max(sh_launches, 1),
                  "byte_model": "per shaded vertex 64 state in + 16 hit + 64 material + 108 indices/attributes; "
                                "64 per continuation ray written; 48 per shadow-ray record (misses counted as hits)"}
    line = {"metric": "Mrays/s", "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator, no datasets)",
            "config": bench_config(world, wl.scene.triangle_count),
            "bvh8_nodes": int(dev.bvh_stats.node_count),
            "tuning": {"values": (tuning or {}).get("tuning", "defaults"), "autotune_trials": (tuning or {}).get("trials", 0)},
            "mpaths_per_s": paths / ms / 1e3,
            "kernel_ms_per_step": {("k_trace" if merged else "k_extend"): ext_ms / args.steps, "k_shade": sh_ms / args.steps,
                                   "k_occlude": oc_ms / args.steps},
            "gpu_launches": int(sum(s.kernel_launches for s in stats)),
            "roofline": roof,
            "roofline_shade": roof_shade,
            "e2e": {"value": e2e_rays / e2e_s / 1e6, "unit": "Mrays/s",
                    "h2d_bytes_per_step": int(C_sizeof_view_params()),
                    "d2h_bytes_per_step": int(W * H * (16 + 16 + 8 + 16 + 8 + 8)),
                    "host_buffers": "page-locked, reused across steps; first-hit AOV copies overlap the later bounces",
                    "clock": "host wall clock around s2_render calls (max over ranks)"},
            "clocks": ck}
    if world == 1 and not args.no_quality:
        line["batched_16_views"] = batched_line(dev, args.steps)
        if GOLDEN_CFG5.exists():
            line["time_to_relmse_0.01"] = quality_line(dev, args)
    if world == 1 and not args.no_quality:
        line["radiance_cache_kernels"] = cache_kernel_line(dev, args.steps)
        line["adjoint"] = adjoint_line(dev)
        line["restir_many_lights"] = restir_line(dev)
        line["vcm_many_lights"] = vcm_line(dev)
    if world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        osc = cpu_oracle(wl)
        pc = params(None, SPP, 0)
        c = cpu_sample(osc, wl, pc, cpu_stride(osc, wl, pc, args.cpu_seconds, threads), threads)
        line["cpu_baseline"] = {"value": c["mrays_per_s"], "unit": "Mrays/s", "cores": threads, "kind": "port",
                                "sample": f"FP32 oracle, every {c['stride']}th pixel ({c['pixels']} pixels) x {SPP} spp, "
                                          f"{c['seconds']:.1f} s"}
    print(json.dumps(line), flush=True)


def batched_views(seed: int = 7, n: int = 16):
    """16 camera views of the terrain with resolutions log-uniform between 256x256 and 1920x1080."""
    from stratum2_b200.scene import look_at_rotation, make_view
    rng = np.random.default_rng(seed)
    views = []
    for _ in range(n):
        w = int(round(np.exp(rng.uniform(np.log(256), np.log(1920)))))
        h = int(round(np.exp(rng.uniform(np.log(256), np.log(1080)))))
        pos = (rng.uniform(-0.9, 0.9), rng.uniform(0.5, 1.2), rng.uniform(1.2, 2.0))
        views.append(make_view(pos, w, h, 45.0, look_at_rotation(pos, (0.0, 0.0, 0.0))))
    return views


def quality_line(dev, args) -> dict:
    """Time to relMSE 0.01 on the learned-cache scene (the terrain workload with 8 area lights,
    1920x1080, path length 3..12, against its FP64 oracle image on a 64x36 pixel subset): the plain
    unbiased path tracer against the radiance-cache forms (paths end in the cache after 1 or 2
    bounces, online training, in the wave entry point and in the batched streaming entry point)."""
    from stratum2_b200.scenegen import terrain_scene
    wl = terrain_scene(area_lights=8)
    dev.upload_scene(wl.scene)
    g = np.load(GOLDEN_CFG5)
    out = {"workload": "terrain 1024^2 + 64 icospheres + 8 area lights, 512x256 sky with 5e3 sun; 1920x1080, path "
                       "length 3..12, Russian roulette",
           "reference_image": f"FP64 oracle, {int(g['spp'])} spp, 64x36 pixel subset (stride 30)",
           "plain": plain_quality(dev, wl, g, args.quality_chunks),
           "cached_1_bounce": cached_quality(dev, wl, g, False, 1, 0.0),
           "cached_2_bounces": cached_quality(dev, wl, g, False, 2, 0.0),
           "batched_cached_2_bounces": cached_quality(dev, wl, g, True, 2, 0.0),
           "cached_2_bounces_regularised": cached_quality(dev, wl, g, False, 2, CACHE_MIN_ROUGHNESS),
           "note": "plain: expected GPU time of the unbiased estimator from the mean relMSE of independent 64-spp "
                   "calls (relMSE ~ 1/spp); cached: measured GPU time of 1-spp frames with online training "
                   f"({CACHE_WARMUP_FRAMES} training frames, then progressive accumulation), including the training "
                   f"frames; the regularised line raises roughness to >= {CACHE_MIN_ROUGHNESS} after the first bounce; "
                   "every estimator samples the environment by its bilinear footprint (S2_FLAG_ENV_FOOTPRINT_PDF)"}
    plain_ms = out["plain"]["ms"]
    for k in ("cached_1_bounce", "cached_2_bounces", "batched_cached_2_bounces", "cached_2_bounces_regularised"):
        if out[k]["ms"] is not None:
            out[k]["fraction_of_plain_time"] = out[k]["ms"] / plain_ms
    return out


def _subset(rad, g):
    x0, y0, st = int(g["rect"][0]), int(g["rect"][1]), int(g["stride"])
    ref = g["mean"]
    return rad[y0::st, x0::st, :3].double().cpu().numpy()[:ref.shape[0], :ref.shape[1]]


def _ref_noise(g):
    ref = g["mean"].astype(np.float64)
    return ref, float(np.mean(g["var_of_mean"].astype(np.float64) / (ref ** 2 + 1e-2)))


def quality_flags():
    from stratum2_b200 import _abi
    return _abi.FLAG_ENV_FOOTPRINT_PDF


def plain_quality(dev, wl, g, chunks: int, chunk: int = 64) -> dict:
    """Plain unbiased path tracing: `chunks` independent `chunk`-spp renders; the expected GPU time
    to relMSE 0.01 is (mean single-chunk relMSE x chunk / 0.01) spp at the measured time per spp (the
    estimator's relMSE falls as 1/spp); the cumulative image's relMSE is reported beside it."""
    import torch

    from stratum2_b200 import _abi
    from stratum2_b200.metrics import relmse
    ref, noise = _ref_noise(g)
    rad = torch.zeros((wl.height, wl.width, 4), dtype=torch.float32, device="cuda")
    aovs = _abi.S2Aovs(rad.data_ptr(), None, None, None, None, None)
    ms, rms, acc = 0.0, [], None
    for k in range(chunks):
        s = dev.render_device(wl.view, params(dev, chunk, 50000 + chunk * k, quality_flags()), aovs)
        ms += s.gpu_ms
        sub = _subset(rad, g)
        rms.append(relmse(sub, ref) - noise)
        acc = sub if acc is None else acc + sub
    per_spp = float(np.mean(rms)) * chunk
    ms_per_spp = ms / (chunks * chunk)
    return {"ms": per_spp / RELMSE_TARGET * ms_per_spp, "measured_to_target": False,
            "relmse_per_spp_mean": per_spp, "relmse_per_spp_median": float(np.median(rms)) * chunk,
            "ms_per_spp": ms_per_spp, "spp_run": chunks * chunk, "gpu_ms_run": ms,
            "relmse_cumulative": relmse(acc / chunks, ref) - noise}


def cached_quality(dev, wl, g, batched: bool, bounces: int, rough: float, max_ms: float = 12000.0) -> dict:
    """Radiance-cache form: a freshly initialised cache, CACHE_WARMUP_FRAMES 1-spp frames that only
    train it, then progressive 1-spp frames (S2_FLAG_ACCUMULATE) until the relMSE against the FP64
    image reaches 0.01 or `max_ms` of GPU time; the GPU time of every frame counts."""
    import torch

    from stratum2_b200 import _abi
    from stratum2_b200.metrics import relmse
    ref, noise = _ref_noise(g)
    rad = torch.zeros((wl.height, wl.width, 4), dtype=torch.float32, device="cuda")
    aovs = _abi.S2Aovs(rad.data_ptr(), None, None, None, None, None)
    dev.cache_init()
    ms, frames, rm, curve = 0.0, 0, float("inf"), []
    while ms < max_ms:
        acc = frames > CACHE_WARMUP_FRAMES
        p = params(dev, 1, 70000 + frames, quality_flags() | _abi.FLAG_RADIANCE_CACHE | (_abi.FLAG_ACCUMULATE if acc else 0))
        p.cache_bounces = bounces
        p.cache_min_roughness = rough
        s = dev.render_views_device([wl.view], p, [aovs]) if batched else dev.render_device(wl.view, p, aovs)
        ms += s.gpu_ms
        frames += 1
        if frames <= CACHE_WARMUP_FRAMES:
            continue
        n = frames - CACHE_WARMUP_FRAMES
        if n % 8 == 0 or n < 8:
            rm = relmse(_subset(rad, g), ref) - noise
            if n in (8, 32, 128, 512, 2048) or rm <= RELMSE_TARGET:
                curve.append([n, round(ms, 1), round(rm, 5)])
            if rm <= RELMSE_TARGET:
                break
    reached = rm <= RELMSE_TARGET
    return {"ms": ms if reached else None, "measured_to_target": reached, "frames": frames, "gpu_ms_run": ms,
            "ms_per_frame": ms / max(frames, 1), "relmse": rm, "curve_frames_ms_relmse": curve,
            "cache_bounces": bounces, "min_roughness": rough, "entry_point": "s2_render_views" if batched else "s2_render"}


def batched_line(dev, steps: int, spp: int = 8) -> dict:
    """The 16-view batched form in one s2_render_views call per step (device AOV buffers)."""
    import torch

    from stratum2_b200 import _abi
    views = batched_views()
    bufs, outs = [], []
    for v in views:
        w, h = v.image_max[0] - v.image_min[0], v.image_max[1] - v.image_min[1]
        t = torch.zeros((h, w, 4), dtype=torch.float32, device="cuda")
        bufs.append(t)
        outs.append(_abi.S2Aovs(t.data_ptr(), None, None, None, None, None))
    dev.render_views_device(views, params(dev, spp, 77), outs)  # warm-up (builds the graphs)
    ms, rays, paths, launches = 0.0, 0, 0, 0
    for k in range(steps):
        s = dev.render_views_device(views, params(dev, spp, 100 + k * spp), outs)
        ms += s.gpu_ms
        rays += s.extension_rays + s.shadow_rays
        paths += s.paths
        launches += s.kernel_launches
    # the same views one s2_render call each, for comparison
    ms_seq, rays_seq = 0.0, 0
    for k in range(steps):
        for v, o in zip(views, outs):
            s = dev.render_device(v, params(dev, spp, 100 + k * spp), o)
            ms_seq += s.gpu_ms
            rays_seq += s.extension_rays + s.shadow_rays
    pixels = sum((v.image_max[0] - v.image_min[0]) * (v.image_max[1] - v.image_min[1]) for v in views)
    return {"views": len(views), "pixels": int(pixels), "spp": spp, "steps": steps,
            "mrays_per_s": rays / ms / 1e3, "mpaths_per_s": paths / ms / 1e3, "ms_per_step": ms / steps,
            "gpu_launches": int(launches), "per_view_calls_mrays_per_s": rays_seq / ms_seq / 1e3}


def cache_kernel_line(dev, steps: int) -> dict:
    """Radiance-cache kernels on their own: inference over 2^21 positions and training steps of
    2^16 records (forward + backward on the tensor cores, table-gradient scatter, Adam on 16.8M
    table and 6,336 weight parameters), device buffers, CUDA-event timing on the library's stream."""
    import torch

    from stratum2_b200 import _abi
    p = _abi.S2CacheParams()
    _abi.lib().s2_cache_default_params(p)
    for k in range(3):
        p.box_min[k], p.box_max[k] = -1.0, 1.0
    dev.cache_init(p)
    stream = torch.cuda.current_stream()
    dev.set_stream(stream.cuda_stream)
    g = torch.Generator(device="cuda").manual_seed(3)
    nq, nt = 1 << 21, 1 << 16
    pos = torch.rand((nq, 4), generator=g, device="cuda") * 2 - 1
    out = torch.empty((nq, 4), device="cuda")
    tpos = torch.rand((nt, 4), generator=g, device="cuda") * 2 - 1
    tgt = torch.rand((nt, 4), generator=g, device="cuda")
    for _ in range(3):
        dev.cache_query_device(pos.data_ptr(), nq, out.data_ptr())
        dev.cache_train_device(tpos.data_ptr(), tgt.data_ptr(), nt)
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record(stream)
    for _ in range(steps):
        dev.cache_query_device(pos.data_ptr(), nq, out.data_ptr())
    e1.record(stream)
    for _ in range(steps):
        dev.cache_train_device(tpos.data_ptr(), tgt.data_ptr(), nt)
    e2.record(stream)
    torch.cuda.synchronize()
    dev.set_stream(None)
    inf_ms, tr_ms = e0.elapsed_time(e1) / steps, e1.elapsed_time(e2) / steps
    flop_q = 2 * 6336
    pk = peaks()
    inf_tflops = flop_q * nq / inf_ms / 1e9
    return {"inference": {"queries": nq, "ms": inf_ms, "mqueries_per_s": nq / inf_ms / 1e3, "tflops": inf_tflops,
                          "tensor_frac_of_measured_bf16": inf_tflops / pk["bf16_tflops"],
                          "table_gather_gbs": 512 * nq / inf_ms / 1e6},
            "training_step": {"records": nt, "ms": tr_ms, "mrecords_per_s": nt / tr_ms / 1e3,
                              "note": "forward + backward + table scatter + Adam over all parameters"}}


def adjoint_line(dev, steps: int = 2) -> dict:
    """Differentiable inverse-rendering workload: the box with 200 level-3 icospheres (256k
    triangles), 1024^2 RGB albedo and 1024^2 roughness textures, a 256x128 environment map; 512x512,
    64 spp, path length up to 4.  Forward (s2_render_diff) and adjoint (s2_render_adjoint, two
    replays per path, texel gradients of all three images) timed on the device."""
    import torch

    from stratum2_b200 import _abi
    from stratum2_b200.scenegen import textured_box_scene
    wl = textured_box_scene(n_random=0, width=512, height=512, tex_res=1024, env_res=(256, 128), spheres=200,
                            sphere_level=3)
    dev.upload_scene(wl.scene)
    p = _abi.S2RenderParams()
    _abi.lib().s2_default_render_params(p)
    p.spp, p.min_path_length, p.max_path_length, p.flags, p.frame_seed = 64, 0, 4, _abi.FLAG_PIXEL_JITTER, 1
    img = torch.empty((512, 512, 4), device="cuda")
    d = torch.rand((512, 512, 4), device="cuda")
    grads = [torch.zeros(im.shape[:2] + (4,), device="cuda") for im in wl.scene.images]
    ptrs = [t.data_ptr() for t in grads]
    dev.render_diff_device(wl.view, p, img.data_ptr())
    dev.render_adjoint_device(wl.view, p, d.data_ptr(), ptrs)
    f_ms = b_ms = 0.0
    rays = 0
    for k in range(steps):
        p.frame_seed = 100 + 64 * k
        s = dev.render_diff_device(wl.view, p, img.data_ptr())
        f_ms += s.gpu_ms
        rays += s.extension_rays + s.shadow_rays
        b_ms += dev.render_adjoint_device(wl.view, p, d.data_ptr(), ptrs).gpu_ms
    paths = 512 * 512 * 64
    return {"workload": "box + 200 icospheres (%d triangles), 1024^2 albedo + roughness textures, 256x128 env; "
                        "512x512, 64 spp, max path length 4" % int(dev.bvh_stats.triangle_count),
            "forward_ms": f_ms / steps, "forward_mrays_per_s": rays / f_ms / 1e3,
            "forward_mpaths_per_s": paths / (f_ms / steps) / 1e3, "adjoint_ms": b_ms / steps,
            "adjoint_mpaths_per_s": paths / (b_ms / steps) / 1e3,
            "gradient_texels": int(sum(t.shape[0] * t.shape[1] for t in grads))}


def vcm_line(dev, iterations: int = 3) -> dict:
    """The VCM renderer (s2_render_vcm) on the many-lights frame: the cfg2 terrain carrying 100k
    emissive triangles (the environment is black in this renderer), 1920x1080, paths of up to 6
    segments (the VCM renderer's default), one light subpath per pixel, power-proportional light
    pick.  Device time per iteration (a light pass and a camera pass) and rays traced per second,
    for path tracing, BPT with the light vertex cache (the reference's default algorithm), the same
    with the DI and light-vertex-cache reservoirs (32 and 8 candidates, both reused), BPT connecting to
    whole light subpaths, and VCM."""
    from stratum2_b200 import _abi
    from stratum2_b200.scenegen import terrain_scene
    wl = terrain_scene(emissive_triangles=100_000, emissive_sigma=2.0)
    dev.upload_scene(wl.scene)
    out = {"workload": "cfg2 terrain + 100k emissive triangles, 1920x1080, max path length 6, "
                       "1 light subpath per pixel, Disney BSDF",
           "kernels": "thread-per-path light and camera megakernels on the shared BVH8 traversal"}
    lvc = _abi.VCM_FLAG_LIGHT_VERTEX_CACHE
    for name, algo, fl in (("path_trace", _abi.VCM_PATH_TRACE, 0),
                           ("bpt_light_vertex_cache", _abi.VCM_BPT, lvc),
                           ("bpt_light_vertex_cache_reservoirs", _abi.VCM_BPT,
                            lvc | _abi.VCM_FLAG_LVC_RIS | _abi.VCM_FLAG_LVC_REUSE | _abi.VCM_FLAG_DI_RIS |
                            _abi.VCM_FLAG_DI_REUSE),
                           ("bpt", _abi.VCM_BPT, 0), ("vcm", _abi.VCM_VCM, 0)):
        p = dev.default_vcm_params()
        p.algorithm, p.vcm_flags, p.iterations = algo, fl, 1
        p.flags = _abi.FLAG_LIGHT_POWER_PICK
        p.frame_seed = 7
        dev.render_vcm(wl.view, wl.width, wl.height, p)  # warm-up
        ms = rays = 0.0
        for k in range(iterations):
            p.frame_seed = 100 + k
            st = dev.render_vcm(wl.view, wl.width, wl.height, p).stats
            ms += st.gpu_ms
            rays += st.extension_rays + st.shadow_rays
        out[name] = {"ms_per_iteration": ms / iterations, "mrays_per_s": rays / ms / 1e3}
    return out


def restir_line(dev, frames: int = 32, ref_spp: int = 1024) -> dict:
    """Many-lights ReSTIR DI: the cfg2 terrain carrying 100k small emissive triangles of lognormal(0, 2)
    power, camera animated over `frames` frames along a seeded Catmull-Rom loop, 1920x1080, 1 spp per
    frame, 32 RIS candidates, screen-space reuse (1 temporal + 5 spatial neighbours within 30 px,
    M-cap 20), direct illumination at the primary vertex (path length 2), lights picked in
    proportion to their power (both estimators; the uniform pick leaves even the reference
    unconverged at these power ratios).  Plain NEE at equal GPU time renders the last view with as
    many samples as one ReSTIR frame's time buys; both last frames are scored by relMSE against
    `ref_spp`-spp plain NEE of that view."""
    import torch

    from stratum2_b200 import _abi, metrics
    from stratum2_b200.scenegen import catmull_rom_views, terrain_scene
    wl = terrain_scene(emissive_triangles=100_000, emissive_sigma=2.0)
    dev.upload_scene(wl.scene)
    W, H = wl.width, wl.height
    views = catmull_rom_views(W, H, frames=frames, seed=11, looping=True)
    rad = torch.zeros((H, W, 4), device="cuda")
    aov = _abi.S2Aovs(rad.data_ptr(), None, None, None, None, None)

    def prm(seed, flags, spp=1):
        p = _abi.S2RenderParams()
        _abi.lib().s2_default_render_params(p)
        p.spp, p.min_path_length, p.max_path_length, p.frame_seed = spp, 2, 2, seed
        p.flags = flags | _abi.FLAG_PIXEL_JITTER | _abi.FLAG_LIGHT_POWER_PICK
        p.restir_candidates, p.restir_spatial, p.restir_spatial_radius, p.restir_max_m = 32, 5, 30.0, 20.0
        return p

    restir = _abi.FLAG_RESTIR_DI | _abi.FLAG_RESTIR_SCREEN
    for v in views[:4]:  # warm-up
        dev.render_device(v, prm(1, restir), aov)
    dev.render_device(views[0], prm(2, 0), aov)  # a call without reuse drops the reservoirs
    ms = rays = 0.0
    for f, v in enumerate(views):
        st = dev.render_device(v, prm(1000 + f, restir), aov)
        ms += st.gpu_ms
        rays += st.extension_rays + st.shadow_rays
    last_restir = rad[..., :3].double().cpu().numpy()
    restir_ms = ms / frames
    ris_1 = dev.render_device(views[-1], prm(4000, _abi.FLAG_RESTIR_DI), aov).gpu_ms  # RIS alone, no reuse
    relmse_ris_1 = rad[..., :3].double().cpu().numpy()
    nee_1 = min(dev.render_device(views[-1], prm(5000 + k, 0), aov).gpu_ms for k in range(3))
    relmse_nee_1 = rad[..., :3].double().cpu().numpy()
    spp_eq = max(1, int(round(restir_ms / nee_1)))
    st = dev.render_device(views[-1], prm(6000, 0, spp_eq), aov)
    last_nee = rad[..., :3].double().cpu().numpy()
    nee_ms = st.gpu_ms
    dev.render_device(views[-1], prm(7000, 0, ref_spp), aov)
    ref = rad[..., :3].double().cpu().numpy()
    relmse_nee_1 = metrics.relmse(relmse_nee_1, ref)
    relmse_ris_1 = metrics.relmse(relmse_ris_1, ref)
    return {"workload": "cfg2 terrain + 100k emissive triangles (power lognormal(0,2)), 32-frame Catmull-Rom camera "
                        "loop, 1920x1080, 1 spp per frame, direct illumination at the primary vertex",
            "restir": "32 RIS candidates, screen-space reuse: 1 temporal + 5 spatial neighbours within 30 px, M-cap 20",
            "light_pick": "power-proportional (alias table), both estimators",
            "restir_ms_per_frame": restir_ms, "restir_mrays_per_s": rays / ms / 1e3,
            "nee_1spp_ms": nee_1, "nee_equal_time_spp": spp_eq, "nee_equal_time_ms": nee_ms,
            "relmse_restir_last_frame": metrics.relmse(last_restir, ref),
            "relmse_nee_equal_time": metrics.relmse(last_nee, ref),
            "relmse_nee_1spp": relmse_nee_1,
            "ris_1spp_ms": ris_1, "relmse_ris_1spp_no_reuse": relmse_ris_1,
            "reference": f"plain NEE, {ref_spp} spp, last view (GPU, power-proportional pick)"}


def C_sizeof_view_params() -> int:
    import ctypes
    from stratum2_b200 import _abi
    return ctypes.sizeof(_abi.S2View) + ctypes.sizeof(_abi.S2RenderParams)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-quality", action="store_true", help="skip the batched and time-to-relMSE measurements")
    ap.add_argument("--no-autotune", action="store_true", help="render with the default tuning")
    ap.add_argument("--quality-chunks", type=int, default=48,
                    help="independent 64-spp renders behind the plain path tracer's time to relMSE 0.01")
    ap.add_argument("--quality-only", action="store_true",
                    help="run only the time-to-relMSE comparison on the learned-cache scene and print it")
    ap.add_argument("--single-frame", type=int, default=0, metavar="SPP",
                    help="render one frame of the workload with SPP samples and exit (profiling)")
    ap.add_argument("--frame-size", default="", metavar="WxH",
                    help="with --single-frame: the frame's extent (default: the workload's 1920x1080); "
                         "the same scene and camera, for small profiling captures")
    ap.add_argument("--cache-kernels", type=int, default=0, metavar="STEPS",
                    help="run the radiance-cache inference and training kernels STEPS times and exit (profiling)")
    ap.add_argument("--cached-frames", type=int, default=0, metavar="N",
                    help="render N 1-spp frames of the learned-cache scene in the 2-bounce radiance-cache form "
                         "and exit (profiling)")
    ap.add_argument("--vcm-only", action="store_true",
                    help="run only the VCM renderer measurement on the many-lights frame and print it")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="run only the differentiable forward and adjoint measurement and print it")
    ap.add_argument("--restir-only", action="store_true",
                    help="run only the many-lights ReSTIR DI versus equal-time NEE comparison and print it")
    args = ap.parse_args()
    if args.cached_frames:
        from stratum2_b200 import Device, _abi
        from stratum2_b200.scenegen import terrain_scene
        dev = Device(0)
        wl = terrain_scene(area_lights=8)
        dev.upload_scene(wl.scene)
        dev.cache_init()
        out = []
        for k in range(args.cached_frames):
            p = params(dev, 1, 50000 + k, _abi.FLAG_RADIANCE_CACHE | (_abi.FLAG_ACCUMULATE if k else 0))
            p.cache_bounces = 2
            p.flags |= _abi.FLAG_ENV_FOOTPRINT_PDF
            r = dev.render(wl.view, wl.width, wl.height, params=p)
            out.append({"gpu_ms": r.stats.gpu_ms, "launches": r.stats.kernel_launches,
                        "extension_rays": r.stats.extension_rays, "shadow_rays": r.stats.shadow_rays})
        print(json.dumps(out))
        return
    if args.cache_kernels:
        from stratum2_b200 import Device
        print(json.dumps(cache_kernel_line(Device(0), args.cache_kernels)))
        return
    if args.vcm_only:
        from stratum2_b200 import Device
        print(json.dumps(vcm_line(Device(0))))
        return
    if args.quality_only:
        from stratum2_b200 import Device
        print(json.dumps(quality_line(Device(0), args)))
        return
    if args.adjoint_only:
        from stratum2_b200 import Device
        print(json.dumps(adjoint_line(Device(0))))
        return
    if args.restir_only:
        from stratum2_b200 import Device
        print(json.dumps(restir_line(Device(0))))
        return
    if args.single_frame:
        from stratum2_b200 import Device
        from stratum2_b200.scenegen import terrain_scene
        dev = Device(0)
        w, h = (int(v) for v in args.frame_size.split("x")) if args.frame_size else (1920, 1080)
        wl = terrain_scene(width=w, height=h)
        dev.upload_scene(wl.scene)
        r = dev.render(wl.view, wl.width, wl.height, params=params(dev, args.single_frame, 0))
        print(json.dumps({"gpu_ms": r.stats.gpu_ms, "extension_rays": r.stats.extension_rays,
                          "shadow_rays": r.stats.shadow_rays}))
        return
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        # one process per GPU: relaunch this command under torchrun with --gpus ranks
        import socket
        with socket.socket() as so:
            so.bind(("127.0.0.1", 0))
            port = so.getsockname()[1]
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
               "--master-addr", "127.0.0.1", "--master-port", str(port), str(Path(__file__).resolve()), *sys.argv[1:]]
        sys.exit(subprocess.call(cmd))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} disagrees with WORLD_SIZE={world} from the launcher")
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
