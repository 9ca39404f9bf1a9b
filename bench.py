"""Benchmark of the wavefront path tracer on one or more B200s.

Workload (the metric's single-GPU configuration): the seeded sphere scene of
1,024,010 FP32 triangles (200 displaced icospheres at subdivision 4 over a
ground quad; 40% Lambert / 30% Trowbridge-Reitz conductor / 30% dielectric; 4
quad lights and a constant environment of 0.5), 1024 x 1024 pixels, max depth 8,
Russian roulette as the reference applies it. Inputs are synthetic (seeded
generator), standing in for the configuration's procedural scene.

A step is one pass of the hot path over one batch: one sample of every pixel
(1,048,576 paths, all bounces, with NEE shadow and MIS rays). `value` is
Msamples/s of the K timed steps rendered as one call of K samples per pixel
(the configuration's frame is one such call of 64 spp), measured with CUDA
events on the launching stream (inputs resident in HBM, L2 flushed before the
call); `per_call_1spp` is the same K steps as K separate one-sample calls with
L2 flushed before each; `e2e` is the metric through the public C ABI with the
step's parameters copied in and the image read back to page-locked host memory
every step. Launch shapes (waves, lanes, blocks) come from the library's
autotuner, run untimed on 8 samples per pixel first.

The `guided` object is the metric's comparison itself: on the hard-indirect
room (2,048,000 clutter triangles of 100 displaced icospheres at subdivision 5,
a 0.5 x 0.5 emitter of radiance 50 facing away from a 0.3-wide slit, glossy
Trowbridge-Reitz floor and walls) at 1024 x 1024, the device time plain path
tracing (autotuned launch shapes) and guided path tracing (the learned guide
trained online from scratch inside the same run, training time included) need
until the relMSE against a converged plain render falls to each target. The
reference render has 4,096 spp instead of 65,536 so that the default run takes
minutes (its own relMSE, about 0.0001 at 0.01 targets, is negligible).

--impl reference times the reference CPU integrator (path_integrator::trace of
the reference sources, compiled as oracle/_ref) on each step's whole workload
(every pixel at one sample) on all host cores; its scene comes from the same
seeded generator compiled into oracle/_ref, so that arm loads nothing of the
product.
"""
from __future__ import annotations

import argparse
import ctypes
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

WORKLOAD = dict(kind=1, seed=1, width=1024, height=1024, num_spheres=200, subdivision=4, max_depth=8)
GUIDED = dict(kind=2, seed=3, num_spheres=100, subdivision=5, max_depth=8)
METRIC = "time to relMSE 0.01: guided vs plain wavefront PT on 1 B200; Msamples/s"
FALLBACK_HBM_GBS = 6650.0


def measured_l2_copy_gbs(buf, mib=32, reps=50):
    """Read + write GB/s of a device copy whose source and destination (2 x `mib` MiB) stay in the 126 MB L2,
    best of three CUDA-event-timed loops of `reps` copies."""
    import torch
    n = mib << 20
    src, dst = buf[:n], buf[n:2 * n]
    dst.copy_(src)
    best = None
    for _ in range(3):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            dst.copy_(src)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        best = ms if best is None else min(best, ms)
    return 2 * n * reps / (best / 1e3) / 1e9


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.rows.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def reference_scene():
    """The workload's scene built by the oracle library alone (no product code imported or loaded)."""
    from oracle import ref
    return ref.RefScene.generated(WORKLOAD["kind"], WORKLOAD["seed"], WORKLOAD["width"], WORKLOAD["height"],
                                  WORKLOAD["num_spheres"], WORKLOAD["subdivision"])


def cpu_reference_frame(R, first_sample, threads):
    """Seconds the reference integrator (oracle/_ref) takes for one step of the workload: every pixel of the
    1024 x 1024 frame at one sample, on `threads` host threads."""
    _, _, sec = R.render(1, first_sample, WORKLOAD["max_depth"], 1.0, 0, threads)
    return sec


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/liboracle_ref.so not built"}))
        return 0
    R = reference_scene()
    threads = os.cpu_count() or 1
    pixels = WORKLOAD["width"] * WORKLOAD["height"]
    for k in range(args.warmup):
        cpu_reference_frame(R, 10_000 + k, threads)
    total_s = 0.0
    for k in range(args.steps):
        total_s += cpu_reference_frame(R, k, threads)
    value = args.steps * pixels / total_s / 1e6
    sample = f"the whole step: all {pixels} pixels of the 1024x1024 frame at 1 spp per step"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Msamples/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_s * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded procedural scene)", "config": config_dict(world),
        "timing": "each step: the reference's path_integrator::trace (oracle/_ref, compiled from the reference "
                  "sources) over every pixel at 1 spp, wall clock, all host threads; scene generated inside "
                  f"oracle/_ref ({R.triangles} triangles)",
        "cpu_baseline": {"value": value, "unit": "Msamples/s", "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


def config_dict(world):
    """The workload of one step, identical for both arms."""
    return {"workload": "sphere field, 1,024,010 triangles, 1024x1024, 1 spp per step, max depth 8",
            "triangles": 1024010, "width": WORKLOAD["width"], "height": WORKLOAD["height"],
            "max_depth": WORKLOAD["max_depth"], "spp_per_step": 1,
            "parallelism": f"replicas x{world} (sample ranges)",
            "l2": "GPU arm: flushed before the timed call; per-step inputs exceed L2 (paths of a wave 0.45-1.8 GB, "
                  "film 59 MB); the 86 MB scene stays resident across steps as in any multi-sample render"}


def guided_leg(rb, device, res, ref_spp, targets, chunk, max_spp, steps_per_wave=12, batch=1 << 18, train_chunks=4,
               lanes=4, learning_rate=1e-3, weight_clip=4.0, guide_seeds=(0, 1, 2, 3, 4)):
    """Device time to each relMSE target: plain vs guided (online training during the first train_chunks
    chunks, then guided sampling with the trained weights). Guided runs once per guide seed (the trained
    guide, and so the time to a target, varies with the weight initialisation and the training order); the
    reported guided time is the median over the seeds."""
    scene = rb.generate_scene(GUIDED["kind"], seed=GUIDED["seed"], width=res, height=res,
                              num_spheres=GUIDED["num_spheres"], subdivision=GUIDED["subdivision"])
    depth = GUIDED["max_depth"]
    ctx = rb.Context(device)
    ctx.upload(scene)
    t0 = time.perf_counter()
    ctx.render(scene.camera, ref_spp, max_depth=depth, seed=1000, want_image=False, paths_per_wave=1 << 22)
    s, _, c = ctx.film()
    ref = s / c[..., None]
    ref_s = time.perf_counter() - t0

    def relmse():
        s, _, c = ctx.film()
        m = s / c[..., None]
        return float(np.mean((m - ref) ** 2 / (ref ** 2 + 1e-2)))

    # plain at its fastest: launch shapes tuned for chunk-sized calls; guided: `lanes` waves per chunk on as
    # many lanes (each lane samples the weights trained after its previous wave)
    plain_tuning, _ = ctx.tune_render(scene.camera, probe_spp=chunk, max_depth=depth, seed=55)
    guided_tuning = dict(paths_per_wave=res * res * chunk // lanes, lanes=lanes, smem_carveout=plain_tuning.smem_carveout)
    out = {}
    for mode, gseed in [("plain", None)] + [("guided", k) for k in guide_seeds]:
        guided = mode == "guided"
        if guided:
            ctx.set_tuning(plain_tuning, **guided_tuning)
            ctx.guide_init(seed=gseed, learning_rate=learning_rate, batch_size=batch, steps_per_wave=steps_per_wave,
                           min_rows=4096, weight_clip=weight_clip)
        ms, spp, left, hit = 0.0, 0, sorted(targets, reverse=True), {}
        while left and spp < max_spp:
            ctx.render(scene.camera, chunk, first_sample=spp, max_depth=depth, seed=7, reset=(spp == 0), guide=guided,
                       train=guided and spp < train_chunks * chunk, want_image=False)
            ms += ctx.stats().elapsed_ms
            spp += chunk
            e = relmse()
            while left and e <= left[0]:
                hit[left.pop(0)] = {"s": ms / 1e3, "spp": spp, "relmse": e}
        if guided:
            st = ctx.guide_stats()
            out.setdefault("guided", []).append(hit)
            out.setdefault("guide", []).append({"seed": gseed, "adam_steps": st.steps, "last_loss": st.last_loss,
                                                "device_error": st.device_error})
        else:
            out["plain"] = hit
    ctx.close()
    res_t = {}
    for t in targets:
        p = out["plain"].get(t)
        runs = [g.get(t) for g in out["guided"]]
        # a seed that never reaches the target within the sample budget counts as infinitely slow; the
        # median exists while more than half of the seeds reach it
        s_all = sorted(g["s"] if g else float("inf") for g in runs)
        spp_all = sorted(g["spp"] if g else float("inf") for g in runs)
        med_s = float(np.median(s_all)) if np.isfinite(np.median(s_all)) else None
        med_spp = float(np.median(spp_all)) if np.isfinite(np.median(spp_all)) else None
        res_t[str(t)] = {"plain_s": p and p["s"], "plain_spp": p and p["spp"], "guided_s": med_s, "guided_spp": med_spp,
                         "speedup": (p["s"] / med_s) if (p and med_s) else None,
                         "guided_runs": [{"seed": k, "s": g and g["s"], "spp": g and g["spp"]}
                                         for k, g in zip(guide_seeds, runs)]}
    return {"workload": f"slit room, {GUIDED['num_spheres'] * 20480 + 18} triangles, {res}x{res}, max depth {depth}, "
                        f"chunks of {chunk} spp; guided: {lanes} waves per chunk on {lanes} lanes, {steps_per_wave} Adam "
                        f"steps (learning rate {learning_rate}, weights clipped at {weight_clip}x their running mean) of up "
                        f"to {batch} samples after each wave of the first {train_chunks} chunks, then guided "
                        f"sampling without training, median over guide seeds {list(guide_seeds)}; plain: autotuned "
                        f"launch shapes {plain_tuning.as_dict()}",
            "reference": f"plain, {ref_spp} spp, FP64 accumulation ({ref_s:.1f} s)", "targets": res_t,
            "guide": out.get("guide"), "timing": "sum of CUDA-event render times; training included in guided_s"}


def photon_waves(res=512, iterations=2):
    """One photon-mapping call (rb_render_photons, `iterations` iterations, one photon per pixel, depth 5,
    radius 0.2) on the sphere field at res x res: the workload of the photon-mapping profile in profiles/."""
    import rainbow_b200 as rb
    scene = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=res, height=res, num_spheres=200, subdivision=4)
    ctx = rb.Context(0)
    ctx.upload(scene)
    t0 = time.perf_counter()
    img = ctx.render_photons(scene.camera, iterations, 5, 0, 0.2, seed=1)
    ms = (time.perf_counter() - t0) * 1e3
    ctx.close()
    print(json.dumps({"ms": ms, "image_mean": float(img.mean())}))
    return 0


def direct_waves(res=1024, spp=2):
    """One direct-lighting call (4 emitter + 4 BSDF samples, staged kernels) of `spp` samples on the sphere
    field: the workload of the direct-lighting profile in profiles/."""
    import rainbow_b200 as rb
    scene = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=res, height=res, num_spheres=200, subdivision=4)
    ctx = rb.Context(0)
    ctx.upload(scene)
    ctx.render(scene.camera, spp, seed=3, want_image=False, direct=(4, 4), paths_per_wave=res * res)
    st = ctx.stats()
    ctx.close()
    print(json.dumps({"ms": st.elapsed_ms, "rays": st.extend_rays, "launches": st.kernel_launches}))
    return 0


def trace_waves(res=512, shadow_test=0):
    """Two one-sample calls on the sphere field at res x res, one lane of one wave (the reduced workload of the
    traversal profile in profiles/: inputs above L2, a few hundred MB on the device)."""
    import rainbow_b200 as rb
    scene = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=res, height=res, num_spheres=200, subdivision=4)
    ctx = rb.Context(0)
    ctx.upload(scene)
    ctx.set_tuning(paths_per_wave=res * res, block_trace=64, block_shade=128, grid_per_sm=8, sort=rb.RB_SORT_RAYS, lanes=1,
                   smem_carveout=76, shadow_test=shadow_test)
    for k in range(2):
        ctx.render(scene.camera, 1, first_sample=k, max_depth=8, reset=True, want_image=False)
    st = ctx.stats()
    ctx.close()
    print(json.dumps({"ms": st.elapsed_ms, "extend_ms": st.extend_ms, "secondary_ms": st.secondary_ms,
                      "traversal_rays": st.extend_rays + st.shadow_rays + st.mis_rays, "extend_rays": st.extend_rays,
                      "secondary_rays": st.shadow_rays + st.mis_rays, "device_error": st.device_error}))
    return 0


def guided_waves(res=1024):
    """Two plain waves, then three guided training waves (2 spp each) on the slit room: the
    workload of the guide-network profile in profiles/."""
    import rainbow_b200 as rb
    scene = rb.generate_scene(GUIDED["kind"], seed=GUIDED["seed"], width=res, height=res,
                              num_spheres=GUIDED["num_spheres"], subdivision=GUIDED["subdivision"])
    ctx = rb.Context(0)
    ctx.upload(scene)
    out = {"plain_ms": [], "guided_ms": []}
    for k in range(2):
        ctx.render(scene.camera, 2, first_sample=2 * k, max_depth=8, seed=7, reset=(k == 0), paths_per_wave=res * res * 2,
                   want_image=False)
        out["plain_ms"].append(ctx.stats().elapsed_ms)
    ctx.guide_init(seed=0, learning_rate=1e-3, batch_size=1 << 18, steps_per_wave=8, min_rows=4096)
    for k in range(3):
        ctx.render(scene.camera, 2, first_sample=2 * k, max_depth=8, seed=7, reset=(k == 0), guide=True, train=True,
                   paths_per_wave=res * res * 2, want_image=False)
        out["guided_ms"].append(ctx.stats().elapsed_ms)
    out["adam_steps"] = ctx.guide_stats().steps
    ctx.close()
    print(json.dumps(out))
    return 0


def config1_leg(rb, device, threads):
    """Configuration 1 as specified: the box room, 256 x 256, 16 spp, depth 5, one render call on the GPU,
    and the same render by the reference CPU integrator (oracle/_ref) on all host cores."""
    scene = rb.generate_scene(rb.RB_SCENE_BOX, seed=0, width=256, height=256)
    ctx = rb.Context(device)
    ctx.upload(scene)
    ctx.render(scene.camera, 16, max_depth=5, seed=1, want_image=False)  # warm-up (graph capture)
    best = min((ctx.render(scene.camera, 16, max_depth=5, seed=2 + k, want_image=False), ctx.stats().elapsed_ms)[1]
               for k in range(3))
    ctx.close()
    samples = 256 * 256 * 16
    out = {"workload": "box room, 32 triangles, 256x256, 16 spp, max depth 5", "gpu_msamples_per_s": samples / best / 1e3,
           "gpu_ms": best}
    try:
        from oracle import ref
        if ref.available():
            _, _, sec = ref.RefScene(scene).render(16, 0, 5, 1.0, 0, threads)
            out.update(cpu_reference_msamples_per_s=samples / sec / 1e6, cpu_reference_s=sec, cpu_cores=threads)
    except Exception as e:  # reported, never required
        out["cpu_reference_error"] = str(e)
    return out


def direct_leg(rb, device, threads, spp=4, rows=(384, 640)):
    """direct_integrator (RB_RENDER_DIRECT, 4 emitter + 4 BSDF samples) on the sphere field (1,024,010
    triangles, 1024 x 1024): one call of `spp` samples per pixel on the GPU, and the reference's own
    direct_integrator on `rows` of the image at 1 spp on all host cores."""
    scene = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=1024, height=1024, num_spheres=200, subdivision=4)
    ctx = rb.Context(device)
    ctx.upload(scene)
    ctx.render(scene.camera, 1, seed=1, want_image=False, direct=(4, 4))  # warm-up (module loading, buffers)
    tuning, _ = ctx.tune_render(scene.camera, probe_spp=1, seed=90, direct=(4, 4))
    best, rays = None, 0
    for k in range(3):
        ctx.render(scene.camera, spp, seed=2 + k, want_image=False, direct=(4, 4))
        st = ctx.stats()
        if best is None or st.elapsed_ms < best:
            best, rays = st.elapsed_ms, st.extend_rays
    ctx.close()
    samples = 1024 * 1024 * spp
    out = {"workload": f"sphere field, {scene.num_triangles} triangles, 1024x1024, {spp} spp, direct lighting with "
                       "4 emitter and 4 BSDF samples", "gpu_msamples_per_s": samples / best / 1e3, "gpu_ms": best,
           "gpu_mrays_per_s": rays / best / 1e3, "tuning": tuning.as_dict()}
    try:
        from oracle import ref
        if ref.available():
            R = ref.RefScene(scene)
            R.set_direct(4, 4)
            _, _, sec = R.render(1, 0, 5, 1.0, 0, threads, rows=rows)
            n = 1024 * (rows[1] - rows[0])
            out.update(cpu_reference_msamples_per_s=n / sec / 1e6, cpu_reference_s=sec, cpu_cores=threads,
                       cpu_sample=f"rows {rows[0]}-{rows[1] - 1} at 1 spp ({n} samples)")
    except Exception as e:  # reported, never required
        out["cpu_reference_error"] = str(e)
    return out


def photons_leg(rb, device, iterations=4, radius=0.2, cpu_res=128, cpu_iterations=2):
    """Stochastic progressive photon mapping (rb_render_photons; photon_mapping_integrator::render) on the
    sphere field (1,024,010 triangles, 1024 x 1024): `iterations` iterations of a visible point per pixel
    and one photon per pixel, max depth 5, initial radius `radius`; the call is synchronous, so its wall
    time covers allocation, all iterations and the image's copy to the host. The reference's own
    photon_mapping_integrator (its parallel loops run in order here: libstdc++'s serial backend) on the
    same scene at cpu_res x cpu_res for cpu_iterations iterations, one host core."""
    scene = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=1024, height=1024, num_spheres=200, subdivision=4)
    ctx = rb.Context(device)
    ctx.upload(scene)
    ctx.render_photons(scene.camera, 1, 5, 0, radius)  # warm-up (module loading)
    best = None
    for k in range(3):
        t0 = time.perf_counter()
        img = ctx.render_photons(scene.camera, iterations, 5, 0, radius, seed=1 + k)
        ms = (time.perf_counter() - t0) * 1e3
        best = ms if best is None else min(best, ms)
    ctx.close()
    items = 1024 * 1024 * iterations
    out = {"workload": f"sphere field, {scene.num_triangles} triangles, 1024x1024, stochastic progressive photon "
                       f"mapping, {iterations} iterations of 1,048,576 visible points and 1,048,576 photons, depth 5, "
                       f"radius {radius}", "gpu_ms": best, "gpu_ms_per_iteration": best / iterations,
           "gpu_mphotons_per_s": items / best / 1e3, "image_mean": float(img.mean())}
    try:
        from oracle import ref
        if ref.available():
            small = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=cpu_res, height=cpu_res, num_spheres=200,
                                      subdivision=4)
            _, sec = ref.RefScene(small).render_photons(cpu_iterations, 5, 0, radius)
            n = cpu_res * cpu_res * cpu_iterations
            out.update(cpu_reference_mphotons_per_s=n / sec / 1e6, cpu_reference_s=sec, cpu_cores=1,
                       cpu_sample=f"{cpu_res}x{cpu_res}, {cpu_iterations} iterations ({n} visible points and photons)")
    except Exception as e:  # reported, never required
        out["cpu_reference_error"] = str(e)
    return out


def subsurface_sphere_field(rb, res):
    """The sphere field (1,024,010 triangles) at res x res with every third material a subsurface material
    (glass lobes over the normalized-diffusion BSSRDF, mean free paths 0.05-0.4, smooth and rough in turn)."""
    scene = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=res, height=res, num_spheres=200, subdivision=4)
    mats = [rb.MaterialDesc.from_buffer_copy(bytes(scene.desc.materials[k])) for k in range(scene.desc.num_materials)]
    for k in range(1, len(mats), 3):
        m = rb.MaterialDesc()
        m.kind, m.remap_roughness, m.ior = rb.RB_MATERIAL_SUBSURFACE, 1, 1.33
        m.reflectance[:], m.transmission[:] = (1.0, 1.0, 1.0), (1.0, 1.0, 1.0)
        m.diffuse[:], m.mfp[:] = (0.8, 0.5, 0.3), (0.4, 0.2, 0.05)
        m.roughness_u = m.roughness_v = 0.0 if (k // 3) % 2 == 0 else 0.2
        mats[k] = m
    return scene.with_materials(mats)


def subsurface_waves(res=512):
    """One 1-spp call of depth 8 on the subsurface sphere field at res x res (waves of res * res paths): the
    workload of the subsurface profile in profiles/."""
    import rainbow_b200 as rb
    scene = subsurface_sphere_field(rb, res)
    ctx = rb.Context(0)
    ctx.upload(scene)
    ctx.render(scene.camera, 1, max_depth=8, seed=3, want_image=False, paths_per_wave=res * res)
    st = ctx.stats()
    ctx.close()
    print(json.dumps({"ms": st.elapsed_ms, "rays": st.extend_rays + st.shadow_rays + st.mis_rays,
                      "launches": st.kernel_launches}))
    return 0


def subsurface_leg(rb, device, threads, spp=4, rows=(448, 576)):
    """Path tracing with subsurface materials: the sphere field (1,024,010 triangles, 1024 x 1024, depth 8)
    with every third material a subsurface material (glass lobes over the normalized-diffusion BSSRDF, mean
    free paths 0.05-0.4, smooth and rough in turn), so a share of the paths takes the k_subsurface stage:
    one call of `spp` samples per pixel with autotuned launch shapes; the reference's own path_integrator on
    `rows` of the image at 1 spp on all host cores."""
    scene = subsurface_sphere_field(rb, 1024)
    ctx = rb.Context(device)
    ctx.upload(scene)
    t, _ = ctx.tune_render(scene.camera, probe_spp=1, max_depth=8, seed=90)
    best, rays = None, 0
    for k in range(2):
        ctx.render(scene.camera, spp, max_depth=8, seed=3 + k, want_image=False)
        st = ctx.stats()
        if best is None or st.elapsed_ms < best:
            best, rays = st.elapsed_ms, st.extend_rays + st.shadow_rays + st.mis_rays
    ctx.close()
    out = {"workload": f"sphere field, {scene.num_triangles} triangles, 1024x1024, {spp} spp, depth 8, every third "
                       "material subsurface (normalized-diffusion BSSRDF)",
           "gpu_msamples_per_s": 1024 * 1024 * spp / best / 1e3, "gpu_ms": best, "gpu_mrays_per_s": rays / best / 1e3,
           "tuning": t.as_dict()}
    try:
        from oracle import ref
        if ref.available():
            _, _, sec = ref.RefScene(scene).render(1, 0, 8, 1.0, 0, threads, rows=rows)
            n = 1024 * (rows[1] - rows[0])
            out.update(cpu_reference_msamples_per_s=n / sec / 1e6, cpu_reference_s=sec, cpu_cores=threads,
                       cpu_sample=f"rows {rows[0]}-{rows[1] - 1} at 1 spp ({n} samples)")
    except Exception as e:  # reported, never required
        out["cpu_reference_error"] = str(e)
    return out


def spheres_s5_leg(rb, device, spp=8):
    """The sphere field at icosphere subdivision 5 (200 spheres, 4,096,002 triangles): one call of `spp`
    samples per pixel with autotuned launch shapes."""
    scene = rb.generate_scene(rb.RB_SCENE_SPHERES, seed=1, width=1024, height=1024, num_spheres=200, subdivision=5)
    ctx = rb.Context(device)
    ctx.upload(scene)
    t, _ = ctx.tune_render(scene.camera, probe_spp=2, max_depth=8, seed=90)
    ctx.render(scene.camera, spp, max_depth=8, seed=3, want_image=False)
    st = ctx.stats()
    ctx.close()
    return {"workload": f"sphere field, {scene.num_triangles} triangles (subdivision 5), 1024x1024, {spp} spp, depth 8",
            "msamples_per_s": 1024 * 1024 * spp / st.elapsed_ms / 1e3,
            "mrays_per_s": (st.extend_rays + st.shadow_rays + st.mis_rays) / st.elapsed_ms / 1e3, "tuning": t.as_dict()}


def config5_leg(rb, device, spp=8):
    """Configuration 5 without guiding: the fog (400 displaced spheres at subdivision 5, 8,192,046 triangles,
    inside an invisible box holding a homogeneous medium), 1920 x 1080, depth 12, volume path tracing, one
    call of `spp` samples per pixel with launch shapes tuned for volume renders."""
    scene = rb.generate_scene(rb.RB_SCENE_FOG, seed=5, width=1920, height=1080, num_spheres=400, subdivision=5)
    ctx = rb.Context(device)
    ctx.upload(scene)
    t, _ = ctx.tune_render(scene.camera, probe_spp=2, max_depth=12, seed=90, volume=True)
    ctx.render(scene.camera, spp, max_depth=12, seed=3, volume=True, want_image=False)
    st = ctx.stats()
    ctx.close()
    return {"workload": f"fog, {scene.num_triangles} triangles, 1920x1080, {spp} spp, depth 12, volume path tracing",
            "msamples_per_s": 1920 * 1080 * spp / st.elapsed_ms / 1e3, "ms": st.elapsed_ms,
            "mrays_per_s": (st.extend_rays + st.shadow_rays + st.mis_rays) / st.elapsed_ms / 1e3, "tuning": t.as_dict()}


def batch_workload(seed=2, count=64):
    """The batched configuration: `count` seeded sphere scenes whose triangle counts are
    log-uniform in [1k, 500k] (displaced icospheres: subdivision and sphere count chosen
    to match), resolutions drawn from {128, 256, 512, 1024} squared, 32 spp, depth 6."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        target = float(np.exp(rng.uniform(np.log(1e3), np.log(5e5))))
        sub = int(np.clip(np.floor(np.log(target / 160.0) / np.log(4.0)), 1, 5))
        spheres = max(1, int(round(target / (20 * 4 ** sub))))
        res = int(rng.choice([128, 256, 512, 1024]))
        out.append(dict(seed=1000 + k, num_spheres=spheres, subdivision=sub, res=res))
    return out


def batched_leg(rb, device, spp=32, depth=6, probe_items=1 << 23):
    """Aggregate Msamples/s and per-scene latency percentiles of one batched render."""
    work = batch_workload()
    scenes = [rb.generate_scene(rb.RB_SCENE_SPHERES, seed=w["seed"], width=w["res"], height=w["res"],
                                num_spheres=w["num_spheres"], subdivision=w["subdivision"]) for w in work]
    tris = [sc.num_triangles for sc in scenes]
    views = [dict(camera=sc.camera, spp=spp, first_sample=0, seed=k) for k, sc in enumerate(scenes)]
    # shortest expected work first: pixels x spp x log(triangles)
    cost = [w["res"] ** 2 * spp * np.log(t) for w, t in zip(work, tris)]
    order = [int(k) for k in np.argsort(cost, kind="stable")]
    ctx = rb.Context(device)
    ctx.batch_upload(scenes)
    tuning, probe_ms = ctx.tune_batch(views, probe_items, max_depth=depth, order=order)
    ms = ctx.batch_render(views, max_depth=depth, order=order)
    st = ctx.stats()
    total_ms = st.elapsed_ms
    ctx.close()
    samples = sum(w["res"] ** 2 * spp for w in work)
    lat = np.sort(ms)
    return {"workload": f"{len(scenes)} sphere scenes, {min(tris)}-{max(tris)} triangles ({sum(tris)} total), "
                        f"resolutions 128^2-1024^2, {spp} spp, depth {depth}, one batched render (shortest first)",
            "msamples_per_s": samples / (total_ms / 1e3) / 1e6, "samples": samples, "ms": total_ms,
            "mrays_per_s": (st.extend_rays + st.shadow_rays + st.mis_rays) / (total_ms / 1e3) / 1e6,
            "scene_latency_ms": {"p50": float(np.percentile(lat, 50)), "p90": float(np.percentile(lat, 90)),
                                 "p99": float(np.percentile(lat, 99)), "max": float(lat[-1])},
            "tuning": tuning.as_dict(), "tuning_probe_ms": probe_ms, "device_error": st.device_error}


def summary_of(extra, batched, guided):
    """The headline figures of the extra legs in a few hundred characters."""
    def pick(d, *keys):
        return {k: (round(d[k], 4) if isinstance(d.get(k), float) else d.get(k)) for k in keys} if isinstance(d, dict) else d
    out = {name: pick(extra.get(name), "gpu_msamples_per_s", "msamples_per_s", "cpu_reference_msamples_per_s", "error")
           for name in ("config1", "direct", "spheres_s5", "config5_plain")}
    out["photons"] = pick(extra.get("photons"), "gpu_mphotons_per_s", "cpu_reference_mphotons_per_s", "error")
    out["subsurface"] = pick(extra.get("subsurface"), "gpu_msamples_per_s", "cpu_reference_msamples_per_s", "error")
    out = {k: {a: b for a, b in v.items() if b is not None} if isinstance(v, dict) else v for k, v in out.items()}
    if isinstance(batched, dict):
        out["batched"] = {k: v for k, v in pick(batched, "msamples_per_s", "error").items() if v is not None}
        if "scene_latency_ms" in batched:
            out["batched"]["latency_ms_p50_p90_max"] = [round(batched["scene_latency_ms"][k], 1) for k in ("p50", "p90", "max")]
    if isinstance(guided, dict) and "targets" in guided:
        out["guided_time_to_relmse"] = {t: {"plain_s": r["plain_s"] and round(r["plain_s"], 4),
                                            "guided_s": r["guided_s"] and round(r["guided_s"], 4),
                                            "speedup": r["speedup"] and round(r["speedup"], 3),
                                            "guided_s_per_seed": [g["s"] and round(g["s"], 4) for g in r["guided_runs"]]}
                                        for t, r in guided["targets"].items()}
    elif isinstance(guided, dict):
        out["guided"] = guided
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=32)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-guided", action="store_true")
    ap.add_argument("--guided-res", type=int, default=1024)
    ap.add_argument("--guided-ref-spp", type=int, default=4096)
    ap.add_argument("--guided-chunk", type=int, default=2)
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--guided-waves", action="store_true",
                    help="only render 2 plain then 3 guided training waves of 2 spp on the slit room (profiling)")
    ap.add_argument("--trace-waves", action="store_true",
                    help="only render two 1-spp calls of the sphere field at 512x512 on one lane (profiling)")
    ap.add_argument("--direct-waves", action="store_true",
                    help="only render one 2-spp direct-lighting call on the sphere field (profiling)")
    ap.add_argument("--photon-waves", action="store_true",
                    help="only render one 2-iteration photon-mapping call on the sphere field at 512x512 (profiling)")
    ap.add_argument("--subsurface-waves", action="store_true",
                    help="only render one 1-spp call of the subsurface sphere field at 512x512 (profiling)")
    ap.add_argument("--no-tune", action="store_true", help="skip the launch-shape autotuner")
    ap.add_argument("--tuning", default=None, help="launch shapes as JSON (skips the autotuner), e.g. "
                    "'{\"block_trace\": 256, \"grid_per_sm\": 16}'")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.guided_waves:
        return guided_waves()
    if args.direct_waves:
        return direct_waves()
    if args.photon_waves:
        return photon_waves()
    if args.subsurface_waves:
        return subsurface_waves()
    if args.trace_waves:
        return trace_waves()

    import torch
    import torch.distributed as dist

    import rainbow_b200 as rb

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    scene = rb.generate_scene(WORKLOAD["kind"], seed=WORKLOAD["seed"], width=WORKLOAD["width"],
                              height=WORKLOAD["height"], num_spheres=WORKLOAD["num_spheres"],
                              subdivision=WORKLOAD["subdivision"])
    W, H, depth = scene.camera.width, scene.camera.height, WORKLOAD["max_depth"]
    pixels = W * H
    ctx = rb.Context(local)
    ctx.upload(scene)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    # each rank renders its own range of sample indices (weak scaling, no data-path collective)
    base = rank * (args.steps + args.warmup + 8)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    tuning = None
    if args.tuning:
        ctx.set_tuning(**json.loads(args.tuning))
        tuning = dict(ctx.tuning().as_dict(), source="--tuning")
    elif not args.no_tune:
        t, probe_ms = ctx.tune_render(scene.camera, probe_spp=min(8, args.steps), max_depth=depth, seed=base + 777)
        tuning = dict(t.as_dict(), probe_spp=min(8, args.steps), probe_ms=probe_ms)
    # warm-up: W untimed steps (one sample of every pixel each)
    ctx.render(scene.camera, spp=args.warmup, first_sample=base + args.steps, max_depth=depth, want_image=False)

    # ---- device-timed steps (value): the K steps as one render call of K samples per pixel
    barrier()
    flush.zero_()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        ctx.render(scene.camera, spp=args.steps, first_sample=base, max_depth=depth, reset=True, want_image=False)
        st = ctx.stats()
        barrier()
    device_ms = st.elapsed_ms
    launches = st.kernel_launches
    rays = st.extend_rays + st.shadow_rays + st.mis_rays
    t = torch.tensor([device_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    value = world * args.steps * pixels / (max_ms / 1e3) / 1e6
    mrays = world * rays / (max_ms / 1e3) / 1e6

    # ---- N > 1: the ranks' films (disjoint sample ranges) summed by one all-reduce over NCCL, then checked on
    # rank 0 against a render of the union of the ranges on its own GPU (outside the timed region)
    film_reduce = None
    if world > 1:
        from rainbow_b200.distributed import reduce_context_film
        before = ctx.film()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        reduce_context_film(ctx, world * args.steps)
        e1.record()
        torch.cuda.synchronize()
        reduced = ctx.film()
        film_reduce = {"ms": e0.elapsed_time(e1), "bytes_per_rank": int(before[0].nbytes + before[1].nbytes + before[2].nbytes)}
        if rank == 0:
            for r in range(world):
                ctx.render(scene.camera, spp=args.steps, first_sample=r * (args.steps + args.warmup + 8), max_depth=depth,
                           reset=(r == 0), want_image=False)
            union = ctx.film()
            rel = float(np.max(np.abs(reduced[0] - union[0]) / np.maximum(np.abs(union[0]), 1e-300)))
            film_reduce.update(counts_equal=bool(np.array_equal(reduced[2], union[2])), max_rel_diff_sums=rel,
                               checked="reduced film vs one-GPU render of the union of the ranks' sample ranges")
        barrier()

    # ---- the same steps as K separate 1-spp calls with L2 flushed before each (reported beside value)
    call_ms = 0.0
    for k in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        ctx.render(scene.camera, spp=1, first_sample=base + k, max_depth=depth, reset=(k == 0), want_image=False)
        call_ms += ctx.stats().elapsed_ms
    per_call = {"value": args.steps * pixels / (call_ms / 1e3) / 1e6, "unit": "Msamples/s",
                "ms_per_step": call_ms / args.steps, "l2": "flushed before every call (256 MiB write)"}

    # ---- end to end through the C ABI with host buffers (params in, image out every step), with the
    # launch shapes tuned for one-sample calls (untimed), as a caller rendering progressively would
    timed_tuning = ctx.tuning()
    # every step: one rb_render_async call (its parameters in by kernel argument), the step's image out to its
    # own page-locked buffer; the calls overlap on the GPU and rb_render_wait ends the run
    imgs = [torch.zeros((H, W, 3), dtype=torch.float32, pin_memory=True) for _ in range(args.steps)]

    def async_calls(n, first):
        for k in range(n):
            p = rb.RenderParams()
            p.camera = scene.camera
            p.spp, p.first_sample, p.max_depth, p.rr_threshold, p.seed = 1, first + k, depth, 1.0, 0
            p.flags = rb.RB_RENDER_RESET if k == 0 else 0
            rb.check(rb.lib().rb_render_async(ctx._h, ctypes.byref(p), ctypes.c_void_p(imgs[k].data_ptr())),
                     "rb_render_async")
        rb.check(rb.lib().rb_render_wait(ctx._h), "rb_render_wait")

    e2e_tuning = None
    if not args.tuning and not args.no_tune:
        # launch shapes for back-to-back one-sample calls (untimed): the tuner's pick for one synchronous call,
        # then the wave sizes and lane counts around it (and the timed call's shapes), each run as the timed
        # loop runs them (overlapping async calls, images read back), the fastest kept
        t1, _ = ctx.tune_render(scene.camera, probe_spp=1, max_depth=depth, seed=base + 999)
        cands = [t1.as_dict(), dict(timed_tuning.as_dict())]
        for ppw in (1 << 18, 1 << 19, 1 << 20):
            for lanes in (2, 4, 8):
                cands.append(dict(t1.as_dict(), paths_per_wave=ppw, lanes=lanes))
                # a one-sample call ends on its longest paths: the tail kernel takes the last bounces
                cands.append(dict(t1.as_dict(), paths_per_wave=ppw, lanes=lanes, tail_bounce=5))
        best = None
        n_probe = min(8, args.steps)
        for c in cands:
            ctx.set_tuning(**c)
            async_calls(2, base + 5000)  # graph capture for these shapes
            t0 = time.perf_counter()
            async_calls(n_probe, base + 6000)
            dt = time.perf_counter() - t0
            if best is None or dt < best[0]:
                best = (dt, c)
        e2e_tuning = dict(best[1], probe_calls=n_probe, probe_ms=best[0] * 1e3, candidates=len(cands))
        ctx.set_tuning(**best[1])
    async_calls(2, base + 7000)  # warm-up: graphs of the chosen shapes
    barrier()
    t0 = time.perf_counter()
    async_calls(args.steps, base)
    barrier()
    e2e_s = time.perf_counter() - t0
    tt = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    e2e_value = world * args.steps * pixels / float(tt.item()) / 1e6
    ctx.set_tuning(timed_tuning)
    h2d = 176  # wave parameter block copied in per call
    d2h = pixels * 3 * 4  # the image (per-pixel means, 3 floats) read back per call

    # ---- roofline of the traversal kernels, from the timed call itself: the kernels time every launch on the
    # device clock (first warp's start to last warp's end, inside the graphs and lanes of the timed run), and a
    # counting pass over exactly the timed samples gives the reference traversal's box and triangle tests
    trav_ms = st.extend_ms + st.secondary_ms
    nl = max(1, st.extend_launches + st.secondary_launches)
    ctx.set_counting(True)
    ctx.render(scene.camera, spp=args.steps, first_sample=base, max_depth=depth, reset=True, want_image=False)
    cst = ctx.stats()
    ctx.set_counting(False)
    trav_rays = cst.extend_rays + cst.shadow_rays + cst.mis_rays
    alg_bytes = 32 * cst.node_visits + 40 * cst.triangle_tests + 48 * trav_rays
    peak, peak_kind = measured_peak_hbm()
    achieved = alg_bytes / (trav_ms / 1e3) / 1e9 if trav_ms > 0 else None
    l2_peak = measured_l2_copy_gbs(flush)
    traffic = None
    prof = os.path.join(ROOT, "profiles", "traversal_sphere_field.json")
    if os.path.exists(prof):
        with open(prof) as f:
            per_ray = json.load(f).get("dram_bytes_per_ray")
        if per_ray:
            traffic = per_ray * trav_rays / nl  # the captured launches' DRAM bytes per ray, per timed launch

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import ref
            if ref.available():
                threads = os.cpu_count() or 1
                sec = cpu_reference_frame(reference_scene(), base, threads)
                cpu = {"value": pixels / sec / 1e6, "unit": "Msamples/s", "cores": threads, "kind": "reference",
                       "sample": f"one step: all {pixels} pixels at 1 spp ({sec:.2f} s)"}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "Msamples/s", "cores": 0, "kind": "reference", "sample": f"failed: {e}"}

    extra = {}
    if rank == 0 and world == 1 and not args.no_batched:
        for name, leg in (("config1", lambda: config1_leg(rb, local, os.cpu_count() or 1)),
                          ("spheres_s5", lambda: spheres_s5_leg(rb, local)),
                          ("config5_plain", lambda: config5_leg(rb, local)),
                          ("direct", lambda: direct_leg(rb, local, os.cpu_count() or 1)),
                          ("photons", lambda: photons_leg(rb, local)),
                          ("subsurface", lambda: subsurface_leg(rb, local, os.cpu_count() or 1))):
            try:
                extra[name] = leg()
            except Exception as e:  # reported, never required for the throughput line
                extra[name] = {"error": str(e)}

    batched = None
    if rank == 0 and world == 1 and not args.no_batched:
        try:
            batched = batched_leg(rb, local)
        except Exception as e:  # reported, never required for the throughput line
            batched = {"error": str(e)}

    guided = None
    if rank == 0 and world == 1 and not args.no_guided:
        try:
            guided = guided_leg(rb, local, args.guided_res, args.guided_ref_spp, (0.01, 0.005), args.guided_chunk, 256)
        except Exception as e:  # reported, never required for the throughput line
            guided = {"error": str(e)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Msamples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": config_dict(world),
            "timing": "K steps = one rb_render call of K samples per pixel, CUDA events on the library's stream",
            "mrays_per_s": mrays, "per_call_1spp": per_call,
            "e2e": {"value": e2e_value, "unit": "Msamples/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "calls": "one rb_render_async per step (1 spp, the step's image read back to page-locked memory), "
                             "rb_render_wait after the last", "tuning": e2e_tuning},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if achieved else None, "traffic": traffic, "peak_source": peak_kind,
                         "kernel": "k_extend + k_trace_secondary (BVH traversal), launches of the timed call",
                         "algorithmic_bytes_per_launch": alg_bytes / nl, "ms_per_launch": trav_ms / nl,
                         "launches": nl, "traversal_ms_summed_over_lanes": trav_ms, "step_ms": device_ms,
                         "step_bound": {"achieved": alg_bytes / (device_ms / 1e3) / 1e9,
                                        "frac": alg_bytes / (device_ms / 1e3) / 1e9 / peak,
                                        "what": "all traversal bytes of the step over the whole step's time"},
                         "l2": {"achieved": achieved, "peak": l2_peak,
                                "frac": achieved / l2_peak if achieved and l2_peak else None,
                                "peak_source": "measured in this run: copy of 32 MiB into 32 MiB, both L2-resident"}},
            "cpu_baseline": cpu, "clocks": clocks.summary(), "gpu_launches": launches, "tuning": tuning,
            "film_reduce": film_reduce,
            **{k: v for k, v in extra.items()},
            "batched": batched, "guided": guided,
            "summary": summary_of(extra, batched, guided),
        }
        # "summary" is the line's last key, so that a reader that keeps only the
        # end of the output still has every leg's headline figures
        print(json.dumps(line))
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
