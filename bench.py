#!/usr/bin/env python
"""small_pt path tracing throughput on B200.

Workload: the single-mesh scene: icosphere subdivided 8x (1,310,720 triangles) with seeded fBm
radial displacement (amplitude 0.05) on a ground quad, one principled material per 1024-triangle
patch (roughness U[0.05,1], metallic Bernoulli(0.3), basecolor U[0,1]^3), a procedural
2048x1024 FP32 HDR sky (gradient + sun lobe of 1e4), rendered at 1024x1024, 256 spp, depth 12.
All inputs are generated from a fixed seed (synthetic data).

One step = one full render of that frame through ks_small_pt_render_device (scene and BVH
resident in HBM, FP64 accumulators on the device).  value = Mrays/s (closest-hit + shadow
queries) over the K timed steps, device time from CUDA events on the library's stream, max over
ranks.  e2e = the same metric through the host-buffer C ABI (scene upload, GPU SBVH build,
render, FP64 image download every step).

Roofline of the closest-hit traversal kernel: algorithmic bytes per query as the CPU oracle counts
them on the same frame (32 B per SBVH node whose bound the reference traversal tests, 48 B per
triangle tested, 48 B of ray and hit I/O), over the kernel's CUDA-event time; beside it the
kernel's own fetch count (128 B per 4-wide node, 48 B per triangle).

time_to_relmse: the glossy scene behind an occluder (the same icosphere made glossy-heavy,
roughness U[0.02,0.2], with an opaque slab between it and the sun) at 1920x1080, depth 12.  The
reference is eight 64x64 crop windows rendered by the CPU oracle at 2048 spp (its own seed) and
accumulated in FP64; plain and guided progressive GPU renders (1 spp per pass, guide trained
online: batches of 2^18 records, Adam lr 1e-2) run until the relative MSE on those crops (eps 1e-2,
reduced in FP64 on the GPU after each pass, outside the timed region) reaches 1e-2, and the CPU
oracle renders the full frame progressively (4 spp per chunk, same sample sequence) to the same
error, timed.

Side configurations, each once per run: the box room (256x256, 64 spp, depth 8) on the GPU and
on the CPU oracle; 64 batched scenes at their full spp (one CUDA-graph launch, autotuned); the
instanced scene (400 instances, 3840x2160, 1024 spp, depth 16) plain and guided.

--impl reference runs the CPU implementation of the path on all host cores (the oracle's
restatement of small_pt over the reference's own SBVH traversal, with the scene, camera and
parameters made by the oracle library, without loading the CUDA library) on the same frame and
configuration, each step one 16-spp interval of the 256-spp render of the full frame.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "icosphere_l8_1310722tris_1024x1024_256spp_depth12_sky2048x1024"
W_RES, H_RES, SPP, BOUNCES = 1024, 1024, 256, 12
# CPU sample: one interval of the frame's samples per step (the full frame, CPU_SPP of the SPP
# samples per pixel, the next interval each step, as SmallPT::run renders its spp intervals)
CPU_SPP = 16


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-steps", type=int, default=None, help="steps of the end-to-end leg (default: --steps)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ttr", action="store_true", help="skip the time-to-relMSE leg")
    ap.add_argument("--no-c4", action="store_true", help="skip the batched multi-scene leg")
    ap.add_argument("--c4-spp-div", type=int, default=1, help="divides the spp of every batched job")
    ap.add_argument("--no-c1", action="store_true", help="skip the box-room leg")
    ap.add_argument("--no-c5", action="store_true", help="skip the instanced-scene leg")
    ap.add_argument("--profile-guided", action="store_true",
                    help="profiling case only: one guided render of the glossy occluded scene at --res x "
                         "(--res * 9 / 16), --spp samples (default 16), then exit")
    ap.add_argument("--profile-unguided", action="store_true",
                    help="with --profile-guided: the same render without the guide")
    ap.add_argument("--c5-spp", type=int, default=1024)
    # reduced frames of the same scene, for profiling captures only (not a bench line)
    ap.add_argument("--spp", type=int, default=None)
    ap.add_argument("--res", type=int, default=None)
    a = ap.parse_args()
    global W_RES, H_RES, SPP, WORKLOAD
    if a.spp or a.res:
        SPP = a.spp or SPP
        W_RES = H_RES = a.res or W_RES
        WORKLOAD = f"icosphere_l8_1310722tris_{W_RES}x{H_RES}_{SPP}spp_depth12_sky2048x1024 (profiling case)"
    return a


def reduce_ranks(pg, torch, seconds, counts, device):
    """Whole-job aggregation over the ranks (replicas): the slowest rank's time (max) and the sums
    of the work counts.  Every rank calls it, in the same order."""
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    r = torch.tensor(counts, dtype=torch.float64, device=device)
    pg.all_reduce(r)
    return float(t.item()), [int(x) for x in r.tolist()]


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def make_generated(ks):
    return ks.Generated("icosphere", 0, level=8, sky=(2048, 1024), resolution=(W_RES, H_RES))


TTR_W, TTR_H, TTR_TARGET, TTR_REF_SPP, TTR_MAX_SPP = 1920, 1080, 1e-2, 2048, 1024
TTR_PRETRAIN_PASSES = 192
# the reference crops: eight 64x64 windows on a 4 x 2 grid over the frame (crop_* semantics of
# small_pt.cpp:25-34), rendered by the CPU oracle at TTR_REF_SPP with their own seed
TTR_CROP = 64
TTR_CROPS = [(int((i + 0.5) * TTR_W / 4) - TTR_CROP // 2, int((j + 0.5) * TTR_H / 2) - TTR_CROP // 2)
             for j in range(2) for i in range(4)]
TTR_REF_SEED, TTR_SEED = 1000, 7
# the CPU arm renders the full frame in chunks of this many samples per pixel, timed
TTR_CPU_CHUNK = 4
TTR_CPU_MAX_SECONDS = 120.0


def oracle_module():
    """tests/oracle_lib (the CPU oracle's binding); used by the CPU legs of this file only."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib
    return oracle_lib


def crop_pixels(W):
    """Frame pixel indices of the reference crops, crop by crop, row-major inside each."""
    import numpy as np
    idx = []
    for x0, y0 in TTR_CROPS:
        ys, xs = np.mgrid[y0:y0 + TTR_CROP, x0:x0 + TTR_CROP]
        idx.append((ys * W + xs).reshape(-1))
    return np.concatenate(idx)


def time_to_relmse(ks, ctx, torch, with_cpu, guide_options=None, guide_params=None):
    """Seconds (and spp) for plain and guided GPU renders, and for the CPU oracle, to reach relMSE
    1e-2 against FP64 CPU reference crops of the glossy occluded scene."""
    import numpy as np
    g = ks.Generated("icosphere", 0, level=8, sky=(2048, 1024), resolution=(TTR_W, TTR_H), roughness=(0.02, 0.2),
                     occluder=True)
    sc = ks.Scene(ctx, g.desc)
    sc.build_bvh()
    cam = ks.camera_perspective(g.camera_to_world, g.vfov, g.aspect)
    n = TTR_W * TTR_H
    idx_np = crop_pixels(TTR_W)
    n_crop = len(idx_np)
    res = {"target_rel_mse": TTR_TARGET, "eps": 1e-2,
           "workload": f"icosphere_l8 glossy (roughness U[0.02,0.2]) behind an occluder slab, {TTR_W}x{TTR_H}, "
                       f"depth {BOUNCES}, 1 spp per GPU pass",
           "timing": "seconds: host wall clock of the render call up to the pass that reached the target, "
                     "minus the time spent in the per-pass error evaluation; device_seconds: the library's "
                     "CUDA-event time of the same render call; cpu: wall clock of the oracle's chunks"}
    # ---- FP64 reference crops from the CPU oracle (the reference's estimator over its SBVH) ----
    ol = oracle_module()
    orc = ol.load()
    osc = orc.scene(g.desc)
    threads = os.cpu_count() or 1
    ref_img = np.zeros((n_crop, 3), np.float64)
    t0 = time.perf_counter()
    ref_paths = 0
    for k, (x0, y0) in enumerate(TTR_CROPS):
        pr = ks.SmallPTParams.make(render_width=TTR_W, render_height=TTR_H, spp=TTR_REF_SPP, bounces=BOUNCES,
                                   rng_seed=TTR_REF_SEED, crop_start_x=x0, crop_start_y=y0, crop_width=TTR_CROP,
                                   crop_height=TTR_CROP)
        a, w, _ = osc.render(cam, pr, threads=threads)
        from imaging import composite
        img = composite(a, w)[y0:y0 + TTR_CROP, x0:x0 + TTR_CROP].reshape(-1, 3)
        ref_img[k * TTR_CROP * TTR_CROP:(k + 1) * TTR_CROP * TTR_CROP] = img
        ref_paths += TTR_CROP * TTR_CROP * TTR_REF_SPP
    ref_s = time.perf_counter() - t0
    res["reference"] = {"kind": "CPU oracle, FP64 accumulation", "crops": [[x, y, TTR_CROP, TTR_CROP] for x, y in TTR_CROPS],
                        "spp": TTR_REF_SPP, "seed": TTR_REF_SEED, "paths": ref_paths, "seconds": ref_s,
                        "cores": threads}
    idx = torch.as_tensor(idx_np, device="cuda")
    ref = torch.as_tensor(ref_img, device="cuda").contiguous()
    acc = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    wts = torch.zeros((n, 2), dtype=torch.float64, device="cuda")

    def crop_error():
        a = acc.index_select(0, idx).contiguous()
        w = wts.index_select(0, idx).contiguous()
        return ctx.rel_mse_device(a.data_ptr(), w.data_ptr(), ref.data_ptr(), n_crop, 1e-2)

    def run(guide, max_passes=None, frozen=False):
        acc.zero_()
        wts.zero_()
        torch.cuda.synchronize()
        p = ks.SmallPTParams.make(render_width=TTR_W, render_height=TTR_H, spp=TTR_MAX_SPP, bounces=BOUNCES,
                                  rng_seed=TTR_SEED, spp_prog_interval=1)
        st = {"cb": 0.0, "hit": None, "last": None, "passes": []}
        t_start = time.perf_counter()

        def cb(spp):
            t_in = time.perf_counter()
            e = crop_error()
            render_s = (t_in - t_start) - st["cb"]
            st["last"] = (spp, render_s, e)
            st["passes"].append(render_s)
            if e <= TTR_TARGET and st["hit"] is None:
                st["hit"] = (spp, render_s, e)
            st["cb"] += time.perf_counter() - t_in
            return st["hit"] is not None or (max_passes is not None and spp >= max_passes)

        opts = None
        if guide is not None:
            kw = dict(train_passes=1 << 20, train_batch=1 << 18, max_records=1 << 20)
            kw.update(guide_options or {})
            if frozen:
                kw.update(train_passes=0, guide_from_pass=0)
            opts = ks.GuideRenderOptions.make(**kw)
        sc.render_device_progress(cam, p, acc.data_ptr(), wts.data_ptr(), cb, guide=guide, options=opts)
        s = sc.stats()
        out = {"spp": None, "seconds": None, "last": {"spp": st["last"][0], "seconds": st["last"][1],
                                                        "rel_mse": st["last"][2]}}
        if st["hit"]:
            out.update(spp=st["hit"][0], seconds=st["hit"][1], rel_mse=st["hit"][2])
        # device time of the whole render call (it stops at the target), from the library's events
        out["device_seconds"] = s.ms_total / 1e3
        pt = [b - a for a, b in zip([0.0] + st["passes"][:-1], st["passes"])]
        out["pass_seconds"] = {"first": pt[0] if pt else None, "median": statistics.median(pt) if pt else None}
        out["mpaths_per_s"] = s.paths / (s.ms_total / 1e3) / 1e6 if s.ms_total > 0 else None
        if guide is not None:
            out.update(train_steps=s.guide_train_steps, records=s.guide_records,
                       ms_guide_infer=s.ms_guide_infer, ms_guide_train=s.ms_guide_train, ms_total=s.ms_total,
                       guide_rows=s.guide_rows)
            if s.ms_guide_infer > 0:
                # guide inference against the dense BF16 tensor peak: 2 x (4 x 64 x 64 + 48 x 64) FLOPs per
                # row evaluated (the tcgen05 GEMMs)
                tflops = s.guide_rows * GUIDE_FLOPS_PER_ROW / (s.ms_guide_infer / 1e3) / 1e12
                peak, kind = measured_bf16_peak()
                out["guide_inference_roofline"] = {"bound": "tensor", "achieved": tflops, "peak": peak,
                                                   "unit": "TFLOP/s", "frac": tflops / peak, "peak_source": kind,
                                                   "rows": s.guide_rows}
        return out

    lo, hi = g.bound
    bound = list(lo - 0.05) + list(hi + 0.05)
    # untimed warm-up of both arms (first-call costs: allocations, module loading)
    run(None, max_passes=2)
    warm = ks.Guide(ctx, bound, seed=2, learning_rate=1e-2)
    run(warm, max_passes=2)
    warm.close()
    plain = run(None)
    gp = dict(seed=1, learning_rate=1e-2)
    gp.update(guide_params or {})
    guide = ks.Guide(ctx, bound, **gp)
    guided = run(guide)
    # the same guide trained further (untimed), then frozen: what a trained proposal gains per
    # sample once its training is paid for (e.g. by an earlier frame of the same scene)
    t0 = time.perf_counter()
    acc.zero_()
    wts.zero_()
    pt = ks.SmallPTParams.make(render_width=TTR_W, render_height=TTR_H, spp=TTR_PRETRAIN_PASSES, bounces=BOUNCES,
                               rng_seed=11, spp_prog_interval=1)
    sc.render_device_progress(cam, pt, acc.data_ptr(), wts.data_ptr(), lambda spp: False, guide=guide,
                              options=ks.GuideRenderOptions.make(**{**dict(train_passes=1 << 20, train_batch=1 << 18,
                                                                              max_records=1 << 20),
                                                                   **(guide_options or {})}))
    torch.cuda.synchronize()
    pre_s = time.perf_counter() - t0
    frozen = run(guide, frozen=True)
    frozen.update(pretrain_passes=TTR_PRETRAIN_PASSES + (guided["last"]["spp"] or 0), pretrain_seconds=pre_s)
    guide.close()
    res.update(plain=plain, guided=guided, guided_pretrained=frozen)
    if with_cpu:
        # the CPU oracle renders the same full frame with the same sample sequence (spp intervals of
        # the TTR_MAX_SPP sequence, as the GPU's 1-spp passes), timed, until its error on the crops
        # reaches the target
        from imaging import composite, rel_mse
        pc = ks.SmallPTParams.make(render_width=TTR_W, render_height=TTR_H, spp=TTR_MAX_SPP, bounces=BOUNCES,
                                   rng_seed=TTR_SEED)
        a = np.zeros((TTR_H, TTR_W, 3), np.float64)
        w = np.zeros((TTR_H, TTR_W, 2), np.float64)
        cpu_s, spp, err, rays, paths = 0.0, 0, None, 0, 0
        while spp < TTR_MAX_SPP and cpu_s < TTR_CPU_MAX_SECONDS:
            t0 = time.perf_counter()
            _, _, cnt, _ = osc.render_range(cam, pc, spp, spp + TTR_CPU_CHUNK, threads=threads, accum=a, weights=w)
            cpu_s += time.perf_counter() - t0
            spp += TTR_CPU_CHUNK
            rays += int(cnt[0]) + int(cnt[1])
            paths += n * TTR_CPU_CHUNK
            img = composite(a.reshape(-1, 3)[idx_np], w.reshape(-1, 2)[idx_np])
            err = rel_mse(img, ref_img)
            if err <= TTR_TARGET:
                break
        res["cpu"] = {"seconds": cpu_s if err is not None and err <= TTR_TARGET else None, "spp": spp,
                      "rel_mse": err, "seconds_run": cpu_s, "cores": threads, "kind": "port",
                      "mpaths_per_s": paths / cpu_s / 1e6, "mrays_per_s": rays / cpu_s / 1e6,
                      "sample": f"the full {TTR_W}x{TTR_H} frame, {TTR_CPU_CHUNK} spp per chunk, error on the "
                                f"reference crops after each chunk (outside the timing)"}
    sc.close()
    return res


def box_room_leg(ks, ctx, torch, with_cpu):
    """The box room (5 wall quads, 2 rotated boxes, a rectangular light; 256x256, 64 spp, depth 8):
    device-timed GPU render and, on the host cores, the CPU oracle on the same full frame."""
    g = ks.Generated("box_room", 0)
    s = ks.Scene(ctx, g.desc)
    s.build_bvh()
    cam = ks.camera_perspective(g.camera_to_world, g.vfov, g.aspect)
    p = ks.SmallPTParams.make(render_width=256, render_height=256, spp=64, bounces=8, clamp_indirect=0.0)
    acc = torch.zeros((256, 256, 3), dtype=torch.float64, device="cuda")
    wts = torch.zeros((256, 256, 2), dtype=torch.float64, device="cuda")
    for _ in range(3):
        s.render_device(cam, p, acc.data_ptr(), wts.data_ptr())
    runs = []
    for _ in range(5):
        acc.zero_()
        wts.zero_()
        s.render_device(cam, p, acc.data_ptr(), wts.data_ptr())
        runs.append(s.stats())
    ms = statistics.median(r.ms_total for r in runs)
    st = runs[0]
    out = {"workload": "box_room: 5 wall quads + 2 rotated boxes + 1 area light (36 triangles), 256x256, 64 spp, "
                       "depth 8, clamp_indirect 0",
           "gpu": {"ms": ms, "mrays_per_s": (st.extension_rays + st.shadow_rays) / ms / 1e3,
                   "mpaths_per_s": st.paths / ms / 1e3, "timing": "median of 5 renders, CUDA events"}}
    if with_cpu:
        orc = oracle_module().load()
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        _, _, cnt = orc.scene(g.desc).render(cam, p, threads=threads)
        cpu_s = time.perf_counter() - t0
        out["cpu"] = {"seconds": cpu_s, "mrays_per_s": (int(cnt[0]) + int(cnt[1])) / cpu_s / 1e6,
                      "mpaths_per_s": 256 * 256 * 64 / cpu_s / 1e6, "cores": threads, "kind": "port",
                      "sample": "the whole frame"}
    s.close()
    return out


def batched_leg(ks, ctx, torch, spp_div):
    """C4: 64 seeded scenes built like the icosphere frame (geodesic spheres, triangles
    log-uniform in [1e4, 2e6]), resolutions from {256^2, 512^2, 1024^2, 1920x1080}, spp from
    {32 .. 512} divided by spp_div; one autotuned batch (one CUDA graph launch) against the same
    jobs rendered one after another."""
    import numpy as np
    rng = np.random.default_rng(4)
    resolutions = [(256, 256), (512, 512), (1024, 1024), (1920, 1080)]
    jobs, keep, tris = [], [], []
    for k in range(64):
        n = float(np.exp(rng.uniform(np.log(1e4), np.log(2e6))))
        f = max(1, int(round(np.sqrt(n / 20.0))))
        W, H = resolutions[int(rng.integers(0, 4))]
        spp = max(1, int(2 ** rng.integers(5, 10)) // spp_div)
        g = ks.Generated("icosphere", 100 + k, frequency=f, sky=(2048, 1024), resolution=(W, H))
        s = ks.Scene(ctx, g.desc, keepalive=g)
        s.build_bvh()
        cam = ks.camera_perspective(g.camera_to_world, g.vfov, g.aspect)
        p = ks.SmallPTParams.make(render_width=W, render_height=H, spp=spp, bounces=BOUNCES, rng_seed=k)
        acc = torch.zeros((H, W, 3), dtype=torch.float64, device="cuda")
        wts = torch.zeros((H, W, 2), dtype=torch.float64, device="cuda")
        jobs.append((s, cam, p, acc, wts))
        keep.append(g)
        tris.append(g.n_triangles)
    desc = [(s, c, p, a.data_ptr(), w.data_ptr()) for s, c, p, a, w in jobs]
    t0 = time.perf_counter()
    opts, tune_ms = ks.batch_autotune(ctx, desc)
    tune_s = time.perf_counter() - t0
    for _, _, _, a, w in jobs:
        a.zero_()
        w.zero_()
    st = ks.batch_render(ctx, desc, capacity=opts.capacity, grid_per_sm=opts.grid_per_sm, use_graph=True)
    seq_ms, seq_rays = 0.0, 0
    for s, c, p, a, w in jobs:
        s.render_device(c, p, a.data_ptr(), w.data_ptr())
        ss = s.stats()
        seq_ms += ss.ms_total
        seq_rays += ss.extension_rays + ss.shadow_rays
    for s, *_ in jobs:
        s.close()
    rays = st.extension_rays + st.shadow_rays
    return {"workload": f"64 seeded geodesic-sphere scenes ({min(tris)}..{max(tris)} triangles, log-uniform), "
                        f"resolutions from 256^2/512^2/1024^2/1920x1080, spp 32..512 / {spp_div}, depth {BOUNCES}",
            "paths": st.paths, "pixels": sum(p.render_width * p.render_height for _, _, p, _, _ in jobs),
            "batched": {"ms": st.ms_total, "mrays_per_s": rays / st.ms_total / 1e3,
                        "mpaths_per_s": st.paths / st.ms_total / 1e3, "graph_launches": st.graph_launches,
                        "iterations": st.iterations, "capacity": opts.capacity, "grid_per_sm": opts.grid_per_sm,
                        "autotune_s": tune_s, "autotune_best_sample_ms": tune_ms},
            "sequential": {"ms": seq_ms, "mrays_per_s": seq_rays / seq_ms / 1e3},
            "speedup": seq_ms / st.ms_total if st.ms_total > 0 else None}


def instanced_leg(ks, ctx, torch, spp):
    """C5: 400 instances of 8 displaced geodesic spheres (50k triangles each) + 64 emitters + the
    sky, 3840x2160, depth 16, at `spp` samples per pixel."""
    g = ks.Generated("instanced", 0, sky=(2048, 1024), resolution=(3840, 2160))
    s = ks.Scene(ctx, g.desc, keepalive=g)
    build_ms = s.build_bvh()
    cam = ks.camera_perspective(g.camera_to_world, g.vfov, g.aspect)
    p = ks.SmallPTParams.make(render_width=3840, render_height=2160, spp=spp, bounces=16)
    acc = torch.zeros((2160, 3840, 3), dtype=torch.float64, device="cuda")
    wts = torch.zeros((2160, 3840, 2), dtype=torch.float64, device="cuda")
    s.render_device(cam, ks.SmallPTParams.make(render_width=3840, render_height=2160, spp=1, bounces=16),
                    acc.data_ptr(), wts.data_ptr())
    acc.zero_()
    wts.zero_()
    s.render_device(cam, p, acc.data_ptr(), wts.data_ptr())
    st = s.stats()
    # the same frame guided (the C5 configuration): 1 spp passes, the guide trained online
    lo, hi = g.bound
    guide = ks.Guide(ctx, list(lo - 0.05) + list(hi + 0.05), seed=1)
    pg = ks.SmallPTParams.make(render_width=3840, render_height=2160, spp=spp, bounces=16, spp_prog_interval=1)
    acc.zero_()
    wts.zero_()
    s.render_guided_device(cam, pg, guide, ks.GuideRenderOptions.make(train_passes=1 << 20, train_batch=1 << 18,
                                                                      max_records=1 << 20),
                           acc.data_ptr(), wts.data_ptr())
    sg = s.stats()
    guide.close()
    s.close()
    flat = sum(len(g.meshes[first + k]["indices"]) for proto, _ in g.instances
               for first, n in [g.prototypes[proto]] for k in range(n))
    return {"workload": f"400 instances x 8 geodesic spheres (50,000 triangles each) + 64 emitters + ground, "
                        f"3840x2160, {spp} spp, depth 16",
            "unique_triangles": g.n_triangles, "instanced_triangles": flat, "bvh_build_ms": build_ms,
            "ms": st.ms_total, "mrays_per_s": (st.extension_rays + st.shadow_rays) / st.ms_total / 1e3,
            "mpaths_per_s": st.paths / st.ms_total / 1e3,
            "guided": {"ms": sg.ms_total, "mrays_per_s": (sg.extension_rays + sg.shadow_rays) / sg.ms_total / 1e3,
                       "mpaths_per_s": sg.paths / sg.ms_total / 1e3, "passes": spp,
                       "train_steps": sg.guide_train_steps, "ms_guide_infer": sg.ms_guide_infer,
                       "ms_guide_train": sg.ms_guide_train}}


def cpu_sample_range(step):
    """Sample indices [s0, s1) of the CPU sample of step `step`: consecutive CPU_SPP-sample intervals
    of the SPP samples per pixel, wrapping around."""
    s0 = (step * CPU_SPP) % SPP
    return s0, s0 + CPU_SPP


def run_cpu(orc, desc, camera, params, steps, warmup, threads):
    """The oracle (CPU restatement of small_pt over the reference SBVH) on the full frame, one
    CPU_SPP-sample interval per step; returns the timed totals."""
    t0 = time.perf_counter()
    sc = orc.scene(desc)
    setup_s = time.perf_counter() - t0
    times, rays = [], []
    for k in range(warmup + steps):
        s0, s1 = cpu_sample_range(k)
        t0 = time.perf_counter()
        _, _, cnt, _ = sc.render_range(camera, params, s0, s1, threads=threads)
        dt = time.perf_counter() - t0
        if k >= warmup:
            times.append(dt)
            rays.append(int(cnt[0]) + int(cnt[1]))
    return dict(seconds=sum(times), rays=sum(rays), steps=steps, setup_s=setup_s, scene=sc,
                sample=f"the full {W_RES}x{H_RES} frame, samples [{CPU_SPP} k, {CPU_SPP} (k + 1)) of its {SPP} "
                       f"per pixel in step k ({W_RES * H_RES * CPU_SPP} paths per step), depth {BOUNCES}")


def oracle_work(sc, camera, params, threads, n_spp=2):
    """Per-query work of the frame's ray queries as the restatement of the reference traversal
    counts it (nodes whose bound is tested, triangles tested), over n_spp samples per pixel of the
    full frame; checked against the reference's own queries on every ray."""
    _, _, cnt, wk = sc.render_range(camera, params, 0, n_spp, threads=threads, count_work=True)
    ext, sh = int(cnt[0]), int(cnt[1])
    return {"ext_queries": ext, "ext_nodes_per_query": wk["ext_nodes"] / ext, "ext_tris_per_query": wk["ext_tris"] / ext,
            "shadow_queries": sh, "shadow_nodes_per_query": wk["shadow_nodes"] / max(sh, 1),
            "shadow_tris_per_query": wk["shadow_tris"] / max(sh, 1), "mismatches": wk["mismatches"],
            "sample": f"the full {W_RES}x{H_RES} frame at samples [0, {n_spp}) of {SPP}"}


def bench_config(world):
    """The workload description both arms print (identical for the same N)."""
    return {"workload": WORKLOAD, "triangles": 1310722, "resolution": [W_RES, H_RES], "spp": SPP, "depth": BOUNCES,
            "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (BVH + triangles + sky > 126 MB)"}


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


GUIDE_FLOPS_PER_ROW = 2 * (4 * 64 * 64 + 48 * 64)


def measured_bf16_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        if "bf16_tflops" in d:
            return d["bf16_tflops"], "measured"
    return 1590.0, "fallback"


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def profile_traffic():
    """DRAM bytes per closest-hit query of the traversal kernel, from the committed ncu summary's
    data file (None if absent)."""
    p = os.path.join(ROOT, "profiles", "k_extend_pt_icosphere_l8.json")
    if not os.path.exists(p):
        return None
    return json.load(open(p)).get("dram_bytes_per_query")


def reference_arm(args):
    """The CPU implementation of the path on all host cores, through the oracle only (scene,
    camera and parameters from the oracle library; the CUDA library is not loaded)."""
    rank, local_rank, world = dist_env()
    if rank != 0:
        return 0
    ol = oracle_module()
    orc = ol.load()
    g = orc.generate("icosphere", 0, level=8, sky=(2048, 1024), resolution=(W_RES, H_RES))
    params = orc.params(render_width=W_RES, render_height=H_RES, spp=SPP, bounces=BOUNCES, rng_seed=0)
    threads = os.cpu_count() or 1
    r = run_cpu(orc, g.desc, g.camera, params, args.steps, args.warmup, threads)
    v = r["rays"] / r["seconds"] / 1e6
    line = {
        "impl": "reference", "metric": "Mrays/s (closest-hit + shadow queries), small_pt on the icosphere frame",
        "value": v, "unit": "Mrays/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * r["seconds"] / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
        "config": bench_config(args.gpus),
        "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": threads, "kind": "port", "sample": r["sample"]},
        "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    rank, local_rank, world = dist_env()
    import numpy as np
    import torch
    torch.cuda.set_device(local_rank)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
        pg = dist
    import keepsake_b200 as ks

    ctx = ks.Context(local_rank)
    if args.profile_guided:
        W = args.res or 512
        H = W * 9 // 16
        gg = ks.Generated("icosphere", 0, level=8, sky=(2048, 1024), resolution=(W, H), roughness=(0.02, 0.2),
                          occluder=True)
        sc = ks.Scene(ctx, gg.desc, keepalive=gg)
        sc.build_bvh()
        lo, hi = gg.bound
        guide = ks.Guide(ctx, list(lo - 0.05) + list(hi + 0.05), seed=1)
        pp = ks.SmallPTParams.make(render_width=W, render_height=H, spp=args.spp or 16, bounces=BOUNCES,
                                   spp_prog_interval=1)
        opts = ks.GuideRenderOptions.make(train_passes=1 << 20, train_batch=1 << 16, max_records=1 << 17)
        acc = torch.zeros((H, W, 3), dtype=torch.float64, device="cuda")
        wts = torch.zeros((H, W, 2), dtype=torch.float64, device="cuda")
        cam = ks.camera_perspective(gg.camera_to_world, gg.vfov, gg.aspect)
        if args.profile_unguided:
            sc.render_device(cam, pp, acc.data_ptr(), wts.data_ptr())
        else:
            sc.render_guided_device(cam, pp, guide, opts, acc.data_ptr(), wts.data_ptr())
        print(json.dumps({"profile_case": "unguided" if args.profile_unguided else "guided", "resolution": [W, H],
                          "stats": sc.stats().as_dict()}))
        guide.close()
        sc.close()
        ctx.close()
        return 0
    g = make_generated(ks)
    cam = ks.camera_perspective(g.camera_to_world, g.vfov, g.aspect)
    # replicas: each rank renders the full frame with its own sampler seed
    params = ks.SmallPTParams.make(render_width=W_RES, render_height=H_RES, spp=SPP, bounces=BOUNCES, rng_seed=rank)
    scene = ks.Scene(ctx, g.desc)
    # GPU SBVH build time: median of warm rebuilds (the first build also loads the builder's kernels)
    build_ms = statistics.median([scene.build_bvh() for _ in range(4)][1:])
    acc = torch.zeros((H_RES, W_RES, 3), dtype=torch.float64, device="cuda")
    wts = torch.zeros((H_RES, W_RES, 2), dtype=torch.float64, device="cuda")

    def step():
        acc.zero_()
        wts.zero_()
        torch.cuda.synchronize()
        scene.render_device(cam, params, acc.data_ptr(), wts.data_ptr())
        return scene.stats()

    for _ in range(args.warmup):
        step()
    clocks = ClockSampler(local_rank)
    clocks.start()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    wall0 = time.perf_counter()
    stats = [step() for _ in range(args.steps)]
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    wall = time.perf_counter() - wall0
    clk = clocks.stop()

    dev_ms = sum(s.ms_total for s in stats)
    rays = sum(s.extension_rays + s.shadow_rays for s in stats)
    paths = sum(s.paths for s in stats)
    if pg:
        dev_ms, (rays, paths) = reduce_ranks(pg, torch, dev_ms, [rays, paths], "cuda")
    value = rays / (dev_ms / 1e3) / 1e6

    # the CPU baseline leg: the oracle on a bounded sample of the same frame (rank 0 at N = 1), and
    # the oracle's count of the frame's per-query work for the roofline
    cpu = owork = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        orc = oracle_module().load()
        threads = os.cpu_count() or 1
        r = run_cpu(orc, g.desc, cam, params, 1, 0, threads)
        cpu = {"value": r["rays"] / r["seconds"] / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "port",
               "sample": r["sample"] + "; oracle restatement of small_pt over the reference cuda/sbvh.cu traversal"}
        owork = oracle_work(r["scene"], cam, params, threads)

    # roofline of the dominant kernel (closest-hit traversal).  Algorithmic bytes per query as the
    # oracle counts them on this frame: 32 B per node whose bound the reference traversal tests +
    # 48 B per triangle tested + 32 B ray read + 16 B hit write; beside it the kernel's own count:
    # 64 B per half of each 128-B 4-wide node fetched + 48 B per triangle tested + 48 B ray/hit I/O.
    ext_ms = sum(s.ms_extend for s in stats)
    shade_ms = sum(s.ms_shade for s in stats)
    shadow_ms = sum(s.ms_shadow for s in stats)
    ext_q = sum(s.extension_rays for s in stats)
    kernel_bytes = sum(s.ext_nodes * 64 + s.ext_tris * 48 for s in stats) + ext_q * (32 + 16)
    launches = sum(s.iterations for s in stats)
    peak, peak_kind = measured_peaks()
    achieved_kernel = kernel_bytes / (ext_ms / 1e3) / 1e9
    tpq = profile_traffic()
    roofline = {"kernel": "k_extend_pt (closest-hit SBVH traversal)", "bound": "hbm", "peak": peak,
                "peak_source": peak_kind, "unit": "GB/s",
                "traffic": (tpq * ext_q / launches) if tpq else None,
                "traffic_source": "profiles/k_extend_pt_icosphere_l8.json (ncu DRAM bytes per query x queries per "
                                  "launch)" if tpq else None,
                "achieved_kernel_counted": achieved_kernel, "frac_kernel_counted": achieved_kernel / peak,
                "kernel_bytes_per_launch": kernel_bytes / launches,
                "kernel_wide_nodes_per_query": sum(s.ext_nodes for s in stats) / 2 / ext_q,
                "kernel_tris_per_query": sum(s.ext_tris for s in stats) / ext_q,
                "share": {"extend": ext_ms / dev_ms, "shade_raygen": shade_ms / dev_ms, "shadow": shadow_ms / dev_ms}}
    if owork:
        bpq = 32.0 * owork["ext_nodes_per_query"] + 48.0 * owork["ext_tris_per_query"] + 48.0
        achieved = ext_q * bpq / (ext_ms / 1e3) / 1e9
        roofline.update(achieved=achieved, frac=achieved / peak, algorithmic_bytes_per_query=bpq,
                        algorithmic_bytes_per_launch=ext_q * bpq / launches,
                        bytes_model="32 B x nodes + 48 B x triangles tested by the reference traversal (counted "
                                    "by the oracle on the same frame) + 48 B of ray and hit I/O",
                        oracle_counts=owork)
    else:
        roofline.update(achieved=achieved_kernel, frac=achieved_kernel / peak,
                        algorithmic_bytes_per_launch=kernel_bytes / launches,
                        bytes_model="the kernel's own fetch count (no CPU leg in this run)")

    # ---- end to end through the host-buffer C ABI ----
    e2e_steps = args.e2e_steps if args.e2e_steps is not None else args.steps
    h2d = sum(m["vertices"].nbytes + m["indices"].nbytes for m in g.meshes)
    h2d += len(g.materials) * ctypes.sizeof(ks.MaterialDesc) + (g.sky_map.nbytes if g.sky_map is not None else 0)
    d2h = W_RES * H_RES * 5 * 8
    e2e_rays, e2e_t = 0, 0.0
    e2e_parts = []
    for k in range(e2e_steps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sc = ks.Scene(ctx, g.desc)
        t1 = time.perf_counter()
        sc.build_bvh()
        t2 = time.perf_counter()
        sc.render(cam, params)
        t3 = time.perf_counter()
        st = sc.stats()
        sc.close()
        t4 = time.perf_counter()
        if k == 0:
            continue  # untimed warm-up step
        e2e_t += t4 - t0
        e2e_rays += st.extension_rays + st.shadow_rays
        e2e_parts.append({"scene_create": t1 - t0, "build": t2 - t1, "render": t3 - t2, "render_device": st.ms_total / 1e3,
                          "destroy": t4 - t3})
    if pg:
        e2e_t, (e2e_rays,) = reduce_ranks(pg, torch, e2e_t, [e2e_rays], "cuda")
    e2e = {"value": e2e_rays / e2e_t / 1e6 if e2e_t > 0 else None, "unit": "Mrays/s", "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h, "steps": e2e_steps, "timing": "host wall clock around synchronous C-ABI calls",
           "step_seconds": {key: statistics.median(p[key] for p in e2e_parts) for key in e2e_parts[0]} if e2e_parts
           else None,
           "step_seconds_max": {key: max(p[key] for p in e2e_parts) for key in e2e_parts[0]} if e2e_parts else None}

    ttr = c1 = c4 = c5 = None
    if rank == 0 and world == 1 and not args.no_c1:
        c1 = box_room_leg(ks, ctx, torch, not args.no_cpu_baseline)
    if rank == 0 and world == 1 and not args.no_ttr:
        ttr = time_to_relmse(ks, ctx, torch, not args.no_cpu_baseline)
    if rank == 0 and world == 1 and not args.no_c4:
        c4 = batched_leg(ks, ctx, torch, max(1, args.c4_spp_div))
    if rank == 0 and world == 1 and not args.no_c5:
        c5 = instanced_leg(ks, ctx, torch, max(1, args.c5_spp))

    if rank == 0:
        line = {
            "metric": "Mrays/s (closest-hit + shadow queries), small_pt on the icosphere frame",
            "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": bench_config(world),
            "bvh_build_ms": build_ms,
            "mpaths_per_s": paths / (dev_ms / 1e3) / 1e6,
            # the two query kinds separately, over the same device time
            "mrays_per_s_extension": sum(s.extension_rays for s in stats) / (dev_ms / 1e3) / 1e6,
            "mrays_per_s_shadow": sum(s.shadow_rays for s in stats) / (dev_ms / 1e3) / 1e6,
            "wall_ms_per_step": 1000.0 * wall / args.steps,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": sum(s.kernel_launches for s in stats),
            "clocks": clk,
            "time_to_relmse": ttr,
            "box_room": c1,
            "batched": c4,
            "instanced": c5,
        }
        print(json.dumps(line), flush=True)
    scene.close()
    ctx.close()
    if pg:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
