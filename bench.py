#!/usr/bin/env python
"""Benchmark of the ESVO ray-casting path on B200.

Workload (one step = one frame): the 1024^3 cave scene (value noise, spacing
64, 5 octaves, 50 % fill, depth 10, DXT1 bricks) and 1920x1080 FP32 primary
rays from a seeded empty voxel in a seeded direction; each rank renders its
own camera (weak scaling, no data-path collective).  `value` is Mrays/s of the
device-resident cast kernel (rays and hits in HBM, L2 flushed between steps);
`e2e` is the same metric through vx_cast_rays_host with pinned host buffers,
copies included.  `--impl reference` times the CPU restatement of the
reference castRay on this host's cores instead.
"""
import argparse
import ctypes as C
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "vbvs--vixen_b200")
METRIC = "Mrays/s on 1 B200, batched vs plain at bit-exact hits; fwd+bwd ms/view"


def load_pkg():
    if "vx_b200" in sys.modules:
        return sys.modules["vx_b200"]
    spec = importlib.util.spec_from_file_location("vx_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["vx_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import vx_oracle
    return vx_oracle


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled while work runs."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
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
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 7:
                continue
            try:
                sm.append(float(p[0]))
                mx.append(float(p[1]))
            except ValueError:
                continue
            for k, n in enumerate(names):
                if p[3 + k].lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def make_workload(vx, R, seed, rank, use_gpu_gen):
    from vx_b200 import workloads as W
    import numpy as np
    spacing, octaves = 64 * R // 1024, 5 if R >= 1024 else 3
    if use_gpu_gen:
        bits = vx.synth_noise_dev(R, spacing, octaves, 0.5, seed, False).cpu().numpy().view(np.uint64)
    else:
        bits = vx.synth_noise(R, spacing, octaves, 0.5, seed, False)
    from vx_b200 import multigpu as M
    wl = W.config2(R=R, seed=seed, bits=bits)
    if rank:
        wl.camera = W.empty_voxel_camera(bits, R, M.rank_seed(seed, rank), 70.0, wl.width, wl.height)
    return wl


def bytes_per_launch(n, iters, grid_reads, dda_steps, hits, color_kind):
    """Algorithmic bytes of one cast launch (per-ray terms counted by the traversal):
    24 ray in + 16 hit record out + colour out (12 B DXT1 texel / 4 B RGBA8) per ray,
    8 per ESVO iteration (one descriptor), 4 per brick-grid lookup, 4 per DDA step
    (one occupancy word), plus the colour fetch of every hit (8 B DXT1 block / 4 B RGBA8)."""
    cout, cin = (12, 8) if color_kind == 2 else ((4, 4) if color_kind == 1 else (0, 0))
    return n * (24 + 16 + cout) + 8 * iters + 4 * grid_reads + 4 * dda_steps + cin * hits


def cpu_baseline(vo, wl, rays, g_hits, budget_s=12.0):
    """Times the oracle (CPU restatement of castRay) on a bounded prefix of the
    frame with every host thread, and checks those rays against the GPU."""
    import numpy as np
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    o = vo.OracleScene.from_dense(wl.bits, wl.R, wl.scene.max_levels)
    build_s = time.perf_counter() - t0
    n = min(rays.shape[0], 1 << 16)
    while True:
        t0 = time.perf_counter()
        oh = o.cast_rays(rays[:n], threads=threads)
        dt = time.perf_counter() - t0
        if dt >= budget_s / 4 or n >= rays.shape[0]:
            break
        n = min(rays.shape[0], n * 4)
    g = g_hits[:n]
    hit = (oh["flags"] & 1).astype(bool)
    mism = int(np.count_nonzero((g["flags"].astype(np.uint32) != oh["flags"]) | (g["brick"] != oh["brick"]) |
                                (g["node"] != oh["node"]) | (g["voxel"].astype(np.uint32) != oh["voxel"]) |
                                (hit & (g["t"].view(np.uint32) != oh["t"].view(np.uint32)))))
    return {"value": n / dt / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "port",
            "sample": f"first {n} rays of the frame ({n / rays.shape[0]:.1%}), {threads} threads, "
                      f"{dt:.2f} s; oracle build {build_s:.1f} s"}, {"checked": n, "mismatches": mism}


def run_reference(args, rank, world):
    """CPU restatement of the reference castRay on all host cores."""
    if rank != 0:
        return 0
    import numpy as np
    vx = load_pkg()
    vo = load_oracle()
    use_gpu = False
    try:
        import torch
        use_gpu = torch.cuda.is_available()
    except Exception:
        pass
    wl = make_workload(vx, args.R, args.seed, 0, use_gpu)
    rays = wl.rays(order="tiled")
    threads = os.cpu_count() or 1
    o = vo.OracleScene.from_dense(wl.bits, wl.R, wl.scene.max_levels)
    n = min(rays.shape[0], 1 << 15)
    while True:  # size one step at about 3 s
        t0 = time.perf_counter()
        o.cast_rays(rays[:n], threads=threads)
        dt = time.perf_counter() - t0
        if dt >= 0.75 or n >= rays.shape[0]:
            break
        n = min(rays.shape[0], n * 4)
    n = min(rays.shape[0], max(1024, int(n * 3.0 / max(dt, 1e-3))))
    for _ in range(args.warmup):
        o.cast_rays(rays[:n], threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        o.cast_rays(rays[:n], threads=threads)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    v = n * args.steps / total / 1e6
    line = {"metric": METRIC, "value": v, "unit": "Mrays/s", "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config_dict(wl, world),
            "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": threads, "kind": "port",
                             "sample": f"first {n} of {rays.shape[0]} rays per step, {threads} threads"},
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_cfg4(args, rank, world):
    """Prints the cfg4 line (see measure_cfg4)."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    res = measure_cfg4(args, rank, world, args.steps, args.warmup)
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        line = {"metric": METRIC, "value": res["batched"]["value"], "unit": "Mrays/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["batched"]["ms_per_frame"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": res.pop("config"),
                # per frame: primary cast, octant counts, offsets, compacted bounce spawn, bounce cast
                "gpu_launches": args.steps * 5}
        line.update(res)
        print(json.dumps(line), flush=True)
    return 0


def measure_cfg4(args, rank, world, steps, warmup):
    """cfg4: 64 scenes (64^3..1024^3; noise 10/50 %, urban 90 %; half DXT1) with one camera
    each (256x256..1920x1080) and 2 cosine-weighted bounce rays per hit.  One frame = primary
    pass, bounce spawn, bounce pass.  Batched: the persistent kernel (autotuned) in a CUDA
    graph; plain: one cast launch per scene and pass.  Both produce identical hits."""
    import numpy as np
    import torch
    import torch.distributed as dist
    local = int(os.environ.get("LOCAL_RANK", "0"))
    vx = load_pkg()
    from vx_b200 import workloads as W
    t_setup = time.perf_counter()
    from vx_b200 import multigpu as M
    specs = W.config4_specs(args.scenes, seed=M.rank_seed(4, rank))
    wls, scenes, rays = [], [], []
    for sp in specs:
        bits = None
        if sp.kind == "noise" and sp.R >= 256:
            spacing = max(4, 64 * sp.R // 1024)
            bits = vx.synth_noise_dev(sp.R, spacing, 5 if spacing >= 64 else 3, sp.fill, sp.seed,
                                      False).cpu().numpy().view(np.uint64)
        wl = W.build_spec(sp, bits)
        scenes.append(vx.Scene(wl.scene))
        rays.append(wl.rays(order="tiled"))
        wl.scene.brick_color = None  # host copies are no longer needed
        wls.append(wl)
    setup_s = time.perf_counter() - t_setup
    begin = np.concatenate([[0], np.cumsum([r.shape[0] for r in rays])]).astype(np.int64)
    n = int(begin[-1])
    d_rays = torch.from_numpy(np.concatenate(rays)).cuda()
    d_begin = torch.from_numpy(begin.astype(np.int32)).cuda()
    d_bbegin = torch.from_numpy((2 * begin).astype(np.int32)).cuda()
    ph = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    bh = torch.zeros((2 * n, 4), dtype=torch.int32, device="cuda")
    bounce = torch.zeros((2 * n, 6), dtype=torch.float32, device="cuda")
    batch = vx.Batch(scenes)
    seed = 77
    # Tune each pass on its own rays: the bounce pass is tuned on the bounce rays of this frame.
    tuning, tune_ms = batch.autotune(d_rays, d_begin, ph)
    vx.spawn_bounce_rays(d_rays, ph, seed, bounce)
    btuning, btune_ms = batch.autotune(bounce, d_bbegin, bh)
    batch.set_tuning(tuning.block, tuning.rays_per_task, tuning.stack_in_shared, tuning.refill)
    batch.set_bounce_tuning(btuning)

    def plain_frame():
        for i, sc in enumerate(scenes):
            a, b = int(begin[i]), int(begin[i + 1])
            sc.cast_rays_dev(d_rays[a:b], ph[a:b])
        vx.spawn_bounce_rays(d_rays, ph, seed, bounce)
        for i, sc in enumerate(scenes):
            a, b = 2 * int(begin[i]), 2 * int(begin[i + 1])
            sc.cast_rays_dev(bounce[a:b], bh[a:b])

    plain_frame()
    torch.cuda.synchronize()
    ref_p, ref_b = ph.cpu().numpy().copy(), bh.cpu().numpy().copy()
    stream = torch.cuda.Stream()

    def capture(compact):
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            if compact:  # the bounce pass casts only the bounce rays of primary hits
                batch.capture_frame_compact(d_rays, d_begin, ph, bounce, bh, seed, stream.cuda_stream)
            else:
                batch.capture_frame(d_rays, d_begin, ph, bounce, d_bbegin, bh, seed, stream.cuda_stream)
            ph.zero_()
            bh.zero_()
            batch.launch_frame(stream.cuda_stream)
        torch.cuda.synchronize()
        return bool(np.array_equal(ph.cpu().numpy(), ref_p) and np.array_equal(bh.cpu().numpy(), ref_b))

    identical_full = capture(False)
    nhit = int(np.count_nonzero(ref_p.view(vx.HIT_DTYPE).reshape(-1)["flags"] & 1))
    rays_per_frame = n + 2 * nhit  # primary + bounce rays of hits (miss slots carry a zero direction)

    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    sampler = ClockSampler(local)
    sampler.start()

    def timed(frame_fn, s):
        with torch.cuda.stream(s):
            for _ in range(warmup):
                frame_fn()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        with torch.cuda.stream(s):
            for a, b in ev:
                flush.zero_()
                a.record(s)
                frame_fn()
                b.record(s)
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in ev]

    plain_ms = timed(plain_frame, stream)
    full_ms = timed(lambda: batch.launch_frame(stream.cuda_stream), stream)
    identical = capture(True) and identical_full
    batched_ms = timed(lambda: batch.launch_frame(stream.cuda_stream), stream)
    clocks = sampler.stop()
    from vx_b200 import multigpu as M
    plain_total, batched_total, full_total = M.max_over_ranks([sum(plain_ms), sum(batched_ms), sum(full_ms)])
    value = world * rays_per_frame * steps / (batched_total / 1e3) / 1e6
    plain_value = world * rays_per_frame * steps / (plain_total / 1e3) / 1e6
    return {"config": {"workload": f"cfg4: {len(specs)} scenes 64^3..1024^3 (noise 10/50%, urban 90%, half DXT1), "
                                   f"one camera each 256x256..1920x1080, 2 bounce rays per hit; batched "
                                   f"persistent kernel in a CUDA graph vs {2 * len(specs)} plain launches",
                       "primary_rays": n, "rays_per_frame": rays_per_frame, "hits": nhit,
                       "ray_order": "primary rays in 8x4-pixel warp tiles (workloads.tile_order)",
                       "scene_R": [sp.R for sp in specs], "setup_s": setup_s,
                       "l2": "flushed before every timed frame (256 MiB write)"},
            "batched": {"value": value, "unit": "Mrays/s", "ms_per_frame": batched_total / steps,
                        "frame": "vx_batch_capture_frame_compact: the bounce pass casts the 2 bounce rays of "
                                 "each primary hit only, per scene grouped by direction octant",
                        "ms_per_frame_uncompacted": full_total / steps,
                        "tuning": tuning.as_dict(), "autotune_best_ms_primary": tune_ms,
                        "bounce_tuning": btuning.as_dict(), "autotune_best_ms_bounce": btune_ms},
            "plain": {"value": plain_value, "unit": "Mrays/s", "ms_per_frame": plain_total / steps,
                      "launches_per_frame": 2 * len(specs) + 1},
            "speedup_batched_vs_plain": plain_total / batched_total,
            "hits_identical_batched_vs_plain": identical, "clocks": clocks}


def measure_cfg3(args, steps, warmup):
    """cfg3: 2048^3 urban lattice (32x32 blocks, 8-voxel streets, heights U[64,1800]), DXT1
    bricks, 3840x2160 primary rays plus one shadow ray per hit toward a seeded light.  One frame =
    primary cast, shadow spawn, shadow cast (plain kernel)."""
    import numpy as np
    import torch
    vx = load_pkg()
    from vx_b200 import workloads as W
    t0 = time.perf_counter()
    wl = W.config3(R=args.R if args.R != 1024 else 2048)
    scene = vx.Scene(wl.scene)
    setup_s = time.perf_counter() - t0
    bricks, nodes, dev_bytes = wl.scene.brick_count, wl.scene.node_count, scene.device_bytes()
    wl.scene.brick_color = None
    rays_np = wl.rays(order="tiled")
    n = rays_np.shape[0]
    rays = torch.from_numpy(rays_np).cuda()
    hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    col = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    shadow = torch.zeros((n, 6), dtype=torch.float32, device="cuda")
    sh = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    L = W.light_dir(3)

    def frame_all_slots():  # shadow rays of all n slots, misses included (zero-direction rays)
        scene.cast_rays_dev(rays, hits, col)
        vx.spawn_shadow_rays(rays, hits, L, shadow)
        scene.cast_rays_dev(shadow, sh)

    def frame():  # the shadow rays of the hits only, compacted on the device
        scene.cast_rays_dev(rays, hits, col)
        scene.cast_shadow_rays_dev(rays, hits, L, sh)

    frame_all_slots()
    torch.cuda.synchronize()
    g = hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1)
    nhit = int(np.count_nonzero(g["flags"] & 1))
    ref_sh = sh.cpu().numpy().copy()
    shit = int(np.count_nonzero(ref_sh.view(vx.HIT_DTYPE).reshape(-1)["flags"] & 1))
    sh.fill_(-1)
    frame()
    torch.cuda.synchronize()
    same = bool(np.array_equal(sh.cpu().numpy(), ref_sh))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for a, b in ev:
            flush.zero_()
            a.record()
            fn()
            b.record()
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in ev) / steps

    ms_all = timed(frame_all_slots)
    ms = timed(frame)
    rays_per_frame = n + nhit
    return {"workload": f"{wl.name}: urban {wl.R}^3 (depth {wl.scene.max_levels}), 32x32 blocks, heights "
                        f"U[64,1800], DXT1; {wl.width}x{wl.height} primary + 1 shadow ray per hit",
            "ray_order": "primary rays in 8x4-pixel warp tiles (workloads.tile_order)",
            "mrays_s": rays_per_frame / (ms / 1e3) / 1e6, "ms_per_frame": ms,
            "frame": "primary cast, then vx_cast_shadow_rays (the shadow rays of hits, compacted)",
            "ms_per_frame_all_slots": ms_all, "shadow_hits_equal_all_slots": same, "primary_rays": n,
            "shadow_rays": nhit, "primary_hit_rate": nhit / n, "shadowed_fraction": shit / max(nhit, 1),
            "bricks": bricks, "nodes": nodes, "scene_device_bytes": dev_bytes, "setup_s": setup_s}


def measure_cfg5(args, rank, world, steps, warmup):
    """cfg5: the 512^3 noise scene (30 % fill), 16 views of 512x512; per variant (per-voxel
    FP32 RGB, FP32 DXT1 endpoints) the forward-with-record time and the forward+adjoint time per
    view (the 16 views as one forward launch and one adjoint launch), the FP64 CPU gradient check
    and central finite differences (h = 1e-3) on 1000 entries."""
    import numpy as np
    import torch
    vx = load_pkg()
    from vx_b200 import workloads as W
    R = 512
    bits = vx.synth_noise_dev(R, 32, 4, 0.30, 5, False).cpu().numpy().view(np.uint64)
    out = {}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for kind, name in ((0, "voxel_rgb"), (1, "dxt1_endpoints")):
        dw = W.config5(R=R, views=16, width=512, height=512, kind=kind, seed=5, bits=bits)
        scene = vx.Scene(dw.wl.scene)
        n = 512 * 512
        attr_d = torch.from_numpy(dw.attr).cuda()
        idx_d = None if dw.dxt_idx is None else torch.from_numpy(dw.dxt_idx.view(np.int32)).cuda()
        tgt_attr = torch.from_numpy(dw.target_attr).cuda()
        # all 16 views in one forward launch and one adjoint launch (view-major buffers)
        V = len(dw.views)
        img_all = torch.zeros((V * n, 3), dtype=torch.float32, device="cuda")
        rec_all = torch.zeros((V * n, 4), dtype=torch.int32, device="cuda")
        tgt_all = torch.zeros((V * n, 3), dtype=torch.float32, device="cuda")
        imgs = [img_all[v * n:(v + 1) * n] for v in range(V)]
        recs = [rec_all[v * n:(v + 1) * n] for v in range(V)]
        tgts = [tgt_all[v * n:(v + 1) * n] for v in range(V)]
        vx.diff_forward_views(scene, dw.views, 512, 512, kind, tgt_attr, idx_d, tgt_all, rec_all)
        grad = torch.zeros_like(attr_d)
        loss = torch.zeros(1, dtype=torch.float32, device="cuda")

        def fwd():
            vx.diff_forward_views(scene, dw.views, 512, 512, kind, attr_d, idx_d, img_all, rec_all)

        def fwdbwd():
            grad.zero_()
            loss.zero_()
            vx.diff_forward_views(scene, dw.views, 512, 512, kind, attr_d, idx_d, img_all, rec_all)
            vx.diff_backward(kind, idx_d, rec_all, img_all, tgt_all, grad, loss)

        def timed(fn):
            for _ in range(warmup):
                fn()
            torch.cuda.synchronize()
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
            for a, b in ev:
                flush.zero_()
                a.record()
                fn()
                b.record()
            torch.cuda.synchronize()
            return sum(a.elapsed_time(b) for a, b in ev) / steps

        f_ms = timed(fwd)
        fb_ms = timed(fwdbwd)
        g = grad.cpu().numpy().astype(np.float64)
        rec_np = [r.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1) for r in recs]
        tgt_np = [t.cpu().numpy() for t in tgts]
        ref = W.adjoint_reference64(dw, rec_np, tgt_np)
        rel64 = float(np.linalg.norm(g - ref) / np.linalg.norm(ref))
        # central finite differences of the GPU forward on 1000 touched entries
        rng = np.random.default_rng(11)
        stride = 3 if kind == 0 else 6
        touched = np.flatnonzero(np.abs(ref) > 1e-4 * np.abs(ref).max())
        fd_err = 0.0
        checked = 0
        for ch in range(stride):
            cand = touched[touched % stride == ch]
            sel = rng.choice(cand, size=min(-(-1000 // stride), cand.size), replace=False)
            h = np.float32(1e-3)
            res = []
            for sgn in (1, -1):
                pert = dw.attr.copy()
                pert[sel] += sgn * h
                pd = torch.from_numpy(pert).cuda()
                dl = np.zeros(dw.attr.shape[0], np.float64)
                for v, pc in enumerate(dw.views):
                    vx.diff_forward(scene, pc, 512, 512, kind, pd, idx_d, imgs[v], recs[v])
                    p64 = imgs[v].cpu().numpy().astype(np.float64)
                    r = rec_np[v]
                    hit = (r["flags"] & 1).astype(bool)
                    key = (r["brick"].astype(np.int64) * 512 + r["voxel"]) if kind == 0 else \
                        (r["brick"].astype(np.int64) * 32 + (r["voxel"].astype(np.int64) >> 4))
                    np.add.at(dl, key[hit] * stride + ch, ((p64 - tgt_np[v].astype(np.float64)) ** 2).sum(1)[hit])
                res.append(dl)
            fd = (res[0] - res[1]) / (2.0 * float(h))
            fd_err = max(fd_err, float(np.max(np.abs(fd[sel] - g[sel]) / np.maximum(np.abs(g[sel]), 1e-6))))
            checked += sel.size
        out[name] = {"fwd_ms_per_view": f_ms / 16, "fwd_bwd_ms_per_view": fb_ms / 16, "ratio": fb_ms / f_ms,
                     "fp64_grad_rel_err": rel64, "fd_max_rel_err": fd_err, "fd_entries": checked,
                     "hit_rate": float(np.mean([(r["flags"] & 1).mean() for r in rec_np])),
                     "attributes": int(dw.attr.shape[0])}
        del scene
    return {"workload": "cfg5: 512^3 noise 30% fill, 16 views 512x512 on an orbit, L2 loss vs targets rendered "
                        "from colours + N(0, 0.05)", **out}


def measure_cfg5_multi(args, rank, world, steps, warmup):
    """cfg5 on N GPUs (strong scaling): the 16 views of a step split over the ranks
    (multigpu.view_range), each rank's forward + adjoint into its own gradient pool, one NCCL sum
    all-reduce of the pool (the adjoint's one exchange); ms per view = max over ranks / 16."""
    import numpy as np
    import torch
    vx = load_pkg()
    from vx_b200 import workloads as W
    from vx_b200 import multigpu as M
    R = 512
    bits = vx.synth_noise_dev(R, 32, 4, 0.30, 5, False).cpu().numpy().view(np.uint64)
    out = {}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for kind, name in ((0, "voxel_rgb"), (1, "dxt1_endpoints")):
        dw = W.config5(R=R, views=16, width=512, height=512, kind=kind, seed=5, bits=bits)
        scene = vx.Scene(dw.wl.scene)
        b, e = M.view_range(len(dw.views), rank, world)
        mine = dw.views[b:e]
        n = 512 * 512 * max(1, len(mine))
        attr_d = torch.from_numpy(dw.attr).cuda()
        idx_d = None if dw.dxt_idx is None else torch.from_numpy(dw.dxt_idx.view(np.int32)).cuda()
        img = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
        rec = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
        tgt = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
        if mine:
            vx.diff_forward_views(scene, mine, 512, 512, kind, torch.from_numpy(dw.target_attr).cuda(), idx_d, tgt,
                                  rec)
        grad = torch.zeros_like(attr_d)

        def step():
            grad.zero_()
            if mine:
                vx.diff_forward_views(scene, mine, 512, 512, kind, attr_d, idx_d, img, rec)
                vx.diff_backward(kind, idx_d, rec, img, tgt, grad)
            M.allreduce_sum_(grad)

        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        torch.distributed.barrier()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for a, bb in ev:
            flush.zero_()
            a.record()
            step()
            bb.record()
        torch.cuda.synchronize()
        ms = M.max_over_ranks([sum(a.elapsed_time(bb) for a, bb in ev) / steps])[0]
        out[name] = {"fwd_bwd_allreduce_ms_per_view": ms / 16, "views_per_rank": len(mine),
                     "gradient_pool_bytes": int(attr_d.numel() * 4)}
        del scene
    return {"workload": "cfg5: 512^3 noise 30% fill, 16 views 512x512 on an orbit split over ranks, gradient "
                        "pool summed by one NCCL all-reduce per step", **out}


def measure_next(args, steps, warmup):
    """The rows beyond the cast (1024^3 cave, seed 2, the cfg2 scene): the device scene
    builder against the host builder, the normal and DXT1 payload encoders, the LOD cut,
    the compressed render and the scene cache file.  Device times are CUDA events."""
    import math
    import tempfile
    import numpy as np
    import torch
    vx = load_pkg()
    from vx_b200 import workloads as W
    R, seed = args.R, args.seed
    out = {"workload": f"cave {R}^3 (depth 10), noise spacing 64, 5 octaves, 50% fill, seed {seed}"}
    ev = lambda: torch.cuda.Event(enable_timing=True)

    def dev_ms(fn, reps=steps):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        a, b = ev(), ev()
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    bits_t = vx.synth_noise_dev(R, 64 * R // 1024, 5 if R >= 1024 else 3, 0.5, seed, False)
    torch.cuda.synchronize()
    # device builder (the call returns when the scene is complete: host clock)
    t = []
    for k in range(3):
        t0 = time.perf_counter()
        sc = vx.scene_from_dense_dev(bits_t, R, 10, vx.VX_COLOR_DXT1, seed ^ 0xD7C1, k == 2)
        t.append(time.perf_counter() - t0)
        if k < 2:
            sc.close()
    bits = bits_t.cpu().numpy().view(np.uint64)
    t0 = time.perf_counter()
    host = vx.build_dense(bits, R, 10)
    host_s = time.perf_counter() - t0
    got = sc.download()
    same = all(np.array_equal(getattr(got, k), getattr(host, k))
               for k in ("nodes", "node_brick", "grid_lookup", "brick_coord", "brick_occ"))
    B = host.brick_count
    out["device_builder"] = {"bricks": B, "nodes": host.node_count, "device_s": min(t[:2]),
                             "device_s_with_dxt1_and_normals": t[2], "host_build_dense_s": host_s,
                             "identical_to_host_builder": bool(same)}
    # payload encoders
    occ_t = torch.from_numpy(host.brick_occ.view(np.int32)).cuda()
    nrm_t = torch.zeros(B * 64, dtype=torch.int64, device="cuda")
    ms = dev_ms(lambda: vx.build_normals_dev(occ_t, nrm_t))
    out["normal_payload"] = {"bricks": B, "device_ms": ms, "mbricks_s": B / ms / 1e3,
                             "equals_scene_payload": bool(np.array_equal(nrm_t.cpu().numpy().view(np.uint64),
                                                                         got.brick_normal.reshape(-1)))}
    nb = min(B, 262144)
    rgba = vx.synth_rgba8(host.brick_coord[:nb], seed)
    rgb_t = torch.from_numpy(np.stack([(rgba >> s_) & 255 for s_ in (0, 8, 16)], -1).astype(np.float32)
                             / np.float32(255.0)).reshape(-1).cuda()
    dxt_t = torch.zeros(nb * 32, dtype=torch.int64, device="cuda")
    occ_sub = occ_t[:nb * 16].contiguous()
    ms = dev_ms(lambda: vx.build_dxt1_dev(rgb_t, occ_sub, dxt_t))
    out["dxt1_encode"] = {"bricks": nb, "colours": "RGBA8 words / 255", "device_ms": ms, "mbricks_s": nb / ms / 1e3}
    del rgb_t, dxt_t, occ_t, nrm_t
    # LOD cut and compressed render on the cfg2 camera
    wl = W.config2(R=R, seed=seed, bits=bits)
    rays = torch.from_numpy(wl.rays(order="tiled")).cuda()
    n = rays.shape[0]
    hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    base = vx.lod_from_camera(math.radians(70.0), wl.height)
    plain_ms = dev_ms(lambda: sc.cast_rays_dev(rays, hits))
    lod_rows = []
    for bias in (0.0, 7.0):
        lod = vx.lod_with_bias(base, bias)
        ms = dev_ms(lambda: sc.cast_rays_dev(rays, hits, lod=lod))
        h = hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1)
        lod_rows.append({"bias": bias, "ray_dir_size": lod.ray_dir_size, "mrays_s": n / ms / 1e3,
                         "lod_hit_fraction": float(np.mean(((h["flags"] & 1) == 1) & (h["brick"] == 0xFFFFFFFF)))})
    out["lod"] = {"rays": n, "castRayScreenSpaceLOD": "70 deg, 1080 rows, times 2^bias",
                  "plain_mrays_s": n / plain_ms / 1e3, "runs": lod_rows}
    img = torch.zeros(n, dtype=torch.int32, device="cuda")
    ms = dev_ms(lambda: sc.render_dev(wl.camera, wl.width, wl.height, img))
    out["compressed_render"] = {"pixels": n, "payloads": "DXT1 colour + DXT normals", "device_ms": ms,
                                "mrays_s": n / ms / 1e3}
    # the reference's published benchmark shape: noise 256^3, 1920x1080 primary rays (context only:
    # the reference's numbers are Vulkan runs on other GPUs, with its own scene instance and camera)
    wl256 = W.config2(R=256, seed=seed)
    s256 = vx.Scene(wl256.scene)
    r256 = torch.from_numpy(wl256.rays(order="tiled")).cuda()
    h256 = torch.zeros((r256.shape[0], 4), dtype=torch.int32, device="cuda")
    c256 = torch.zeros((r256.shape[0], 3), dtype=torch.float32, device="cuda")
    ms = dev_ms(lambda: s256.cast_rays_dev(r256, h256, c256))
    out["noise256_1080p"] = {"workload": "noise 256^3 (50% fill, DXT1), 1920x1080 primary rays, plain cast",
                             "mrays_s": r256.shape[0] / ms / 1e3, "ms_per_frame": ms,
                             "published_context": "the reference's published runs of this shape: 4,573 / 4,688 "
                                                  "Mrays/s uncompressed / DXT, RTX 4080 Laptop, Vulkan (not "
                                                  "comparable hardware or scene instance)"}
    s256.close()
    del r256, h256, c256
    # scene cache file
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "cave.vxsc")
        t0 = time.perf_counter()
        sc.save(path)
        save_s = time.perf_counter() - t0
        size = os.path.getsize(path)
        t0 = time.perf_counter()
        sl = vx.Scene.load(path)
        torch.cuda.synchronize()
        load_s = time.perf_counter() - t0
        h2 = torch.zeros_like(hits)
        sl.cast_rays_dev(rays, h2)
        sc.cast_rays_dev(rays, hits)
        torch.cuda.synchronize()
        out["scene_cache"] = {"format": "VXSC", "bytes": size, "save_s": save_s, "load_s": load_s,
                              "hits_equal_after_load": bool(torch.equal(hits, h2))}
        sl.close()
    sc.close()
    return out


def measure_tour(args):
    """One pass over every kernel of the library on the cfg2 scene (1024^3 cave) and small
    companions, each step timed with CUDA events (mean of 3 after 1 warm-up): noise synthesis,
    device builder with both payloads, the RGBA8 builder, plain / counting / LOD casts, the
    compressed render, per-hit normal decode, the payload encoders, the batched kernels (static
    and refilling lanes, bounce and shadow spawn, the no-allocation entry point, a frame with
    bounce compaction) and the adjoint pair.  Meant as the command an ncu launch list or a per-kernel capture runs."""
    import math
    import numpy as np
    import torch
    vx = load_pkg()
    from vx_b200 import workloads as W
    out = {}

    def ev_ms(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    R, seed = 1024, 2
    holder = {}
    out["synth_noise_1024"] = ev_ms(lambda: holder.__setitem__("bits", vx.synth_noise_dev(R, 64, 5, 0.5, seed, False)))
    bits = holder["bits"]
    t0 = time.perf_counter()
    sc = vx.scene_from_dense_dev(bits, R, 10, vx.VX_COLOR_DXT1, seed ^ 0xD7C1, True)
    torch.cuda.synchronize()
    out["device_build_1024_dxt1_normals_host_clock"] = (time.perf_counter() - t0) * 1e3
    bits256 = vx.synth_noise_dev(256, 16, 3, 0.5, 3, False)
    sc_rgba = vx.scene_from_dense_dev(bits256, 256, 8, vx.VX_COLOR_RGBA8, 3, False)
    bits_np = bits.cpu().numpy().view(np.uint64)
    cam = W.empty_voxel_camera(bits_np, R, seed, 70.0, 1920, 1080)
    rays = torch.from_numpy(vx.camera_rays(cam, 1920, 1080)[W.tile_order(1920, 1080)]).cuda()
    n = rays.shape[0]
    hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    color = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    counters = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    out["cast_1080p"] = ev_ms(lambda: sc.cast_rays_dev(rays, hits, color))
    out["cast_1080p_counters"] = ev_ms(lambda: sc.cast_rays_dev(rays, hits, color, counters))
    lod = vx.lod_with_bias(vx.lod_from_camera(math.radians(70.0), 1080), 7.0)
    out["cast_1080p_lod_bias7"] = ev_ms(lambda: sc.cast_rays_dev(rays, hits, lod=lod))
    img = torch.zeros(n, dtype=torch.int32, device="cuda")
    out["render_1080p_dxt1_normals"] = ev_ms(lambda: sc.render_dev(cam, 1920, 1080, img, hits))
    nrm = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    out["hit_normals_1080p"] = ev_ms(lambda: sc.hit_normals_dev(hits, nrm))
    a = sc.download()
    B = a.brick_count
    occ = torch.from_numpy(a.brick_occ.view(np.int32).reshape(-1)).cuda()
    nout = torch.zeros(B * 64, dtype=torch.int64, device="cuda")
    out["normal_payload_1024"] = ev_ms(lambda: vx.build_normals_dev(occ, nout))
    nb = min(B, 262144)
    rgba = vx.synth_rgba8(a.brick_coord[:nb], seed)
    rgb = torch.from_numpy(np.stack([(rgba >> s_) & 255 for s_ in (0, 8, 16)], -1).astype(np.float32)
                           / np.float32(255.0)).reshape(-1).cuda()
    dout = torch.zeros(nb * 32, dtype=torch.int64, device="cuda")
    occ_sub = occ[:nb * 16].contiguous()
    out["dxt1_payload_262k"] = ev_ms(lambda: vx.build_dxt1_dev(rgb, occ_sub, dout))
    del a, occ, nout, rgb, dout, occ_sub
    # batched: the cave frame and 2^18 random rays through the 256^3 RGBA8 scene
    r2 = torch.from_numpy(W.random_rays(262144, 256, seed=9)).cuda()
    brays = torch.cat([rays, r2])
    begin = torch.tensor([0, n, n + r2.shape[0]], dtype=torch.int32, device="cuda")
    bh = torch.zeros((brays.shape[0], 4), dtype=torch.int32, device="cuda")
    batch = vx.Batch([sc, sc_rgba])
    batch.set_tuning(256, 32, 1, 0)
    out["batch_static"] = ev_ms(lambda: batch.cast(brays, begin, bh))
    bounce = torch.zeros((2 * brays.shape[0], 6), dtype=torch.float32, device="cuda")
    out["spawn_bounce"] = ev_ms(lambda: vx.spawn_bounce_rays(brays, bh, 77, bounce))
    bbegin = begin * 2
    bbh = torch.zeros((bounce.shape[0], 4), dtype=torch.int32, device="cuda")
    batch.set_tuning(128, 256, 0, 24)
    out["batch_refill_bounce"] = ev_ms(lambda: batch.cast(bounce, bbegin, bbh))
    shadow = torch.zeros_like(brays)
    out["spawn_shadow"] = ev_ms(lambda: vx.spawn_shadow_rays(brays, bh, [0.3, 0.8, 0.5], shadow))
    out["batch_noalloc"] = ev_ms(lambda: vx.cast_batch_noalloc([sc, sc_rgba], brays, begin, bh))
    # a frame with bounce compaction (hit count, chunk scan, compacted spawn, scene offsets)
    batch.set_tuning(256, 32, 1, 0)
    batch.set_bounce_tuning(vx.BatchTuning(128, 256, 0, 24))
    fs = torch.cuda.Stream()
    torch.cuda.synchronize()
    with torch.cuda.stream(fs):
        batch.capture_frame_compact(brays, begin, bh, bounce, bbh, 77, fs.cuda_stream)
        out["frame_compact"] = ev_ms(lambda: batch.launch_frame(fs.cuda_stream))
    batch.close()
    del bounce, bbh, shadow, brays, bh
    # adjoint pair on a 256^3 scene, 4 views of 512x512, per-voxel RGB and DXT1 endpoints
    bits_d = vx.synth_noise_dev(256, 16, 3, 0.30, 5, False)
    sd = vx.scene_from_dense_dev(bits_d, 256, 8, vx.VX_COLOR_NONE, 0, False)
    Bd = int(sd.info().brick_count)
    c = 128.0
    views = [W.look_camera([c + 243 * math.cos(t), c + 20.0, c + 243 * math.sin(t)],
                           [-243 * math.cos(t), -20.0, -243 * math.sin(t)], 60.0, 512, 512)
             for t in (0.3, 1.9, 3.5, 5.1)]
    V, npx = len(views), 512 * 512
    gen = torch.Generator(device="cuda").manual_seed(5)
    for kind, name, per in ((0, "rgb", Bd * 512 * 3), (1, "dxt1_endpoints", Bd * 32 * 6)):
        attr = torch.rand(per, device="cuda", generator=gen)
        idx = None if kind == 0 else torch.randint(-2 ** 31, 2 ** 31 - 1, (Bd * 32,), device="cuda",
                                                   dtype=torch.int32, generator=gen)
        imgs = torch.zeros((V * npx, 3), dtype=torch.float32, device="cuda")
        rec = torch.zeros((V * npx, 4), dtype=torch.int32, device="cuda")
        tgt = torch.rand((V * npx, 3), device="cuda", generator=gen)
        grad = torch.zeros_like(attr)
        loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        out[f"diff_forward_4x512_{name}"] = ev_ms(
            lambda: vx.diff_forward_views(sd, views, 512, 512, kind, attr, idx, imgs, rec))
        out[f"diff_backward_4x512_{name}"] = ev_ms(lambda: vx.diff_backward(kind, idx, rec, imgs, tgt, grad, loss))
    sd.close()
    sc_rgba.close()
    sc.close()
    return {"workload": "kernel tour: cave 1024^3 (cfg2 scene, DXT1 + normals), 1920x1080 tiled rays, "
                        "256^3 RGBA8 companion with 2^18 random rays, 256^3 adjoint scene with 4 views of 512x512",
            "ms": out}


def config_dict(wl, world):
    return {"workload": f"{wl.name}: cave {wl.R}^3 (depth {wl.scene.max_levels}), value noise spacing "
                        f"{64 * wl.R // 1024}, 5 octaves, 50% fill, DXT1 bricks, {wl.width}x{wl.height} FP32 "
                        f"primary rays per rank, plain cast kernel",
            "ray_order": "8x4-pixel warp tiles in 32x8 blocks (vx_render's order; workloads.tile_order)",
            "rays_per_step_per_gpu": wl.width * wl.height, "bricks": int(wl.scene.brick_count),
            "nodes": int(wl.scene.node_count), "parallelism": f"replicated scene, {world} camera(s)",
            "l2": "flushed between timed steps (256 MiB write)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="vx", choices=["vx", "reference"])
    ap.add_argument("--R", type=int, default=1024)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="cfg2", choices=["cfg2", "cfg3", "cfg4", "cfg5", "next", "tour"],
                    help="cfg2: plain cast of the 1024^3 cave frame (with the cfg4, cfg5 and next-row results "
                         "attached at N=1); cfg4: 64-scene batched frame vs plain; cfg5: forward / adjoint ms per "
                         "view; next: device builder, payload encoders, LOD cut, compressed render, cache file; "
                         "tour: every kernel once, CUDA-event times per step (the command for ncu captures)")
    ap.add_argument("--no-extra", action="store_true",
                    help="cfg2 only: skip the attached batched (cfg4), adjoint (cfg5) and next-row measurements")
    ap.add_argument("--scenes", type=int, default=64, help="cfg4: number of scenes")
    ap.add_argument("--split-views", action="store_true",
                    help="cfg5: split the views over the ranks and all-reduce the gradient (default when N > 1; "
                         "needs a process group, i.e. torchrun, also for N = 1)")
    ap.add_argument("--soak-seconds", type=float, default=1.5,
                    help="untimed launches before timing so clocks reach steady state")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "cfg4":
        return run_cfg4(args, rank, world)
    if args.workload == "cfg3":
        import torch
        torch.cuda.set_device(local)
        res = measure_cfg3(args, args.steps, args.warmup)
        if rank == 0:
            line = {"metric": METRIC, "value": res["mrays_s"], "unit": "Mrays/s", "n_gpus": 1, "steps": args.steps,
                    "warmup": args.warmup, "ms_per_step": res["ms_per_frame"], "higher_is_better": True,
                    "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                    # per frame: primary cast, shadow hit count, scan, compacted spawn, shadow cast
                    "config": {"workload": res.pop("workload")}, "gpu_launches": args.steps * 5}
            line.update(res)
            print(json.dumps(line), flush=True)
        return 0
    if args.workload == "tour":
        import torch
        torch.cuda.set_device(local)
        res = measure_tour(args)
        if rank == 0:
            print(json.dumps({"workload": "tour", "tour": res}), flush=True)
        return 0
    if args.workload == "next":
        res = measure_next(args, args.steps, args.warmup)
        if rank == 0:
            print(json.dumps({"workload": "next", "next_rows": res}), flush=True)
        return 0
    if args.workload == "cfg5" and (world > 1 or args.split_views):
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
        res = measure_cfg5_multi(args, rank, world, args.steps, args.warmup)
        dist.destroy_process_group()
        if rank == 0:
            a = res["voxel_rgb"]
            print(json.dumps({"metric": METRIC, "value": a["fwd_bwd_allreduce_ms_per_view"], "unit": "ms/view",
                              "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                              "ms_per_step": a["fwd_bwd_allreduce_ms_per_view"] * 16, "higher_is_better": False,
                              "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                              "config": {"workload": res.pop("workload")}, "adjoint": res,
                              "gpu_launches": args.steps * 2}), flush=True)
        return 0
    if args.workload == "cfg5":
        import torch
        torch.cuda.set_device(local)
        res = measure_cfg5(args, rank, world, args.steps, args.warmup)
        if rank == 0:
            a = res["voxel_rgb"]
            print(json.dumps({"metric": METRIC, "value": a["fwd_bwd_ms_per_view"], "unit": "ms/view", "n_gpus": 1,
                              "steps": args.steps, "warmup": args.warmup,
                              "ms_per_step": a["fwd_bwd_ms_per_view"] * 16, "higher_is_better": False,
                              "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                              "config": {"workload": res.pop("workload")}, "adjoint": res,
                              "gpu_launches": args.steps * 2}), flush=True)  # per fwd+bwd step: 1 forward, 1 adjoint
        return 0

    import numpy as np
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    vx = load_pkg()
    wl = make_workload(vx, args.R, args.seed, rank, True)
    scene = vx.Scene(wl.scene)
    rays_np = wl.rays(order="tiled")
    n = rays_np.shape[0]
    rays = torch.from_numpy(rays_np).cuda()
    hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    color = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    counters = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()

    # Counting pass (untimed): per-ray work for the algorithmic-byte count.
    scene.cast_rays_dev(rays, hits, color, counters)
    torch.cuda.synchronize()
    cnt = counters.cpu().numpy().view(vx.COUNTER_DTYPE).reshape(-1)
    g_hits = hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1).copy()
    nhit = int(np.count_nonzero(g_hits["flags"] & 1))
    tot = {k: int(cnt[k].astype(np.int64).sum()) for k in cnt.dtype.names}
    # Bytes the kernel has to move (iterations after a detected cycle repeat
    # data already read and are not counted) and, for reference, the bytes of
    # the full 500-iteration reference loop.
    algo_bytes = bytes_per_launch(n, tot["run_iters"], tot["run_grid_reads"], tot["run_dda_steps"], nhit,
                                  scene.color_kind)
    ref_bytes = bytes_per_launch(n, tot["iters"], tot["grid_reads"], tot["dda_steps"], nhit, scene.color_kind)

    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    sampler = ClockSampler(local)
    sampler.start()
    t_soak = time.perf_counter()
    for _ in range(args.warmup):
        scene.cast_rays_dev(rays, hits, color)
    torch.cuda.synchronize()
    while time.perf_counter() - t_soak < args.soak_seconds:  # clocks to steady state before timing
        for _ in range(20):
            scene.cast_rays_dev(rays, hits, color)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.zero_()
        ev0[k].record(stream)
        scene.cast_rays_dev(rays, hits, color)
        ev1[k].record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in zip(ev0, ev1)]
    total_ms = sum(step_ms)

    # e2e through the host-buffer entry point: pinned rays in, hits + texels out.
    rays_h = torch.from_numpy(rays_np).pin_memory()
    hits_h = torch.zeros((n, 4), dtype=torch.int32).pin_memory()
    col_h = torch.zeros((n, 3), dtype=torch.float32).pin_memory()
    L = vx.lib()

    def e2e_call():
        vx.check(L.vx_cast_rays_host(scene.handle, C.c_void_p(rays_h.data_ptr()), n, 0.0, vx.FLT_MAX,
                                     C.c_void_p(hits_h.data_ptr()), C.c_void_p(col_h.data_ptr()),
                                     C.c_void_p(stream.cuda_stream)))

    for _ in range(args.warmup):
        e2e_call()
    e0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    e1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.zero_()
        e0[k].record(stream)
        e2e_call()
        e1[k].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    e2e_ms = sum(a.elapsed_time(b) for a, b in zip(e0, e1))
    e2e_same = bool(np.array_equal(hits_h.numpy().view(np.uint8), g_hits.view(np.uint8).reshape(n, 16)))

    from vx_b200 import multigpu as M
    total_ms, e2e_ms = M.max_over_ranks([total_ms, e2e_ms])
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0

    value = M.aggregate_throughput(n * args.steps, world, total_ms / 1e3) / 1e6
    e2e_value = M.aggregate_throughput(n * args.steps, world, e2e_ms / 1e3) / 1e6
    mean_s = statistics.mean(step_ms) / 1e3
    peak, peak_kind = measured_peaks()
    achieved = algo_bytes / mean_s / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "cast_kernel_traffic.json")
    if os.path.exists(tf):
        try:
            with open(tf) as f:
                d = json.load(f)
            if d.get("workload") == wl.name:
                traffic = d.get("dram_bytes_per_launch")
        except Exception:
            pass
    line = {"metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_dict(wl, world),
            "e2e": {"value": e2e_value, "unit": "Mrays/s", "h2d_bytes_per_step": world * n * 24,
                    "d2h_bytes_per_step": world * n * (16 + 12), "hits_equal_device_path": e2e_same},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": algo_bytes,
                         "reference_loop_bytes_per_launch": ref_bytes,
                         "per_ray": {k: v / n for k, v in tot.items()},
                         "kernel": "vx::cast_kernel", "kernel_ms_mean": mean_s * 1e3},
            "gpu_launches": args.steps, "hit_rate": nhit / n,
            "clocks": clocks}
    if world == 1 and not args.no_cpu_baseline:
        vo = load_oracle()
        cb, parity = cpu_baseline(vo, wl, rays_np, g_hits)
        line["cpu_baseline"] = cb
        line["parity_sample"] = parity
    if world == 1 and not args.no_extra:
        del scene
        torch.cuda.empty_cache()
        extra_steps, extra_warmup = max(3, min(args.steps, 5)), max(2, min(args.warmup, 3))
        b = measure_cfg4(args, rank, world, extra_steps, extra_warmup)
        line["batched"] = {"workload": b["config"]["workload"], "rays_per_frame": b["config"]["rays_per_frame"],
                           "batched_mrays_s": b["batched"]["value"], "plain_mrays_s": b["plain"]["value"],
                           "speedup_batched_vs_plain": b["speedup_batched_vs_plain"],
                           "batched_ms_per_frame": b["batched"]["ms_per_frame"],
                           "batched_ms_per_frame_uncompacted": b["batched"]["ms_per_frame_uncompacted"],
                           "hits_identical": b["hits_identical_batched_vs_plain"], "tuning": b["batched"]["tuning"],
                           "steps": extra_steps}
        torch.cuda.empty_cache()
        line["adjoint"] = measure_cfg5(args, rank, world, extra_steps, extra_warmup)
        torch.cuda.empty_cache()
        line["next_rows"] = measure_next(args, extra_steps, extra_warmup)
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
