#!/usr/bin/env python
"""Benchmark of the ESVO ray-casting path on B200.

Headline (default, one step = one frame): the batched frame of 64 scenes
(64^3..1024^3; noise at 10/50 % fill, urban lattices at 90 %; half of them
with DXT1 bricks), one camera each (256x256..1920x1080) and two
cosine-weighted bounce rays per primary hit.  The frame runs as one CUDA
graph: the persistent batched cast of every primary ray, the compaction of
the bounce rays of hits, the batched bounce cast.  `value` is Mrays/s of that
frame (primary rays + bounce rays of hits) with every input resident in HBM;
the plain arm casts the same rays with one launch per scene and pass; `e2e`
is the same frame through vx_batch_launch_frame_host with pinned host
buffers.  The line also carries the 1024^3 cave frame (cfg2), the 2048^3
urban frame with shadow rays (cfg3), the adjoint (cfg5) and the rows beyond
the cast.  `--impl reference` times the CPU restatement of the reference
castRay (the oracle) on this host's cores over a sample of the same frame,
its inputs built on the oracle side without the product library.
"""
import argparse
import concurrent.futures as cf
import ctypes as C
import glob
import hashlib
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "vbvs--vixen_b200")
METRIC = "Mrays/s on 1 B200, batched vs plain at bit-exact hits; fwd+bwd ms/view"
CFG4_SEED = 77  # bounce-ray seed of the batched frame


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
    d = os.path.join(ROOT, "oracle")
    if d not in sys.path:
        sys.path.insert(0, d)
    import vx_oracle
    return vx_oracle


def load_oracle_workloads():
    load_oracle()
    import workloads_ref
    return workloads_ref


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def source_hash():
    """sha256 over the library's CUDA / C++ sources: identifies the build a profile was taken of."""
    h = hashlib.sha256()
    for p in sorted(glob.glob(os.path.join(PKG_DIR, "csrc", "*"))):
        with open(p, "rb") as f:
            h.update(os.path.basename(p).encode() + b"\0" + f.read())
    return h.hexdigest()[:16]


def profiled_traffic(kernel, workload):
    """DRAM bytes per launch of `kernel` on `workload` from profiles/dram_traffic.json, only when
    the entry was captured from the current sources (else None)."""
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic.json")) as f:
            entries = json.load(f)
    except Exception:
        return None
    want = source_hash()
    for e in entries:
        if e.get("kernel") == kernel and e.get("workload") == workload and e.get("source_sha256") == want:
            return e.get("dram_bytes_per_launch")
    return None


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
        return self

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


def bytes_per_launch(n, iters, grid_reads, dda_steps, hits, color_kind):
    """Algorithmic bytes of one cast launch (per-ray terms counted by the traversal):
    24 ray in + 16 hit record out + colour out (12 B DXT1 texel / 4 B RGBA8) per ray,
    8 per ESVO iteration (one descriptor), 4 per brick-grid lookup, 4 per DDA step
    (one occupancy word), plus the colour fetch of every hit (8 B DXT1 block / 4 B RGBA8)."""
    cout, cin = (12, 8) if color_kind == 2 else ((4, 4) if color_kind == 1 else (0, 0))
    return n * (24 + 16 + cout) + 8 * iters + 4 * grid_reads + 4 * dda_steps + cin * hits


def counter_totals(vx, counters):
    cnt = counters.cpu().numpy().view(vx.COUNTER_DTYPE).reshape(-1)
    return {k: int(cnt[k].astype(np.int64).sum()) for k in cnt.dtype.names}


def events_ms(fn, steps, warmup, flush, stream=None):
    """Per-step CUDA-event times of fn on `stream` (the current stream by default), L2 flushed
    before every step."""
    import torch
    s = stream or torch.cuda.current_stream()
    with torch.cuda.stream(s):
        for _ in range(warmup):
            fn()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    with torch.cuda.stream(s):
        for a, b in ev:
            flush.zero_()
            a.record(s)
            fn()
            b.record(s)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def mismatches(g, o, g_col=None, o_col=None, cnt=None):
    """Per-field mismatch counts of product hit records g against oracle records o (t compared as
    bits on hits; texels as bits; counters when given)."""
    hit = (o["flags"] & 1).astype(bool)
    m = {"flags": int(np.count_nonzero(g["flags"].astype(np.uint32) != o["flags"])),
         "brick": int(np.count_nonzero(g["brick"] != o["brick"])),
         "node": int(np.count_nonzero(g["node"] != o["node"])),
         "voxel": int(np.count_nonzero(g["voxel"].astype(np.uint32) != o["voxel"])),
         "scale": int(np.count_nonzero(g["scale"].astype(np.int32) != o["scale"])),
         "t": int(np.count_nonzero(hit & (g["t"].view(np.uint32) != o["t"].view(np.uint32))))}
    if g_col is not None:
        m["texel"] = int(np.count_nonzero(np.any(g_col.view(np.uint32) != o_col.view(np.uint32), axis=1)))
    if cnt is not None:
        m["iters"] = int(np.count_nonzero(cnt["iters"].astype(np.uint32) != o["iters"]))
        m["dda_steps"] = int(np.count_nonzero(cnt["dda_steps"].astype(np.uint32) != o["dda_steps"]))
    return m


def oracle_scenes(vo, frames, threads=None):
    """Oracle octrees of (bits, R, max_levels) triples, built concurrently (each build is one
    C++ call that releases the interpreter lock)."""
    with cf.ThreadPoolExecutor(max_workers=threads or min(16, os.cpu_count() or 1)) as ex:
        return list(ex.map(lambda f: vo.OracleScene.from_dense(f[0], f[1], f[2]), frames))


# ---------------------------------------------------------------------------
# cfg4: the batched frame (headline)
# ---------------------------------------------------------------------------

def cfg4_config(specs):
    n = sum(s.width * s.height for s in specs)
    return {"workload": f"cfg4: {len(specs)} scenes 64^3..1024^3 (noise 10/50%, urban 90%, half DXT1), one camera "
                        f"each 256x256..1920x1080, 2 cosine-weighted bounce rays per primary hit; one frame = batched "
                        f"primary cast + bounce compaction + batched bounce cast in one CUDA graph",
            "primary_rays": n, "scenes": len(specs), "scene_R": [s.R for s in specs],
            "ray_order": "primary rays in 8x4-pixel warp tiles of 32x8 blocks (vx_render's order)",
            "rays_counted": "primary rays + the 2 bounce rays of every primary hit",
            "l2": "flushed before every timed frame (256 MiB write)", "parallelism": "replicated scenes, weak scaling"}


def cfg4_sample(begin, target):
    """Global primary indices of a stride sample of about `target` rays over every scene."""
    n = int(begin[-1])
    stride = max(1, n // max(1, target))
    return np.arange(0, n, stride, dtype=np.int64)


def oracle_cfg4_pass(vo, wr, oscenes, rays_all, begin, idx, threads, pool=None):
    """The oracle's frame over sampled primary rays idx (global indices): primary casts per scene,
    the bounce rays of the hits, their casts.  The casts run as chunks of at most 2048 rays of one
    scene on `threads` host threads (one oracle thread per chunk).  Returns (primary records, bounce
    records (2 per sampled ray), bounce rays, seconds)."""
    t0 = time.perf_counter()
    own = pool is None
    pool = pool or cf.ThreadPoolExecutor(max_workers=threads)

    def cast_all(rays, scene_of, out, sel_mask=None):
        jobs = []
        for s in np.unique(scene_of if sel_mask is None else scene_of[sel_mask]):
            sel = np.flatnonzero((scene_of == s) if sel_mask is None else ((scene_of == s) & sel_mask))
            for c in range(0, sel.size, 2048):
                part = sel[c:c + 2048]
                jobs.append((part, pool.submit(oscenes[s].cast_rays, rays[part], 0.0, 3.4028234663852886e38, 1)))
        for part, fut in jobs:
            out[part] = fut.result()

    sc = np.searchsorted(begin, idx, side="right") - 1
    prim_rays = rays_all[idx]
    prim = np.zeros(idx.size, vo.HIT_DTYPE)
    cast_all(prim_rays, sc, prim)
    bounce = wr.spawn_bounce(prim_rays, prim, CFG4_SEED, idx.astype(np.uint64))
    bsc = np.repeat(sc, 2)
    brec = np.zeros(bounce.shape[0], vo.HIT_DTYPE)
    live = np.repeat((prim["flags"] & 1).astype(bool), 2)
    cast_all(bounce, bsc, brec, live)
    dead = np.flatnonzero(~live)
    if dead.size:  # zero-direction rays: the invalid record, as the cast writes it
        brec[dead] = oscenes[0].cast_rays(bounce[dead], threads=1)
    if own:
        pool.shutdown()
    return prim, brec, bounce, time.perf_counter() - t0


def measure_cfg4(args, rank, world, steps, warmup, with_cpu):
    """The batched frame against the plain launches, the per-pass roofline, e2e through host
    buffers, and (with_cpu) the oracle on a sample of the frame's rays."""
    import torch
    import torch.distributed as dist
    vx = load_pkg()
    from vx_b200 import workloads as W
    from vx_b200 import multigpu as M
    local = int(os.environ.get("LOCAL_RANK", "0"))
    t_setup = time.perf_counter()
    specs = W.config4_specs(args.scenes, seed=M.rank_seed(4, rank))
    scenes, rays, frames = [], [], []
    for sp in specs:
        bits = None
        if sp.kind == "noise" and sp.R >= 256:
            spacing = max(4, 64 * sp.R // 1024)
            bits = vx.synth_noise_dev(sp.R, spacing, 5 if spacing >= 64 else 3, sp.fill, sp.seed,
                                      False).cpu().numpy().view(np.uint64)
        wl = W.build_spec(sp, bits)
        scenes.append(vx.Scene(wl.scene))
        rays.append(wl.rays(order="tiled"))
        frames.append((wl.bits, wl.R, wl.scene.max_levels))
        wl.scene.brick_color = None
    setup_s = time.perf_counter() - t_setup
    begin = np.concatenate([[0], np.cumsum([r.shape[0] for r in rays])]).astype(np.int64)
    n = int(begin[-1])
    rays_all = np.concatenate(rays)
    del rays
    d_rays = torch.from_numpy(rays_all).cuda()
    d_begin = torch.from_numpy(begin.astype(np.int32)).cuda()
    d_bbegin = torch.from_numpy((2 * begin).astype(np.int32)).cuda()
    ph = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    bh = torch.zeros((2 * n, 4), dtype=torch.int32, device="cuda")
    bounce = torch.zeros((2 * n, 6), dtype=torch.float32, device="cuda")
    batch = vx.Batch(scenes)
    # each pass tuned on its own rays (the bounce pass on this frame's bounce rays)
    tuning, tune_ms = batch.autotune(d_rays, d_begin, ph)
    vx.spawn_bounce_rays(d_rays, ph, CFG4_SEED, bounce)
    btuning, btune_ms = batch.autotune(bounce, d_bbegin, bh)
    batch.set_tuning(**tuning.as_dict())
    batch.set_bounce_tuning(btuning)
    stream = torch.cuda.Stream()

    def capture(compact):
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            if compact:
                batch.capture_frame_compact(d_rays, d_begin, ph, bounce, bh, CFG4_SEED, stream.cuda_stream)
            else:
                batch.capture_frame(d_rays, d_begin, ph, bounce, d_bbegin, bh, CFG4_SEED, stream.cuda_stream)
            ph.zero_()
            bh.zero_()
            batch.launch_frame(stream.cuda_stream)
        torch.cuda.synchronize()
        return ph.cpu().numpy().copy(), bh.cpu().numpy().copy()

    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    sampler = ClockSampler(local).start()
    full_p, full_b = capture(False)
    if world > 1:
        dist.barrier()
    full_ms = events_ms(lambda: batch.launch_frame(stream.cuda_stream), steps, warmup, flush, stream)
    ref_p, ref_b = capture(True)
    identical_compact = bool(np.array_equal(ref_p, full_p) and np.array_equal(ref_b, full_b))
    del full_p, full_b
    cb, slot = batch.frame_compaction()
    h2 = int(cb[-1])  # bounce rays of hits in the compacted frame
    g_p = ref_p.view(vx.HIT_DTYPE).reshape(-1)
    nhit = int(np.count_nonzero(g_p["flags"] & 1))
    rays_per_frame = n + 2 * nhit
    if world > 1:
        dist.barrier()
    batched_ms = events_ms(lambda: batch.launch_frame(stream.cuda_stream), steps, warmup, flush, stream)

    # Plain arm: one launch per scene and pass over the same rays: the primary rays, then the
    # compacted bounce rays of hits (left in `bounce` by the batched frame; the plain frame does no
    # spawning or compaction of its own, which favours it).
    pbh = torch.zeros((max(h2, 1), 4), dtype=torch.int32, device="cuda")

    def plain_frame():
        for i, sc in enumerate(scenes):
            a, b = int(begin[i]), int(begin[i + 1])
            if b > a:
                sc.cast_rays_dev(d_rays[a:b], ph[a:b])
        for i, sc in enumerate(scenes):
            a, b = int(cb[i]), int(cb[i + 1])
            if b > a:
                sc.cast_rays_dev(bounce[a:b], pbh[a:b])

    if world > 1:
        dist.barrier()
    plain_ms = events_ms(plain_frame, steps, warmup, flush, stream)
    torch.cuda.synchronize()
    identical_plain = bool(np.array_equal(ph.cpu().numpy(), ref_p)) and \
        bool(np.array_equal(pbh[:h2].cpu().numpy(), ref_b[slot.astype(np.int64)]))

    # Counting passes and per-pass kernel times (roofline): each pass as its own batched launch
    # with the frame's tuning for it; the bounce pass over the compacted rays.
    d_cb = torch.from_numpy(cb.astype(np.int32)).cuda()
    cnt_p = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    cnt_b = torch.zeros((max(h2, 1), 4), dtype=torch.int32, device="cuda")
    batch.cast(d_rays, d_begin, ph, cnt_p)
    batch.set_tuning(**btuning.as_dict())
    batch.cast(bounce[:h2], d_cb, pbh, cnt_b)
    torch.cuda.synchronize()
    tot_p = counter_totals(vx, cnt_p)
    tot_b = counter_totals(vx, cnt_b[:h2])
    bounce_pass_ms = events_ms(lambda: batch.cast(bounce[:h2], d_cb, pbh), steps, warmup, flush, stream)
    batch.set_tuning(**tuning.as_dict())
    primary_pass_ms = events_ms(lambda: batch.cast(d_rays, d_begin, ph), steps, warmup, flush, stream)
    del cnt_p, cnt_b
    clocks = sampler.stop()

    # e2e: the frame from pinned host buffers (rays in; primary and bounce hits out) through
    # vx_batch_launch_frame_host, the frame captured in parts so that the copies of each part
    # overlap the casts of its neighbours; the whole frame's host call for comparison.
    rays_h = torch.from_numpy(rays_all).pin_memory()
    ph_h = torch.zeros((n, 4), dtype=torch.int32).pin_memory()
    bh_h = torch.zeros((2 * n, 4), dtype=torch.int32).pin_memory()
    with torch.cuda.stream(stream):
        batch.capture_frame_compact(d_rays, d_begin, ph, bounce, bh, CFG4_SEED, stream.cuda_stream)
    whole_ms = events_ms(lambda: batch.launch_frame_host(rays_h, ph_h, bh_h, stream.cuda_stream), steps, warmup,
                         flush, stream)
    whole_same = bool(np.array_equal(ph_h.numpy(), ref_p) and np.array_equal(bh_h.numpy(), ref_b))
    ph_h.zero_(), bh_h.zero_()
    with torch.cuda.stream(stream):
        batch.capture_frame_parts(d_rays, d_begin, ph, bounce, bh, CFG4_SEED, args.e2e_parts, stream.cuda_stream)
    torch.cuda.synchronize()
    e2e_ms = events_ms(lambda: batch.launch_frame_host(rays_h, ph_h, bh_h, stream.cuda_stream), steps, warmup,
                       flush, stream)
    e2e_same = bool(np.array_equal(ph_h.numpy(), ref_p) and np.array_equal(bh_h.numpy(), ref_b))
    del rays_h, ph_h, bh_h
    batch_total, plain_total, full_total, e2e_total, whole_total = M.max_over_ranks(
        [sum(batched_ms), sum(plain_ms), sum(full_ms), sum(e2e_ms), sum(whole_ms)])

    peak, peak_kind = measured_peaks()
    passes = {}
    for name, tot, nr, ms, tn, kern in (("primary", tot_p, n, primary_pass_ms, tuning, "primary"),
                                        ("bounce", tot_b, h2, bounce_pass_ms, btuning, "bounce")):
        algo = bytes_per_launch(nr, tot["run_iters"], tot["run_grid_reads"], tot["run_dda_steps"], 0, 0)
        mean_s = statistics.mean(ms) / 1e3
        kname = "vx::batch_refill_kernel" if tn.refill else "vx::batch_kernel"
        passes[name] = {"kernel": kname, "rays": nr, "tuning": tn.as_dict(), "kernel_ms_mean": mean_s * 1e3,
                        "launches": 2 if tn.budget else 1,  # a budgeted pass: all rays, then the set-aside ones
                        "algorithmic_bytes_per_launch": algo, "achieved_gbs": algo / mean_s / 1e9,
                        "mrays_s": nr / mean_s / 1e6,
                        "per_ray": {k: v / max(nr, 1) for k, v in tot.items()}}
    dom = max(passes, key=lambda k: passes[k]["kernel_ms_mean"])
    d = passes[dom]
    workload_key = f"cfg4_{dom}_pass"
    roofline = {"bound": "hbm", "achieved": d["achieved_gbs"], "peak": peak, "unit": "GB/s",
                "frac": d["achieved_gbs"] / peak, "traffic": profiled_traffic(d["kernel"], workload_key),
                "peak_source": peak_kind, "kernel": f"{d['kernel']} ({dom} pass of the frame)",
                "kernel_ms_mean": d["kernel_ms_mean"], "algorithmic_bytes_per_launch": d["algorithmic_bytes_per_launch"],
                "traffic_source": f"profiles/dram_traffic.json entry '{workload_key}' for the current sources, "
                                  f"else null", "passes": passes}
    out = {"config": cfg4_config(specs),
           "value": world * rays_per_frame * steps / (batch_total / 1e3) / 1e6,
           "ms_per_frame": batch_total / steps,
           "frame": {"primary_rays": n, "primary_hits": nhit, "bounce_rays": 2 * nhit, "rays_per_frame": rays_per_frame,
                     "setup_s": setup_s, "graph": "vx_batch_capture_frame_compact"},
           "roofline": roofline,
           "e2e": {"value": world * rays_per_frame * steps / (e2e_total / 1e3) / 1e6, "unit": "Mrays/s",
                   "h2d_bytes_per_step": world * n * 24, "d2h_bytes_per_step": world * n * (16 + 32),
                   "call": f"vx_batch_launch_frame_host on the frame captured in {args.e2e_parts} parts "
                           f"(vx_batch_capture_frame_parts; pinned buffers; rays in, primary and bounce hits out, "
                           f"overlapped with the other parts' casts)", "hits_equal_device_path": e2e_same,
                   "ms_per_frame": e2e_total / steps,
                   "whole_frame": {"value": world * rays_per_frame * steps / (whole_total / 1e3) / 1e6,
                                   "ms_per_frame": whole_total / steps, "hits_equal_device_path": whole_same,
                                   "call": "vx_batch_launch_frame_host on the frame of vx_batch_capture_frame_compact "
                                           "(primary hits copied out during the bounce pass)"}},
           "batched": {"mrays_s": world * rays_per_frame * steps / (batch_total / 1e3) / 1e6,
                       "ms_per_frame": batch_total / steps, "tuning": tuning.as_dict(), "bounce_tuning": btuning.as_dict(),
                       "autotune_best_ms_primary": tune_ms, "autotune_best_ms_bounce": btune_ms},
           "plain": {"mrays_s": world * rays_per_frame * steps / (plain_total / 1e3) / 1e6,
                     "ms_per_frame": plain_total / steps, "launches_per_frame": 2 * len(specs),
                     "rays": "the same primary rays and compacted bounce rays of hits as the batched frame"},
           "launches_per_frame": 6 + int(tuning.budget > 0) + int(btuning.budget > 0),
           "speedup_batched_vs_plain": plain_total / batch_total,
           "uncompacted_batched_ms_per_frame": full_total / steps,
           "compaction_gain": full_total / batch_total,
           "hits_identical": {"batched_vs_plain": identical_plain, "compacted_vs_uncompacted_frame": identical_compact},
           "clocks": clocks}
    if with_cpu:
        vo = load_oracle()
        wr = load_oracle_workloads()
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        osc = oracle_scenes(vo, frames)
        build_s = time.perf_counter() - t0
        target, spent = 1 << 15, 0.0
        while True:
            idx = cfg4_sample(begin, target)
            prim, brec, _, dt = oracle_cfg4_pass(vo, wr, osc, rays_all, begin, idx, threads)
            spent += dt
            if dt >= 2.0 or idx.size >= n or spent > 20.0:
                break
            target = int(target * min(16.0, max(2.0, 6.0 / max(dt, 1e-3))))
        live = np.repeat((prim["flags"] & 1).astype(bool), 2)
        counted = idx.size + int(live.sum())
        bslots = (2 * idx[:, None] + np.arange(2)[None, :]).reshape(-1)
        mp = mismatches(g_p[idx], prim)
        mb = mismatches(ref_b.view(vx.HIT_DTYPE).reshape(-1)[bslots], brec)
        out["cpu_baseline"] = {"value": counted / dt / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "port",
                               "sample": f"every {int(begin[-1]) // max(idx.size, 1)}th primary ray of the frame "
                                         f"({idx.size} rays over all {len(specs)} scenes) and the 2 bounce rays of "
                                         f"each of its hits ({int(live.sum())}); {counted} rays in {dt:.2f} s on "
                                         f"{threads} threads; oracle octree builds {build_s:.1f} s"}
        out["parity_sample"] = {"primary_rays": int(idx.size), "bounce_rays": int(bslots.size),
                                "primary_mismatches": mp, "bounce_mismatches": mb,
                                "fields": "flags, brick, node, voxel, scale, t bits"}
        it_ref = float(np.mean(prim["iters"]))
        out["iterations_per_primary_ray"] = {
            "reference_loop": it_ref, "kernel_executed": passes["primary"]["per_ray"]["run_iters"],
            "note": "the reference loop runs rays caught in a repeating state to its 500-iteration cap; the kernel "
                    "detects the repeat exactly and stops, so part of the ratio to the CPU baseline is algorithmic"}
        del osc
    batch.close()
    del scenes, d_rays, ph, bh, bounce, pbh
    torch.cuda.empty_cache()
    return out


def run_cfg4_pass(args):
    """One launch of each pass of the batched frame over the first `--scenes` scenes of the frame,
    with fixed tunings (both passes: block 256, 32 rays per task, shared-memory stack, static
    lanes, no iteration budget; what the default run's autotuner picks on this frame).  The
    command for ncu captures of the frame's kernels on a small case: after the frame's graph, each
    of --steps steps launches the primary pass, then the bounce pass over the compacted bounce
    rays."""
    import torch
    vx = load_pkg()
    from vx_b200 import workloads as W
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    specs = W.config4_specs(64, seed=4)[:args.scenes]
    scenes, rays = [], []
    for sp in specs:
        bits = None
        if sp.kind == "noise" and sp.R >= 256:
            spacing = max(4, 64 * sp.R // 1024)
            bits = vx.synth_noise_dev(sp.R, spacing, 5 if spacing >= 64 else 3, sp.fill, sp.seed,
                                      False).cpu().numpy().view(np.uint64)
        wl = W.build_spec(sp, bits)
        scenes.append(vx.Scene(wl.scene))
        rays.append(wl.rays(order="tiled"))
    begin = np.concatenate([[0], np.cumsum([r.shape[0] for r in rays])]).astype(np.int64)
    n = int(begin[-1])
    d_rays = torch.from_numpy(np.concatenate(rays)).cuda()
    d_begin = torch.from_numpy(begin.astype(np.int32)).cuda()
    ph = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    bh = torch.zeros((2 * n, 4), dtype=torch.int32, device="cuda")
    bounce = torch.zeros((2 * n, 6), dtype=torch.float32, device="cuda")
    batch = vx.Batch(scenes)
    batch.set_tuning(256, 32, 1, 0)
    batch.set_bounce_tuning(vx.BatchTuning(256, 32, 1, 0, 0))
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        batch.capture_frame_compact(d_rays, d_begin, ph, bounce, bh, CFG4_SEED, s.cuda_stream)
        batch.launch_frame(s.cuda_stream)
    torch.cuda.synchronize()
    cb, _ = batch.frame_compaction()
    h2 = int(cb[-1])
    d_cb = torch.from_numpy(cb.astype(np.int32)).cuda()
    pbh = torch.zeros((max(h2, 1), 4), dtype=torch.int32, device="cuda")
    times = []
    for _ in range(max(1, args.steps)):  # each step: the primary pass, then the bounce pass
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        batch.set_tuning(256, 32, 1, 0)
        ev[0].record()
        batch.cast(d_rays, d_begin, ph)
        ev[1].record()
        batch.set_tuning(256, 32, 1, 0, 0)
        ev[2].record()
        batch.cast(bounce[:h2], d_cb, pbh)
        ev[3].record()
        torch.cuda.synchronize()
        times.append((ev[0].elapsed_time(ev[1]), ev[2].elapsed_time(ev[3])))
    print(json.dumps({"workload": "cfg4-passes", "scenes": len(specs), "primary_rays": n, "bounce_rays": h2,
                      "primary_ms": [t[0] for t in times], "bounce_ms": [t[1] for t in times],
                      "source_sha256": source_hash()}), flush=True)
    return 0


def run_cfg4(args, rank, world):
    """Prints the headline line: the batched frame (cfg4), with cfg2, cfg3, cfg5 and the next rows
    attached at N = 1."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    res = measure_cfg4(args, rank, world, args.steps, args.warmup,
                       with_cpu=(world == 1 and rank == 0 and not args.no_cpu_baseline))
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "value": res.pop("value"), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res.pop("ms_per_frame"), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": res.pop("config"),
            # per timed frame: batched primary cast, bin counts, per-scene scans, bases, compacted scatter,
            # batched bounce cast, and the second launch of each pass whose tuning has an iteration budget
            "gpu_launches": args.steps * res.pop("launches_per_frame")}
    line.update(res)
    if world == 1 and not args.no_extra:
        extra_steps, extra_warmup = max(3, min(args.steps, 10)), max(3, min(args.warmup, 3))
        line["cfg2"] = measure_cfg2(args, 0, 1, extra_steps, extra_warmup, with_cpu=not args.no_cpu_baseline)
        torch.cuda.empty_cache()
        line["cfg3"] = measure_cfg3(args, extra_steps, extra_warmup, with_oracle=not args.no_cpu_baseline)
        torch.cuda.empty_cache()
        line["adjoint"] = measure_cfg5(args, 0, 1, extra_steps, extra_warmup)
        torch.cuda.empty_cache()
        line["next_rows"] = measure_next(args, extra_steps, extra_warmup)
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# cfg2: the 1024^3 cave frame, plain cast
# ---------------------------------------------------------------------------

def cfg2_config(R, width, height, world):
    return {"workload": f"cfg2_cave{R}_dxt1_{width}x{height}: cave {R}^3 (depth 10), value noise spacing "
                        f"{64 * R // 1024}, 5 octaves, 50% fill, DXT1 bricks, {width}x{height} FP32 primary rays per "
                        f"rank, plain cast kernel",
            "ray_order": "8x4-pixel warp tiles in 32x8 blocks (vx_render's order)",
            "rays_per_step_per_gpu": width * height, "parallelism": f"replicated scene, {world} camera(s)",
            "l2": "flushed between timed steps (256 MiB write)"}


def measure_cfg2(args, rank, world, steps, warmup, with_cpu):
    """The cave frame through the plain cast kernel: device Mrays/s, e2e through vx_cast_rays_host,
    the kernel's roofline, and the oracle on a sample (every field, the texel included)."""
    import torch
    import torch.distributed as dist
    vx = load_pkg()
    from vx_b200 import workloads as W
    from vx_b200 import multigpu as M
    local = int(os.environ.get("LOCAL_RANK", "0"))
    R, seed = args.R, args.seed
    spacing = 64 * R // 1024
    bits = vx.synth_noise_dev(R, spacing, 5 if R >= 1024 else 3, 0.5, seed, False).cpu().numpy().view(np.uint64)
    wl = W.config2(R=R, seed=seed, bits=bits)
    if rank:
        wl.camera = W.empty_voxel_camera(bits, R, M.rank_seed(seed, rank), 70.0, wl.width, wl.height)
    scene = vx.Scene(wl.scene)
    rays_np = wl.rays(order="tiled")
    n = rays_np.shape[0]
    rays = torch.from_numpy(rays_np).cuda()
    hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    color = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    counters = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    scene.cast_rays_dev(rays, hits, color, counters)  # counting pass (untimed)
    torch.cuda.synchronize()
    tot = counter_totals(vx, counters)
    cnt = counters.cpu().numpy().view(vx.COUNTER_DTYPE).reshape(-1)
    g_hits = hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1).copy()
    g_col = color.cpu().numpy().copy()
    nhit = int(np.count_nonzero(g_hits["flags"] & 1))
    algo = bytes_per_launch(n, tot["run_iters"], tot["run_grid_reads"], tot["run_dda_steps"], nhit, scene.color_kind)
    ref_bytes = bytes_per_launch(n, tot["iters"], tot["grid_reads"], tot["dda_steps"], nhit, scene.color_kind)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    sampler = ClockSampler(local).start()
    t_soak = time.perf_counter()
    while time.perf_counter() - t_soak < args.soak_seconds:  # clocks to steady state before timing
        for _ in range(20):
            scene.cast_rays_dev(rays, hits, color)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    step_ms = events_ms(lambda: scene.cast_rays_dev(rays, hits, color), steps, warmup, flush)
    rays_h = torch.from_numpy(rays_np).pin_memory()
    hits_h = torch.zeros((n, 4), dtype=torch.int32).pin_memory()
    col_h = torch.zeros((n, 3), dtype=torch.float32).pin_memory()
    L = vx.lib()
    stream = torch.cuda.current_stream()

    def e2e_call():
        vx.check(L.vx_cast_rays_host(scene.handle, C.c_void_p(rays_h.data_ptr()), n, 0.0, vx.FLT_MAX,
                                     C.c_void_p(hits_h.data_ptr()), C.c_void_p(col_h.data_ptr()),
                                     C.c_void_p(stream.cuda_stream)))

    e2e_ms = events_ms(e2e_call, steps, warmup, flush)
    clocks = sampler.stop()
    e2e_same = bool(np.array_equal(hits_h.numpy().view(np.uint8), g_hits.view(np.uint8).reshape(n, 16)))
    total_ms, e2e_total = M.max_over_ranks([sum(step_ms), sum(e2e_ms)])
    mean_s = statistics.mean(step_ms) / 1e3
    peak, peak_kind = measured_peaks()
    out = {"config": cfg2_config(R, wl.width, wl.height, world),
           "value": M.aggregate_throughput(n * steps, world, total_ms / 1e3) / 1e6, "unit": "Mrays/s",
           "ms_per_frame": total_ms / steps, "steps": steps,
           "bricks": int(wl.scene.brick_count), "nodes": int(wl.scene.node_count), "hit_rate": nhit / n,
           "e2e": {"value": M.aggregate_throughput(n * steps, world, e2e_total / 1e3) / 1e6, "unit": "Mrays/s",
                   "h2d_bytes_per_step": world * n * 24, "d2h_bytes_per_step": world * n * (16 + 12),
                   "hits_equal_device_path": e2e_same},
           "roofline": {"bound": "hbm", "achieved": algo / mean_s / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": algo / mean_s / 1e9 / peak,
                        "traffic": profiled_traffic("vx::cast_kernel", wl.name), "peak_source": peak_kind,
                        "algorithmic_bytes_per_launch": algo, "reference_loop_bytes_per_launch": ref_bytes,
                        "per_ray": {k: v / n for k, v in tot.items()}, "kernel": "vx::cast_kernel",
                        "kernel_ms_mean": mean_s * 1e3},
           "clocks": clocks}
    if with_cpu:
        vo = load_oracle()
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        o = vo.OracleScene.from_dense(bits, R, wl.scene.max_levels)
        build_s = time.perf_counter() - t0
        m = min(n, 1 << 16)
        while True:
            t0 = time.perf_counter()
            oh = o.cast_rays(rays_np[:m], threads=threads)
            dt = time.perf_counter() - t0
            if dt >= 3.0 or m >= n:
                break
            m = min(n, m * 4)
        o_col = vo.hit_texels_dxt(wl.scene.brick_color, oh)
        out["cpu_baseline"] = {"value": m / dt / 1e6, "unit": "Mrays/s", "cores": threads, "kind": "port",
                               "sample": f"first {m} rays of the frame ({m / n:.1%}), {threads} threads, {dt:.2f} s; "
                                         f"oracle build {build_s:.1f} s"}
        out["parity_sample"] = {"checked": m, "mismatches": mismatches(g_hits[:m], oh, g_col[:m], o_col, cnt[:m]),
                                "fields": "flags, brick, node, voxel, scale, t bits, DXT1 texel bits, iteration and "
                                          "DDA-step counters"}
    del scene, rays, hits, color, counters
    torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------------------
# cfg3: the 2048^3 urban frame with shadow rays
# ---------------------------------------------------------------------------

def cfg3_config(R, width, height):
    return {"workload": f"cfg3_urban{R}_dxt1_{width}x{height}: urban {R}^3 (depth 11), 32x32 blocks, 8-voxel "
                        f"streets, heights U[64,1800], DXT1 bricks; {width}x{height} primary rays + 1 shadow ray per "
                        f"hit toward a seeded light; one frame = primary cast + compacted shadow pass",
            "ray_order": "primary rays in 8x4-pixel warp tiles (vx_render's order)",
            "l2": "flushed before every timed frame (256 MiB write)"}


def measure_cfg3(args, steps, warmup, with_oracle):
    """The urban frame: primary cast (plain kernel, DXT1 texel out), then vx_cast_shadow_rays (the
    shadow rays of hits, compacted on the device).  ms/frame, Mrays/s, the primary kernel's roofline,
    and the oracle on a stride sample of the frame (primary record + texel, and the shadow record)."""
    import torch
    vx = load_pkg()
    from vx_b200 import workloads as W
    t0 = time.perf_counter()
    wl = W.config3(R=args.R3)
    scene = vx.Scene(wl.scene)
    setup_s = time.perf_counter() - t0
    rays_np = wl.rays(order="tiled")
    n = rays_np.shape[0]
    rays = torch.from_numpy(rays_np).cuda()
    hits = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    col = torch.zeros((n, 3), dtype=torch.float32, device="cuda")
    cnt = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    sh = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    L = W.light_dir(3)
    scene.cast_rays_dev(rays, hits, col, cnt)
    scene.cast_shadow_rays_dev(rays, hits, L, sh)
    torch.cuda.synchronize()
    tot = counter_totals(vx, cnt)
    g = hits.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1).copy()
    g_col = col.cpu().numpy().copy()
    g_sh = sh.cpu().numpy().view(vx.HIT_DTYPE).reshape(-1).copy()
    del cnt
    nhit = int(np.count_nonzero(g["flags"] & 1))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def frame():
        scene.cast_rays_dev(rays, hits, col)
        scene.cast_shadow_rays_dev(rays, hits, L, sh)

    ms = statistics.mean(events_ms(frame, steps, warmup, flush))
    prim_ms = events_ms(lambda: scene.cast_rays_dev(rays, hits, col), steps, warmup, flush)
    mean_s = statistics.mean(prim_ms) / 1e3
    algo = bytes_per_launch(n, tot["run_iters"], tot["run_grid_reads"], tot["run_dda_steps"], nhit, scene.color_kind)
    peak, peak_kind = measured_peaks()
    out = {"config": cfg3_config(wl.R, wl.width, wl.height), "mrays_s": (n + nhit) / (ms / 1e3) / 1e6,
           "ms_per_frame": ms, "steps": steps, "primary_rays": n, "shadow_rays": nhit, "primary_hit_rate": nhit / n,
           "shadowed_fraction": float(np.count_nonzero(g_sh["flags"] & 1)) / max(nhit, 1),
           "bricks": int(wl.scene.brick_count), "nodes": int(wl.scene.node_count),
           "scene_device_bytes": scene.device_bytes(), "setup_s": setup_s,
           "roofline": {"bound": "hbm", "kernel": "vx::cast_kernel (primary pass)", "kernel_ms_mean": mean_s * 1e3,
                        "achieved": algo / mean_s / 1e9, "peak": peak, "unit": "GB/s",
                        "frac": algo / mean_s / 1e9 / peak, "peak_source": peak_kind,
                        "traffic": profiled_traffic("vx::cast_kernel", wl.name),
                        "algorithmic_bytes_per_launch": algo, "per_ray": {k: v / n for k, v in tot.items()}}}
    del scene, rays, hits, col, sh
    torch.cuda.empty_cache()
    if with_oracle:
        vo = load_oracle()
        wr = load_oracle_workloads()
        t0 = time.perf_counter()
        o = vo.OracleScene.from_dense(wl.bits, wl.R, wl.scene.max_levels)
        build_s = time.perf_counter() - t0
        idx = np.arange(0, n, max(1, n // 65536), dtype=np.int64)
        oh = o.cast_rays(rays_np[idx], threads=0)
        o_col = vo.hit_texels_dxt(wl.scene.brick_color, oh)
        so = o.cast_rays(wr.spawn_shadow(rays_np[idx], oh, L), threads=0)
        out["parity_sample"] = {"checked": int(idx.size), "stride": int(n // 65536), "oracle_build_s": build_s,
                                "primary_mismatches": mismatches(g[idx], oh, g_col[idx], o_col),
                                "shadow_mismatches": mismatches(g_sh[idx], so),
                                "fields": "flags, brick, node, voxel, scale, t bits (+ DXT1 texel bits on primaries)"}
    return out


# ---------------------------------------------------------------------------
# Reference arm: the oracle (CPU restatement of castRay) on this host's cores
# ---------------------------------------------------------------------------

def run_reference(args, rank, world):
    """The reference's CPU path over a bounded sample of the same frame, every input built on the
    oracle side (oracle/workloads_ref.py) without loading the product library.  Under torchrun only
    rank 0 runs."""
    if rank != 0:
        return 0
    vo = load_oracle()
    wr = load_oracle_workloads()
    threads = os.cpu_count() or 1
    t_setup = time.perf_counter()
    if args.workload == "cfg2":
        fr = wr.cfg2(R=args.R, seed=args.seed)
        rays_all = fr.rays()
        o = fr.scene()
        config = cfg2_config(args.R, fr.width, fr.height, world)

        def step(idx):
            o.cast_rays(rays_all[idx], threads=threads)
            return idx.size
        n = rays_all.shape[0]
        sample_of = lambda m: np.arange(m, dtype=np.int64)  # noqa: E731  (the frame's first m rays)
        what = "first {m} of {n} rays of the frame per step"
    else:
        specs = wr.cfg4_specs(args.scenes, seed=4)
        frames = [wr.cfg4_frame(sp, threads) for sp in specs]
        rays = [f.rays() for f in frames]
        begin = np.concatenate([[0], np.cumsum([r.shape[0] for r in rays])]).astype(np.int64)
        rays_all = np.concatenate(rays)
        del rays
        osc = oracle_scenes(vo, [(f.bits, f.R, f.max_levels) for f in frames])
        for f in frames:
            f.bits = None
        config = cfg4_config(specs)
        n = int(begin[-1])

        pool = cf.ThreadPoolExecutor(max_workers=threads)

        def step(idx):
            prim, _, _, _ = oracle_cfg4_pass(vo, wr, osc, rays_all, begin, idx, threads, pool)
            return idx.size + 2 * int(np.count_nonzero(prim["flags"] & 1))
        sample_of = lambda m: cfg4_sample(begin, m)  # noqa: E731
        what = "every (n / {m})th primary ray of the frame over all scenes, and the 2 bounce rays of each hit, per step"
    setup_s = time.perf_counter() - t_setup
    m = 1 << 13
    while True:  # size one step at about 1 s
        t0 = time.perf_counter()
        step(sample_of(m))
        dt = time.perf_counter() - t0
        if dt >= 0.25 or m >= n:
            break
        m = min(n, m * 4)
    m = min(n, max(1024, int(m * 1.0 / max(dt, 1e-3))))
    idx = sample_of(m)
    for _ in range(args.warmup):
        step(idx)
    times, units = [], 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        units = step(idx)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    v = units * args.steps / total / 1e6
    sample = what.format(m=m, n=n) + f"; {units} rays per step, {threads} threads; setup {setup_s:.1f} s"
    line = {"metric": METRIC, "value": v, "unit": "Mrays/s", "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": config,
            "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


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
    (multigpu.view_range), each rank's forward + adjoint into its own gradient pool, then the
    adjoint's one exchange: the touched entries of every rank all-gathered and summed in rank
    order (multigpu.sparse_allreduce_); ms per view = max over ranks / 16."""
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

        touched = [0]

        def step():
            grad.zero_()
            if mine:
                vx.diff_forward_views(scene, mine, 512, 512, kind, attr_d, idx_d, img, rec)
                vx.diff_backward(kind, idx_d, rec, img, tgt, grad)
            # the exchange: only the gradient entries this rank's hit records touched
            entries = M.touched_entries(rec, kind) if mine else torch.zeros(0, dtype=torch.int64, device="cuda")
            touched[0] = int(entries.numel())
            M.sparse_allreduce_(grad, entries)

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
        out[name] = {"fwd_bwd_exchange_ms_per_view": ms / 16, "views_per_rank": len(mine),
                     "gradient_pool_bytes": int(attr_d.numel() * 4),
                     "exchange": "sparse all-gather of the touched (index, value) pairs (multigpu.sparse_allreduce_)",
                     "touched_entries_rank0": touched[0], "exchange_bytes_per_rank": touched[0] * 12}
        del scene
    return {"workload": "cfg5: 512^3 noise 30% fill, 16 views 512x512 on an orbit split over ranks, the touched "
                        "gradient entries all-gathered and summed per step", **out}


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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="vx", choices=["vx", "reference"])
    ap.add_argument("--workload", default="cfg4",
                    choices=["cfg4", "cfg2", "cfg3", "cfg5", "next", "tour", "cfg4-passes"],
                    help="cfg4 (default): the 64-scene batched frame vs plain launches, with cfg2, cfg3, cfg5 and the "
                         "next rows attached at N=1; cfg2: plain cast of the 1024^3 cave frame; cfg3: the 2048^3 "
                         "urban frame with shadow rays; cfg5: forward / adjoint ms per view; next: device builder, "
                         "payload encoders, LOD cut, compressed render, cache file; tour: every kernel once, "
                         "CUDA-event times per step (the command for ncu captures); cfg4-passes: one launch of "
                         "each pass of the batched frame over --scenes scenes (ncu captures of its kernels)")
    ap.add_argument("--R", type=int, default=1024, help="cfg2 / next: grid side of the cave scene")
    ap.add_argument("--R3", type=int, default=2048, help="cfg3: grid side of the urban scene")
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--scenes", type=int, default=64, help="cfg4: number of scenes")
    ap.add_argument("--e2e-parts", type=int, default=32,
                    help="cfg4: parts of the frame whose host copies overlap the other parts' casts (e2e)")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the oracle legs (CPU baseline and parity samples)")
    ap.add_argument("--no-extra", action="store_true",
                    help="cfg4 only: skip the attached cfg2, cfg3, adjoint and next-row measurements")
    ap.add_argument("--split-views", action="store_true",
                    help="cfg5: split the views over the ranks and all-reduce the gradient (default when N > 1; "
                         "needs a process group, i.e. torchrun, also for N = 1)")
    ap.add_argument("--soak-seconds", type=float, default=1.5,
                    help="cfg2: untimed launches before timing so clocks reach steady state")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if args.workload not in ("cfg4", "cfg2"):
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": f"the reference arm times cfg4 (default) or "
                                                                      f"cfg2, not {args.workload}"}), flush=True)
            return 0
        return run_reference(args, rank, world)
    if args.workload == "cfg4":
        return run_cfg4(args, rank, world)
    if args.workload == "cfg4-passes":
        return run_cfg4_pass(args)
    import torch
    torch.cuda.set_device(local)
    if args.workload == "cfg2":
        import torch.distributed as dist
        from datetime import timedelta
        if world > 1:
            dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
        res = measure_cfg2(args, rank, world, args.steps, args.warmup,
                           with_cpu=(world == 1 and not args.no_cpu_baseline))
        if world > 1:
            dist.destroy_process_group()
        if rank == 0:
            line = {"metric": METRIC, "value": res.pop("value"), "unit": res.pop("unit"), "n_gpus": world,
                    "steps": args.steps, "warmup": args.warmup, "ms_per_step": res.pop("ms_per_frame"),
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                    "data": "synthetic", "config": res.pop("config"), "gpu_launches": args.steps}
            line.update(res)
            print(json.dumps(line), flush=True)
        return 0
    if args.workload == "cfg3":
        res = measure_cfg3(args, args.steps, args.warmup, with_oracle=not args.no_cpu_baseline)
        if rank == 0:
            line = {"metric": METRIC, "value": res["mrays_s"], "unit": "Mrays/s", "n_gpus": 1, "steps": args.steps,
                    "warmup": args.warmup, "ms_per_step": res["ms_per_frame"], "higher_is_better": True,
                    "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                    # per frame: primary cast, shadow hit count, scan, compacted spawn, shadow cast
                    "config": res.pop("config"), "gpu_launches": args.steps * 5}
            line.update(res)
            print(json.dumps(line), flush=True)
        return 0
    if args.workload == "tour":
        res = measure_tour(args)
        if rank == 0:
            print(json.dumps({"workload": "tour", "tour": res}), flush=True)
        return 0
    if args.workload == "next":
        res = measure_next(args, args.steps, args.warmup)
        if rank == 0:
            print(json.dumps({"workload": "next", "next_rows": res}), flush=True)
        return 0
    if world > 1 or args.split_views:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
        res = measure_cfg5_multi(args, rank, world, args.steps, args.warmup)
        dist.destroy_process_group()
        if rank == 0:
            a = res["voxel_rgb"]
            print(json.dumps({"metric": METRIC, "value": a["fwd_bwd_exchange_ms_per_view"], "unit": "ms/view",
                              "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                              "ms_per_step": a["fwd_bwd_exchange_ms_per_view"] * 16, "higher_is_better": False,
                              "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                              "config": {"workload": res.pop("workload")}, "adjoint": res,
                              "gpu_launches": args.steps * 2}), flush=True)
        return 0
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


if __name__ == "__main__":
    sys.exit(main())
