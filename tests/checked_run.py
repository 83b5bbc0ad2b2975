"""Runs one of every device path of the library and saves the outputs (used by
test_gpu_checked.py under both builds).  Usage: python checked_run.py OUT.npz"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)


def main(out_path):
    import torch
    from conftest import load_vx
    vx = load_vx()
    from vx_b200 import workloads as W
    torch.cuda.set_device(0)
    out = {}
    enabled, v0 = vx.bounds_checks()
    out["enabled"] = np.array([int(enabled)])
    # plain cast, RGBA8, camera + random + degenerate rays, counters
    wl = W.config1(R=128, width=64, height=64, seed=41)
    s = vx.Scene(wl.scene)
    nan, inf = np.float32(np.nan), np.float32(np.inf)
    degen = np.array([[3, 3, 3, 0, 0, 0], [1, 1, 1, nan, 1, 0], [inf, 1, 1, -1, 0, 0], [64, 64, -1, 0, 0, 1],
                      [0, 0, 0, 1, 1, 1], [128, 128, 128, -1, -1, -1]], np.float32)
    rays = np.concatenate([wl.rays(), W.random_rays(20000, 128, seed=42), degen])
    r = torch.from_numpy(rays).cuda()
    n = r.shape[0]
    h = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    c = torch.zeros((n, 1), dtype=torch.int32, device="cuda")
    k = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    s.cast_rays_dev(r, h, c, k)
    lod_h = torch.zeros_like(h)
    s.cast_rays_dev(r, lod_h, None, None, lod=(0.1, 0.05))
    out.update(plain_hits=h.cpu().numpy(), plain_col=c.cpu().numpy(), plain_cnt=k.cpu().numpy(),
               lod_hits=lod_h.cpu().numpy())
    # DXT scene with normals: render and per-hit normals
    wl2 = W.config2(R=128, width=96, height=64, seed=43)
    import dataclasses
    a2 = dataclasses.replace(wl2.scene, brick_normal=vx.build_normals(wl2.scene.brick_occ.reshape(-1, 16)))
    s2 = vx.Scene(a2)
    npx = wl2.width * wl2.height
    img = torch.zeros(npx, dtype=torch.int32, device="cuda")
    rh = torch.zeros((npx, 4), dtype=torch.int32, device="cuda")
    s2.render_dev(wl2.camera, wl2.width, wl2.height, img, rh)
    nrm = torch.zeros((npx, 3), dtype=torch.float32, device="cuda")
    s2.hit_normals_dev(rh, nrm)
    out.update(render_img=img.cpu().numpy(), render_hits=rh.cpu().numpy(), normals=nrm.cpu().numpy())
    # batched cast (static and refilling lanes) with bounce rays
    specs = W.config4_specs(6, seed=44, r_range=(6, 7.4), res_lo=(48, 40), res_hi=(128, 96))
    wls = [W.build_spec(sp) for sp in specs]
    scenes = [vx.Scene(w.scene) for w in wls]
    rl = [w.rays() for w in wls]
    begin = np.concatenate([[0], np.cumsum([x.shape[0] for x in rl])]).astype(np.int32)
    br = torch.from_numpy(np.concatenate(rl)).cuda()
    bb = torch.from_numpy(begin).cuda()
    batch = vx.Batch(scenes)
    for tune in ((256, 32, 1, 0, 3), (128, 64, 0, 16, 0)):
        batch.set_tuning(*tune)
        bh = torch.zeros((br.shape[0], 4), dtype=torch.int32, device="cuda")
        batch.cast(br, bb, bh)
        out[f"batch_{tune[3]}"] = bh.cpu().numpy()
    bounce = torch.zeros((2 * br.shape[0], 6), dtype=torch.float32, device="cuda")
    vx.spawn_bounce_rays(br, bh, 5, bounce)
    bbh = torch.zeros((bounce.shape[0], 4), dtype=torch.int32, device="cuda")
    batch.cast(bounce, torch.from_numpy(2 * begin).cuda(), bbh)
    out["bounce_hits"] = bbh.cpu().numpy()
    # the frame with bounce compaction, and the compacted shadow pass
    fh = torch.zeros_like(bh)
    fbh = torch.zeros_like(bbh)
    fs = torch.cuda.Stream()
    torch.cuda.synchronize()
    with torch.cuda.stream(fs):
        batch.capture_frame_compact(br, bb, fh, bounce, fbh, 5, fs.cuda_stream)
        batch.launch_frame(fs.cuda_stream)
    torch.cuda.synchronize()
    out.update(frame_hits=fh.cpu().numpy(), frame_bounce_hits=fbh.cpu().numpy())
    sh = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
    s.cast_shadow_rays_dev(r, h, [0.3, 0.8, 0.5], sh)
    srays = torch.zeros((n, 6), dtype=torch.float32, device="cuda")
    vx.spawn_shadow_rays(r, h, [0.3, 0.8, 0.5], srays)
    sh_all = torch.zeros_like(sh)
    s.cast_rays_dev(srays, sh_all)
    out.update(shadow_hits=sh.cpu().numpy(), shadow_hits_all_slots=sh_all.cpu().numpy())
    # adjoint
    dw = W.config5(R=128, views=3, width=64, height=48, kind=1, seed=45)
    s5 = vx.Scene(dw.wl.scene)
    attr = torch.from_numpy(dw.attr).cuda()
    idx = torch.from_numpy(dw.dxt_idx.view(np.int32)).cuda()
    m = 3 * 64 * 48
    dimg = torch.zeros((m, 3), dtype=torch.float32, device="cuda")
    drec = torch.zeros((m, 4), dtype=torch.int32, device="cuda")
    vx.diff_forward_views(s5, dw.views, 64, 48, 1, attr, idx, dimg, drec)
    grad = torch.zeros_like(attr)
    vx.diff_backward(1, idx, drec, dimg, torch.zeros_like(dimg), grad)
    out.update(diff_img=dimg.cpu().numpy(), diff_rec=drec.cpu().numpy(), diff_grad_nonzero=np.array(
        [int((grad != 0).sum().item())]))
    # device builder
    bits = vx.synth_noise_dev(128, 16, 3, 0.3, 46, False)
    sd = vx.scene_from_dense_dev(bits, 128, 7, vx.VX_COLOR_DXT1, 1, True)
    dh = torch.zeros((4096, 4), dtype=torch.int32, device="cuda")
    sd.cast_rays_dev(torch.from_numpy(W.random_rays(4096, 128, seed=47)).cuda(), dh)
    out["devbuild_hits"] = dh.cpu().numpy()
    torch.cuda.synchronize()
    out["violations"] = np.array([vx.bounds_checks()[1]])
    np.savez(out_path, **out)


if __name__ == "__main__":
    main(sys.argv[1])
