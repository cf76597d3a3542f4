#!/usr/bin/env python3
"""Trains the search-proposal network on the GPU and writes its VSBP file.

    python vid.stab_b200/train_pnet.py --out vid.stab_b200/vidstab_b200/data/pnet_1080p.vsbp

1. Training pairs: 1920x1080 camera-walk clips (the 1080p benchmark's
   generator, held-out seeds) run through a plain detector with the field
   log on; each coarse and fine field the full search ran on gives its
   network input and its full-search result as the label.
2. Training: the library's own forward and backward kernels under a torch
   autograd Function, Adam on fp32 master weights, bf16 weights in the
   kernels.
3. Calibration on a validation clip: the confidence threshold and the SAD
   bound of the fallback.
4. Evaluation on a third clip: field agreement with the full search
   (verify mode) and frames/s of the plain and the proposal detectors.

Prints one JSON summary line.
"""
import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--train-seeds", default="101,102,103,104")
    ap.add_argument("--frames", type=int, default=150)
    ap.add_argument("--pairs", type=int, default=200000)
    ap.add_argument("--val-seed", type=int, default=201)
    ap.add_argument("--eval-seed", type=int, default=301)
    ap.add_argument("--eval-frames", type=int, default=100)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--radius", type=float, default=2.0)
    ap.add_argument("--coarse-weight", type=float, default=3.0)
    ap.add_argument("--trans-sigma", type=float, default=3.0)
    ap.add_argument("--rot-sigma", type=float, default=0.2)
    ap.add_argument("--conf-target", type=float, default=0.999)
    ap.add_argument("--conf-sweep", default="")
    ap.add_argument("--val-agreement", type=float, default=1.0)
    ap.add_argument("--train-shake", default="",
                    help="per training seed, a factor on the camera-walk step sizes")
    a = ap.parse_args()

    import torch
    import vidstab_b200 as V
    from vidstab_b200 import pnet
    from vidstab_b200 import synthetic as S

    W, H = a.width, a.height
    t0 = time.time()
    xs, labs = [], []
    seeds = [int(v) for v in a.train_seeds.split(",")]
    shakes = [float(v) for v in a.train_shake.split(",")] if a.train_shake else [1.0] * len(seeds)
    for sd, k in zip(seeds, shakes):
        clip = S.clip(W, H, a.frames, seed=sd, device="cuda", trans_sigma=a.trans_sigma * k,
                      rot_sigma_deg=a.rot_sigma * k)
        x, lab = pnet.field_log(clip, W, H, cap=a.pairs)
        xs.append(x)
        labs.append(lab)
        del clip
    x = torch.cat(xs)
    lab = np.concatenate(labs)
    keep = min(len(lab), a.pairs)
    x, lab = x[:keep], lab[:keep]
    t_data = time.time() - t0

    sizes = {}
    det = V.MotionDetector(W, H, V.PF_YUV420P)
    sizes[0] = det.md.fieldscoarse.fieldSize
    sizes[1] = det.md.fieldsfine.fieldSize
    det.close()

    t1 = time.time()
    log = []
    master = pnet.train(x, lab, steps=a.steps, batch=a.batch, lr=a.lr, radius=a.radius,
                        coarse_weight=a.coarse_weight,
                        log=lambda r: (log.append(r), print("step %d loss %.4f hit %.3f" % r,
                                                           flush=True)))
    torch.cuda.synchronize()
    t_train = time.time() - t1
    bits, f32 = pnet.master_bits(master)
    params = pnet.params_to_device(bits, f32)

    vclip = S.clip(W, H, 60, seed=a.val_seed, device="cuda", trans_sigma=a.trans_sigma,
                   rot_sigma_deg=a.rot_sigma)
    vx, vlab = pnet.field_log(vclip, W, H, cap=60 * 500)
    cal = pnet.calibrate(params, vx, vlab, sizes, radius=a.radius, target=a.conf_target)
    blob = pnet.pack_blob(bits, f32, pnet.SCALE, a.radius, cal["conf_min"], cal["match_bound"])
    # the confidence threshold: the lowest fallback rate among the thresholds
    # whose field agreement with the full search on the validation clip is
    # complete (the ring and SAD-bound checks stay on)
    sweep = []
    for cm in sorted({round(cal["conf_min"], 3), 2.0, 0.0, -2.0, -4.0}, reverse=True):
        det = V.MotionDetector(W, H, V.PF_YUV420P)
        pnet.set_proposal(det, blob, conf_min=cm, verify=True)
        rec = np.zeros(60 * 512 + 64, V.LM_DTYPE)
        cnt = np.zeros(60, np.int32)
        det.run(60, vclip.data_ptr(), W * H, W, True, rec, cnt)
        st = pnet.proposal_stats(det)
        det.close()
        sweep.append({"conf_min": cm, "agreement": st["agreement"],
                      "fallback_rate": st["fallback_rate"]})
    good = [r for r in sweep if r["agreement"] is not None and r["agreement"] >= a.val_agreement]
    if good:
        pick = min(good, key=lambda r: (r["fallback_rate"], -r["conf_min"]))
        cal["conf_min"] = pick["conf_min"]
    cal["sweep"] = sweep
    del vclip
    blob = pnet.pack_blob(bits, f32, pnet.SCALE, a.radius, cal["conf_min"], cal["match_bound"])
    os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
    with open(a.out, "wb") as f:
        f.write(blob)

    ev = evaluate(blob, W, H, a.eval_seed, a.eval_frames, a.trans_sigma, a.rot_sigma,
                  [float(v) for v in a.conf_sweep.split(",")] if a.conf_sweep else ())
    ev_shake = evaluate(blob, W, H, a.eval_seed + 1, a.eval_frames // 2, 8.0, 0.5)
    print(json.dumps({"pairs": int(len(lab)), "pairs_used": int((lab["use"] == 1).sum()),
                      "coarse_pairs": int(((lab["use"] == 1) & (lab["kind"] == 0)).sum()),
                      "data_s": t_data, "train_s": t_train, "steps": a.steps,
                      "final_loss": log[-1][1] if log else None, "calibration": cal,
                      "eval": ev, "eval_large_shake": ev_shake, "out": a.out}))


def evaluate(blob, W, H, seed, n, trans_sigma=3.0, rot_sigma=0.2, conf_sweep=()):
    """agreement (verify mode) and frames/s of plain vs proposal detectors"""
    import torch
    import vidstab_b200 as V
    from vidstab_b200 import pnet
    from vidstab_b200 import synthetic as S
    clip = S.clip(W, H, n, seed=seed, device="cuda", trans_sigma=trans_sigma,
                  rot_sigma_deg=rot_sigma)
    res = {}
    rec = np.zeros(n * 512 + 64, V.LM_DTYPE)
    cnt = np.zeros(n, np.int32)

    def timed(det):
        det.run(n, clip.data_ptr(), W * H, W, True, rec, cnt)  # warm-up pass
        torch.cuda.synchronize()
        t = time.perf_counter()
        tot = det.run(n, clip.data_ptr(), W * H, W, True, rec, cnt)
        torch.cuda.synchronize()
        return n / (time.perf_counter() - t), rec[:tot].copy(), cnt.copy()

    plain = V.MotionDetector(W, H, V.PF_YUV420P)
    res["plain_fps"], prec, pcnt = timed(plain)
    res["plain_kernel_ms"] = pnet.kernel_ms(
        plain, lambda: plain.run(n, clip.data_ptr(), W * H, W, True, rec, cnt))
    plain.close()
    runs = [("learned", blob, float("nan"), False), ("learned_fine_net", blob, float("nan"), True),
            ("zero", pnet.zero_blob(), float("nan"), False)]
    runs += [("learned_conf%g" % cm, blob, cm, False) for cm in conf_sweep]
    for name, b, cm, fnet in runs:
        det = V.MotionDetector(W, H, V.PF_YUV420P)
        pnet.set_proposal(det, b, conf_min=cm, verify=True, fine_net=fnet)
        det.run(n, clip.data_ptr(), W * H, W, True, rec, cnt)
        st = pnet.proposal_stats(det)
        det.close()
        det = V.MotionDetector(W, H, V.PF_YUV420P)
        pnet.set_proposal(det, b, conf_min=cm, fine_net=fnet)
        fps, lrec, lcnt = timed(det)
        kms = pnet.kernel_ms(det, lambda: det.run(n, clip.data_ptr(), W * H, W, True, rec, cnt))
        det.close()
        res[name] = {"fps": fps, "agreement": st["agreement"], "fallback_rate": st["fallback_rate"],
                     "searched": st["searched"], "stats": st, "kernel_ms": kms,
                     "frames_identical": frames_identical(prec, pcnt, lrec, lcnt), "frames": n}
    return res


def frames_identical(a, ca, b, cb):
    """number of frames whose LocalMotions are identical in both runs"""
    oa = np.concatenate([[0], np.cumsum(ca)])
    ob = np.concatenate([[0], np.cumsum(cb)])
    same = 0
    for k in range(len(ca)):
        if ca[k] == cb[k] and np.array_equal(a[oa[k]:oa[k + 1]], b[ob[k]:ob[k + 1]]):
            same += 1
    return same


if __name__ == "__main__":
    main()
