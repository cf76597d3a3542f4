#!/usr/bin/env python3
"""Benchmark of the motion-detection pass (vidstabdetect) on B200.

Workload: the 1080p headline configuration -- a seeded synthetic 300-frame
1920x1080 YUV420p clip (4-octave value-noise scene with blobs and edges, camera
random walk with translation steps N(0,3 px), rotation N(0,0.2 deg), zoom
N(0,0.2 %), sensor noise sigma 2), default settings (stepsize 6, accuracy 15,
shakiness 5, mincontrast 0.25).  One step = the detect pass over the whole clip.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

* value: frames/s with the clip resident in HBM, through the library's frame
  loop vsb_detect_run over device frames (the results of
  vsb_motion_detection_device frame by frame; no host copies of frames);
* e2e: frames/s through the same frame loop with the frames in pinned host
  memory (vsMotionDetection's results frame by frame; the luma copy to the
  device and the per-field results back are inside the timed region);
* roofline: the dominant kernel (the coarse SAD search) against the measured
  packed-SAD throughput of this GPU, and the prefilter against HBM;
* cpu_baseline: the reference's own CPU detect (compiled from its sources,
  oracle/_ref) on this host's cores over a bounded sample of the same clip;
* learned: the learned-proposal detector on the same clip (frames/s in HBM
  and from host frames, field agreement with the exact full search over
  every field, frames identical to the plain path);
* batched: 64 concurrent streams of mixed resolution through one batch,
  aggregate frames/s, against the same streams through single-stream
  detectors one after another;
* large_shake_4k: 16 streams of 4K with large camera steps through the
  learned proposal inside the batched persistent kernel, against the plain
  batch, and learned and plain detectors stepped together; field agreement
  with the exact search, record by record;
* per_frame: vsMotionDetection once per frame from pinned host frames (the
  drop-in's call sequence);
* pruned_search: the exact pruned strategy on the clip in HBM, checked
  against the reference;
* second_pass: vsLocalmotions2Transforms' per-frame fit over the clip's
  motions, against the reference's.

With --gpus N (torchrun), every rank runs an independent clip (seed + rank):
no data moves between GPUs; the time is the max over ranks.

Every timed step's LocalMotions (all frames of the clip) are compared with
the reference's CPU detect of the same clip (oracle/_ref, compiled from the
reference's sources; the C restatement where that build is absent).

Profiling modes (no JSON line; an NVTX range around the last frames or
steps, for ncu --nvtx --nvtx-include "detect/" or "batch/"):

  python bench.py --profile detect [--width 1920 --height 1080]
      [--profile-frames 4] [--profiled 1] [--search dense|pruned]
      [--proposal default|PATH] [--conf-min X] [--host-profile]
  python bench.py --profile batch [--mix 64|small] [--profile-frames 4] [--profiled 1]

"detect" runs the per-frame API over a clip in device memory
(vsb_motion_detection_device); "batch" steps the 64-stream mix with the
per-step batch API.  The frames (steps) before the range prime the detector
(first frame, autotuning).
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "vid.stab_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))

import numpy as np  # noqa: E402


def records_per_frame(width, height):
    """an upper bound of the LocalMotions one frame gives (every coarse and
    fine field; fine fields are at least 16 pixels apart)"""
    return 256 + (width // 16 + 1) * (height // 16 + 1)

METRIC = "1080p detect frames/s: plain GPU (bit-exact) vs learned-proposal (≥99.5% agree)"
W, H = 1920, 1080
PUBLISHED_FPS = 1000.0 / 4.43  # docs/simd.md: 1080p detect, AVX2, 19 threads, Ryzen 9 9900X
WORKLOAD = ("plain GPU detect, 300-frame 1920x1080 YUV420p synthetic clip (value noise + blobs + "
            "edges, camera random walk), stepsize 6, accuracy 15, shakiness 5, mincontrast 0.25")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--frames", type=int, default=300)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batch-frames", type=int, default=120)
    ap.add_argument("--no-shake4k", action="store_true")
    ap.add_argument("--shake4k-frames", type=int, default=120)
    ap.add_argument("--side-steps", type=int, default=2,
                    help="timed steps of the batched and 4K arms (each a whole 120-frame run)")
    ap.add_argument("--side-warmup", type=int, default=1)
    ap.add_argument("--no-per-frame", action="store_true")
    ap.add_argument("--no-pruned", action="store_true")
    ap.add_argument("--no-second-pass", action="store_true")
    ap.add_argument("--profile", choices=["none", "detect", "batch"], default="none")
    ap.add_argument("--width", type=int, default=W)
    ap.add_argument("--height", type=int, default=H)
    ap.add_argument("--profile-frames", type=int, default=4)
    ap.add_argument("--profiled", type=int, default=1)
    ap.add_argument("--search", choices=["dense", "pruned"], default="dense")
    ap.add_argument("--proposal", default=None)
    ap.add_argument("--conf-min", type=float, default=float("nan"))
    ap.add_argument("--host-profile", action="store_true")
    ap.add_argument("--mix", choices=["64", "small"], default="64")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def reduce_max(vals, dist, device):
    """Each of vals, maxed over the ranks in one all-reduce (vals as they are
    without a process group): every rank's timed totals become the slowest
    rank's."""
    if not dist:
        return [float(v) for v in vals]
    import torch
    t = torch.tensor([float(v) for v in vals], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def aggregate_fps(frames_per_step, steps, world, seconds):
    """whole-job frames/s: every rank's frames over the slowest rank's time"""
    return frames_per_step * steps * world / seconds


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def make_clip(n, seed, device):
    from vidstab_b200 import synthetic as S
    return S.clip(W, H, n, seed=seed, device=device)


def cpu_reference(frames_np, seconds, threads):
    """The reference's CPU detect over a bounded prefix of the clip; returns
    (frames/s, frames used, seconds)."""
    import oracle as O
    if not O.ref_available():
        return None
    probe = min(6, len(frames_np))
    _, _, el = O.ref_clip(frames_np[:probe], 1, threads=threads)
    per = el / max(probe - 1, 1)
    n = int(min(len(frames_np), max(probe, seconds / max(per, 1e-4))))
    _, _, el = O.ref_clip(frames_np[:n], 1, threads=threads)
    return n / el, n, el


class Clocks:
    """nvidia-smi samples during a timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.f = None

    def start(self, busy=None):
        """starts sampling every 100 ms; busy() (GPU work) runs until the
        first sample has arrived (at most 5 s), so that the timed region
        that follows is sampled from its start"""
        try:
            self.f = tempfile.NamedTemporaryFile(mode="w+")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.proc.poll() is None:
            if os.path.getsize(self.f.name) > 0:
                break
            if busy:
                busy()
            else:
                time.sleep(0.05)
        self.skip = self._lines()

    def _lines(self):
        with open(self.f.name) as g:
            return len(g.read().splitlines())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.seek(0)
        sm, mx, reasons = [], 0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        # only the samples taken after start() returned: the timed region
        for line in self.f.read().splitlines()[getattr(self, "skip", 0):]:
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    f = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(f):
        d = json.load(open(f))
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def traffic_from_profile(name):
    """dram bytes per launch recorded by the committed ncu summary"""
    f = os.path.join(REPO, "profiles", name)
    if not os.path.exists(f):
        return None
    for line in open(f):
        if line.strip().startswith("dram_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


LM_FIELDS = ("vx", "vy", "fx", "fy", "fsize", "contrast", "match")


def same_records(a, b):
    """LocalMotions equality over all seven fields, in order (the predicate of
    tests/test_determinism.c:356-361 of the reference)"""
    return len(a) == len(b) and all(np.array_equal(a[k], b[k]) for k in LM_FIELDS)


def reference_records(frames_np, threads, pformat=1, **kw):
    """LocalMotions of the reference's CPU detect over a clip (the C
    restatement where the reference build is absent): records, per-frame
    counts, checker name"""
    import oracle as O
    if O.ref_available():
        r, c, _ = O.ref_clip(frames_np, pformat, threads=threads, **kw)
        return r, c, "reference (oracle/_ref)"
    r, c = O.oracle_clip(frames_np, pformat, **kw)
    return r, c, "oracle restatement"


def frames_identical(a, ca, b, cb):
    """frames whose LocalMotions are identical in two runs"""
    oa = np.concatenate([[0], np.cumsum(ca)])
    ob = np.concatenate([[0], np.cumsum(cb)])
    return int(sum(1 for k in range(len(ca)) if ca[k] == cb[k] and
                   np.array_equal(a[oa[k]:oa[k + 1]], b[ob[k]:ob[k + 1]])))


def fields_identical(a, ca, b, cb):
    """records of run b reproduced exactly by run a (frames with equal counts,
    record by record over all seven fields)"""
    oa = np.concatenate([[0], np.cumsum(ca)])
    ob = np.concatenate([[0], np.cumsum(cb)])
    same = 0
    for k in range(len(cb)):
        if ca[k] != cb[k] or cb[k] == 0:
            continue
        x, y = a[oa[k]:oa[k + 1]], b[ob[k]:ob[k + 1]]
        eq = np.ones(len(y), bool)
        for f in ("vx", "vy", "fx", "fy", "fsize", "contrast", "match"):
            eq &= x[f] == y[f]
        same += int(eq.sum())
    return same


def learned_arm(V, clip, host_np, nfr, steps, warmup, timed):
    """The learned-proposal detector (the packaged 1080p network) on the same
    clip: frames/s with the clip in HBM and from pinned host frames, field
    agreement with the exact full search (verify mode, every field of the
    clip), frames whose LocalMotions equal the plain detector's, and the
    per-frame device time of its kernels."""
    from vidstab_b200 import pnet
    blob = pnet.load_blob()
    rec = np.zeros(nfr * records_per_frame(W, H) + 64, V.LM_DTYPE)
    cnt = np.zeros(nfr, np.int32)

    def fresh(with_blob, verify=False):
        d = V.MotionDetector(W, H, V.PF_YUV420P)
        if with_blob:
            pnet.set_proposal(d, blob, verify=verify)
        return d

    d = fresh(True, verify=True)
    d.run(nfr, clip.data_ptr(), W * H, W, True, rec, cnt)
    st = pnet.proposal_stats(d)
    d.close()
    d = fresh(False)
    tp = d.run(nfr, clip.data_ptr(), W * H, W, True, rec, cnt)
    prec, pcnt = rec[:tp].copy(), cnt.copy()
    d.close()
    d = fresh(True)
    tl = d.run(nfr, clip.data_ptr(), W * H, W, True, rec, cnt)
    same = frames_identical(prec, pcnt, rec[:tl], cnt)
    d.close()
    dd, dh = fresh(True), fresh(True)
    for _ in range(warmup):
        dd.run(nfr, clip.data_ptr(), W * H, W, True, rec, cnt)
    td = timed(lambda: dd.run(nfr, clip.data_ptr(), W * H, W, True, rec, cnt), steps)
    for _ in range(max(1, warmup // 2)):
        dh.run(nfr, host_np.ctypes.data, W * H, W, False, rec, cnt)
    th = timed(lambda: dh.run(nfr, host_np.ctypes.data, W * H, W, False, rec, cnt), steps)
    nk = min(nfr, 60)
    kms = pnet.kernel_ms(dd, lambda: [dd.detect_device(clip.data_ptr() + k * W * H, W)
                                      for k in range(nk)])
    dd.close()
    dh.close()
    return {"value": nfr * steps / sum(td), "unit": "frames/s",
            "e2e": nfr * steps / sum(th),
            "agreement": st["agreement"], "fields_verified": st["verified"],
            "fallback_rate": st["fallback_rate"], "coarse_fallbacks": st["coarse_fell_back"],
            "fine_fallbacks": st["fine_fell_back"],
            "frames_identical_to_plain": same, "frames": nfr,
            "stage_ms_per_frame": kms,
            "stage_ms_note": "CUDA events around each stage on the detector's stream, per-frame "
                             "API, no frame overlap; they include host launch gaps, so they bound "
                             "the kernels from above (kernel durations: the ncu launch list)",
            "network": "packaged 1080p proposal network (vidstab_b200/data/pnet_1080p.vsbp) on "
                       "tcgen05: coarse fields by the network; fine fields take the dense search"}


def batched_arm(V, steps, warmup, timed, frames):
    """64 concurrent streams, resolutions 640x360 / 1280x720 / 1920x1080 /
    3840x2160 in ratio 4:3:2:1 (26/19/13/6 streams), each a camera-walk clip
    of its own seed, through one batch (persistent kernel per stage from
    captured CUDA graphs), against the same streams run one after another
    through single-stream detectors on the same GPU, and through the same
    detectors stepped together by one host thread (vsb_detect_multi).
    Every stream's batch output is compared with its own detector's, and
    the first stream of each resolution with the reference's CPU detect."""
    from vidstab_b200 import synthetic as S
    classes = [(640, 360, 26), (1280, 720, 19), (1920, 1080, 13), (3840, 2160, 6)]
    sizes = [(w, h) for w, h, n in classes for _ in range(n)]
    clips = [S.clip(w, h, frames, seed=5000 + i, device="cuda") for i, (w, h) in enumerate(sizes)]
    ptrs = [c.data_ptr() for c in clips]
    fb = [w * h for w, h in sizes]
    pitches = [w for w, _ in sizes]
    n = len(sizes)
    per = [records_per_frame(w, h) for w, h in sizes]
    out = np.zeros(frames * sum(per) + 64, V.LM_DTYPE)
    counts = np.zeros(frames * n, np.int32)
    b = V.Batch([w for w, _ in sizes], [h for _, h in sizes])
    tot = b.run(ptrs, fb, pitches, frames, True, out, counts)  # fresh streams: the parity run
    cm = counts.reshape(frames, n).copy()
    pos = np.concatenate([[0], np.cumsum(cm.ravel())])

    def batch_stream(s):
        return np.concatenate([out[pos[k * n + s]:pos[k * n + s + 1]] for k in range(frames)])

    mine = [batch_stream(s) for s in range(n)]
    for _ in range(warmup):
        b.run(ptrs, fb, pitches, frames, True, out, counts)
    l0 = b.launches()
    tb = timed(lambda: b.run(ptrs, fb, pitches, frames, True, out, counts), steps)
    launches = (b.launches() - l0) // max(steps, 1)
    b.close()
    # every stream through a detector of its own, one after another; the
    # first (untimed) pass checks every stream against the batch
    dets = [V.MotionDetector(w, h, V.PF_YUV420P) for w, h in sizes]
    rec = np.zeros(frames * max(per) + 64, V.LM_DTYPE)
    cnt = np.zeros(frames, np.int32)
    same = 0
    for s in range(n):
        t = dets[s].run(frames, ptrs[s], fb[s], pitches[s], True, rec, cnt)
        same += int(np.array_equal(cm[:, s], cnt) and same_records(mine[s], rec[:t]))

    def run_all():
        for s in range(n):
            dets[s].run(frames, ptrs[s], fb[s], pitches[s], True, rec, cnt)

    # the first stream of each resolution against the reference's CPU detect
    ref_same, checker = [], None
    first = 0
    for w, h, k in classes:
        r, c, checker = reference_records(clips[first].cpu().numpy(), host_cores())
        ref_same.append("%dx%d: %s" % (w, h, "identical" if np.array_equal(c, cm[:, first]) and
                                        same_records(r, mine[first]) else "DIFFERENT"))
        first += k
    for _ in range(warmup):
        run_all()
    ts = timed(run_all, steps)
    # the same detectors stepped together by one host thread (vsb_detect_multi)
    mout = np.zeros(frames * sum(per) + 64, V.LM_DTYPE)
    mcnt = np.zeros(frames * n, np.int32)
    for _ in range(warmup):
        V.detect_multi(dets, ptrs, fb, pitches, frames, True, mout, mcnt)
    tm = timed(lambda: V.detect_multi(dets, ptrs, fb, pitches, frames, True, mout, mcnt), steps)
    for d in dets:
        d.close()
    agg = n * frames * steps / sum(tb)
    seq = n * frames * steps / sum(ts)
    multi = n * frames * steps / sum(tm)
    return {"value": agg, "unit": "frames/s (all streams)", "streams": n,
            "frames_per_stream": frames, "records": int(tot), "steps": steps, "warmup": warmup,
            "streams_checked_identical": "%d of %d (batch vs each stream's own detector, all "
                                         "frames)" % (same, n),
            "reference_check": {"checker": checker, "streams": ref_same},
            "single_stream_detectors_sequential": seq, "speedup": agg / seq,
            "detectors_stepped_together": multi,
            "persistent_launches_per_step": int(launches),
            "workload": "64 streams 26x640x360 + 19x1280x720 + 13x1920x1080 + 6x3840x2160, "
                        "camera-walk clips (seed per stream), defaults of the 1080p clip"}


def shake4k_arm(V, steps, warmup, timed, frames):
    """16 streams of 3840x2160 with large camera steps (N(0,8 px), N(0,0.5
    deg)), shakiness 10: the learned proposal inside the batched persistent
    kernel (network passes, global-motion prior, narrowed searches and the
    dense search of fallbacks as work items of the same kernel; two graph
    launches per step) against the plain batch on the same GPU, with the
    learned detectors and the plain detectors stepped together by one host
    thread beside them; field agreement of the learned streams with the
    exact full search (verify mode of the detectors, and the batch's records
    against the plain detectors' record by record)."""
    from vidstab_b200 import pnet
    from vidstab_b200 import synthetic as S
    n, w, h = 16, 3840, 2160
    clips = S.clips_shared_world(w, h, frames, list(range(7001, 7001 + n)), 7000,
                                 trans_sigma=8.0, rot_sigma_deg=0.5, device="cuda")
    ptrs = [c.data_ptr() for c in clips]
    fb, pt = [w * h] * n, [w] * n
    blob = pnet.load_blob()
    out = np.zeros(frames * n * records_per_frame(w, h) + 64, V.LM_DTYPE)
    counts = np.zeros(frames * n, np.int32)

    def dets(learned, verify=False):
        ds = [V.MotionDetector(w, h, V.PF_YUV420P, shakiness=10) for _ in range(n)]
        if learned:
            for d in ds:
                pnet.set_proposal(d, blob, verify=verify)
        return ds

    # agreement and identity with the plain path, from fresh detectors
    ds = dets(True, verify=True)
    tl = V.detect_multi(ds, ptrs, fb, pt, frames, True, out, counts)
    lrec, lcnt = out[:tl].copy(), counts.copy()
    st = [pnet.proposal_stats(d) for d in ds]
    for d in ds:
        d.close()
    ds = dets(False)
    tp = V.detect_multi(ds, ptrs, fb, pt, frames, True, out, counts)
    prec, pcnt = out[:tp].copy(), counts.copy()
    same = frames_identical(prec, pcnt, lrec, lcnt)
    for d in ds:
        d.close()
    res = {}
    for name, learned in (("learned", True), ("plain_multi", False)):
        ds = dets(learned)
        for _ in range(warmup):
            V.detect_multi(ds, ptrs, fb, pt, frames, True, out, counts)
        t = timed(lambda: V.detect_multi(ds, ptrs, fb, pt, frames, True, out, counts), steps)
        res[name] = n * frames * steps / sum(t)
        for d in ds:
            d.close()
    b = V.Batch([w] * n, [h] * n, shakiness=10)
    for _ in range(warmup):
        b.run(ptrs, fb, pt, frames, True, out, counts)
    t = timed(lambda: b.run(ptrs, fb, pt, frames, True, out, counts), steps)
    res["plain_batch"] = n * frames * steps / sum(t)
    b.close()
    # the learned persistent batch: parity run from fresh streams, then timed
    b = V.Batch([w] * n, [h] * n, shakiness=10)
    b.set_proposal(blob)
    tb = b.run(ptrs, fb, pt, frames, True, out, counts)
    brec, bcnt = out[:tb].copy(), counts.copy()
    bst = b.proposal_stats()
    b_same_plain = frames_identical(brec, bcnt, prec, pcnt)
    b_fields = fields_identical(brec, bcnt, prec, pcnt)
    b_same_learned = frames_identical(brec, bcnt, lrec, lcnt)
    launches0 = b.launches()
    for _ in range(warmup):
        b.run(ptrs, fb, pt, frames, True, out, counts)
    t = timed(lambda: b.run(ptrs, fb, pt, frames, True, out, counts), steps)
    res["learned_batch"] = n * frames * steps / sum(t)
    per_step = (b.launches() - launches0) / float((warmup + steps) * frames)
    b.close()
    ver = sum(x["verified"] for x in st)
    return {"value": res["learned_batch"], "unit": "frames/s (all streams)",
            "impl": "learned proposal inside the batched persistent kernel",
            "plain_batch_persistent": res["plain_batch"],
            "speedup_vs_plain_batch": res["learned_batch"] / res["plain_batch"],
            "persistent_launches_per_step": per_step,
            "agreement": b_fields / max(1, int(pcnt.sum())),
            "agreement_basis": "records of the plain detectors (exact full search) reproduced by "
                               "the learned batch, record by record",
            "fields": int(pcnt.sum()),
            "stream_frames_identical_to_plain": b_same_plain,
            "stream_frames_identical_to_learned_detectors": b_same_learned,
            "stream_frames": n * frames,
            "coarse_fallback_rate": bst["coarse_fell_back"] / max(1, bst["coarse_searched"]),
            "fine_fallback_rate": bst["fine_fell_back"] / max(1, bst["fine_searched"]),
            "learned_detectors_stepped": {
                "value": res["learned"], "agreement": sum(x["identical"] for x in st) / ver
                if ver else None, "fields_verified": ver,
                "stream_frames_identical_to_plain": same},
            "plain_detectors_stepped": res["plain_multi"],
            "workload": "16 streams 3840x2160, %d frames each, camera steps N(0,8 px) and "
                        "N(0,0.5 deg), zoom N(0,0.2%%), shakiness 10, one shared scene" % frames}


def second_pass_arm(V, recs, counts, width, height, steps, warmup, timed):
    """The second pass (vsLocalmotions2Transforms' fit: one transform per
    frame, one GPU warp per frame) over the clip's LocalMotions: frames/s with
    the records resident in device memory (value) and from host records
    through vsb_motions_to_transforms (e2e, copies included), against the
    reference's vsLocalmotions2Transforms on the same records (single-threaded
    there); parity per frame against the reference's transforms."""
    import ctypes as C
    import torch
    import oracle as O
    L = V.lib()
    recs = np.ascontiguousarray(recs, V.LM_DTYPE)
    counts = np.asarray(counts, np.int64)
    n = len(counts)
    first = np.zeros(n + 1, np.int64)
    first[1:] = np.cumsum(counts)
    d_recs = torch.from_numpy(recs.view(np.uint8).copy()).cuda()
    d_first = torch.from_numpy(first).cuda()
    d_out = torch.zeros(n * V.TRANSFORM_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    maxn = int(counts.max()) if n else 0

    def run_dev():
        rc = L.vsb_motions_to_transforms_device(d_recs.data_ptr(), d_first.data_ptr(), n, maxn,
                                                width, height, 0.0, 0, d_out.data_ptr(), None,
                                                None, st)
        assert rc == 0, L.vsb_last_error()

    host_out = np.zeros(n, V.TRANSFORM_DTYPE)

    def run_host():
        rc = L.vsb_motions_to_transforms(recs.ctypes.data, first.ctypes.data, n, width, height,
                                         0.0, 0, host_out.ctypes.data, None, None)
        assert rc == 0, L.vsb_last_error()

    for _ in range(max(3, warmup)):
        run_dev()
        run_host()
    dev_t = timed(run_dev, steps)
    host_t = timed(run_host, steps)
    dev_out = d_out.cpu().numpy().view(V.TRANSFORM_DTYPE)
    res = {"value": n * len(dev_t) / sum(dev_t), "unit": "frames/s",
           "e2e": n * len(host_t) / sum(host_t),
           "kernel_ms": 1000.0 * min(dev_t), "frames": n, "records": int(len(recs)),
           "h2d_bytes_per_step": int(recs.nbytes + first.nbytes),
           "d2h_bytes_per_step": int(n * V.TRANSFORM_DTYPE.itemsize),
           "launches_per_step": 1,
           "workload": "the 300-frame clip's LocalMotions (as detected), similarity model, "
                       "smoothZoom 0, lens estimate off"}
    mine = np.stack([dev_out["x"], dev_out["y"], dev_out["alpha"], dev_out["zoom"],
                     dev_out["extra"].astype(np.float64)], 1)
    if O.ref_available():
        R = O.ref()
        R.vsref_motions_to_transforms.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                                  C.c_int, C.c_double, C.c_int, C.c_int,
                                                  C.c_void_p, C.c_void_p]
        TD = np.dtype([("x", "<f8"), ("y", "<f8"), ("alpha", "<f8"), ("zoom", "<f8"),
                       ("barrel", "<f8"), ("rshutter", "<f8"), ("extra", "<i4"), ("pad", "<i4")])
        ref = np.zeros(n, TD)
        best = None
        for _ in range(3):
            el = C.c_double()
            R.vsref_motions_to_transforms(width, height, recs.ctypes.data, first.ctypes.data, n,
                                          0.0, 0, 0, ref.ctypes.data, C.byref(el))
            best = el.value if best is None else min(best, el.value)
        refrows = np.stack([ref["x"], ref["y"], ref["alpha"], ref["zoom"],
                            ref["extra"].astype(np.float64)], 1)
        res["reference"] = {"value": n / best, "unit": "frames/s", "cores": 1,
                            "kind": "reference",
                            "sample": "the same %d frames, vsLocalmotions2Transforms (best of 3)"
                                      % n}
        res["parity"] = {"checker": "reference (oracle/_ref)",
                         "frames_identical": int((mine == refrows).all(1).sum()),
                         "extra_identical": bool(np.array_equal(mine[:, 4], refrows[:, 4])),
                         "max_abs_diff": float(np.abs(mine[:, :4] - refrows[:, :4]).max())
                         if n else 0.0,
                         "host_equals_device": bool(np.array_equal(host_out.view(np.uint8),
                                                                   dev_out.view(np.uint8)))}
    return res


def run_reference(args):
    """The reference's own CPU detect (oracle/_ref, compiled from its
    sources) over the same 300-frame clip the GPU arm runs (same generator,
    seed and device), every step the whole clip, all host threads."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference build (oracle/_ref) not present"}))
        return 0
    cores = host_cores()
    n = args.frames
    device = "cpu"
    try:
        import torch
        if torch.cuda.is_available():
            device = "cuda"
    except Exception:
        pass
    clip = make_clip(n, seed=1, device=device)
    frames = clip.cpu().numpy()
    del clip
    for _ in range(args.warmup):
        O.ref_clip(frames[:3], 1, threads=cores)
    times = []
    for _ in range(args.steps):
        _, _, el = O.ref_clip(frames, 1, threads=cores)
        times.append(el)
    fps = n / statistics.median(times)
    sample = ("the whole %d-frame 1920x1080 clip per step, the clip the GPU arm times "
              "(seed 1, generated on %s)" % (n, device))
    print(json.dumps({
        "metric": METRIC, "value": fps, "unit": "frames/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * statistics.median(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": fps / PUBLISHED_FPS,
        "dtype": "u8", "data": "synthetic", "impl": "reference",
        "config": {"workload": WORKLOAD, "frames_per_step": n, "width": W, "height": H},
        "cpu_baseline": {"value": fps, "unit": "frames/s", "cores": cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": fps, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


def profile_detect(a):
    """NVTX range "detect" around the last a.profiled frames of the per-frame
    API over a clip in device memory"""
    import ctypes as C
    import torch
    import vidstab_b200 as V
    from vidstab_b200 import synthetic as S
    w, h = a.width, a.height
    n = max(a.profile_frames, a.profiled + 2)
    clip = S.clip(w, h, n, seed=1, device="cuda")
    torch.cuda.synchronize()
    V.lib().vsb_set_default_search_mode(1 if a.search == "pruned" else 0)
    det = V.MotionDetector(w, h, V.PF_YUV420P)
    if a.proposal:
        from vidstab_b200 import pnet
        blob = pnet.load_blob(None if a.proposal == "default" else a.proposal)
        pnet.set_proposal(det, blob, conf_min=a.conf_min)
    L = V.lib()
    L.vsb_host_profile.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    L.vsb_host_profile.restype = None
    first = n - a.profiled
    records = 0
    for k in range(n):
        if k == first:
            torch.cuda.synchronize()
            L.vsb_host_profile(None, None, 1)
            torch.cuda.nvtx.range_push("detect")
        records += len(det.detect_device(clip.data_ptr() + k * w * h, w))
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    if a.host_profile:
        sec = (C.c_double * 4)()
        nf = C.c_long()
        L.vsb_host_profile(sec, C.byref(nf), 0)
        per = [1e6 * v / max(nf.value, 1) for v in sec]
        print("per frame (us): device stage A %.1f, host A %.1f, device stage B %.1f, host B %.1f,"
              " total %.1f" % (per[0], per[1], per[2], per[3], sum(per)))
    det.close()
    print("frames %d (%d in the range), %d local motions" % (n, a.profiled, records))
    return 0


def profile_batch(a):
    """NVTX range "batch" around the last a.profiled steps of a batch of
    camera-walk streams stepped with the per-step API"""
    import ctypes as C
    import torch
    import vidstab_b200 as V
    from vidstab_b200 import synthetic as S
    mixes = {"64": [(640, 360, 26), (1280, 720, 19), (1920, 1080, 13), (3840, 2160, 6)],
             "small": [(640, 360, 4), (1280, 720, 2), (1920, 1080, 1)]}
    sizes = [(w, h) for w, h, n in mixes[a.mix] for _ in range(n)]
    steps = max(a.profile_frames, a.profiled + 2)
    clips = [S.clip(w, h, steps, seed=5000 + i, device="cuda") for i, (w, h) in enumerate(sizes)]
    torch.cuda.synchronize()
    pitches = [w for w, _ in sizes]
    b = V.Batch([w for w, _ in sizes], [h for _, h in sizes])
    L = V.lib()
    L.vsb_host_profile.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    first = steps - a.profiled
    records = 0
    try:
        for k in range(steps):
            if k == first:
                torch.cuda.synchronize()
                L.vsb_host_profile(None, None, 1)
                torch.cuda.nvtx.range_push("batch")
            planes = [c.data_ptr() + k * w * h for c, (w, h) in zip(clips, sizes)]
            records += sum(len(r) for r in b.detect(planes, pitches, True))
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        sec = (C.c_double * 4)()
        nf = C.c_long()
        L.vsb_host_profile(sec, C.byref(nf), 0)
        per = [1e3 * v / max(nf.value / len(sizes), 1) for v in sec]
        print("per step (ms): stage A %.2f, host A %.2f, stage B %.2f, host B %.2f"
              % (per[0], per[1], per[2], per[3]))
        print("streams %d, steps %d (%d in the range), %d local motions, grid %s"
              % (len(sizes), steps, a.profiled, records, b.grid()))
    finally:
        b.close()
    return 0


def main():
    args = parse()
    if args.profile == "detect":
        return profile_detect(args)
    if args.profile == "batch":
        return profile_batch(args)
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import vidstab_b200 as V
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    L = V.lib()
    L.vsb_counters.argtypes = [C.POINTER(C.c_longlong)] * 3

    def counters():
        a, b, c = C.c_longlong(), C.c_longlong(), C.c_longlong()
        L.vsb_counters(C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    nfr = args.frames
    clip = make_clip(nfr, seed=1 + rank, device="cuda")
    torch.cuda.synchronize()
    host = torch.empty(clip.shape, dtype=torch.uint8).pin_memory()
    host.copy_(clip.cpu())
    host_np = host.numpy()

    # one detector per arm, initialised before timing (vsMotionDetectInit:
    # device buffers, tiling lookup); each step runs the clip's frames through
    # it in C and copies every LocalMotion into a preallocated record buffer
    rec = np.zeros(nfr * records_per_frame(W, H) + 64, V.LM_DTYPE)
    cnt = np.zeros(nfr, np.int32)
    det_dev = V.MotionDetector(W, H, V.PF_YUV420P)
    det_host = V.MotionDetector(W, H, V.PF_YUV420P)

    def run_device():
        return det_dev.run(nfr, clip.data_ptr(), W * H, W, True, rec, cnt)

    def run_host():
        return det_host.run(nfr, host_np.ctypes.data, W * H, W, False, rec, cnt)

    # the reference's LocalMotions of the whole clip as a detector that has
    # already run it sees it (every timed step follows a warm-up pass, so
    # frame 0 is searched against the clip's last frame): the reference
    # detects [last frame, frame 0, ..., last frame] and its first frame's
    # (empty) result is dropped.  Every rank checks its own clip.
    primed = np.concatenate([host_np[-1:], host_np])
    ref_rec, ref_cnt, checker = reference_records(primed, max(1, host_cores() // world))
    assert ref_cnt[0] == 0
    ref_cnt = ref_cnt[1:]
    checks = {"device": [], "host": [], "per_frame": []}

    def check(kind, cnt_now, total):
        checks[kind].append(bool(total == len(ref_rec) and np.array_equal(cnt_now, ref_cnt) and
                                 same_records(rec[:total], ref_rec)))

    def timed(fn, steps, after=None):
        """CUDA-event time of each of `steps` calls of fn, bracketed by a
        barrier and a device synchronize on both sides; after(result) runs
        outside the timed region"""
        ts = []
        for _ in range(steps):
            if dist:
                dist.barrier()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            r = fn()
            e1.record()
            torch.cuda.synchronize()
            if dist:
                dist.barrier()
            ts.append(e0.elapsed_time(e1) / 1000.0)
            if after:
                after(r)
        return ts

    for _ in range(max(1, args.warmup)):  # at least one pass: the parity check expects it
        run_device()
    # clocks sampled over both timed loops (clip in HBM, then host frames)
    clocks = Clocks(local)
    clocks.start(busy=run_device)
    l0, _, _ = counters()
    dev_times = timed(run_device, args.steps, lambda t: check("device", cnt, t))
    l1, _, _ = counters()
    for _ in range(max(1, args.warmup // 2)):
        run_host()
    _, h0, d0 = counters()
    host_times = timed(run_host, args.steps, lambda t: check("host", cnt, t))
    _, h1, d1 = counters()
    clk = clocks.stop()
    det_dev.close()
    det_host.close()
    # the drop-in's per-frame path: one vsMotionDetection call per frame
    # (what vidstabdetect calls), pinned host frames, no overlap between frames
    per_frame = None
    if not args.no_per_frame:
        det_pf = V.MotionDetector(W, H, V.PF_YUV420P)

        def run_pf():
            return det_pf.run_frames(nfr, host_np.ctypes.data, W * H, W, False, rec, cnt)

        for _ in range(max(1, args.warmup // 2)):
            run_pf()
        p0, _, _ = counters()
        pf_times = timed(run_pf, args.steps, lambda t: check("per_frame", cnt, t))
        p1, _, _ = counters()
        det_pf.close()
        (tot_pf,) = reduce_max([sum(pf_times)], dist, "cuda")
        per_frame = {"value": aggregate_fps(nfr, args.steps, world, tot_pf), "unit": "frames/s",
                     "launches_per_frame": (p1 - p0) / float(nfr * args.steps),
                     "api": "vsMotionDetection once per frame, pinned host frames, each call "
                            "returning the frame's motions (vsb_detect_frames)"}
    # the exact pruned strategy (vsb_set_search_mode 1: a partial-sum bound
    # removes candidates that cannot win) on the same clip in HBM, checked
    # against the same reference records; it runs without frame overlap
    pruned = None
    if not args.no_pruned:
        V.lib().vsb_set_default_search_mode(1)
        det_pr = V.MotionDetector(W, H, V.PF_YUV420P)
        V.lib().vsb_set_default_search_mode(-1)

        def run_pr():
            return det_pr.run(nfr, clip.data_ptr(), W * H, W, True, rec, cnt)

        for _ in range(max(1, args.side_warmup)):
            run_pr()
        pr_ok = []
        pr_times = timed(run_pr, args.side_steps,
                         lambda t: pr_ok.append(bool(t == len(ref_rec) and
                                                     np.array_equal(cnt, ref_cnt) and
                                                     same_records(rec[:t], ref_rec))))
        det_pr.close()
        (tot_pr,) = reduce_max([sum(pr_times)], dist, "cuda")
        pruned = {"value": aggregate_fps(nfr, args.side_steps, world, tot_pr),
                  "unit": "frames/s", "identical_to_reference": all(pr_ok),
                  "api": "vsb_detect_run with the pruned strategy, clip in HBM (no frame "
                         "overlap: the pruned search shares its scratch between stages)"}
    tot_dev = sum(dev_times)
    tot_host = sum(host_times)
    tot_dev, tot_host = reduce_max([tot_dev, tot_host], dist, "cuda")
    value = aggregate_fps(nfr, args.steps, world, tot_dev)
    e2e = aggregate_fps(nfr, args.steps, world, tot_host)
    identical = all(checks["device"]) and all(checks["host"]) and all(checks["per_frame"])
    (all_ranks,) = reduce_max([0.0 if identical else 1.0], dist, "cuda")
    parity = {"frames": nfr, "records": int(len(ref_rec)), "checker": checker,
              "steps_checked": {k: len(v) for k, v in checks.items()},
              "identical": bool(identical), "all_ranks_identical": all_ranks == 0.0,
              "checked": "the LocalMotions of every timed step (value, e2e and per_frame "
                         "loops), all frames, all seven fields, against the checker's detect "
                         "of the same clip after a pass over it (its first frame searched "
                         "against its last, as in a step after warm-up)"}

    def timed_local(fn, steps):
        """CUDA-event time of fn on this rank alone (no barrier)"""
        ts = []
        for _ in range(steps):
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1) / 1000.0)
        return ts

    learned = None
    batched = None
    if rank == 0 and not args.no_learned:
        learned = learned_arm(V, clip, host_np, nfr, args.steps, args.warmup, timed_local)
    if rank == 0 and not args.no_batched:
        batched = batched_arm(V, args.side_steps, args.side_warmup, timed_local, args.batch_frames)
    second = None
    if rank == 0 and not args.no_second_pass:
        second = second_pass_arm(V, ref_rec, ref_cnt, W, H, args.steps, args.warmup, timed_local)
    shake4k = None
    if rank == 0 and not args.no_shake4k:
        shake4k = shake4k_arm(V, args.side_steps, args.side_warmup, timed_local,
                              args.shake4k_frames)

    # per-kernel device time on the detector's stream (separate, instrumented pass)
    roof = None
    roof_hbm = None
    kernel_ms = None
    tiling = None
    if rank == 0:
        det = V.MotionDetector(W, H, V.PF_YUV420P)
        L.vsb_set_kernel_timing.argtypes = [C.c_void_p, C.c_int]
        L.vsb_kernel_times.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.vsb_set_kernel_timing(C.byref(det.md), 1)
        nk = min(nfr, 60)
        for k in range(nk):
            det.detect_device(clip.data_ptr() + k * W * H, W)
        ms = (C.c_double * 6)()
        cnt = (C.c_long * 6)()
        L.vsb_kernel_times(C.byref(det.md), ms, cnt)
        fc = det.md.fieldscoarse
        tiling = {}
        for name, fine in (("coarse", 0), ("fine", 1)):
            desc = (C.c_int * 8)()
            L.vsb_search_tiling(C.byref(det.md), fine, desc)
            kern = {5: "k_sweep", 6: "k_fine"}.get(desc[1], "k_lattice")
            tiling[name] = {"kernel": kern,
                            "layout": desc[1], "lattice_cols_per_tile": desc[2],
                            "lattice_rows_per_tile": desc[3], "strips": desc[4],
                            "threads": desc[5], "smem": desc[6],
                            ("ctas" if desc[1] == 5 else "ctas_per_field"): desc[7]}
            if desc[1] == 6:
                tiling[name]["lattice_rows_per_thread"] = desc[4]
                tiling[name]["strips"] = tiling[name].pop("ctas_per_field")
        bdesc = (C.c_int * 4)()
        L.vsb_blur_tiling(C.byref(det.md), bdesc)
        fused = bool(bdesc[3])
        tiling["prefilter"] = ("k_blurmm: blur + field min/max, one launch, 128x8 warp blocks"
                               if fused else "k_blur_fast tile %dx%d + k_minmax_planar"
                               % (bdesc[0], bdesc[1]))
        det.close()
        kernel_ms = {n: (ms[i] / cnt[i] if cnt[i] else None) for i, n in
                     enumerate(["blur", "field_minmax", "coarse_search", "fine_search"])}
        peak_sad = C.c_double()
        L.vsb_sad_peak(0, C.byref(peak_sad))
        # algorithmic work of one coarse launch: every coarse field, every
        # lattice candidate plus the refinement candidates, size^2 byte SADs
        K = fc.maxShift // fc.stepSize
        lattice = (2 * K + 1) ** 2
        refine, s = 0, fc.stepSize
        while s > 1:
            h = s // 2
            side = (2 * (s - h)) // h + 1
            refine += side * side - 1
            s = h
        ops = fc.fieldNum * (lattice + refine) * fc.fieldSize ** 2
        t_coarse = kernel_ms["coarse_search"] * 1e-3
        achieved = ops / t_coarse / 1e12
        peak = peak_sad.value / 1e12
        kname = tiling["coarse"]["kernel"]
        roof = {"kernel": "%s (coarse SAD search, 1080p)" % kname, "bound": "int-alu",
                "achieved": achieved, "peak": peak, "unit": "Tbyte-absdiff/s", "frac": achieved / peak,
                "traffic": traffic_from_profile("%s_coarse_1080p.md" % kname),
                "algorithmic_per_launch": ops,
                "peak_source": "measured live: register-only vabsdiff4 loop (vsb_sad_peak)"}
        hbm, src = peaks()
        bb = 2.0 * W * H
        t_blur = kernel_ms["blur"] * 1e-3
        pname = "k_blurmm" if fused else "k_blur_fast"
        roof_hbm = {"kernel": "%s (prefilter%s, 1080p)" % (pname, " + field min/max" if fused
                                                             else ""), "bound": "hbm",
                    "achieved": bb / t_blur / 1e9, "peak": hbm, "unit": "GB/s",
                    "frac": bb / t_blur / 1e9 / hbm, "peak_source": src,
                    "traffic": traffic_from_profile("%s_1080p.md" % pname)}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        cores = host_cores()
        r = cpu_reference(host_np, args.cpu_seconds, cores)
        if r:
            fps, n, el = r
            cpu = {"value": fps, "unit": "frames/s", "cores": cores, "kind": "reference",
                   "sample": "first %d frames of the same clip (%.1f s)" % (n, el)}
            r1 = cpu_reference(host_np, min(args.cpu_seconds, 5.0), 1)
            if r1:
                cpu["one_thread"] = {"value": r1[0], "unit": "frames/s", "cores": 1,
                                     "sample": "first %d frames of the same clip (%.1f s)"
                                               % (r1[1], r1[2])}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * tot_dev / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": value / PUBLISHED_FPS,
            "dtype": "u8", "data": "synthetic",
            "config": {"workload": WORKLOAD, "frames_per_step": nfr, "width": W, "height": H,
                       "l2": "inputs (%d MB of luma) larger than L2" % (nfr * W * H // 2**20),
                       "parallelism": "replicas x%d (independent clips, no collective)" % world,
                       "timed_step": "the clip's frames through one initialised detector's "
                                     "frame loop (vsb_detect_run: vsMotionDetection's results "
                                     "frame by frame, consecutive frames overlapped on the "
                                     "GPU, records copied out)",
                       "vs_baseline_ref": "docs/simd.md 1080p AVX2 19-thread figure (4.43 ms/frame)"},
            "e2e": {"value": e2e, "unit": "frames/s",
                    "h2d_bytes_per_step": (h1 - h0) // max(args.steps, 1),
                    "d2h_bytes_per_step": (d1 - d0) // max(args.steps, 1)},
            "gpu_launches": l1 - l0,
            "roofline": roof, "roofline_hbm": roof_hbm, "kernel_ms": kernel_ms,
            "tiling": tiling,
            "learned": learned, "batched": batched, "large_shake_4k": shake4k,
            "second_pass": second,
            "cpu_baseline": cpu, "clocks": clk, "parity": parity, "per_frame": per_frame,
            "pruned_search": pruned,
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
