#!/usr/bin/env python3
"""Profiling driver for the detect pass.

Runs the per-frame detect API over a seeded synthetic clip resident in device
memory (vsb_motion_detection_device) and wraps the last frames in an NVTX
range named "detect", so a profiler can be limited to those launches:

    ncu --nvtx --nvtx-include "detect/" --set full --clock-control none \
        -k regex:k_lattice -c 1 -o out python vid.stab_b200/prof_detect.py

    python vid.stab_b200/prof_detect.py [--width 1920 --height 1080]
        [--frames 4] [--profiled 1] [--search dense|pruned]
        [--proposal default|PATH] [--conf-min X] [--host-profile]

The frames before the range prime the detector (first frame, autotuning);
the range covers --profiled frames.  --proposal gives the detector a search
proposal network (the packaged one for "default"); --host-profile prints the
per-frame wall time of the device stages and the host parts over the range.
"""
import argparse
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--frames", type=int, default=4)
    ap.add_argument("--profiled", type=int, default=1)
    ap.add_argument("--search", choices=["dense", "pruned"], default="dense")
    ap.add_argument("--proposal", default=None)
    ap.add_argument("--conf-min", type=float, default=float("nan"))
    ap.add_argument("--host-profile", action="store_true")
    a = ap.parse_args()
    import torch
    import vidstab_b200 as V
    from vidstab_b200 import synthetic as S
    W, H = a.width, a.height
    n = max(a.frames, a.profiled + 2)
    clip = S.clip(W, H, n, seed=1, device="cuda")
    torch.cuda.synchronize()
    V.lib().vsb_set_default_search_mode(1 if a.search == "pruned" else 0)
    det = V.MotionDetector(W, H, V.PF_YUV420P)
    if a.proposal:
        from vidstab_b200 import pnet
        blob = pnet.load_blob(None if a.proposal == "default" else a.proposal)
        pnet.set_proposal(det, blob, conf_min=a.conf_min)
    import ctypes as C
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
        records += len(det.detect_device(clip.data_ptr() + k * W * H, W))
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


if __name__ == "__main__":
    sys.exit(main())
