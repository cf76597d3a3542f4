#!/usr/bin/env python3
"""Profiling driver for the detect pass.

Runs the per-frame detect API over a seeded synthetic clip resident in device
memory (vsb_motion_detection_device) and wraps the last frames in an NVTX
range named "detect", so a profiler can be limited to those launches:

    ncu --nvtx --nvtx-include "detect/" --set full --clock-control none \
        -k regex:k_lattice -c 1 -o out python vid.stab_b200/prof_detect.py

    python vid.stab_b200/prof_detect.py [--width 1920 --height 1080]
        [--frames 4] [--profiled 1] [--search dense|pruned]

The frames before the range prime the detector (first frame, autotuning);
the range covers --profiled frames.
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
    first = n - a.profiled
    records = 0
    for k in range(n):
        if k == first:
            torch.cuda.synchronize()
            torch.cuda.nvtx.range_push("detect")
        records += len(det.detect_device(clip.data_ptr() + k * W * H, W))
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    det.close()
    print("frames %d (%d in the range), %d local motions" % (n, a.profiled, records))
    return 0


if __name__ == "__main__":
    sys.exit(main())
