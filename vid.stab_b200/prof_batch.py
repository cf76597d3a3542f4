#!/usr/bin/env python3
"""Profiling driver for the batched multi-stream detect.

Runs a batch of camera-walk streams (the benchmark's 64-stream mix by
default) resident in device memory, stepping it with the per-step API, and
wraps the last steps in an NVTX range named "batch", so a profiler can be
limited to the persistent kernel's launches of those steps:

    ncu --nvtx --nvtx-include "batch/" --section SpeedOfLight --section WarpStateStats \\
        --clock-control none -k regex:k_batch -c 2 -o out python vid.stab_b200/prof_batch.py

    python vid.stab_b200/prof_batch.py [--mix 64|small] [--steps 4] [--profiled 1]

Each step is two launches of the persistent kernel: stage A (blur, min/max,
coarse search of every stream) and stage B (fine search).  The steps before
the range prime the streams (first frame, tuning at creation).
"""
import argparse
import ctypes as C
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

MIXES = {
    "64": [(640, 360, 26), (1280, 720, 19), (1920, 1080, 13), (3840, 2160, 6)],
    "small": [(640, 360, 4), (1280, 720, 2), (1920, 1080, 1)],
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--mix", choices=sorted(MIXES), default="64")
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--profiled", type=int, default=1)
    a = ap.parse_args()
    import torch
    import vidstab_b200 as V
    from vidstab_b200 import synthetic as S
    sizes = [(w, h) for w, h, n in MIXES[a.mix] for _ in range(n)]
    steps = max(a.steps, a.profiled + 2)
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


if __name__ == "__main__":
    sys.exit(main())
