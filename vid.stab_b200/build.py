#!/usr/bin/env python3
"""Builds libvidstab_b200.so in-tree (vid.stab_b200/lib/).

Host C is compiled with gcc, the kernels with nvcc for sm_100a only.  The C
files whose floating-point results decide output bits (the coarse-to-fine
model, the trimmed means, the overlay line positions) are compiled with the
floating-point flags of the reference's shipped build (-O3 -msse2
-ffast-math); everything else with strict IEEE arithmetic.

    python vid.stab_b200/build.py [--verbose] [--ptxas-v]
"""
import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libvidstab_b200.so")
INCLUDE = os.path.join(REPO, "include")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
CC = shutil.which("gcc", path="/usr/bin:/bin") or "gcc"

STRICT_C = ["vs_runtime.c", "vs_frameinfo.c", "vs_vector.c", "vs_serialize.c",
            "vs_motiondetect.c", "vs_ext.c", "vs_batch.c", "vs_pnet.c", "vs_l2t.c"]
REFFP_C = ["vs_transform.c", "vs_motionmodel.c", "vs_draw.c"]
CU = ["vsb_device.cu", "vsb_noalloc.cu", "vsb_batch.cu", "vsb_pnet.cu", "vsb_l2t.cu"]
# the second pass follows the reference's rounding step by step: no fused
# multiply-adds there
CU_EXTRA = {"vsb_l2t.cu": ["--fmad=false"]}

COMMON_C = ["-std=gnu99", "-O3", "-DNDEBUG", "-fPIC", "-Wall", "-fvisibility=hidden",
            "-I" + INCLUDE, "-I" + CSRC, "-I" + os.path.join(CUDA_HOME, "include")]
REFFP_FLAGS = ["-msse2", "-ffast-math"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC,-fvisibility=hidden", "-I" + INCLUDE, "-I" + CSRC]


def run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise SystemExit("build failed: " + " ".join(cmd[:3]) + " ...")
    out = (r.stdout + r.stderr).strip()
    if out and verbose:
        print(out)
    return out


def newer(src_list, target):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in src_list)


def headers():
    hs = [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    hs += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    return hs


def build(verbose=False, ptxas_v=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdrs = headers()
    objs = []
    for f in STRICT_C + REFFP_C:
        src = os.path.join(CSRC, f)
        if not os.path.exists(src):
            continue
        obj = os.path.join(BUILD, f[:-2] + ".o")
        objs.append(obj)
        if force or newer([src] + hdrs, obj):
            flags = COMMON_C + (REFFP_FLAGS if f in REFFP_C else [])
            run([CC] + flags + ["-c", src, "-o", obj], verbose)
    jobs = []
    for f in CU:
        src = os.path.join(CSRC, f)
        if not os.path.exists(src):
            continue
        obj = os.path.join(BUILD, f[:-3] + ".cu.o")
        objs.append(obj)
        if force or ptxas_v or newer([src] + hdrs, obj):
            extra = ["-Xptxas", "-v"] if ptxas_v else []
            jobs.append([NVCC] + NVCC_FLAGS + CU_EXTRA.get(f, []) + extra + ["-c", src, "-o", obj])
    # the CUDA translation units compile independently: one nvcc each, in parallel
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for out in ex.map(lambda cmd: run(cmd, verbose), jobs):
            if ptxas_v and out:
                print(out)
    if force or newer(objs, LIB):
        run([NVCC, "-shared", "-cudart", "static", "-gencode", "arch=compute_100a,code=sm_100a",
             "-o", LIB, "-Xlinker", "--no-undefined"] + objs + ["-lpthread", "-lm", "-ldl", "-lrt"], verbose)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose, a.ptxas_v, a.force))
