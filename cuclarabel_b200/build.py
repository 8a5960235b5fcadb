"""Builds libclgpu.so (the sm_100a CUDA library) in place.

    python -m cuclarabel_b200.build

nvcc cross-compiles for sm_100a without a GPU.  Objects are cached under
cuclarabel_b200/_build and relinked when a source or header changes.
"""
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libclgpu.so")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC",
          "-I" + os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers():
    return (glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp"))
            + glob.glob(os.path.join(ROOT, "include", "*.h")))


def build_pack(verbose=False):
    """The CPython extension that packs a batch's problem structs
    (csrc/pack.c), compiled in place with the host compiler."""
    import sysconfig
    src = os.path.join(CSRC, "pack.c")
    out = os.path.join(HERE, "_pack" + sysconfig.get_config_var("EXT_SUFFIX"))
    deps = [src, os.path.join(ROOT, "include", "clgpu.h")]
    if os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(d) for d in deps):
        return out
    cc = os.environ.get("CC", shutil.which("gcc") or "cc")
    cmd = [cc, "-O2", "-shared", "-fPIC", "-I" + sysconfig.get_paths()["include"],
           "-I" + os.path.join(ROOT, "include"), src, "-o", out]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    return out


def build(verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    hdr_mtime = max([os.path.getmtime(h) for h in _headers()] + [0])
    objs = []
    for src in _sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if (os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
                and os.path.getmtime(obj) >= hdr_mtime and not ptxas_info):
            continue
        cmd = [NVCC] + ARCH + COMMON + ["-c", src, "-o", obj]
        if src.endswith(".cu") and ptxas_info:
            cmd += ["-Xptxas", "-v"]
        if verbose or ptxas_info:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    try:
        build_pack(verbose)
    except (OSError, subprocess.CalledProcessError) as e:  # no host compiler or headers:
        print("packer not built (%s); batches pack in Python" % e, file=sys.stderr)
    need_link = (not os.path.exists(LIB)
                 or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs))
    if need_link:
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
    print("built", LIB)
