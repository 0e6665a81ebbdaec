"""Builds libcbmv.so (the CUDA kernels and C ABI) in-tree for sm_100a.

    python -m cbmv_b200.build        # or __graft_entry__.build()

Each csrc/*.cu is compiled with nvcc -gencode arch=compute_100a,code=sm_100a
into csrc/_build/, then linked into cbmv_b200/libcbmv.so next to this file.
Objects are rebuilt when their source or any csrc header is newer.
"""
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libcbmv.so")
BUILD = os.path.join(CSRC, "_build")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# hidden visibility: only the C ABI of include/cbmv.h (default visibility
# there) is exported, no C++ internals or kernel stubs
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(os.path.dirname(HERE), "include", "cbmv.h")]


def _compile(src, newest_header, flags_changed):
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    if not flags_changed and os.path.exists(obj) and \
            os.path.getmtime(obj) >= max(os.path.getmtime(src), newest_header):
        return obj, ""
    cmd = [NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed on %s:\n%s%s" % (src, r.stdout, r.stderr))
    return obj, (r.stdout + r.stderr).strip()


def build(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    newest = max(os.path.getmtime(h) for h in _headers())
    # objects compiled with other flags are stale too
    stamp = os.path.join(BUILD, "flags.txt")
    flags = " ".join([NVCC] + ARCH + FLAGS)
    changed = not os.path.exists(stamp) or open(stamp).read() != flags
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, newest, changed), srcs))
    with open(stamp, "w") as f:
        f.write(flags)
    objs = [o for o, _ in results]
    for o, msg in results:
        if msg and verbose:
            print(msg, file=sys.stderr)
    if changed or not os.path.exists(OUT) or os.path.getmtime(OUT) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    return OUT


if __name__ == "__main__":
    print(build(verbose=True))
