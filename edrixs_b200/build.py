"""Build libedx.so (all CUDA kernels + the C ABI) in-tree for sm_100a with nvcc.

The shared library is written next to this file so that it travels with the source tree;
``edrixs_b200._lib`` loads it from there and raises if it is missing.
"""
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libedx.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + [os.path.join(ROOT, "include", "edx.h")]
    return all(os.path.getmtime(d) <= t for d in deps)


def build(force=False, verbose=False, extra=()):
    """Compile every .cu to an object in parallel (one nvcc per source), then link."""
    if not force and up_to_date():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    host_cc = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    flags = [nvcc(), "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-ccbin", host_cc, *ARCH,
             "-I", os.path.join(ROOT, "include"), *extra]
    jobs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        jobs.append((src, obj, flags + ["-c", src, "-o", obj]))

    def run(job):
        src, obj, cmd = job
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, r

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        results = list(ex.map(run, jobs))
    for src, r in results:
        if verbose or r.returncode != 0:
            sys.stdout.write(r.stdout)
            sys.stderr.write(r.stderr)
        if r.returncode != 0:
            raise subprocess.CalledProcessError(r.returncode, f"nvcc {os.path.basename(src)}")
    link = [nvcc(), "-shared", "-ccbin", host_cc, *ARCH, "-cudart", "static", "-o", LIB + ".tmp",
            *[obj for _, obj, _ in jobs]]
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])
