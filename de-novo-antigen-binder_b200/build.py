"""Build libbinder_b200.so (the sm_100a kernels + C ABI) in-tree.

    python de-novo-antigen-binder_b200/build.py [--force] [--verbose]

Each csrc/*.cu (and the host-only csrc/*.cpp) is compiled by nvcc for sm_100a
into _build/*.o (in parallel, skipped when up to date) and linked with a static CUDA runtime into
de-novo-antigen-binder_b200/libbinder_b200.so.
"""
import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libbinder_b200.so"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
                     "-I", str(INCLUDE), "-I", str(CSRC)]


def nvcc():
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _deps():
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.inc")) + \
        sorted(INCLUDE.glob("*.h"))


def _stale(target, sources):
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def build(force=False, verbose=False, extra_flags=()):
    BUILD.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    deps = _deps()
    jobs = []
    for src in sources:
        obj = BUILD / (src.stem + ".o")
        if force or _stale(obj, [src] + deps):
            jobs.append((src, obj))

    def compile_one(job):
        src, obj = job
        cmd = [nvcc()] + NVCC_FLAGS + list(extra_flags) + ["-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, r

    failed = []
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for src, r in ex.map(compile_one, jobs):
            if r.returncode != 0:
                failed.append((src, r.stdout + r.stderr))
            elif verbose and (r.stdout or r.stderr):
                print(r.stdout + r.stderr)
    if failed:
        for src, log in failed:
            sys.stderr.write(f"--- nvcc failed on {src.name} ---\n{log}\n")
        raise RuntimeError("nvcc build failed")
    objs = [BUILD / (s.stem + ".o") for s in sources]
    if force or jobs or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-Xlinker", "--no-undefined", "-o", str(LIB)] + \
            [str(o) for o in objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
