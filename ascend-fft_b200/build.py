"""Build libbfly_b200.so in-tree for sm_100a.

CUDA translation units are compiled by nvcc with `-gencode arch=compute_100a,code=sm_100a`,
host units by g++, and everything is linked into bfly/_lib/libbfly_b200.so next to the Python
package (the CUDA runtime is linked statically).  Objects go to _build/; a unit is rebuilt only
when it or a header is newer than its object.

    python ascend-fft_b200/build.py [--force] [--jobs N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIBDIR = PKG / "bfly" / "_lib"
LIB = LIBDIR / "libbfly_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCLUDES = ["-I", str(ROOT / "include"), "-I", str(CSRC)]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found (CUDA 12.9 toolkit required)")


def sources():
    cu = sorted(CSRC.glob("*.cu"))
    cpp = sorted(CSRC.glob("*.cpp"))
    return cu, cpp


def headers():
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + \
        list((ROOT / "include").rglob("*.h*"))


def stale(src: Path, obj: Path, deps) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(h.stat().st_mtime > t for h in deps)


def compile_one(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stderr


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    LIBDIR.mkdir(parents=True, exist_ok=True)
    cu, cpp = sources()
    deps = headers()
    cmds, objs = [], []
    for src in cu:
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if force or stale(src, obj, deps):
            cmds.append([nvcc(), "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC",
                         "-Xptxas", "-v" if verbose else "-O3", *INCLUDES, "-c", str(src), "-o", str(obj)])
    for src in cpp:
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if force or stale(src, obj, deps):
            cmds.append(["g++", "-std=c++17", "-O2", "-fPIC", "-Wall", "-Wextra", *INCLUDES,
                         "-c", str(src), "-o", str(obj)])
    if cmds:
        with cf.ThreadPoolExecutor(max_workers=jobs or min(len(cmds), os.cpu_count() or 4)) as ex:
            for out in ex.map(compile_one, cmds):
                if verbose and out:
                    print(out, file=sys.stderr)
    if cmds or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        compile_one([nvcc(), "-shared", *ARCH, "-cudart", "static", "-o", str(tmp),
                     *[str(o) for o in objs], "-lpthread", "-ldl", "-lrt"])
        os.replace(tmp, LIB)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.force, a.jobs, a.verbose))


if __name__ == "__main__":
    main()
