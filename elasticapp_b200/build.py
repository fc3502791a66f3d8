"""Build libelastica_b200.so (the C-ABI + sm_100a kernels) in-tree with nvcc.

Usage: ``python -m elasticapp_b200.build [--force] [--verbose-ptxas]``.
The shared library lands next to this file so it travels with the repository
snapshot; object files go to ``elasticapp_b200/_build/`` (git-ignored).
"""
from __future__ import annotations

import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libelastica_b200.so")

# (object name, source, extra nvcc flags)
SOURCES = [
    ("eb_capi.o", "eb_capi.cu", []),
    ("rod_step_fp64.o", "rod_step_fp64.cu", ["-DEB_FAST_FP64"]),
    ("rod_step_fp64_reference.o", "rod_step_fp64.cu", ["--fmad=false"]),
    ("rod_block_fp64.o", "rod_block_fp64.cu", []),
    ("rod_block_mixed.o", "rod_block_mixed.cu", []),
    ("rod_energy.o", "rod_energy.cu", []),
    # rounded as written (no contracted multiply-adds): capsules, boxes and
    # candidate pairs bit-identical to a scalar FP64 evaluation
    ("contact.o", "contact.cu", ["--fmad=false"]),
    ("box_pairs_noalloc.o", "box_pairs_noalloc.cu", []),
    # joint loads rounded as written, like the CPU restatement
    ("connection.o", "connection.cu", ["--fmad=false"]),
    ("serve.o", "serve.cu", []),
    ("partition.o", "partition.cu", []),
]
HEADERS = ["eb_internal.h", "rod_math.cuh", "bulk_copy.cuh", "contact.h", "eb_host.h", "joint.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_compiler() -> list[str]:
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def common_flags() -> list[str]:
    return ARCH + host_compiler() + [
        "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
        "-Xcompiler", "-fPIC,-fvisibility=hidden,-O2",
        "-I", os.path.join(ROOT, "include"), "-I", CSRC,
    ]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose_ptxas: bool = False, quiet: bool = True) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "elastica_b200.h")]
    objs, cmds = [], []
    for oname, src, extra in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, oname)
        objs.append(obj)
        if force or verbose_ptxas or _stale(obj, [path] + headers):
            cmd = [nvcc()] + common_flags() + extra + ["-c", path, "-o", obj]
            if verbose_ptxas:
                cmd += ["-Xptxas", "-v"]
            if not quiet:
                print(" ".join(cmd))
            cmds.append(cmd)
    # the translation units compile independently: one nvcc per core
    workers = max(1, min(len(cmds), os.cpu_count() or 1))
    with concurrent.futures.ThreadPoolExecutor(max_workers=workers) as pool:
        for done in pool.map(lambda c: subprocess.run(c, check=False), cmds):
            if done.returncode != 0:
                raise subprocess.CalledProcessError(done.returncode, done.args)
    if force or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + host_compiler() + ["-shared", "-cudart", "static", "-o", LIB] + objs
        if not quiet:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    args = ap.parse_args(argv)
    print(build(force=args.force, verbose_ptxas=args.verbose_ptxas, quiet=False))
    return 0


if __name__ == "__main__":
    sys.exit(main())
