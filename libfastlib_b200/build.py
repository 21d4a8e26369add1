"""Builds libwahgpu.so in-tree for sm_100a (and nothing else).

    python -m libfastlib_b200.build

nvcc cross-compiles without a GPU present.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "nvcc")


def _sources():
    d = os.path.join(HERE, "csrc")
    return [os.path.join(d, f) for f in sorted(os.listdir(d))]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(p) > t for p in deps)


def build_lib(force: bool = False, verbose: bool = False) -> str:
    out = os.path.join(HERE, "libwahgpu.so")
    deps = _sources() + [os.path.join(ROOT, "include", "wahgpu.h")]
    if not force and not _stale(out, deps):
        return out
    cmd = [NVCC, "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC,-O3",
           "-shared", "-I" + os.path.join(ROOT, "include"),
           "-o", out, os.path.join(HERE, "csrc", "wah_api.cu"),
           os.path.join(HERE, "csrc", "wah_index.cu"), os.path.join(HERE, "csrc", "wah_build.cu"),
           os.path.join(HERE, "csrc", "wah_server.cu"),
           os.path.join(HERE, "csrc", "wah_noalloc.cu"), os.path.join(HERE, "csrc", "wah_idxfile.cu")]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return out


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    print(build_lib(force="--force" in argv, verbose=True))


if __name__ == "__main__":
    main()
