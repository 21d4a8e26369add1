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


UNITS = ["wah_api", "wah_index", "wah_build", "wah_server", "wah_noalloc", "wah_idxfile"]


def build_lib(force: bool = False, verbose: bool = False) -> str:
    """Compiles the translation units in parallel (one nvcc each, objects
    under _build/) and links them into libwahgpu.so."""
    from concurrent.futures import ThreadPoolExecutor
    out = os.path.join(HERE, "libwahgpu.so")
    deps = _sources() + [os.path.join(ROOT, "include", "wahgpu.h")]
    if not force and not _stale(out, deps):
        return out
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    flags = ["-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC,-O3",
             "-I" + os.path.join(ROOT, "include")]
    cmds = [[NVCC, *flags, "-c", "-o", os.path.join(objdir, u + ".o"), os.path.join(HERE, "csrc", u + ".cu")]
            for u in UNITS]
    if verbose:
        for c in cmds:
            print(" ".join(c))
    with ThreadPoolExecutor(len(cmds)) as ex:
        for r in list(ex.map(lambda c: subprocess.run(c), cmds)):
            if r.returncode:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    link = [NVCC, *ARCH, "-shared", "-o", out, *[os.path.join(objdir, u + ".o") for u in UNITS]]
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True)
    return out


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    print(build_lib(force="--force" in argv, verbose=True))


if __name__ == "__main__":
    main()
