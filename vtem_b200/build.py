"""Build of the vtem_b200 CUDA library (``vtem_b200/_lib/libvtem_b200.so``).

Every ``csrc/*.cu`` is compiled by nvcc for sm_100a only and linked into one
shared library with a plain C ABI (``include/vtem_b200.h``).  The IAF scan
is compiled with ``--fmad=false`` so that its float64 arithmetic rounds
operation by operation, like the reference kernel run without contraction.

Usage: ``python -m vtem_b200.build [--force]``
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_lib", "obj")
LIB = os.path.join(HERE, "_lib", "libvtem_b200.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-O3",
          "-I", os.path.join(ROOT, "include"), "-I", CSRC]
# per-file extra flags
EXTRA = {
    "iaf.cu": ["--fmad=false"],
}
CUTLASS_INC = None


def _cutlass_include():
    """CuTe/CUTLASS header tree vendored with flashinfer (headers only)."""
    global CUTLASS_INC
    if CUTLASS_INC is None:
        try:
            import flashinfer  # noqa: F401
            base = os.path.dirname(flashinfer.__file__)
        except Exception:
            base = None
        cand = [os.path.join(base, "data", "cutlass", "include")] if base else []
        CUTLASS_INC = next((c for c in cand if os.path.isdir(os.path.join(c, "cute"))), "")
    return CUTLASS_INC


def _deps(src):
    """Headers a translation unit depends on (local includes, one level)."""
    deps = [src, os.path.join(ROOT, "include", "vtem_b200.h")]
    for h in os.listdir(CSRC):
        if h.endswith(".cuh"):
            deps.append(os.path.join(CSRC, h))
    return deps


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src, force):
    name = os.path.basename(src)
    obj = os.path.join(OBJ, name.replace(".cu", ".o"))
    if not force and not _stale(obj, _deps(src)):
        return obj, None
    cmd = [NVCC] + ARCH + COMMON + EXTRA.get(name, []) + ["-c", src, "-o", obj]
    cut = _cutlass_include()
    if cut:
        cmd[1:1] = ["-I", cut]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed on %s:\n%s\n%s" % (name, " ".join(cmd), r.stderr))
    return obj, r.stderr


def build(force=False, verbose=False):
    """Compile and link; returns the library path."""
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(s, force), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for _, err in results:
            if err:
                print(err)
    if force or _stale(LIB, objs):
        libdir = os.path.join(CUDA, "lib64")
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + [
            "-L", libdir, "-lcusolver", "-lcudart", "-Xlinker", "-rpath=" + libdir]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.force, a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
