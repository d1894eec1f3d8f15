"""Build recipe for ``oracle/_ref``: the reference's own CUDA kernels, compiled
for the host as the checker of the CUDA product (test infrastructure).

The reference keeps every kernel as a C source string inside a Python-2
module and compiles it at run time through PyCUDA (vtem/utils/kernel_utils.py:
136-142), templated with ``%(type)s``.  This script reads those strings where
they lie in the read-only reference tree, applies the same ``%`` templating
the reference applies, and compiles each kernel with g++ against
``ref_shim.hpp`` (a CPU execution model of CUDA threads).  All outputs go to
``oracle/_ref/`` (git-ignored, never committed).

Usage:  python oracle/build_ref.py [--reference /path/to/reference]
        (default: $VTEM_REFERENCE_ROOT, else the container's mount point)
Needs the reference tree; on a machine without it, the prebuilt
``oracle/_ref/libvtem_ref.so`` is used as is.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# where the read-only reference tree is mounted in the build container;
# VTEM_REFERENCE_ROOT or --reference override it
DEFAULT_REF = "/root/reference"


def reference_root() -> str:
    """The reference tree to read the kernel strings from."""
    return os.environ.get("VTEM_REFERENCE_ROOT", DEFAULT_REF)


class _Types(dict):
    """Template dictionary: every ``%(...)s`` key not named maps to double."""

    def __missing__(self, key):
        return "double"


# (symbol, module path, template-building function, template variable, type map)
KERNELS = [
    ("iaf_linear", "vtem/ensemble_encode.py", "get_IAF_kernel_linear", {}),
    ("iaf_linear_rt", "vtem/ensemble_encode.py", "get_IAF_kernel_linear_rt", {}),
    ("compute_q", "vtem/dirichlet.py", "get_compute_q_kernel", {}),
    ("compute_G", "vtem/dirichlet.py", "get_G_kernel", {}),
    ("diag_add", "vtem/dirichlet.py", "get_diag_add_kernel", {}),
    ("reconstruct", "vtem/dirichlet.py", "get_reconstruct_kernel", {}),
    ("put_norm", "vtem/vrf.py", "get_put_norm_kernel", {}),
    ("gabor", "vtem/vrf.py", "get_gabor_kernel", {}),
    ("cs", "vtem/vrf.py", "get_cs_kernel", {}),
    ("fft2Ds", "vtem/vrf.py", "get_fft2Ds_kernel", {"type": "pycuda::complex<double>"}),
    ("Ds2fft", "vtem/vrf.py", "get_Ds2fft_kernel", {"type": "pycuda::complex<double>"}),
    ("filter2rec", "vtem/vrf.py", "get_filter2rec_kernel",
     {"type": "pycuda::complex<double>", "typef": "double"}),
    ("rnn3_update", "vtem/neural_network.py", "get_rnn3_update_func", {}),
    ("sq", "vtem/utils/linalg.py", "_get_sq_kernel", {}),
]

_CTYPE = {"double": "d", "float": "f", "int": "i", "unsigned int": "u"}


def extract_template(src: str, func: str) -> str:
    """The first triple-quoted string in the body of ``def func(``."""
    m = re.search(r"^def %s\(" % re.escape(func), src, re.M)
    if not m:
        raise KeyError(func)
    body = src[m.end():]
    end = re.search(r"^(def |class |@)", body, re.M)
    if end:
        body = body[:end.start()]
    s = re.search(r'"""(.*?)"""', body, re.S)
    if not s:
        raise KeyError("template in " + func)
    return s.group(1)


def parse_signature(code: str):
    """(kernel name, [(c type, is_pointer)]) of the single __global__ kernel."""
    m = re.search(r"__global__\s+void\s+(\w+)\s*\((.*?)\)\s*\{", code, re.S)
    name, params = m.group(1), m.group(2)
    args = []
    for p in params.split(","):
        p = " ".join(p.split())
        ptr = "*" in p
        base = p.replace("*", " ").split()
        ctype = " ".join(base[:-1])
        args.append((ctype, ptr))
    return name, args


def generate(ref_root: str):
    os.makedirs(OUT, exist_ok=True)
    manifest = {}
    sources = []
    for sym, path, func, types in KERNELS:
        with open(os.path.join(ref_root, path)) as f:
            src = f.read()
        code = extract_template(src, func) % _Types(types)
        # the shim header supplies pycuda::complex; drop the PyCUDA include
        code = code.replace("#include <pycuda/pycuda-complex.hpp>", "")
        kname, args = parse_signature(code)
        unpack = []
        for i, (ct, ptr) in enumerate(args):
            t = ct + ("*" if ptr else "")
            unpack.append("*(%s*)args[%d]" % (t, i))
        cpp = os.path.join(OUT, "k_%s.cpp" % sym)
        with open(cpp, "w") as f:
            f.write('#include "ref_shim.hpp"\n')
            f.write("// generated from %s:%s by oracle/build_ref.py\n" % (path, func))
            f.write("namespace ns_%s {\n%s\n}\n" % (sym, code))
            f.write('extern "C" void ref_launch_%s(unsigned gx, unsigned gy, unsigned bx, '
                    'unsigned by, void** args, int os_threads) {\n' % sym)
            f.write("  vt_launch({gx, gy, 1}, {bx, by, 1}, [&]() { ns_%s::%s(%s); }, os_threads);\n}\n"
                    % (sym, kname, ", ".join(unpack)))
        sources.append(cpp)
        manifest[sym] = {"kernel": kname, "source": "%s:%s" % (path, func),
                         "args": [("p" if p else _CTYPE.get(c, "?")) + ":" + c for c, p in args]}
    with open(os.path.join(OUT, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1)
    return sources


def compile_all(sources):
    lib = os.path.join(OUT, "libvtem_ref.so")
    cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fPIC",
           "-shared", "-w", "-I", HERE, "-o", lib, os.path.join(HERE, "ref_shim.cpp")]
    cmd += sources + ["-lpthread"]
    subprocess.check_call(cmd)
    return lib


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=reference_root())
    a = ap.parse_args(argv)
    if not os.path.isdir(os.path.join(a.reference, "vtem")):
        print("reference tree not found at %s; keeping prebuilt oracle/_ref" % a.reference)
        return 0
    lib = compile_all(generate(a.reference))
    print(lib)
    return 0


if __name__ == "__main__":
    sys.exit(main())
