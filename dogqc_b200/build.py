"""Builds ``libdogqc_b200.so`` (the CUDA engine and its C ABI) in-tree for sm_100a.

``python -m dogqc_b200.build`` or ``dogqc_b200.build.build()``; rebuilds only when a
source is newer than the library.  The compiler is nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3``; no GPU is needed.

The device headers the per-pipeline kernel generator compiles against at run
time (NVRTC, sm_100a) are embedded into the library as string literals
(``_build/dq_jit_embed.inc``), so the library needs no source tree at run time.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libdogqc_b200.so")
SOURCES = ["dq_kernels.cu", "dq_import.cu", "dq_runtime.cu", "dq_noalloc.cu", "dq_jit.cpp"]
HEADERS = ["dq_device.h", "dq_common.cuh", "dq_jit.h", os.path.join("..", "..", "include", "dogqc_b200.h")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# in-memory headers of generated kernels: (include name, file)
EMBED = [("dq_common.cuh", os.path.join(CSRC, "dq_common.cuh")),
         ("dq_device.h", os.path.join(CSRC, "dq_device.h")),
         ("../../include/dogqc_b200.h", os.path.join(ROOT, "include", "dogqc_b200.h"))]
DELIM = "DQSRC"


def _write_embed(build_dir):
    parts = []
    for name, path in EMBED:
        with open(path) as f:
            text = f.read()
        if (")%s\"" % DELIM) in text:
            raise RuntimeError("%s contains the raw-string delimiter" % path)
        parts.append((name, text))
    out = ["// written by dogqc_b200/build.py: device headers of generated kernels",
           "static const int kEmbedCount = %d;" % len(parts),
           "static const char* const kEmbedNames[] = {%s};" % ", ".join('"%s"' % n for n, _ in parts),
           "static const char* const kEmbedText[] = {"]
    for _, text in parts:
        out.append('R"%s(%s)%s",' % (DELIM, text, DELIM))
    out.append("};")
    path = os.path.join(build_dir, "dq_jit_embed.inc")
    data = "\n".join(out) + "\n"
    if not os.path.exists(path) or open(path).read() != data:
        with open(path, "w") as f:
            f.write(data)


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    raise RuntimeError("nvcc not found")


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    for f in SOURCES + HEADERS:
        if os.path.getmtime(os.path.join(CSRC, f)) > t:
            return True
    return False


def build(force=False, verbose=False):
    if not force and not _stale():
        return LIB
    objs = []
    build_dir = os.path.join(HERE, "_build")
    os.makedirs(build_dir, exist_ok=True)
    _write_embed(build_dir)
    for src in SOURCES:
        obj = os.path.join(build_dir, os.path.splitext(src)[0] + ".o")
        cmd = [_nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
               "-I", os.path.join(ROOT, "include"), "-I", build_dir, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s" % (src, r.stderr[-4000:]))
        if verbose:
            sys.stderr.write(r.stderr)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [_nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs, "-lnvrtc", "-ldl"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s" % r.stderr[-4000:])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
