"""Build libsalvus_b200.so in-tree with nvcc for sm_100a.

    python -m salvus_b200.build        (or salvus_b200.build.build())

The shared object is written next to this file so that it travels with the
source tree; nothing is installed into site-packages.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libsalvus_b200.so")

SOURCES = ["abi.cu", "noalloc.cu", "server.cpp", "host_geometry.cpp", "host_mesh.cpp",
           "host_simplex.cpp", "host_coupling.cpp",
           "host_exodus.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
         "-Xptxas", "-O3", "-ccbin", "/usr/bin/g++"]


def _stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    for root, _, files in os.walk(CSRC):
        for f in files:
            if os.path.getmtime(os.path.join(root, f)) > t:
                return True
    hdr = os.path.join(HERE, "..", "include", "salvus_b200.h")
    return os.path.getmtime(hdr) > t


def build(force=False, verbose=True, extra=()):
    if not force and not _stale():
        return OUT
    srcs = [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    objs = []
    procs = []
    os.makedirs(os.path.join(HERE, "_build"), exist_ok=True)
    for s in srcs:
        o = os.path.join(HERE, "_build", os.path.basename(s) + ".o")
        cmd = ["nvcc", "-c", s, "-o", o] + ARCH + FLAGS + list(extra)
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((subprocess.Popen(cmd), s))
        objs.append(o)
    for pr, s in procs:
        if pr.wait() != 0:
            raise RuntimeError(f"nvcc failed on {s}")
    link = ["nvcc", "-shared", "-o", OUT] + objs + ARCH + ["-ccbin", "/usr/bin/g++", "-lcudart"]
    if verbose:
        print(" ".join(link), flush=True)
    subprocess.check_call(link)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, extra=[a for a in sys.argv[1:] if a != "--force"])
