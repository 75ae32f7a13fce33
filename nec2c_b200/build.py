"""Build recipe for libnec2c_cuda.so (in-tree, sm_100a only).

CUDA sources under csrc/ are compiled with nvcc for sm_100a, the C host layer
under host/ with gcc (-std=gnu11, like the reference), and both are linked
into nec2c_b200/lib/libnec2c_cuda.so with the CUDA runtime linked statically.
Incremental: an object is rebuilt only when its source or a header is newer.
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
OBJ = os.path.join(HERE, "lib", "obj")
LIB = os.path.join(HERE, "lib", "libnec2c_cuda.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(ROOT, "include", "nec2c_cuda.h"))
    return hs


def _stale(src, obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in [src] + deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r.stdout + r.stderr


def build(verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    deps = _headers()
    jobs = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith(".cu"):
            src, obj = os.path.join(CSRC, f), os.path.join(OBJ, f[:-3] + ".o")
            cmd = [NVCC] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                                   "-I" + CSRC, "-I" + os.path.join(ROOT, "include")]
            cmd += ["-c", src, "-o", obj]
            jobs.append((src, obj, cmd))
    for f in sorted(os.listdir(HOST)):
        if f.endswith(".c"):
            src, obj = os.path.join(HOST, f), os.path.join(OBJ, "host_" + f[:-2] + ".o")
            cmd = ["gcc", "-O2", "-std=gnu11", "-fPIC", "-pthread", "-Wall", "-Wno-unused-function",
                   "-I" + os.path.join(ROOT, "include"), "-c", src, "-o", obj]
            jobs.append((src, obj, cmd))
    todo = [j for j in jobs if _stale(j[0], j[1], deps)]
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for out in ex.map(lambda j: _run(j[2]), todo):
            if verbose and out.strip():
                print(out)
    objs = [j[1] for j in jobs]
    if todo or not os.path.exists(LIB):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs + ["-lm", "-lpthread"])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
