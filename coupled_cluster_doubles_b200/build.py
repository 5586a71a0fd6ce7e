"""In-tree build of the package's native libraries.

libccdgpu.so   CUDA kernels + C ABI (include/ccdgpu.h), nvcc for sm_100a only.
libccdhost.so  host problem builder (include/ccdhost.h), g++.

Both land next to this file so that they travel with the source tree.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(REPO, "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
GXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _newer(target, sources):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources)


def _sources(d, exts):
    out = []
    for root, _, files in os.walk(d):
        out += [os.path.join(root, f) for f in files if f.endswith(exts)]
    return out


def build_host(force=False):
    """Links against libccdgpu.so (device channel construction), found next to it at run time."""
    out = os.path.join(HERE, "libccdhost.so")
    src = os.path.join(CSRC, "host", "ccd_system.cpp")
    gpu = os.path.join(HERE, "libccdgpu.so")
    deps = [src, gpu, os.path.join(CSRC, "host", "channel_order.h"),
            os.path.join(INC, "ccdhost.h"), os.path.join(INC, "ccdgpu.h")]
    if not force and _newer(out, deps):
        return out
    subprocess.run([GXX, "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-Wall",
                    "-I" + INC, "-I" + os.path.join(CSRC, "host"), src, "-o", out,
                    "-L" + HERE, "-lccdgpu", "-Wl,-rpath,$ORIGIN"], check=True)
    return out


def build_gpu(force=False, verbose=False):
    out = os.path.join(HERE, "libccdgpu.so")
    srcs = [os.path.join(CSRC, "ccdgpu.cu"), os.path.join(CSRC, "ccd_noalloc.cu")]
    deps = _sources(CSRC, (".cu", ".cuh")) + [os.path.join(INC, "ccdgpu.h"),
                                              os.path.join(CSRC, "host", "channel_order.h")]
    if not force and _newer(out, deps):
        return out
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "--shared", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fopenmp", "-I" + INC, "-I" + CSRC, *srcs, "-o", out, "-lgomp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    # Point nvcc at the system compiler (the image's default CXX lacks libgomp).
    env = dict(os.environ)
    env.pop("CXX", None)
    env.pop("CC", None)
    if os.path.exists("/usr/bin/g++"):
        cmd += ["-ccbin", "/usr/bin/g++"]
    subprocess.run(cmd, check=True, env=env)
    return out


def build_all(force=False):
    gpu = build_gpu(force)
    return build_host(force), gpu


if __name__ == "__main__":
    import sys
    print(build_gpu(force=True, verbose="-v" in sys.argv))
    print(build_host(force=True))
