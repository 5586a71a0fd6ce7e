"""Builds the oracle (test infrastructure only).

build_oracle()  compiles oracle/ccd_oracle.c into oracle/libccdoracle.so (always possible).
build_ref()     compiles the unmodified reference sources into oracle/_ref/ (ccd.exe and the
                golden-vector harness) with oracle/ref/Makefile, only where the reference
                tree is present; elsewhere the prebuilt files are used as they are.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
# The reference sources; CCD_REF_SRC overrides the default location.
REF_SRC = os.environ.get("CCD_REF_SRC", "/root/reference/src")
GXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
GCC = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"


def _newer(target, sources):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources)


def build_oracle(force=False):
    out = os.path.join(HERE, "libccdoracle.so")
    src = os.path.join(HERE, "ccd_oracle.c")
    hdr = os.path.join(REPO, "include", "ccdgpu.h")
    if not force and _newer(out, [src, hdr]):
        return out
    cmd = [GCC, "-O3", "-std=c11", "-fopenmp", "-fPIC", "-shared", "-Wall",
           "-I" + os.path.join(REPO, "include"), src, "-o", out, "-lm"]
    subprocess.run(cmd, check=True)
    return out


def build_ref():
    """Returns the directory of the reference build, or None if neither the sources nor a
    previous build are available."""
    out = os.path.join(HERE, "_ref")
    if os.path.isdir(REF_SRC):
        subprocess.run(["make", "-s", "-C", os.path.join(HERE, "ref"), "-j8", "REF_SRC=" + REF_SRC],
                       check=True)
    if os.path.exists(os.path.join(out, "ccd.exe")):
        return out
    return None


if __name__ == "__main__":
    print(build_oracle(force=True))
    print(build_ref())
