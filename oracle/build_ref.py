"""Build the reference's own FP64 ERI code into ``oracle/_ref/libref_int2e.so``.

Test infrastructure only: the library built here is a checker for the ERI
oracle and the CUDA ERI kernel, never part of the product path.

The reference ships ``pyscf_ipu/electron_repulsion/cpu_int2e_sph.cpp``, an FP64
host build of its libcint port (``#define dtype double``, cpu_int2e_sph.cpp:16-18),
normally compiled with the Graphcore Poplar SDK (direct.sh:4).  Poplar is not
available here, so this script copies the source into a temporary directory,
drops the unconditional Poplar includes / ``using namespace`` lines
(cpu_int2e_sph.cpp:8-14) and every ``#ifdef __cplusplus`` block that drives a
Poplar device (the IPU self-test harnesses, e.g. cpu_int2e_sph.cpp:531-598,
7881-7923), and compiles the rest with g++.  Nothing from the reference is
copied into this repository; the source is read where it lies.

Usage: python oracle/build_ref.py [--src REFERENCE_ROOT]
"""
import argparse
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
OUT_LIB = os.path.join(OUT_DIR, "libref_int2e.so")
REL = os.path.join("pyscf_ipu", "electron_repulsion", "cpu_int2e_sph.cpp")
POPLAR_WORDS = ("poplar", "Device", "Engine", "Graph", "engine.", "graph.", "program::")


def strip_poplar(text):
    lines = text.split("\n")
    out = []
    i = 0
    while i < len(lines):
        ln = lines[i]
        s = ln.strip()
        if s.startswith("#include <poplar") or s.startswith("using namespace poplar"):
            i += 1
            continue
        if s.startswith("#ifdef __cplusplus"):
            depth, j = 1, i + 1
            while j < len(lines) and depth:
                t = lines[j].strip()
                if t.startswith("#if"):
                    depth += 1
                elif t.startswith("#endif"):
                    depth -= 1
                j += 1
            block = "\n".join(lines[i:j])
            if any(w in block for w in POPLAR_WORDS):
                i = j
                continue
        out.append(ln)
        i += 1
    head = "#include <cassert>\n#include <vector>\n#include <algorithm>\n#include <iostream>\n"
    return head + "\n".join(out)


def build(src_root, quiet=False):
    src = os.path.join(src_root, REL)
    if not os.path.exists(src):
        raise FileNotFoundError(src)
    os.makedirs(OUT_DIR, exist_ok=True)
    with open(src) as f:
        text = strip_poplar(f.read())
    tmp = tempfile.mkdtemp(prefix="ref_int2e_")
    try:
        cpp = os.path.join(tmp, "cpu_int2e_sph_stripped.cpp")
        with open(cpp, "w") as f:
            f.write(text)
        cmd = ["g++", "-O2", "-shared", "-fPIC", "-fpermissive", "-w", cpp, "-o", OUT_LIB, "-lquadmath"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("reference ERI build failed:\n" + r.stderr[-4000:])
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    if not quiet:
        print("built", OUT_LIB)
    return OUT_LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=os.environ.get("PYSCF_IPU_REFERENCE", "/root/reference"))
    a = ap.parse_args()
    build(a.src)
