"""Build libb200dft.so (sm_100a) and the test-only host-check library in-tree.

    python pyscf-ipu_b200/csrc/build.py [--force]

Outputs (git-ignored, shipped with the tree):
    pyscf-ipu_b200/b200dft/_lib/libb200dft.so           product kernels + C ABI
    pyscf-ipu_b200/b200dft/_lib/libb200dft_hostcheck.so CPU build of the kernel math (tests)
"""
import argparse
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(os.path.dirname(HERE), "b200dft")
OUT = os.path.join(PKG, "_lib")
INC = os.path.join(os.path.dirname(os.path.dirname(HERE)), "include")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + HERE, "-I" + INC,
          "--expt-relaxed-constexpr", "-Wno-deprecated-gpu-targets"]
LIB_SRCS = ["capi.cu", "eri.cu", "jk.cu", "jk_symv.cu", "xc.cu", "scf.cu", "setup.cu", "xc_direct.cu", "xc_tc.cu", "learned.cu",
            "grad.cu", "blocks.cu"]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed: " + " ".join(cmd))
    return r


def build(force=False, verbose=False, jobs=None):
    os.makedirs(OUT, exist_ok=True)
    deps = glob.glob(os.path.join(HERE, "*.cu")) + glob.glob(os.path.join(HERE, "*.cuh")) + \
        glob.glob(os.path.join(HERE, "*.hpp")) + glob.glob(os.path.join(INC, "*.h"))
    lib = os.path.join(OUT, "libb200dft.so")
    if force or _newer(lib, deps):
        objs = []
        procs = []
        for s in LIB_SRCS:
            o = os.path.join(OUT, s.replace(".cu", ".o"))
            objs.append(o)
            cmd = [NVCC] + ARCH + COMMON + ["-dc" if False else "-c", os.path.join(HERE, s), "-o", o]
            if verbose:
                cmd += ["-Xptxas", "-v"]
            procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        for cmd, p in procs:
            out = p.communicate()[0]
            if p.returncode != 0:
                sys.stderr.write(out)
                raise RuntimeError("nvcc failed: " + " ".join(cmd))
            if verbose:
                sys.stdout.write(out)
        _run([NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart"])
        for o in objs:
            os.remove(o)
    hc = os.path.join(OUT, "libb200dft_hostcheck.so")
    if force or _newer(hc, deps):
        _run([NVCC, "-O2", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-I" + HERE,
              "-Wno-deprecated-gpu-targets", os.path.join(HERE, "hostcheck.cu"), "-o", hc])
    return lib, hc


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
