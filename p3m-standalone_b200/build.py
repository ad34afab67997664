"""Build the p3mg CUDA library in-tree for sm_100a.

    python p3m-standalone_b200/build.py [--verbose-ptxas] [--host]

Produces ``p3m-standalone_b200/libp3mg.so`` (the C ABI of include/p3mg.h)
from ``csrc/*.cu`` with explicit nvcc commands, and -- with ``--host`` --
the drop-in command-line program ``p3m-standalone_b200/p3m_gpu`` from
``host/*.c`` linked against it.  Objects go to ``_build/`` next to this file.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
           "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]
# Per-file flags.  The FP32 pair force flushes single-precision denormals:
# its reciprocals, square roots and exponentials then need no denormal
# handling, and none of its FP32 values comes near 1e-38 (distances are
# >= 1e-3 of the cell, forces and energies are O(q^2 / rcut^2) and above).
FILE_FLAGS = {"p3mg_pairs.cu": ["-ftz=true"]}


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    return r.returncode, " ".join(cmd), r.stdout


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose_ptxas=False, host=False, force=False, jobs=None):
    bdir = os.path.join(HERE, "_build")
    os.makedirs(bdir, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))
    headers = glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    objs, cmds = [], []
    for s in srcs:
        o = os.path.join(bdir, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            extra = (["-Xptxas", "-v"] if verbose_ptxas else []) + FILE_FLAGS.get(os.path.basename(s), [])
            cmds.append([NVCC] + ARCH + CUFLAGS + extra + ["-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count()) as ex:
        for rc, cmd, out in ex.map(_run, cmds):
            if out.strip() and (rc or verbose_ptxas):
                sys.stdout.write(out)
            if rc:
                raise RuntimeError("nvcc failed: " + cmd)
    lib = os.path.join(HERE, "libp3mg.so")
    if force or cmds or _stale(lib, objs):
        rc, cmd, out = _run([NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart"])
        if rc:
            sys.stdout.write(out)
            raise RuntimeError("link failed: " + cmd)
    if host:
        hsrc = sorted(glob.glob(os.path.join(HERE, "host", "*.c")))
        exe = os.path.join(HERE, "p3m_gpu")
        if hsrc and (force or _stale(exe, hsrc + [lib] + glob.glob(os.path.join(HERE, "host", "*.h")))):
            cmd = ["gcc", "-O2", "-std=c99", "-D_GNU_SOURCE", "-I" + os.path.join(ROOT, "include"), "-o", exe] + hsrc + [
                "-L" + HERE, "-lp3mg", "-Wl,-rpath,$ORIGIN", "-lm"]
            rc, cmd_s, out = _run(cmd)
            if rc:
                sys.stdout.write(out)
                raise RuntimeError("host build failed: " + cmd_s)
    return lib


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--host", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(verbose_ptxas=a.verbose_ptxas, host=a.host, force=a.force))
