"""Build libcfem.so (sm_100a) in-tree with nvcc.

Usage: python -m cloudfem_b200.csrc.build [--force]

The library is a plain shared object with a C ABI (include/cfem.h); the
CUDA runtime is linked statically so the .so only needs the driver.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
INCLUDE = os.path.join(ROOT, "include")
OUT = os.path.join(os.path.dirname(HERE), "libcfem.so")
SOURCES = ["cfem_core.cu", "cfem_pattern.cu", "cfem_assemble.cu",
           "cfem_dirichlet.cu", "cfem_solve.cu", "cfem_complex.cu", "cfem_em.cu",
           "cfem_faces.cu"]
HEADERS = ["cfem_common.cuh", "cfem_tables.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(HERE, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(INCLUDE, "cfem.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    """Compile every .cu to an object, then link libcfem.so."""
    if not force and not _stale():
        return OUT
    nvcc = _nvcc()
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        cmd = [nvcc, *ARCH, *FLAGS, "-I", INCLUDE, "-I", HERE,
               "-DCFEM_BUILD", "-c", os.path.join(HERE, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                            stderr=subprocess.STDOUT,
                                            text=True)))
        objs.append(obj)
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stderr.write(out)
        if p.returncode != 0:
            failed.append(src)
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    tmp = OUT + ".tmp"
    link = [nvcc, *ARCH, "-shared", "-o", tmp, *objs, "-cudart", "static",
            "-Xcompiler", "-fPIC"]
    subprocess.run(link, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
