"""Build libcsffci_b200.so (all CUDA sources in csrc/) in-tree for sm_100a.

    python pyscf-forge_b200/build.py [--force]

Uses nvcc directly (-gencode arch=compute_100a,code=sm_100a -lineinfo); the
CUDA runtime is linked statically, so the library only needs the driver.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
INC = os.path.abspath(os.path.join(HERE, "..", "include"))
LIB = os.path.join(HERE, "libcsffci_b200.so")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-I" + INC]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def sources():
    return sorted(glob.glob(os.path.join(SRC, "*.cu")))


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(SRC, "*.cuh")) + glob.glob(os.path.join(INC, "*.h"))
    return all(os.path.getmtime(d) <= t for d in deps)


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    nvcc = _nvcc()
    # headers are shared: an object is rebuilt when its source or any header
    # is newer than it; translation units compile in parallel
    hdr_t = max([os.path.getmtime(h) for h in glob.glob(os.path.join(SRC, "*.cuh")) +
                 glob.glob(os.path.join(INC, "*.h"))] + [0.0])
    objs, cmds = [], []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr_t):
            cmds.append([nvcc] + NVCC_FLAGS + ["-c", src, "-o", obj])
    from concurrent.futures import ThreadPoolExecutor
    workers = max(1, min(len(cmds), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=workers) as ex:
        futs = []
        for cmd in cmds:
            if verbose:
                print(" ".join(cmd))
            futs.append(ex.submit(subprocess.check_call, cmd))
        for f in futs:
            f.result()
    cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB + ".tmp"] + objs
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
