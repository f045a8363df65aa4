"""Build libf2m_b200.so and F2M.solver.exe in-tree with nvcc for sm_100a."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libf2m_b200.so")
CLI = os.path.join(HERE, "bin", "F2M.solver.exe")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall"]
SOURCES = ["f2m_kernels.cu", "f2m_grid.cu", "f2m_smooth.cu", "f2m_probe.cu", "f2m_sort.cu",
           "f2m_runtime.cu"]


def _nvcc():
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    p = os.path.join(cuda, "bin", "nvcc")
    return p if os.path.exists(p) else "nvcc"


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(verbose_ptxas=False):
    from concurrent.futures import ThreadPoolExecutor
    nvcc = _nvcc()
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    cmds, objs = [], []
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        extra = ["-Xptxas", "-v"] if (verbose_ptxas and src.endswith(".cu")) else []
        lang = ["-x", "cu"] if src.endswith(".cpp") else []
        cmds.append([nvcc] + ARCH + FLAGS + extra + lang + ["-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    # the translation units are independent: compile them side by side
    with ThreadPoolExecutor(max_workers=len(cmds)) as ex:
        for f in [ex.submit(_run, c) for c in cmds]:
            f.result()
    _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs)
    _run([nvcc] + ARCH + FLAGS + ["-o", CLI, os.path.join(CSRC, "f2m_cli.cpp"), "-L" + HERE,
                                  "-lf2m_b200", "-Xlinker", "-rpath=$ORIGIN/.."])
    return LIB


if __name__ == "__main__":
    build(verbose_ptxas="-v" in sys.argv)
