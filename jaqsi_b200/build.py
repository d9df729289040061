"""Build libjqsim.so in-tree with nvcc for sm_100a.

The library is the only native artefact of the package: the host planner
(csrc/planner.cpp) and the kernels plus C ABI (csrc/jqsim.cu).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libjqsim.so")
SOURCES = ["planner.cpp", "jit.cpp", "jqsim.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    path = os.path.join(cuda, "bin", "nvcc")
    return path if os.path.exists(path) else "nvcc"


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "jqsim.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the library if a source is newer than it; return its path."""
    if not force and not needs_build():
        return LIB
    cmd = [
        _nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared",
        "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
        "--expt-relaxed-constexpr", "-I", os.path.join(HERE, "..", "include"),
        *[os.path.join(CSRC, s) for s in SOURCES],
        "-o", LIB + ".tmp", "-lcudart", "-ldl", "-lpthread",
    ]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
