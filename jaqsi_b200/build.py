"""Build libjqsim.so in-tree with nvcc for sm_100a.

The library is the only native artefact of the package: the host planner
(csrc/planner.cpp), the NVRTC specialiser (csrc/jit.cpp) and the kernels plus
C ABI (csrc/jqsim.cu).  Each source compiles to its own object under
jaqsi_b200/_build (in parallel); an object is rebuilt when its source, or any
header it may include, is newer than it, and the library is relinked when an
object changed.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(HERE, "..", "include")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libjqsim.so")
SOURCES = ["planner.cpp", "jit.cpp", "jqsim.cu", "pulse.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr"]


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    path = os.path.join(cuda, "bin", "nvcc")
    return path if os.path.exists(path) else "nvcc"


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(INCLUDE, "jqsim.h"))
    return [h for h in hs if os.path.exists(h)]


def _obj(src: str) -> str:
    return os.path.join(OBJDIR, src + ".o")


def _stale(src: str) -> bool:
    obj = _obj(src)
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in [os.path.join(CSRC, src)] + _headers())


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(_stale(s) for s in SOURCES) or any(os.path.getmtime(_obj(s)) > t for s in SOURCES)


def _compile(src: str, verbose: bool) -> None:
    cmd = [_nvcc(), *ARCH, *FLAGS, "-I", INCLUDE, "-c", os.path.join(CSRC, src), "-o", _obj(src) + ".tmp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(_obj(src) + ".tmp", _obj(src))


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile what changed and relink; return the library's path."""
    if not force and not needs_build():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    todo = [s for s in SOURCES if force or _stale(s)]
    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        for f in [ex.submit(_compile, s, verbose) for s in todo]:
            f.result()
    cmd = [_nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", *[_obj(s) for s in SOURCES], "-o", LIB + ".tmp",
           "-lcudart", "-ldl", "-lpthread"]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
