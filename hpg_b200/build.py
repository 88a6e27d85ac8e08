"""Build the native libraries of hpg_b200 in-tree.

    python -m hpg_b200.build          # or hpg_b200.build.build()

Products (git-ignored, shipped with the source tree):
  hpg_b200/lib/libhpgb.so   sm_100a CUDA device library (C ABI, include/hpgb.h)
  hpg_b200/lib/libhpg.so    C++ hpg:: API over the C ABI (hpg_b200/cpp)
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "hpg_b200")
CSRC = os.path.join(PKG, "csrc")
CPP = os.path.join(PKG, "cpp")
LIB = os.path.join(PKG, "lib")
OBJ = os.path.join(PKG, "_build")
INCLUDE = os.path.join(ROOT, "include")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-I" + INCLUDE, "-I" + CSRC,
]


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT,
                       text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed:\n" + " ".join(cmd) + "\n" + r.stdout)
    return r.stdout


def _newer(target, sources):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources)


def _headers(d, exts):
    out = []
    for name in sorted(os.listdir(d)):
        if name.endswith(exts):
            out.append(os.path.join(d, name))
    return out


def build_device(verbose=False, force=False):
    """Compile hpg_b200/csrc/*.cu for sm_100a and link libhpgb.so."""
    os.makedirs(LIB, exist_ok=True)
    os.makedirs(OBJ, exist_ok=True)
    sources = _headers(CSRC, (".cu",))
    headers = _headers(CSRC, (".cuh", ".h")) + [os.path.join(INCLUDE, "hpgb.h")]
    target = os.path.join(LIB, "libhpgb.so")
    if not force and _newer(target, sources + headers):
        return target

    def compile_one(src):
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        if force or not _newer(obj, [src] + headers):
            out = _run([NVCC] + NVCC_FLAGS + ["-Xptxas", "-v", "-c", src, "-o", obj]
                       if verbose else [NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj])
            if verbose:
                print(out)
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, sources))
    tmp = target + ".tmp"
    # --no-undefined: a declaration without a definition fails the build
    # here instead of the library's load on the device
    _run([NVCC] + ARCH + ["-shared", "-o", tmp] + objs +
         ["-L" + os.path.join(CUDA_HOME, "lib64"), "-lcufft",
          "-Xlinker", "--no-undefined",
          "-Xlinker", "-rpath=" + os.path.join(CUDA_HOME, "lib64")])
    os.replace(tmp, target)
    return target


def build_cpp(verbose=False, force=False):
    """Compile the C++ hpg:: API (hpg_b200/cpp) into libhpg.so."""
    src_dir = os.path.join(CPP, "src")
    inc_dir = os.path.join(CPP, "include")
    if not os.path.isdir(src_dir):
        return None
    sources = _headers(src_dir, (".cc",))
    headers = []
    for d, _, files in os.walk(inc_dir):
        headers += [os.path.join(d, f) for f in files]
    target = os.path.join(LIB, "libhpg.so")
    if not force and _newer(target, sources + headers + [os.path.join(LIB, "libhpgb.so")]):
        return target
    tmp = target + ".tmp"
    _run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-I" + inc_dir,
          "-I" + INCLUDE, "-o", tmp] + sources +
         ["-L" + LIB, "-lhpgb", "-Wl,-rpath,$ORIGIN"])
    os.replace(tmp, target)
    return target


def build(verbose=False, force=False):
    dev = build_device(verbose=verbose, force=force)
    cpp = build_cpp(verbose=verbose, force=force)
    return dev, cpp


if __name__ == "__main__":
    force = "--force" in sys.argv
    verbose = "-v" in sys.argv
    print(build(verbose=verbose, force=force))
