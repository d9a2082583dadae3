"""Builds libstarsh_b200.so in place (stars-h_b200/libstarsh_b200.so).

Host C files are compiled with gcc, CUDA files with nvcc for sm_100a only
(`-gencode arch=compute_100a,code=sm_100a`), and everything is linked into
one shared library with a static CUDA runtime and -Bsymbolic, so that the
library's own symbols win over a STARS-H library loaded in the same
process.

    python stars-h_b200/build.py [--force]
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libstarsh_b200.so")

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]
CC_FLAGS = ["-std=gnu11", "-O2", "-fPIC", "-Wall", "-Wno-unused-function",
            "-I", INCLUDE, "-I", CSRC]


def _sources():
    c = sorted(f for f in os.listdir(CSRC) if f.endswith(".c"))
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    return c, cu


def _headers_mtime():
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC)
             if f.endswith((".h", ".cuh"))]
    paths += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return max(os.path.getmtime(p) for p in paths)


def _compile(src, force, hdr_time):
    obj = os.path.join(OBJ, src + ".o")
    path = os.path.join(CSRC, src)
    if (not force and os.path.exists(obj)
            and os.path.getmtime(obj) > max(os.path.getmtime(path), hdr_time)):
        return obj
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCC_FLAGS + ["-c", path, "-o", obj]
    else:
        cmd = ["gcc"] + CC_FLAGS + ["-c", path, "-o", obj]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    return obj


def build(force=False):
    os.makedirs(OBJ, exist_ok=True)
    c, cu = _sources()
    hdr_time = _headers_mtime()
    try:
        with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
            objs = list(ex.map(lambda s: _compile(s, force, hdr_time), c + cu))
    except RuntimeError:
        # no stale library may outlive a failed build
        if os.path.exists(LIB):
            os.remove(LIB)
        raise
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) > max(os.path.getmtime(o) for o in objs)):
        return LIB
    script = os.path.join(OBJ, "exports.map")
    with open(script, "w") as f:
        # Only the STARS-H API and the B200 entry points are exported.
        f.write("{ global: starsh_*; array_*; local: *; };\n")
    cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs + \
          ["-Xlinker", "-Bsymbolic", "-Xlinker", "--version-script=" + script,
           "-ldl", "-lpthread", "-lm"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
