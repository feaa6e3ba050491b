"""Build recipe of the CUDA library (cupf_b200/libcupf.so, sm_100a) and the
phase_field command-line driver (cupf_b200/phase_field).

    python cupf_b200/build.py [--force] [--verbose]

Built in-tree so the binaries travel with the repository; nvcc cross-compiles
on a machine without a GPU.  Objects go to cupf_b200/_build/.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
OUT = os.path.join(HERE, "libcupf.so")
EXE = os.path.join(HERE, "phase_field")
EXE2D = os.path.join(HERE, "phase_field_2d")
OBJ = os.path.join(HERE, "_build")
CU_SOURCES = [os.path.join(HERE, "csrc", f)
              for f in ("cupf_capi.cu", "cupf_server.cu", "cupf_noalloc.cu", "cupf_ek2d.cu",
                        "cupf_dense.cu")]
CPP_SOURCES = [os.path.join(HERE, "host", f) for f in
               ("host_util.cpp", "qoi.cpp", "phase_field.cpp", "npz_writer.cpp", "h5_writer.cpp",
                "host_capi.cpp", "ek2d_host.cpp", "substrate.cpp")]
MAIN = os.path.join(HERE, "host", "main.cpp")
MAIN2D = os.path.join(HERE, "host", "ek2d_main.cpp")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
                  "--expt-relaxed-constexpr"]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-function"]


def _deps():
    hdrs = []
    for sub in ("csrc", "host"):
        d = os.path.join(HERE, sub)
        hdrs += [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".cuh", ".h"))]
    return hdrs + [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))
                   if f.endswith(".h")] + [__file__]


def _newer(target, sources):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources)


def _run(cmd, verbose=False):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)


def build(force=False, verbose=False):
    deps = _deps()
    allsrc = CU_SOURCES + CPP_SOURCES + [MAIN, MAIN2D]
    if not force and all(_newer(t, allsrc + deps) for t in (OUT, EXE, EXE2D)):
        return OUT
    os.makedirs(OBJ, exist_ok=True)
    jobs = []
    objs = []
    for s in CU_SOURCES:
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        objs.append(o)
        if force or not _newer(o, [s] + deps):
            jobs.append([NVCC] + NVFLAGS + (["-Xptxas", "-v"] if verbose else []) +
                        ["-c", s, "-o", o])
    for s in CPP_SOURCES + [MAIN, MAIN2D]:
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        if s not in (MAIN, MAIN2D):
            objs.append(o)
        if force or not _newer(o, [s] + deps):
            jobs.append(["g++"] + CXXFLAGS + ["-I", "/usr/local/cuda/include", "-c", s, "-o", o])
    with ThreadPoolExecutor(max_workers=8) as ex:
        list(ex.map(lambda c: _run(c, verbose), jobs))
    _run([NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart"])
    for exe, main in ((EXE, "main.cpp.o"), (EXE2D, "ek2d_main.cpp.o")):
        _run(["g++", "-o", exe, os.path.join(OBJ, main), "-L", HERE, "-lcupf",
              "-Wl,-rpath,$ORIGIN", "-L/usr/local/cuda/lib64", "-lcudart",
              "-Wl,-rpath,/usr/local/cuda/lib64"])
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
