"""Build the B200 gridder in place.

    python rang-core_b200/build.py

produces, next to the Python package `rang` in this directory:

* `rang/librang_wgrid_b200.so` — the CUDA library with the C ABI of
  include/rang_wgridder.h, compiled for sm_100a only;
* `rang/_core.<abi>.so` — the pybind11 module `rang._core` bound to it.

The device code is compiled with `--fmad=false` and the host code with
`-ffp-contract=off`: the binning arithmetic must round exactly as the
reference's, so no multiply-add is fused except the explicit fma() calls
that restate the reference's `mul_add`.
"""

import os
import subprocess
import sys
import sysconfig
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
CSRC = HERE / "csrc"
PKG = HERE / "rang"
INCLUDE = REPO / "include"
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
LIB = PKG / "librang_wgrid_b200.so"

CU_SOURCES = ["wgrid_plan.cu", "wgrid_capi.cu", "wgrid_weights.cu", "wgrid_gram.cu", "wgrid_solver.cu", "nn_kernels.cu",
              "nn_conv_tc.cu"]
CXX_SOURCES = ["wgrid_setup.cpp", "msv4_codec.cpp"]
HEADERS = ["wgrid_common.h", "wgrid_device.cuh", "wgrid_fast.cuh", "wgrid_f64.cuh", "wgrid_plan.h", "wgrid_setup.h",
           "kernel_db.inc", "nn_conv_tc.h"]


def ext_path():
    return PKG / ("_core" + sysconfig.get_config_var("EXT_SUFFIX"))


def _stale(target, deps):
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd):
    print(" ".join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def build_lib(force=False, jobs=None):
    deps = [CSRC / s for s in CU_SOURCES + CXX_SOURCES + HEADERS] + [INCLUDE / "rang_wgridder.h", INCLUDE / "rang_weights.h", INCLUDE / "rang_gram.h", INCLUDE / "rang_nn.h", INCLUDE / "rang_msv4.h",
            INCLUDE / "rang_solver.h"]
    deps.append(Path(__file__))
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = HERE / "_build"
    objdir.mkdir(exist_ok=True)
    common = ["-O3", "-std=c++17", f"-I{INCLUDE}", f"-I{CSRC}"]
    objs = []
    procs = []
    for src in CU_SOURCES:
        obj = objdir / (src + ".o")
        cmd = [NVCC, *ARCH, "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC,-ffp-contract=off",
               "-Xptxas", "-warn-spills", *common, "-c", CSRC / src, "-o", obj]
        print(" ".join(str(c) for c in cmd), flush=True)
        procs.append(subprocess.Popen([str(c) for c in cmd]))
        objs.append(obj)
    for src in CXX_SOURCES:
        obj = objdir / (src + ".o")
        cmd = ["g++", "-fPIC", "-ffp-contract=off", *common, f"-I{CUDA / 'include'}", "-c", CSRC / src, "-o", obj]
        print(" ".join(str(c) for c in cmd), flush=True)
        procs.append(subprocess.Popen([str(c) for c in cmd]))
        objs.append(obj)
    for p in procs:
        if p.wait() != 0:
            raise SystemExit("compilation failed")
    _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs, f"-L{CUDA / 'lib64'}", "-lcufft",
          "-Xlinker", f"-rpath,{CUDA / 'lib64'}"])
    return LIB


def build_ext(force=False):
    target = ext_path()
    deps = [CSRC / "pyext.cpp", INCLUDE / "rang_wgridder.h", INCLUDE / "rang_weights.h", INCLUDE / "rang_gram.h", LIB, Path(__file__)]
    if not force and not _stale(target, deps):
        return target
    import pybind11

    py_inc = sysconfig.get_paths()["include"]
    _run(["g++", "-O2", "-shared", "-fPIC", "-std=c++17", f"-I{INCLUDE}", f"-I{pybind11.get_include()}",
          f"-I{py_inc}", CSRC / "pyext.cpp", "-o", target, f"-L{PKG}", "-lrang_wgrid_b200",
          "-Wl,-rpath,$ORIGIN"])
    return target


def build(force=False):
    build_lib(force)
    build_ext(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
