"""Build libplanck_fock.so (sm_100a) in-tree.

nvcc compiles the ten bra-class translation units of pfk_classes.cu, the
setup kernels and the C ABI in parallel into _build/, then links the shared
library next to this file.  Objects are rebuilt when any source under csrc/
or include/ is newer than them.

    python build.py [-j N] [--force]
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(REPO, "_build", "pfk")
LIB = os.path.join(HERE, "libplanck_fock.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + CSRC,
         "-I" + os.path.join(REPO, "include")]


DEVICE_DEPS = ["pfk_device.cuh", "pfk_internal.h", "rys_table_data.inc", "../../include/planck_fock.h"]
DEPS = {
    "pfk_classes.cu": DEVICE_DEPS + ["pfk_kernels.cuh", "pfk_os.cuh"],
    "pfk_setup.cu": DEVICE_DEPS + ["pfk_kernels.cuh", "pfk_setup.h"],
    "pfk_api.cu": DEVICE_DEPS + ["pfk_setup.h", "../../include/planck_fock.h"],
    "pfk_onee.cu": DEVICE_DEPS + ["pfk_kernels.cuh", "pfk_os.cuh"],
    "pfk_mlp.cu": ["../../include/planck_fock.h"],
    "pfk_checkpoint.cu": ["../../include/planck_fock.h"],
    "pfk_scf.cu": ["../../include/planck_fock.h", "pfk_internal.h", "pfk_device.cuh"],
}


# Class ranges per translation unit (class c = X(X+1)/2 + Y for bra pair
# class X >= ket pair class Y): one unit per class, so the 55 classes compile
# in parallel.
CLASS_UNITS = [(c, c + 1) for c in range(55)]


def _units():
    units = [("pfk_classes.cu", f"classes_{b}_{e}.o", [f"-DPFK_CLASS_BEGIN={b}", f"-DPFK_CLASS_END={e}"])
             for b, e in reversed(CLASS_UNITS)]
    units += [("pfk_setup.cu", "setup.o", []), ("pfk_api.cu", "api.o", []), ("pfk_onee.cu", "onee.o", []),
              ("pfk_mlp.cu", "mlp.o", []), ("pfk_checkpoint.cu", "checkpoint.o", []), ("pfk_scf.cu", "scf.o", [])]
    return units


def _newest(src):
    files = [os.path.join(CSRC, src)] + [os.path.join(CSRC, d) for d in DEPS[src]] + [os.path.abspath(__file__)]
    return max(os.path.getmtime(f) for f in files)


def _compile(src, obj, extra, verbose):
    cmd = [NVCC] + ARCH + FLAGS + extra + ["-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src} {extra}:\n{r.stderr[-6000:]}")
    return r.stderr


def build(jobs=None, force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    todo = []
    for src, obj, extra in _units():
        path = os.path.join(BUILD, obj)
        if force or not os.path.exists(path) or os.path.getmtime(path) < _newest(src):
            todo.append((src, path, extra))
    logs = {}
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count()) as ex:
            futs = {ex.submit(_compile, s, o, e, verbose): (s, o) for s, o, e in todo}
            for f in cf.as_completed(futs):
                logs[futs[f][1]] = f.result()
    objs = [os.path.join(BUILD, o) for _, o, _ in _units()]
    if todo or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lcublas", "-lcusolver"]
        subprocess.check_call(cmd)
    return LIB, logs


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true", help="print ptxas register/spill report")
    a = ap.parse_args()
    lib, logs = build(a.j, a.force, a.verbose)
    if a.verbose:
        for k, v in logs.items():
            print("==", k)
            print(v)
    print(lib)
    sys.exit(0)
