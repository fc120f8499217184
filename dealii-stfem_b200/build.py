"""Builds libstmg_cuda.so for sm_100a in-tree (dealii-stfem_b200/).

  python dealii-stfem_b200/build.py [-j N]

Each .cu / .cc under csrc/ is compiled by nvcc to an object in
dealii-stfem_b200/build/ and linked into dealii-stfem_b200/libstmg_cuda.so.
Objects are rebuilt when their source or any header changed.
"""
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "build")
LIB = os.path.join(HERE, "libstmg_cuda.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
         "-I", os.path.join(REPO, "include"), "-I", CSRC]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        [os.path.join(REPO, "include", "stmg.h")]


def _compile(src, extra):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest_dep = max(os.path.getmtime(p) for p in _headers() + [src])
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep:
        return obj, None
    cmd = [NVCC] + FLAGS + extra + ["-c", src, "-o", obj]
    if src.endswith(".cc"):
        cmd[1:1] = ["-x", "cu"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, r.stdout + r.stderr
    return obj, None


def build(jobs=8, verbose_ptxas=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cc")))
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    objs, errors = [], []
    with cf.ThreadPoolExecutor(jobs) as ex:
        for obj, err in ex.map(lambda s: _compile(s, extra), srcs):
            objs.append(obj)
            if err:
                errors.append(err)
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB] + objs + ["-lcudart"]
        subprocess.run(cmd, check=True)
    return LIB


CPP_TESTS = [(os.path.join(REPO, "tests", "cpp", "shim_test.cc"), os.path.join(REPO, "tests", "cpp", "build", "shim_test"))]


def build_cpp_tests():
    """Host C++ programs of tests/cpp (the drop-in classes of
    include/stmg_dealii.hpp over the C ABI), linked against the in-tree
    library with a relative run path so they run wherever the tree is."""
    cuda = os.path.dirname(os.path.dirname(NVCC))
    for src, exe in CPP_TESTS:
        os.makedirs(os.path.dirname(exe), exist_ok=True)
        deps = [src, LIB, os.path.join(REPO, "include", "stmg_dealii.hpp"), os.path.join(REPO, "include", "stmg.h")]
        if os.path.exists(exe) and os.path.getmtime(exe) >= max(os.path.getmtime(d) for d in deps):
            continue
        cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(REPO, "include"), "-I",
               os.path.join(cuda, "include"), src, "-L", HERE, "-lstmg_cuda", "-L", os.path.join(cuda, "lib64"),
               "-lcudart", "-Wl,-rpath,$ORIGIN/../../../dealii-stfem_b200", "-o", exe]
        subprocess.run(cmd, check=True)


if __name__ == "__main__":
    jobs = int(sys.argv[sys.argv.index("-j") + 1]) if "-j" in sys.argv else 8
    print(build(jobs, verbose_ptxas="--ptxas-v" in sys.argv))
    build_cpp_tests()
