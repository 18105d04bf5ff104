"""Build step of the CUDA library libtcg_b200.so (in-tree, sm_100a).

api.cu (C-ABI, orchestration, generic kernels), subspace.cu (the dense
Davidson subspace step on cuBLAS / cuSOLVER) and one instance of fast_inst.cu
per compiled cubic grid size are compiled in parallel into tc_b200/_build/
and linked into tc_b200/libtcg_b200.so.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "libtcg_b200.so")
SRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
FAST_SIZES = (12, 16, 24, 32, 36, 40, 48)
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]


def sources():
    return [os.path.join(SRC, f) for f in sorted(os.listdir(SRC)) if f.endswith((".cu", ".cuh"))] + \
        [os.path.join(HERE, "..", "include", "tcg.h")]


def stale():
    if not os.path.exists(SO):
        return True
    t = os.path.getmtime(SO)
    return any(os.path.getmtime(s) > t for s in sources())


def _units():
    units = [(os.path.join(SRC, "api.cu"), os.path.join(OBJ, "api.o"), []),
             (os.path.join(SRC, "subspace.cu"), os.path.join(OBJ, "subspace.o"), [])]
    for n in FAST_SIZES:
        units.append((os.path.join(SRC, "fast_inst.cu"), os.path.join(OBJ, f"fast_{n}.o"), [f"-DTCG_FAST_N={n}"]))
    return units


def build(force=False, verbose=False, jobs=None):
    if not force and not stale():
        return SO
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(OBJ, exist_ok=True)

    def compile_one(u):
        src, obj, extra = u
        cmd = [nvcc, *CFLAGS, *extra, "-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src} {extra}:\n{r.stderr}")
        return obj

    units = _units()
    jobs = jobs or min(len(units), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(compile_one, units))
    cmd = [nvcc, *ARCH, "-shared", "-o", SO + ".tmp", *objs, "-lcublas", "-lcusolver"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(SO + ".tmp", SO)
    return SO


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(SO)
