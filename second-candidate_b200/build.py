"""Builds libscgpu.so in-tree with nvcc for sm_100a (no JIT, no torch)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libscgpu.so")
SOURCES = ["search_u4.cu", "search_u2.cu", "search_u8.cu", "search_sel.cu", "api.cu", "tables.cu", "tables_tc.cu", "search.cu",
           "encode.cu", "rerank.cu", "server.cu", "coarse.cu", "encode_tc.cu", "train.cu", "build_index.cu", "gt.cu", "select_warp.cu", "merge_warp.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if not f.endswith(".o")] + \
        [os.path.join(ROOT, "include", "scg.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, jobs=None, out=None, defines=()):
    """Compiles every source for sm_100a (in parallel) and links libscgpu.so
    in-tree (or at `out`, with extra -D `defines`); does nothing when the
    in-tree library is newer than every source."""
    lib = out or LIB
    if out is None and not force and not _stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    objdir = os.path.dirname(lib) if out else CSRC
    objs = [os.path.join(objdir, src.replace(".cu", ".o")) for src in SOURCES]
    dflags = ["-D" + d for d in defines]
    cmds = [[NVCC] + FLAGS + dflags + ["-I", os.path.join(ROOT, "include"), "-c", os.path.join(CSRC, src), "-o", obj]
            for src, obj in zip(SOURCES, objs)]
    if verbose:
        for c in cmds:
            print(" ".join(c), file=sys.stderr)
    jobs = jobs or min(len(cmds), max(1, os.cpu_count() or 1))
    with ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds))
    for c, r in zip(cmds, results):
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise subprocess.CalledProcessError(r.returncode, c)
    tmp = lib + ".tmp"
    subprocess.run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp] + objs + ["-lcudart"], check=True)
    os.replace(tmp, lib)
    for o in objs:
        os.remove(o)
    return lib


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
