"""Builds puzzlesearch_b200/libpsb200.so (sm_100a) from puzzlesearch_b200/csrc.

    python -m puzzlesearch_b200.build [--verbose]

Each .cu file is compiled by nvcc in parallel (-gencode arch=compute_100a,
code=sm_100a), then linked into one shared library with the CUDA runtime
linked statically.  The library travels with the repository, so a machine
with a GPU needs no compiler.
"""
import argparse
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.environ.get("PSB_BUILD_DIR") or os.path.join(HERE, "_build")
LIB = os.environ.get("PSB_LIB_OUT") or os.path.join(HERE, "libpsb200.so")
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    cand = os.environ.get("PSB_NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def host_compiler():
    # The system g++: a compiler wrapper that links libstdc++ statically would
    # clash with the libstdc++ already loaded into a Python process.
    return os.environ.get("PSB_HOST_CXX", "/usr/bin/g++")


def flags(verbose):
    f = GENCODE + ["-O3", "-lineinfo", "-std=c++17", "-ccbin", host_compiler(),
                   "-Xcompiler", "-fPIC,-O3", "-I" + os.path.join(HERE, "..", "include")]
    if verbose:
        f += ["-Xptxas", "-v"]
    return f


def compile_one(src, verbose):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    deps = [src] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".cuh", ".h"))]
    deps.append(os.path.join(HERE, "..", "include", "psb200.h"))
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj, ""
    cmd = [nvcc()] + flags(verbose) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
    return obj, r.stderr


def build(verbose=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    sources = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))
    logs = []
    with concurrent.futures.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: compile_one(s, verbose), sources))
    objs = [o for o, _ in results]
    logs = [l for _, l in results if l]
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc()] + GENCODE + ["-shared", "-ccbin", host_compiler(), "-Xcompiler", "-fPIC",
                                    "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    return LIB, "\n".join(logs)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true", help="pass -Xptxas -v and print its report")
    args = ap.parse_args()
    lib, log = build(args.verbose)
    if log:
        print(log)
    print(lib)


if __name__ == "__main__":
    sys.exit(main())
