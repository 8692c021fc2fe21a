"""Build the in-tree shared library ``semtex_b200/libsemtex_b200.so``.

Host sources are compiled with g++, kernels with nvcc for sm_100a only;
objects go to ``semtex_b200/_build`` and are rebuilt when a source or any
header under ``csrc`` is newer than the object.
"""

from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsemtex_b200.so")
BIN = os.path.join(HERE, "bin")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-Wno-unused-function"]


def _sources():
    cpp = sorted(glob.glob(os.path.join(CSRC, "host", "*.cpp")))
    cu = sorted(glob.glob(os.path.join(CSRC, "kernels", "*.cu"))) + sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    return cpp, cu


def _headers_mtime():
    hs = glob.glob(os.path.join(CSRC, "**", "*.h*"), recursive=True)
    hs += glob.glob(os.path.join(HERE, "..", "include", "*.h"))
    hs += glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True)
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _obj(src):
    rel = os.path.relpath(src, CSRC).replace(os.sep, "_")
    return os.path.join(BUILD, rel + ".o")


def _compile(src, ptxas_verbose=False):
    obj = _obj(src)
    if src.endswith(".cu"):
        cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
               "-I", CSRC, "-c", src, "-o", obj]
        if ptxas_verbose:
            cmd.insert(1, "-Xptxas=-v")
    else:
        cmd = ["g++", *CXXFLAGS, "-I", CSRC, "-I", "/usr/local/cuda/include", "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    cpp, cu = _sources()
    hdr = _headers_mtime()
    todo = []
    for s in cpp + cu:
        o = _obj(s)
        if force or ptxas_verbose or not os.path.exists(o) or \
                os.path.getmtime(o) < max(os.path.getmtime(s), hdr):
            todo.append(s)
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for obj, err in ex.map(lambda s: _compile(s, ptxas_verbose), todo):
            if err.strip() and (verbose or "warning" in err):
                print(err, file=sys.stderr)
    objs = [_obj(s) for s in cpp + cu]
    relinked = False
    if todo or not os.path.exists(LIB):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        relinked = True
    # the `elliptic` and `dns` programs over the library (semtex_b200/bin)
    os.makedirs(BIN, exist_ok=True)
    for src in sorted(glob.glob(os.path.join(CSRC, "cli", "*.cpp"))):
        exe = os.path.join(BIN, os.path.splitext(os.path.basename(src))[0])
        if force or relinked or not os.path.exists(exe) or os.path.getmtime(exe) < max(os.path.getmtime(src), hdr):
            cmd = ["g++", *CXXFLAGS, "-I", CSRC, src, "-o", exe, "-L", HERE, "-lsemtex_b200",
                   "-Wl,-rpath,$ORIGIN/.."]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"program build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
            if r.stderr.strip() and "warning" in r.stderr:
                print(r.stderr, file=sys.stderr)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True,
                ptxas_verbose="--ptxas" in sys.argv))
