"""Builds libculs_b200.so in-tree: every CUDA source for sm_100a with nvcc,
the host C++ with g++, and the rewriting library embedded as a byte array.

    python -m culs_b200.build [--force] [--jobs N]
"""
import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INC = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "libculs_b200.so"
CLI = PKG / "gpuls"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
                  "-I", str(INC), "-I", str(CSRC)]
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-I", str(INC), "-I", str(CSRC),
            "-I", "/usr/local/cuda/include"]


def _newer(out: Path, deps) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _embed_library():
    src = PKG / "data" / "rwlib.bin"
    out = BUILD / "rwlib_blob.c"
    if not _newer(out, [src, Path(__file__)]):
        return out
    data = src.read_bytes()
    lines = ["/* generated from culs_b200/data/rwlib.bin by culs_b200/build.py */",
             "#include <stddef.h>",
             f"const size_t culs_rwlib_blob_size = {len(data)};",
             "const unsigned char culs_rwlib_blob[] = {"]
    for i in range(0, len(data), 24):
        lines.append(",".join(str(b) for b in data[i:i + 24]) + ",")
    lines.append("};")
    out.write_text("\n".join(lines) + "\n")
    return out


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def build(force=False, jobs=None, verbose=False):
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INC.glob("*.h"))
    blob = _embed_library()
    tasks = []
    objs = []
    for cu in sorted(CSRC.glob("*.cu")):
        o = BUILD / (cu.stem + ".cu.o")
        objs.append(o)
        if force or _newer(o, [cu] + headers + [Path(__file__)]):
            tasks.append([NVCC] + NVFLAGS + ["-c", str(cu), "-o", str(o)])
    for cpp in sorted(CSRC.glob("host_*.cpp")):
        o = BUILD / (cpp.stem + ".cpp.o")
        objs.append(o)
        if force or _newer(o, [cpp] + headers):
            tasks.append(["g++"] + CXXFLAGS + ["-c", str(cpp), "-o", str(o)])
    bo = BUILD / "rwlib_blob.o"
    objs.append(bo)
    if force or _newer(bo, [blob]):
        tasks.append(["gcc", "-O1", "-fPIC", "-c", str(blob), "-o", str(bo)])
    with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for r in ex.map(_run, tasks):
            if verbose and (r.stderr.strip()):
                print(r.stderr, file=sys.stderr)
    if force or tasks or not LIB.exists():
        _run([NVCC] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] + ["-lpthread"])
    cli_src = CSRC / "gpuls_main.cpp"
    if cli_src.exists() and (force or _newer(CLI, [cli_src, LIB] + headers)):
        _run(["g++"] + CXXFLAGS + [str(cli_src), "-o", str(CLI), "-L", str(PKG), "-lculs_b200",
                                   "-Wl,-rpath,$ORIGIN"])
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, jobs=a.jobs, verbose=a.verbose))


if __name__ == "__main__":
    main()
