"""Build libbssn_b200.so in-tree for sm_100a with nvcc.

Usage: python -m nrpy_b200.build [--jobs N] [--verbose-ptxas]
The library lands next to this file (nrpy_b200/libbssn_b200.so); object files go to
nrpy_b200/_build/ and are rebuilt only when a source or header is newer.
"""

import argparse
import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libbssn_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["abi.cu", "setup.cu", "pointwise.cu", "boundary.cu", "mol.cu", "reductions.cu", "batch.cu",
           "adjoint.cu", "diagnostics.cu", "checkpoint.cu"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def flags(ptxas_verbose: bool = False):
    f = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                f"-I{ROOT / 'include'}", f"-I{CSRC}"]
    if ptxas_verbose:
        f += ["-Xptxas", "-v"]
    return f


def _newest_dep(src: str) -> float:
    """Newest modification time among a source and the headers it can include."""
    deps = [CSRC / src, CSRC / "bssn_common.cuh"] + list((ROOT / "include").glob("*.h"))
    if src == "pointwise.cu":
        deps += [p for p in (CSRC / "gen").glob("bssn_*.cuh") if not p.name.startswith("bssn_adj_")]
    if src == "adjoint.cu":
        deps += list((CSRC / "gen").glob("bssn_adj_*.cuh"))
    return max(p.stat().st_mtime for p in deps)


def build(jobs: int = 0, ptxas_verbose: bool = False, force: bool = False) -> pathlib.Path:
    BUILD.mkdir(exist_ok=True)
    cc = nvcc()

    def one(src: str) -> pathlib.Path:
        obj = BUILD / (src + ".o")
        if force or ptxas_verbose or not obj.exists() or obj.stat().st_mtime < _newest_dep(src):
            cmd = [cc] + flags(ptxas_verbose) + ["-c", str(CSRC / src), "-o", str(obj)]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
            if ptxas_verbose:
                sys.stderr.write(r.stderr)
        return obj

    with cf.ThreadPoolExecutor(max_workers=jobs or len(SOURCES)) as ex:
        objs = list(ex.map(one, SOURCES))
    if force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [cc] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=0)
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.jobs, a.verbose_ptxas, a.force))
