"""Build libbssn_b200.so in-tree for sm_100a with nvcc.

Usage: python -m nrpy_b200.build [--jobs N] [--verbose-ptxas] [--fd-order 4|8]
The library lands next to this file: nrpy_b200/libbssn_b200.so (4th-order finite differences)
or nrpy_b200/libbssn_b200_fd8.so (8th order, NGHOSTS = 5). Object files go to nrpy_b200/_build/
(_build_fd8/) and are rebuilt only when a source or header is newer.
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
FD_ORDERS = (4, 8)


def lib_path(fd_order: int = 4) -> pathlib.Path:
    return PKG / ("libbssn_b200.so" if fd_order == 4 else f"libbssn_b200_fd{fd_order}.so")


def build_dir(fd_order: int = 4) -> pathlib.Path:
    return PKG / ("_build" if fd_order == 4 else f"_build_fd{fd_order}")


LIB = lib_path(4)
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["abi.cu", "setup.cu", "pointwise.cu", "boundary.cu", "mol.cu", "reductions.cu", "batch.cu",
           "adjoint.cu", "diagnostics.cu", "checkpoint.cu"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def flags(ptxas_verbose: bool = False, fd_order: int = 4):
    f = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                f"-DBSSN_B200_FD_ORDER={fd_order}", f"-I{ROOT / 'include'}", f"-I{CSRC}"]
    if ptxas_verbose:
        f += ["-Xptxas", "-v"]
    return f


def _newest_dep(src: str, fd_order: int = 4) -> float:
    """Newest modification time among a source and the headers it can include."""
    deps = [CSRC / src, CSRC / "bssn_common.cuh"] + list((ROOT / "include").glob("*.h"))
    if src == "pointwise.cu":
        gen = [p for p in (CSRC / "gen").glob("bssn_*.cuh") if not p.name.startswith("bssn_adj_")]
        deps += [p for p in gen if p.name.endswith(f"_fd{fd_order}.cuh") == (fd_order != 4) and
                 (fd_order != 4 or "_fd" not in p.name)]
    if src == "adjoint.cu":
        deps += list((CSRC / "gen").glob("bssn_adj_*.cuh"))
    return max(p.stat().st_mtime for p in deps)


def build(jobs: int = 0, ptxas_verbose: bool = False, force: bool = False, fd_order: int = 4) -> pathlib.Path:
    if fd_order not in FD_ORDERS:
        raise ValueError(f"fd_order {fd_order}: generated algebra exists for {FD_ORDERS}")
    bdir, lib = build_dir(fd_order), lib_path(fd_order)
    bdir.mkdir(exist_ok=True)
    cc = nvcc()

    def one(src: str) -> pathlib.Path:
        obj = bdir / (src + ".o")
        if force or ptxas_verbose or not obj.exists() or obj.stat().st_mtime < _newest_dep(src, fd_order):
            cmd = [cc] + flags(ptxas_verbose, fd_order) + ["-c", str(CSRC / src), "-o", str(obj)]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
            if ptxas_verbose:
                sys.stderr.write(r.stderr)
        return obj

    with cf.ThreadPoolExecutor(max_workers=jobs or len(SOURCES)) as ex:
        objs = list(ex.map(one, SOURCES))
    if force or not lib.exists() or any(o.stat().st_mtime > lib.stat().st_mtime for o in objs):
        cmd = [cc] + ARCH + ["-shared", "-o", str(lib)] + [str(o) for o in objs] + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return lib


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=0)
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--fd-order", type=int, default=4, choices=FD_ORDERS)
    a = ap.parse_args()
    print(build(a.jobs, a.verbose_ptxas, a.force, a.fd_order))
