"""Build the reference oracle: generate the reference's BHaH BSSN C projects and compile them.

Test infrastructure only (never shipped, never on the product path).

Recipe
------
1. Import shims for four packages the reference imports but never calls on this path
   (appdirs -> platformdirs, black.format_str -> identity, nrpypn -> empty stubs,
   clang-format -> ``cat``). They are written under ``oracle/_ref/shim``.
2. ``oracle/ref_project.py`` runs the reference's own generators (nrpy, read from the
   reference checkout) to emit one project per variant into ``oracle/_ref/<variant>/project``.
3. Every generated ``*.c`` except ``main.c``, plus ``oracle/ref_harness.c``, is compiled
   with gcc (the generated Makefile is NOT used: its OpenMP probe fails under GNU make 4.3)
   into ``oracle/_ref/<variant>/libref_<isa>.so`` with the generated Makefile's own
   flags (``-std=gnu99 -O2 -fopenmp``), once per ISA level so that the library also
   runs on hosts without AVX-512.

Variants
--------
  sphaxi : Spherical, symmetry_axes="2" (axisymmetric; the 72x12x2 workload)
  sph3d  : Spherical, full 3-D (batched and adjoint workloads)
  sinh3d : SinhSpherical, full 3-D (the 256x64x64 workloads)
  sph3dck: sph3d plus write_checkpoint/read_checkpoint (checkpoint file parity)
  sph3d8, sinh3d8, sphaxi8: sph3d, sinh3d and sphaxi with 8th-order finite differences
           (NGHOSTS = 5)
  sinhaxi, sinhaxi8: SinhSpherical, symmetry_axes="2", 4th and 8th order
  sinhcyl, sinhcyl8: SinhCylindrical, symmetry_axes="1" (axisymmetric about z), 4th and
           8th order; blackhole_spectroscopy's coordinates (its project uses fd_order 8)
  sinh3d_cuda: sinh3d emitted by the reference's CUDA path (``--cuda``), compiled with nvcc
           for sm_100a (relocatable device code, the generated Makefile's flags with
           ``-arch=sm_100a``) together with ``oracle/ref_harness_cuda.cu`` into
           ``oracle/_ref/sinh3d_cuda/libref_cuda.so``: the reference's own GPU step, timed
           beside this library's on the B200 (built by default after the C variants; it
           needs nvcc, not a GPU, to build)

Usage: python oracle/gen_ref.py [--variants sphaxi,sph3d,sinh3d,sinh3d_cuda] [--reference DIR]
"""

import argparse
import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
REF_OUT = HERE / "_ref"
VARIANTS = {
    "sphaxi": ["--coord", "Spherical", "--axisym"],
    "sph3d": ["--coord", "Spherical"],
    "sinh3d": ["--coord", "SinhSpherical"],
    "sph3dck": ["--coord", "Spherical", "--checkpoint"],
    "sph3d8": ["--coord", "Spherical", "--fd-order", "8"],
    "sinh3d8": ["--coord", "SinhSpherical", "--fd-order", "8"],
    "sphaxi8": ["--coord", "Spherical", "--axisym", "--fd-order", "8"],
    "sinhaxi": ["--coord", "SinhSpherical", "--axisym"],
    "sinhaxi8": ["--coord", "SinhSpherical", "--axisym", "--fd-order", "8"],
    "sinhcyl": ["--coord", "SinhCylindrical", "--axisym"],
    "sinhcyl8": ["--coord", "SinhCylindrical", "--axisym", "--fd-order", "8"],
}
# Variants emitted by the reference's CUDA path (built with nvcc; not in the default list).
CUDA_VARIANTS = {
    "sinh3d_cuda": ["--coord", "SinhSpherical", "--cuda"],
}
# Extra compiler definitions of a variant's harness build.
HARNESS_DEFS = {"sph3dck": ["-DREF_HAS_CHECKPOINT"]}
ISAS = {"avx512": "-march=x86-64-v4", "avx2": "-march=x86-64-v3"}


def write_shims(shim: pathlib.Path) -> None:
    (shim / "nrpypn").mkdir(parents=True, exist_ok=True)
    (shim / "bin").mkdir(parents=True, exist_ok=True)
    (shim / "appdirs.py").write_text("from platformdirs import user_cache_dir  # noqa: F401\n")
    (shim / "black.py").write_text(
        "class Mode:\n    def __init__(self, *a, **k):\n        pass\n\n\n"
        "FileMode = Mode\n\n\ndef format_str(s, mode=None):\n    return s\n"
    )
    (shim / "nrpypn" / "__init__.py").write_text("")
    (shim / "nrpypn" / "NRPyPN_shortcuts.py").write_text(
        "S1U = S2U = chi1U = chi2U = n12U = n21U = p1U = p2U = [0, 0, 0]\nm1 = m2 = r = 0\n"
    )
    (shim / "nrpypn" / "PN_p_r.py").write_text("class PN_p_r:\n    pass\n")
    (shim / "nrpypn" / "PN_p_t.py").write_text("class PN_p_t:\n    pass\n")
    cf_path = shim / "bin" / "clang-format"
    cf_path.write_text("#!/bin/sh\ncat\n")
    cf_path.chmod(0o755)


def generate(variant: str, reference: pathlib.Path, shim: pathlib.Path) -> pathlib.Path:
    vdir = REF_OUT / variant
    proj = vdir / "project"
    vdir.mkdir(parents=True, exist_ok=True)
    env = dict(os.environ)
    env["PYTHONPATH"] = f"{shim}:{reference}"
    env["PATH"] = f"{shim / 'bin'}:{env.get('PATH', '')}"
    cmd = [sys.executable, str(HERE / "ref_project.py"), "--project-dir", str(proj)] + {**VARIANTS, **CUDA_VARIANTS}[variant]
    with open(vdir / "generate.log", "w") as log:
        subprocess.run(cmd, cwd=vdir, env=env, stdout=log, stderr=subprocess.STDOUT, check=True)
    return proj


def compile_variant(variant: str, proj: pathlib.Path, jobs: int) -> None:
    vdir = REF_OUT / variant
    sources = sorted(p for p in proj.rglob("*.c") if p.name != "main.c")
    sources.append(HERE / "ref_harness.c")
    for isa, march in ISAS.items():
        objdir = vdir / f"obj_{isa}"
        objdir.mkdir(exist_ok=True)
        base = ["gcc", "-std=gnu99", "-O2", march, "-fopenmp", "-fPIC", "-w", f"-I{proj}"] + HARNESS_DEFS.get(variant, [])

        def one(src: pathlib.Path) -> pathlib.Path:
            rel = src.relative_to(proj) if proj in src.parents else pathlib.Path(src.name)
            obj = objdir / (str(rel).replace("/", "__") + ".o")
            subprocess.run(base + ["-c", str(src), "-o", str(obj)], check=True)
            return obj

        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            objs = list(ex.map(one, sources))
        lib = vdir / f"libref_{isa}.so"
        subprocess.run(
            ["gcc", "-shared", "-fopenmp", "-o", str(lib)] + [str(o) for o in objs] + ["-lm"], check=True
        )
        shutil.rmtree(objdir)
        print(f"built {lib}")


def compile_cuda_variant(variant: str, proj: pathlib.Path, jobs: int) -> None:
    """nvcc build of a CUDA project: every generated .cu (not main.cu) with the generated
    Makefile's NVCCFLAGS for sm_100a, its .cc files with the host compiler, and the CUDA
    harness, linked into one shared library (device link included)."""
    vdir = REF_OUT / variant
    objdir = vdir / "obj_cuda"
    objdir.mkdir(exist_ok=True)
    cu = sorted(p for p in proj.rglob("*.cu") if p.name != "main.cu") + [HERE / "ref_harness_cuda.cu"]
    cc = sorted(proj.rglob("*.cc"))
    nv = ["nvcc", "-O2", "-arch=sm_100a", "--relocatable-device-code=true", "-allow-unsupported-compiler",
          "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp", "-Xcompiler", "-march=x86-64-v3", "-w", f"-I{proj}"]
    cxx = ["g++", "-O2", "-fPIC", "-fopenmp", "-march=x86-64-v3", "-w", f"-I{proj}", "-I/usr/local/cuda/include"]

    def one(src: pathlib.Path) -> pathlib.Path:
        rel = src.relative_to(proj) if proj in src.parents else pathlib.Path(src.name)
        obj = objdir / (str(rel).replace("/", "__") + ".o")
        base = nv if src.suffix == ".cu" else cxx
        subprocess.run(base + ["-c", str(src), "-o", str(obj)], check=True)
        return obj

    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(one, cu + cc))
    lib = vdir / "libref_cuda.so"
    subprocess.run(["nvcc", "-shared", "-arch=sm_100a", "--relocatable-device-code=true", "-Xcompiler", "-fopenmp",
                    "-o", str(lib)] + [str(o) for o in objs] + ["-lm"], check=True)
    shutil.rmtree(objdir)
    print(f"built {lib}")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--variants", default=",".join(list(VARIANTS) + list(CUDA_VARIANTS)))
    ap.add_argument("--reference", default=os.environ.get("NRPY_REFERENCE", str(HERE.parent.parent / "reference")),
                    help="the nrpy checkout (default: $NRPY_REFERENCE, else ../reference beside this repository)")
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 4)
    args = ap.parse_args()
    reference = pathlib.Path(args.reference)
    if not (reference / "nrpy").is_dir():
        raise SystemExit(f"reference checkout not found at {reference}")
    shim = REF_OUT / "shim"
    write_shims(shim)
    for v in args.variants.split(","):
        proj = generate(v, reference, shim)
        if v in CUDA_VARIANTS:
            compile_cuda_variant(v, proj, args.jobs)
        else:
            compile_variant(v, proj, args.jobs)


if __name__ == "__main__":
    main()
