"""The reference's generated project, linked against libbssn_b200, against the same project built alone (B200).

The two_blackholes_collide-style project that the oracle generated (Spherical 3-D) keeps
its own main(), parameter-file parser, CodeParameter defaults, grid set-up driver
(numerical_grids_and_timestep) and griddata_free. Every other function comes from
libbssn_b200, linked as a shared library: grid, rfm, bcstruct, CFL timestep, initial data,
MoL storage and RK4 step, diagnostics.

One change to the generated sources is needed. Its BHAH_MALLOC and BHAH_FREE macros are
mapped to CUDA managed memory, so the gridfunctions that main() allocates itself are usable
on the device. The library's memory convention is that gridfunctions are device arrays.

Both executables run the same parameter file: the project's default 72x12x2 grid to t = 0.1
(15 RK4 steps), with diagnostics every 0.05. Their output files must have the same names and
identical comment lines. Numbers must agree to 1e-12 for coordinates and times, and to 1e-8
of each column's largest magnitude for H, M^2 and the integrals (plus 1e-12 for columns at
rounding noise), or to 10 times the spread between two compilations of the reference
itself where that is larger.

The same is done for the SinhCylindrical project set up as blackhole_spectroscopy.py sets
it up (axisymmetric about z), at convergence factor 0.1 (a 40x2x120 grid), to t = 0.1. That
project bakes symmetry_axes = "1" into its generated code; with the library the symmetry is
a run-time switch, so the linked build adds one constructor that calls
bssn_b200_set_symmetry_axes("1") before main().
"""

import pathlib
import re
import shutil
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = pathlib.Path(__file__).resolve().parents[1]
OWN = ["main.c", "cmdline_input_and_parfile_parser.c", "commondata_struct_set_to_default.c",
       "params_struct_set_to_default.c", "numerical_grids_and_timestep.c", "griddata_free.c"]
CUDA = pathlib.Path("/usr/local/cuda")

MANAGED = r'''
#include <cuda_runtime.h>
static inline void *bhah_managed_malloc(size_t sz) {
  void *p = NULL;
  if (cudaMallocManaged(&p, sz, cudaMemAttachGlobal) != cudaSuccess) return NULL;
  return p;
}
static inline void bhah_any_free(void *p) {
  struct cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) == cudaSuccess && (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged)) {
    cudaFree(p);
  } else {
    cudaGetLastError();
    free(p);
  }
}
#define BHAH_MALLOC(a, sz) do { a = (BHAH_TYPEOF(a)) bhah_managed_malloc(sz); } while(0);
#define BHAH_FREE(a) do { if (a) { bhah_any_free((void*)(a)); (a) = NULL; } } while (0);
'''


def run(cmd, cwd):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, f"{cmd[:3]} failed:\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}"
    return r


def read(path):
    comments, rows = [], []
    for line in path.read_text().splitlines():
        (comments if line.startswith("#") else rows).append(line)
    return comments, np.array([[float(x) for x in r.split()] for r in rows])


SYMMETRY_CTOR = r'''
int bssn_b200_set_symmetry_axes(const char *axes);
__attribute__((constructor)) static void set_symmetry(void) { bssn_b200_set_symmetry_axes("@AXES@"); }
'''

# (oracle variant, convergence factor on the command line, symmetry axes the project bakes in)
PROJECTS = [("sph3d", "1.0", ""), ("sinhcyl", "0.1", "1")]


@pytest.fixture(scope="module", params=PROJECTS, ids=[p[0] for p in PROJECTS])
def runs(request, tmp_path_factory, cuda):
    from nrpy_b200 import lib as L

    variant, conv, axes = request.param
    PROJECT = ROOT / "oracle" / "_ref" / variant / "project"
    if not (PROJECT / "main.c").exists():
        pytest.skip(f"oracle/_ref/{variant}/project not generated")
    if L.FD_ORDER != 4:
        pytest.skip("the projects are 4th order")
    lib = ROOT / "nrpy_b200" / "libbssn_b200.so"
    base = tmp_path_factory.mktemp(f"dropin_{variant}")
    par = (PROJECT / "bssn_ref.par").read_text()
    par = re.sub(r"^t_final = .*$", "t_final = 0.1", par, flags=re.M)
    par = re.sub(r"^diagnostics_output_every = .*$", "diagnostics_output_every = 0.05", par, flags=re.M)
    # the generated project alone
    ref_src = base / "ref_src"
    shutil.copytree(PROJECT, ref_src)
    srcs = sorted(str(p) for p in ref_src.rglob("*.c"))
    run(["gcc", "-std=gnu99", "-O2", "-march=native", "-fopenmp", "-w", f"-I{ref_src}", "-o", "ref_exe"] + srcs + ["-lm"],
        base)
    # and built a second way (no FMA contraction, baseline x86-64): the reference's own
    # compile-to-compile spread
    run(["gcc", "-std=gnu99", "-O2", "-ffp-contract=off", "-fopenmp", "-w", f"-I{ref_src}", "-o", "ref2_exe"] + srcs
        + ["-lm"], base)
    # the same project with the library
    own_src = base / "own_src"
    shutil.copytree(PROJECT, own_src)
    defs = (own_src / "BHaH_defines.h").read_text()
    lines = defs.splitlines()
    i_m = next(i for i, ln in enumerate(lines) if ln.startswith("#define BHAH_MALLOC(a, sz)"))
    i_f = next(i for i, ln in enumerate(lines) if ln.startswith("#define BHAH_FREE(a)"))
    lines[i_m] = MANAGED
    lines[i_f] = ""
    (own_src / "BHaH_defines.h").write_text("\n".join(lines) + "\n")
    extra = []
    if axes:
        (own_src / "set_symmetry.c").write_text(SYMMETRY_CTOR.replace("@AXES@", axes))
        extra = [str(own_src / "set_symmetry.c")]
    run(["gcc", "-std=gnu99", "-O2", "-fopenmp", "-w", f"-I{own_src}", f"-I{CUDA / 'include'}", "-o", "own_exe"]
        + [str(own_src / f) for f in OWN] + extra
        + [f"-L{lib.parent}", f"-Wl,-rpath,{lib.parent}", "-lbssn_b200", f"-L{CUDA / 'lib64'}", "-lcudart", "-lm"],
        base)
    out = {}
    for name in ("ref", "ref2", "own"):
        d = base / f"run_{name}"
        d.mkdir()
        (d / "bssn_ref.par").write_text(par)
        run([str(base / f"{name}_exe"), "bssn_ref.par", conv], d)
        out[name] = d
    return out


def test_same_output_files(runs):
    names_ref = sorted(p.name for p in runs["ref"].iterdir() if p.name.startswith("out"))
    names_own = sorted(p.name for p in runs["own"].iterdir() if p.name.startswith("out"))
    assert names_ref and names_own == names_ref
    assert len([n for n in names_ref if n.startswith("out1d-y")]) >= 2  # at least two output times


def _deviations(d_ref_dir, d_other_dir):
    """Per output file: the absolute deviations of the values from the reference run, each
    column's largest magnitude, and an absolute floor (1e-12 for out3d, whose |Lambda|
    integrals are rounding noise in every build at t = 0). Comment lines and coordinates are
    checked on the way (identical; 1e-12)."""
    dev = {}
    for f in sorted(p for p in d_ref_dir.iterdir() if p.name.startswith("out")):
        c_ref, d_ref = read(f)
        c_oth, d_oth = read(d_other_dir / f.name)
        assert c_oth == c_ref, f.name
        assert d_oth.shape == d_ref.shape, f.name
        if f.name.startswith("out3d"):
            dev[f.name] = (np.abs(d_oth - d_ref), np.abs(d_ref).max(axis=0), 1e-12)
            continue
        ncoord = 1 if f.name.startswith(("out0d", "out1d")) else 2
        np.testing.assert_allclose(d_oth[:, :ncoord], d_ref[:, :ncoord], rtol=1e-12, atol=1e-12, err_msg=f.name)
        dev[f.name] = (np.abs(d_oth[:, ncoord:] - d_ref[:, ncoord:]), np.abs(d_ref[:, ncoord:]).max(axis=0), 0.0)
    return dev


def test_same_numbers(runs):
    """Values within 1e-8 of each column's largest magnitude, or within 10 times the spread
    between two compilations of the reference itself where that is larger. The SinhCylindrical
    centre point sits next to the axis, where H is a difference of terms about 1/rho^2 larger
    than H itself: there the two reference builds differ by about 4e-7 of the column."""
    own = _deviations(runs["ref"], runs["own"])
    ref2 = _deviations(runs["ref"], runs["ref2"])
    report, bad = {}, {}
    for name, (diff, scale, floor) in own.items():
        d2 = ref2[name][0]
        allowed = np.maximum(1e-8 * scale, 10.0 * d2.max(axis=0)) + floor
        report[name] = (float((diff / (scale + 1e-300)).max()), float((d2 / (scale + 1e-300)).max()))
        if np.any(diff > allowed):
            bad[name] = report[name]
    print({k: f"{a:.2e} (reference spread {b:.2e})" for k, (a, b) in report.items()})
    assert not bad, bad
