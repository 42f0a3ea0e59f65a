"""ctypes access to the reference oracle (oracle/_ref/<variant>/libref_<isa>.so).

Test infrastructure only: the libraries are the reference's own generated BHaH C
(emitted by nrpy's generators and compiled by oracle/gen_ref.py) plus the thin C harness
oracle/ref_harness.c. Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg as the checker / baseline; never by the product.

Variants: "sphaxi" (Spherical, symmetry_axes="2"), "sph3d" (Spherical, 3-D),
"sinh3d" (SinhSpherical, 3-D).
"""

import ctypes as C
import os
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
NGHOSTS = 3
NUM_EVOL_GFS = 24
NUM_AUXEVOL_GFS = 6


def cpu_isa() -> str:
    try:
        flags = open("/proc/cpuinfo").read()
    except OSError:
        return "avx2"
    return "avx512" if " avx512f" in flags else "avx2"


def lib_path(variant: str, isa: str = None) -> pathlib.Path:
    return REF_DIR / variant / f"libref_{isa or cpu_isa()}.so"


def available(variant: str) -> bool:
    return lib_path(variant).exists()


_LIBS = {}


def _load(variant: str, isa: str = None) -> C.CDLL:
    key = (variant, isa or cpu_isa())
    if key in _LIBS:
        return _LIBS[key]
    p = lib_path(variant, isa)
    if not p.exists():
        raise FileNotFoundError(f"oracle library {p} missing; run `python oracle/gen_ref.py`")
    lib = C.CDLL(str(p))
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.c_int
    lib.ref_create.restype = vp
    lib.ref_create.argtypes = [ip, ip, ip] + [C.c_double] * 7 + [ip]
    for f in ("ref_y_n", "ref_auxevol", "ref_k_odd"):
        getattr(lib, f).restype = dp
        getattr(lib, f).argtypes = [vp]
    lib.ref_xx.restype = dp
    lib.ref_xx.argtypes = [vp, ip]
    lib.ref_rfm.restype = dp
    lib.ref_rfm.argtypes = [vp, ip]
    lib.ref_N.argtypes = [vp, ip]
    for f in ("ref_dt", "ref_time"):
        getattr(lib, f).restype = C.c_double
        getattr(lib, f).argtypes = [vp]
    lib.ref_param_double.restype = C.c_double
    lib.ref_param_double.argtypes = [vp, ip]
    lib.ref_nn.argtypes = [vp]
    lib.ref_num_inner.argtypes = [vp]
    lib.ref_inner.restype = vp
    lib.ref_inner.argtypes = [vp]
    lib.ref_num_pure_outer.argtypes = [vp, ip, ip]
    lib.ref_pure_outer.restype = vp
    lib.ref_pure_outer.argtypes = [vp, ip, ip]
    lib.ref_evol_gf_parity.restype = C.POINTER(C.c_int8)
    for f in ("ref_Ricci", "ref_bc_radiation"):
        getattr(lib, f).argtypes = [vp, dp, dp]
    lib.ref_rhs.argtypes = [vp, dp, dp, dp]
    for f in ("ref_bc_extrap", "ref_bc_inner", "ref_enforce"):
        getattr(lib, f).argtypes = [vp, dp]
    lib.ref_step.argtypes = [vp, ip]
    lib.ref_constraints.argtypes = [vp, dp, dp, dp]
    lib.ref_dV.restype = C.c_double
    lib.ref_dV.argtypes = [vp, ip, ip, ip]
    lib.ref_diagnostics.argtypes = [vp, ip, C.c_double, C.c_double]
    lib.ref_initial_data.argtypes = [vp]
    lib.ref_nghosts.argtypes = []
    lib.ref_set_clock.argtypes = [vp, ip, C.c_double]
    lib.ref_commondata.restype = vp
    lib.ref_commondata.argtypes = [vp]
    lib.ref_t_0.restype = C.c_double
    lib.ref_t_0.argtypes = [vp]
    lib.ref_nn_0.argtypes = [vp]
    if hasattr(lib, "ref_write_checkpoint"):
        lib.ref_write_checkpoint.argtypes = [vp, C.c_double]
        lib.ref_read_checkpoint.argtypes = [vp]
        lib.ref_checkpoint_every.restype = C.c_double
        lib.ref_checkpoint_every.argtypes = [vp]
        lib.ref_offsetof_commondata_checkpoint_every.restype = C.c_size_t
        lib.ref_offsetof_commondata_checkpoint_every.argtypes = []
    lib.ref_destroy.argtypes = [vp]
    for f in ("ref_sizeof_commondata", "ref_sizeof_params", "ref_sizeof_bc_struct", "ref_sizeof_griddata",
              "ref_sizeof_innerpt", "ref_sizeof_outerpt", "ref_offsetof_params_Nxx0", "ref_offsetof_params_invdxx0",
              "ref_offsetof_params_hash", "ref_offsetof_commondata_eta", "ref_offsetof_commondata_dt",
              "ref_offsetof_commondata_bc", "ref_offsetof_commondata_nn"):
        getattr(lib, f).restype = C.c_size_t
        getattr(lib, f).argtypes = []
    _LIBS[key] = lib
    return lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


class RefGrid:
    """One grid of the reference project: set-up exactly as its generated main().

    ``isa`` picks the build ("avx512" or "avx2"; default: the host's best). The reference's
    loops over i0 advance by the SIMD width and write whole vectors: with AVX-512 (8 doubles)
    the last vector of a row runs 4 points past its interior end when Nxx0 = 1 (mod 8), into
    the first interior point of the next row, which another OpenMP thread may already have
    written. The AVX2 build (4 doubles) never runs past the end of a row."""

    def __init__(self, variant: str, Nxx, grid_physical_size: float, SINHW: float = 0.2, BH1_mass: float = 0.5,
                 BH1_posn_z: float = 0.5, BH2_mass: float = 0.5, BH2_posn_z: float = -0.5, CFL_FACTOR: float = 0.5,
                 outer_bc_type: str = "radiation", isa: str = None):
        self.variant = variant
        self.lib = _load(variant, isa)
        self.h = self.lib.ref_create(int(Nxx[0]), int(Nxx[1]), int(Nxx[2]), grid_physical_size, SINHW, BH1_mass,
                                     BH1_posn_z, BH2_mass, BH2_posn_z, CFL_FACTOR,
                                     1 if outer_bc_type == "extrapolation" else 0)
        self.N = tuple(self.lib.ref_N(self.h, d) for d in range(3))
        self.nghosts = self.lib.ref_nghosts()
        self.ntot = self.N[0] * self.N[1] * self.N[2]

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # views of the reference's own arrays (copied out)
    def _arr(self, ptr, n):
        return np.ctypeslib.as_array(ptr, shape=(n,)).copy()

    def y_n(self) -> np.ndarray:
        return self._arr(self.lib.ref_y_n(self.h), NUM_EVOL_GFS * self.ntot)

    def set_y_n(self, y: np.ndarray) -> None:
        dst = np.ctypeslib.as_array(self.lib.ref_y_n(self.h), shape=(NUM_EVOL_GFS * self.ntot,))
        dst[:] = y

    def xx(self):
        return [self._arr(self.lib.ref_xx(self.h, d), self.N[d]) for d in range(3)]

    def rfm_field(self, k: int, n: int) -> np.ndarray:
        return self._arr(self.lib.ref_rfm(self.h, k), n)

    @property
    def dt(self) -> float:
        return self.lib.ref_dt(self.h)

    @property
    def time(self) -> float:
        return self.lib.ref_time(self.h)

    def param(self, which: int) -> float:
        return self.lib.ref_param_double(self.h, which)

    # operators on caller arrays
    def ricci(self, in_gfs: np.ndarray) -> np.ndarray:
        aux = np.zeros(NUM_AUXEVOL_GFS * self.ntot)
        self.lib.ref_Ricci(self.h, _dp(in_gfs), _dp(aux))
        return aux

    def rhs(self, aux: np.ndarray, in_gfs: np.ndarray) -> np.ndarray:
        rhs = np.zeros(NUM_EVOL_GFS * self.ntot)
        self.lib.ref_rhs(self.h, _dp(aux), _dp(in_gfs), _dp(rhs))
        return rhs

    def bc_radiation(self, gfs: np.ndarray, rhs: np.ndarray) -> None:
        self.lib.ref_bc_radiation(self.h, _dp(gfs), _dp(rhs))

    def bc_extrap(self, gfs: np.ndarray) -> None:
        self.lib.ref_bc_extrap(self.h, _dp(gfs))

    def bc_inner(self, gfs: np.ndarray) -> None:
        self.lib.ref_bc_inner(self.h, _dp(gfs))

    def enforce(self, gfs: np.ndarray) -> None:
        self.lib.ref_enforce(self.h, _dp(gfs))

    def step(self, n: int = 1) -> None:
        self.lib.ref_step(self.h, n)

    def constraints(self, in_gfs: np.ndarray, aux: np.ndarray) -> np.ndarray:
        """Returns (3, ntot): H, M^2, |Lambda| (interior points written)."""
        ndiag = self.lib.ref_num_diag_gfs()
        diag = np.zeros(ndiag * self.ntot)
        self.lib.ref_constraints(self.h, _dp(in_gfs), _dp(aux), _dp(diag))
        d = diag.reshape(ndiag, self.ntot)
        return np.stack([d[self.lib.ref_diag_index(k)] for k in range(3)])

    def initial_data(self) -> None:
        """Recompute the generated initial_data() into y_n."""
        self.lib.ref_initial_data(self.h)

    def diagnostics(self, nn: int, time: float, output_every: float) -> None:
        """The generated diagnostics() driver at the present state (files in the current directory)."""
        self.lib.ref_diagnostics(self.h, int(nn), float(time), float(output_every))

    def commondata_bytes(self) -> bytes:
        """The raw bytes of the project's commondata_struct."""
        return C.string_at(self.lib.ref_commondata(self.h), self.lib.ref_sizeof_commondata())

    def set_clock(self, nn: int, time: float) -> None:
        self.lib.ref_set_clock(self.h, int(nn), float(time))

    def nn(self) -> int:
        return self.lib.ref_nn(self.h)

    def t_0(self) -> float:
        return self.lib.ref_t_0(self.h)

    def nn_0(self) -> int:
        return self.lib.ref_nn_0(self.h)

    def write_checkpoint(self, checkpoint_every: float) -> None:
        """The generated write_checkpoint() (checkpoint-enabled variant; current directory)."""
        self.lib.ref_write_checkpoint(self.h, float(checkpoint_every))

    def read_checkpoint(self) -> int:
        """The generated read_checkpoint(): 0 without a file, 1 after restoring commondata and y_n."""
        return self.lib.ref_read_checkpoint(self.h)

    def checkpoint_every(self) -> float:
        return self.lib.ref_checkpoint_every(self.h)

    def dV(self) -> np.ndarray:
        G = self.nghosts
        out = np.zeros((self.N[2], self.N[1], self.N[0]))
        for i2 in range(G, self.N[2] - G):
            for i1 in range(G, self.N[1] - G):
                for i0 in range(G, self.N[0] - G):
                    out[i2, i1, i0] = self.lib.ref_dV(self.h, i0, i1, i2)
        return out

    def interior_dV(self) -> np.ndarray:
        """The reference's volume element sqrt(det gammahat) dxx0 dxx1 dxx2 on the interior
        (shape (N2-2G, N1-2G, N0-2G)), from its own rfm arrays (|f0' f0^2 f1| dxx0 dxx1 dxx2,
        Spherical family), spot-checked against its dV() at a few points."""
        G = self.nghosts
        N0, N1, N2 = self.N
        f0, f0_D0, f1 = self.rfm_field(0, N0), self.rfm_field(1, N0), self.rfm_field(4, N1)
        x0, x1, x2 = self.xx()
        dvol = abs((x0[1] - x0[0]) * (x1[1] - x1[0]) * (x2[1] - x2[0]))
        dV = np.abs(f0_D0[None, None, :] * f0[None, None, :] ** 2 * f1[None, :, None]) * dvol
        dV = np.ascontiguousarray(np.broadcast_to(dV, (N2, N1, N0))[G:-G, G:-G, G:-G])
        rng = np.random.default_rng(0)
        for _ in range(4):
            i0, i1, i2 = (int(rng.integers(G, n - G)) for n in (N0, N1, N2))
            ref_dv = self.lib.ref_dV(self.h, i0, i1, i2)
            if abs(dV[i2 - G, i1 - G, i0 - G] - ref_dv) > 1e-12 * abs(ref_dv):
                raise RuntimeError("volume element differs from the reference's dV()")
        return dV

    def h_l2(self, y: np.ndarray, dV: np.ndarray = None) -> float:
        """sqrt(sum over the interior of H^2 dV): the reference's Ricci_eval + constraints_eval
        and its volume-integration measure, on state y."""
        G = self.nghosts
        dV = self.interior_dV() if dV is None else dV
        H = self.constraints(y, self.ricci(y))[0].reshape(self.N[2], self.N[1], self.N[0])[G:-G, G:-G, G:-G]
        return float(np.sqrt((H**2 * dV).sum()))

    def bcstruct(self):
        """(inner: structured array dstpt/srcpt/parity, outer: {(gz,dirn): array i0,i1,i2,FACEX0..2})."""
        inner_dt = np.dtype([("dstpt", "<i4"), ("srcpt", "<i4"), ("parity", "i1", (10,)), ("_pad", "V2")])
        outer_dt = np.dtype([("i0", "<i2"), ("i1", "<i2"), ("i2", "<i2"), ("FACEX0", "i1"), ("FACEX1", "i1"),
                             ("FACEX2", "i1"), ("_pad", "V1")])
        assert inner_dt.itemsize == self.lib.ref_sizeof_innerpt()
        assert outer_dt.itemsize == self.lib.ref_sizeof_outerpt()
        ni = self.lib.ref_num_inner(self.h)
        buf = (C.c_char * (ni * inner_dt.itemsize)).from_address(self.lib.ref_inner(self.h))
        inner = np.frombuffer(bytes(buf), dtype=inner_dt)
        outer = {}
        for gz in range(self.nghosts):
            for d in range(3):
                n = self.lib.ref_num_pure_outer(self.h, gz, d)
                if n:
                    b = (C.c_char * (n * outer_dt.itemsize)).from_address(self.lib.ref_pure_outer(self.h, gz, d))
                    outer[(gz, d)] = np.frombuffer(bytes(b), dtype=outer_dt)
                else:
                    outer[(gz, d)] = np.zeros(0, dtype=outer_dt)
        return inner, outer


def cuda_available(variant: str = "sinh3d_cuda") -> bool:
    return (REF_DIR / variant / "libref_cuda.so").exists()


_CUDA_LIBS = {}


def _load_cuda(variant: str) -> C.CDLL:
    if variant in _CUDA_LIBS:
        return _CUDA_LIBS[variant]
    p = REF_DIR / variant / "libref_cuda.so"
    if not p.exists():
        raise FileNotFoundError(f"reference CUDA library {p} missing; run `python oracle/gen_ref.py --variants {variant}`")
    lib = C.CDLL(str(p))
    vp, ip, dp = C.c_void_p, C.c_int, C.POINTER(C.c_double)
    lib.refc_create.restype = vp
    lib.refc_create.argtypes = [ip, ip, ip] + [C.c_double] * 7
    lib.refc_N.argtypes = [vp, ip]
    lib.refc_dt.restype = C.c_double
    lib.refc_dt.argtypes = [vp]
    lib.refc_nn.argtypes = [vp]
    lib.refc_set_y_n.argtypes = [vp, dp]
    lib.refc_get_y_n.argtypes = [vp, dp]
    lib.refc_steps.restype = C.c_double
    lib.refc_steps.argtypes = [vp, ip]
    lib.refc_destroy.argtypes = [vp]
    _CUDA_LIBS[variant] = lib
    return lib


class RefCudaGrid:
    """One SinhSpherical grid of the reference's own CUDA build (nrpy --cuda, sm_100a): set up
    as its generated main() and numerical_grids_and_timestep() do, stepped by its generated
    MoL_step_forward_in_time on the current GPU."""

    def __init__(self, Nxx, grid_physical_size: float, SINHW: float = 0.2, BH1_mass: float = 0.5,
                 BH1_posn_z: float = 0.5, BH2_mass: float = 0.5, BH2_posn_z: float = -0.5, CFL_FACTOR: float = 0.5,
                 variant: str = "sinh3d_cuda"):
        self.lib = _load_cuda(variant)
        self.h = self.lib.refc_create(int(Nxx[0]), int(Nxx[1]), int(Nxx[2]), grid_physical_size, SINHW, BH1_mass,
                                      BH1_posn_z, BH2_mass, BH2_posn_z, CFL_FACTOR)
        self.N = tuple(self.lib.refc_N(self.h, d) for d in range(3))
        self.ntot = self.N[0] * self.N[1] * self.N[2]

    @property
    def dt(self) -> float:
        return self.lib.refc_dt(self.h)

    def y_n(self) -> np.ndarray:
        out = np.zeros(NUM_EVOL_GFS * self.ntot)
        if self.lib.refc_get_y_n(self.h, _dp(out)) != 0:
            raise RuntimeError("reference CUDA build: device-to-host copy failed")
        return out

    def set_y_n(self, y: np.ndarray) -> None:
        y = np.ascontiguousarray(y, dtype=np.float64)
        if self.lib.refc_set_y_n(self.h, _dp(y)) != 0:
            raise RuntimeError("reference CUDA build: host-to-device copy failed")

    def steps(self, n: int) -> float:
        """n generated MoL_step_forward_in_time calls; device milliseconds (CUDA events)."""
        ms = self.lib.refc_steps(self.h, int(n))
        if ms < 0:
            raise RuntimeError("reference CUDA build: a CUDA error occurred during the steps")
        return ms

    def close(self):
        if self.h:
            self.lib.refc_destroy(self.h)
            self.h = None


def struct_layout(variant: str) -> dict:
    lib = _load(variant)
    names = ["sizeof_commondata", "sizeof_params", "sizeof_bc_struct", "sizeof_griddata", "sizeof_innerpt",
             "sizeof_outerpt", "offsetof_params_Nxx0", "offsetof_params_invdxx0", "offsetof_params_hash",
             "offsetof_commondata_eta", "offsetof_commondata_dt", "offsetof_commondata_bc", "offsetof_commondata_nn"]
    return {n: int(getattr(lib, "ref_" + n)()) for n in names}


def set_threads(n: int) -> None:
    os.environ["OMP_NUM_THREADS"] = str(n)


# Perturbation amplitudes per gridfunction: every term of the RHS is exercised when all 24
# fields are nonzero and smooth. alpha and cf are scaled multiplicatively to stay positive.
def perturbed_state(rg: "RefGrid", seed: int = 1, amp: float = 0.05) -> np.ndarray:
    """Reference initial data plus seeded smooth perturbations of all 24 gridfunctions,
    with the reference's own extrapolation + inner boundary conditions applied."""
    rng = np.random.default_rng(seed)
    y = rg.y_n().reshape(NUM_EVOL_GFS, rg.N[2], rg.N[1], rg.N[0])
    x0, x1, x2 = rg.xx()
    X0 = x0[None, None, :]
    X1 = x1[None, :, None]
    X2 = x2[:, None, None]
    x0max = max(abs(x0).max(), 1e-300)
    for gf in range(NUM_EVOL_GFS):
        k0, k1, k2 = rng.uniform(0.5, 2.0, 3)
        p0, p1, p2 = rng.uniform(0, 2 * np.pi, 3)
        a = amp * rng.uniform(0.5, 1.0)
        field = np.sin(k0 * np.pi * X0 / x0max + p0) * np.cos(k1 * X1 + p1) * np.cos(k2 * X2 + p2)
        if gf in (6, 10):  # alpha, cf
            y[gf] *= 1.0 + a * field
        else:
            y[gf] += a * field
    flat = np.ascontiguousarray(y.reshape(-1))
    rg.bc_extrap(flat)
    return flat
