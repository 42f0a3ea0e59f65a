"""ctypes binding of libbssn_b200.so (the C ABI in include/bssn_b200.h).

The struct classes mirror the C layouts field by field. Loading fails loudly when the
library has not been built: there is no fallback implementation.

The interior finite-difference order is chosen per process by the environment variable
BSSN_B200_FD_ORDER (4, the default: libbssn_b200.so; 8: libbssn_b200_fd8.so). NGHOSTS, and
with it the bc_info_struct / bc_struct layouts, follow it; load() checks that the library was
built for the same order.
"""

import ctypes as C
import os
import pathlib

REAL = C.c_double
FD_ORDER = int(os.environ.get("BSSN_B200_FD_ORDER", "4"))
if FD_ORDER not in (4, 8):
    raise ValueError(f"BSSN_B200_FD_ORDER={FD_ORDER}: libbssn_b200 is built for 4 and 8")
NGHOSTS = FD_ORDER // 2 + 1
NUM_EVOL_GFS = 24
NUM_AUXEVOL_GFS = 6
NUM_DIAG_GFS = 3
# The generated project's diagnostic gridfunctions (BSSN_B200_DIAG_*GF of bssn_b200.h).
DIAG_GFS = ["DIAG_GRIDINDEX", "DIAG_HAMILTONIAN", "DIAG_LAMBDA_CONSTRAINT", "DIAG_LAPSE", "DIAG_MSQUARED",
            "DIAG_RBARDD00", "DIAG_RBARDD01", "DIAG_RBARDD02", "DIAG_RBARDD11", "DIAG_RBARDD12", "DIAG_RBARDD22",
            "DIAG_W"]
TOTAL_NUM_DIAG_GFS = len(DIAG_GFS)
MAXNUMGRIDS = 15
SPHERICAL = 1307621703
SINHSPHERICAL = 579707936
SINHCYLINDRICAL = 1325205359
COORD_HASH = {"Spherical": SPHERICAL, "SinhSpherical": SINHSPHERICAL, "SinhCylindrical": SINHCYLINDRICAL}

GF_NAMES = [
    "aDD00", "aDD01", "aDD02", "aDD11", "aDD12", "aDD22", "alpha", "betU0", "betU1", "betU2",
    "cf", "hDD00", "hDD01", "hDD02", "hDD11", "hDD12", "hDD22", "lambdaU0", "lambdaU1",
    "lambdaU2", "trK", "vetU0", "vetU1", "vetU2",
]
GF = {n: i for i, n in enumerate(GF_NAMES)}
# evol_gf_parity of the generated BHaH_defines.h
EVOL_GF_PARITY = [4, 5, 6, 7, 8, 9, 0, 1, 2, 3, 0, 4, 5, 6, 7, 8, 9, 1, 2, 3, 0, 1, 2, 3]


class Timespec(C.Structure):
    _fields_ = [("tv_sec", C.c_long), ("tv_nsec", C.c_long)]


class CommondataStruct(C.Structure):
    _fields_ = [
        ("BH1_mass", REAL), ("BH1_posn_x", REAL), ("BH1_posn_y", REAL), ("BH1_posn_z", REAL),
        ("BH2_mass", REAL), ("BH2_posn_x", REAL), ("BH2_posn_y", REAL), ("BH2_posn_z", REAL),
        ("CFL_FACTOR", REAL), ("KreissOliger_strength_gauge", REAL),
        ("KreissOliger_strength_nongauge", REAL), ("convergence_factor", REAL),
        ("diagnostics_output_every", REAL), ("dt", REAL), ("eta", REAL), ("t_0", REAL),
        ("t_final", REAL), ("time", REAL), ("start_wallclock_time", Timespec),
        ("outer_bc_type", C.c_char * 50), ("NUMGRIDS", C.c_int), ("nn", C.c_int), ("nn_0", C.c_int),
        ("output_progress_every", C.c_int),
    ]


class CheckpointCommondata(C.Structure):
    """commondata_struct of a project that registers checkpointing (checkpoint files begin with it)."""
    _fields_ = [
        ("BH1_mass", REAL), ("BH1_posn_x", REAL), ("BH1_posn_y", REAL), ("BH1_posn_z", REAL),
        ("BH2_mass", REAL), ("BH2_posn_x", REAL), ("BH2_posn_y", REAL), ("BH2_posn_z", REAL),
        ("CFL_FACTOR", REAL), ("KreissOliger_strength_gauge", REAL),
        ("KreissOliger_strength_nongauge", REAL), ("checkpoint_every", REAL), ("convergence_factor", REAL),
        ("diagnostics_output_every", REAL), ("dt", REAL), ("eta", REAL), ("t_0", REAL),
        ("t_final", REAL), ("time", REAL), ("start_wallclock_time", Timespec),
        ("outer_bc_type", C.c_char * 50), ("NUMGRIDS", C.c_int), ("nn", C.c_int), ("nn_0", C.c_int),
        ("output_progress_every", C.c_int),
    ]


class ParamsStruct(C.Structure):
    _fields_ = [
        ("AMPL", REAL), ("AMPLRHO", REAL), ("AMPLZ", REAL), ("Cart_originx", REAL), ("Cart_originy", REAL),
        ("Cart_originz", REAL), ("PI", REAL), ("RHOMAX", REAL), ("RMAX", REAL), ("SINHW", REAL), ("SINHWRHO", REAL),
        ("SINHWZ", REAL), ("ZMAX", REAL), ("ZMIN", REAL), ("dxx0", REAL), ("dxx1", REAL), ("dxx2", REAL),
        ("grid_hole_radius", REAL), ("grid_physical_size", REAL), ("invdxx0", REAL), ("invdxx1", REAL),
        ("invdxx2", REAL), ("xmax", REAL), ("xmin", REAL), ("xxmax0", REAL), ("xxmax1", REAL),
        ("xxmax2", REAL), ("xxmin0", REAL), ("xxmin1", REAL), ("xxmin2", REAL), ("ymax", REAL),
        ("ymin", REAL), ("zmax", REAL), ("zmin", REAL), ("grid_rotates", C.c_bool), ("is_host", C.c_bool),
        ("CoordSystemName", C.c_char * 100), ("gridname", C.c_char * 100), ("CoordSystem_hash", C.c_int),
        ("Nxx0", C.c_int), ("Nxx1", C.c_int), ("Nxx2", C.c_int), ("Nxx_plus_2NGHOSTS0", C.c_int),
        ("Nxx_plus_2NGHOSTS1", C.c_int), ("Nxx_plus_2NGHOSTS2", C.c_int), ("grid_idx", C.c_int),
    ]


class RfmStruct(C.Structure):
    _fields_ = [(n, C.POINTER(REAL)) for n in (
        "f0_of_xx0", "f0_of_xx0__D0", "f0_of_xx0__DD00", "f0_of_xx0__DDD000",
        "f1_of_xx1", "f1_of_xx1__D1", "f1_of_xx1__DD11")]


class InnerptBcStruct(C.Structure):
    _fields_ = [("dstpt", C.c_int), ("srcpt", C.c_int), ("parity", C.c_int8 * 10)]


class OuterptBcStruct(C.Structure):
    _fields_ = [("i0", C.c_short), ("i1", C.c_short), ("i2", C.c_short),
                ("FACEX0", C.c_int8), ("FACEX1", C.c_int8), ("FACEX2", C.c_int8)]


class BcInfoStruct(C.Structure):
    _fields_ = [
        ("num_inner_boundary_points", C.c_int),
        ("num_pure_outer_boundary_points", (C.c_int * 3) * NGHOSTS),
        ("bc_loop_bounds", ((C.c_int * 6) * 6) * NGHOSTS),
    ]


class BcStruct(C.Structure):
    _fields_ = [
        ("inner_bc_array", C.POINTER(InnerptBcStruct)),
        ("pure_outer_bc_array", C.POINTER(OuterptBcStruct) * (NGHOSTS * 3)),
        ("bc_info", BcInfoStruct),
    ]


class MoLGridfunctionsStruct(C.Structure):
    _fields_ = [(n, C.POINTER(REAL)) for n in (
        "y_n_gfs", "y_nplus1_running_total_gfs", "k_odd_gfs", "k_even_gfs", "auxevol_gfs")]


class GriddataStruct(C.Structure):
    _fields_ = [
        ("xx", C.POINTER(REAL) * 3),
        ("bcstruct", BcStruct),
        ("gridfuncs", MoLGridfunctionsStruct),
        ("params", ParamsStruct),
        ("rfmstruct", C.POINTER(RfmStruct)),
    ]


class BssnError(RuntimeError):
    """A libbssn_b200 call returned a nonzero status."""


def _lib_path() -> pathlib.Path:
    env = os.environ.get("BSSN_B200_LIB")
    if env:
        return pathlib.Path(env)
    name = "libbssn_b200.so" if FD_ORDER == 4 else f"libbssn_b200_fd{FD_ORDER}.so"
    return pathlib.Path(__file__).resolve().parent / name


_LIB = None

# (name, restype, argtypes) of every C-ABI symbol; used for binding and by the export test.
PR = C.POINTER(REAL)
PCD = C.POINTER(CommondataStruct)
PP = C.POINTER(ParamsStruct)
PRFM = C.POINTER(RfmStruct)
PBC = C.POINTER(BcStruct)
PGD = C.POINTER(GriddataStruct)
PMOL = C.POINTER(MoLGridfunctionsStruct)
XX = PR * 3
V = C.c_void_p
SIGNATURES = [
    ("commondata_struct_set_to_default", None, [PCD]),
    ("params_struct_set_to_default", None, [PCD, PGD]),
    ("numerical_grid_params_Nxx_dxx_xx", None, [PCD, PP, XX, C.c_int * 3, C.c_bool]),
    ("rfm_precompute_malloc", None, [PCD, PP, PRFM]),
    ("rfm_precompute_defines", None, [PCD, PP, PRFM, XX]),
    ("rfm_precompute_free", None, [PCD, PP, PRFM]),
    ("bcstruct_set_up", None, [PCD, PP, XX, PBC]),
    ("bcstruct_free", None, [PBC]),
    ("cfl_limited_timestep", None, [PCD, PP, XX]),
    ("initial_data", None, [PCD, PGD]),
    ("MoL_malloc_y_n_gfs", None, [PCD, PP, PMOL]),
    ("MoL_malloc_intermediate_stage_gfs", None, [PCD, PP, PMOL]),
    ("MoL_free_intermediate_stage_gfs", None, [PMOL]),
    ("Ricci_eval", None, [PP, PRFM, PR, PR]),
    ("rhs_eval", None, [PCD, PP, PRFM, PR, PR, PR]),
    ("apply_bcs_outerradiation_and_inner", None, [PCD, PP, PBC, XX, PR, PR, PR, PR]),
    ("apply_bcs_outerextrap_and_inner", None, [PCD, PP, PBC, PR]),
    ("apply_bcs_inner_only", None, [PCD, PP, PBC, PR]),
    ("enforce_detgammabar_equals_detgammahat", None, [PP, PRFM, PR, PR]),
    ("MoL_step_forward_in_time", None, [PCD, PGD]),
    ("constraints_eval", None, [PCD, PP, PRFM, PR, PR, PR]),
    ("diagnostics", None, [PCD, PGD]),
    ("diagnostic_gfs_set", None, [PCD, PGD, C.POINTER(PR)]),
    ("diagnostics_nearest", None, [PCD, PGD, C.POINTER(PR)]),
    ("diagnostics_volume_integration", None, [PCD, PGD, C.POINTER(PR)]),
    ("progress_indicator", None, [PCD, PGD]),
    ("bssn_b200_diagnostics", C.c_int, [PCD, PGD, V]),
    ("bssn_b200_last_error", C.c_char_p, []),
    ("bssn_b200_version", C.c_char_p, []),
    ("bssn_b200_fd_order", C.c_int, []),
    ("bssn_b200_set_symmetry_axes", C.c_int, [C.c_char_p]),
    ("bssn_b200_ricci_eval", C.c_int, [PP, PRFM, PR, PR, V]),
    ("bssn_b200_rhs_eval", C.c_int, [PCD, PP, PRFM, PR, PR, PR, V]),
    ("bssn_b200_rhs_eval_mixed", C.c_int, [PCD, PP, PRFM, PR, PR, PR, V]),
    ("bssn_b200_apply_bcs_outerradiation_and_inner", C.c_int, [PCD, PP, PBC, XX, PR, PR, PR, PR, V]),
    ("bssn_b200_apply_bcs_outerextrap_and_inner", C.c_int, [PP, PBC, PR, V]),
    ("bssn_b200_apply_bcs_inner_only", C.c_int, [PP, PBC, PR, C.c_int, C.POINTER(C.c_int8), V]),
    ("bssn_b200_enforce_detgammabar_equals_detgammahat", C.c_int, [PP, PRFM, PR, V]),
    ("bssn_b200_constraints_eval", C.c_int, [PCD, PP, PRFM, PR, PR, PR, V]),
    ("bssn_b200_constraint_integrals", C.c_int, [PP, PRFM, PR, C.POINTER(C.c_double), V]),
    ("bssn_b200_constraint_integrals_noalloc", C.c_int, [PP, PRFM, PR, C.POINTER(C.c_double), V]),
    ("bssn_b200_mol_step", C.c_int, [PCD, PGD, C.c_int, C.c_int, V]),
    ("bssn_b200_stepper_create", C.c_int, [PCD, PGD, C.c_int, C.c_int, C.c_int, V, C.POINTER(V)]),
    ("bssn_b200_stepper_run", C.c_int, [V, C.c_int]),
    ("bssn_b200_stepper_destroy", C.c_int, [V]),
    ("bssn_b200_stepper_kernel_nodes", C.c_int, [V, C.POINTER(C.c_ulonglong)]),
    ("bssn_b200_kernel_launches", C.c_ulonglong, []),
    ("bssn_b200_rhs_fused_stage", C.c_int, [PCD, PGD, C.c_int, C.c_int, V]),
    ("bssn_b200_fp64_fma_rate", C.c_int, [C.c_int, C.POINTER(C.c_double), V]),
    ("bssn_b200_batch_create", C.c_int, [C.c_int, C.POINTER(PCD), C.POINTER(PGD), C.c_int, C.c_int, C.c_int, V,
                                         C.POINTER(V)]),
    ("bssn_b200_batch_run", C.c_int, [V, C.c_int]),
    ("bssn_b200_batch_info", C.c_int, [V, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                       C.POINTER(C.c_ulonglong)]),
    ("bssn_b200_batch_tile_fill", C.c_int, [V, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    ("bssn_b200_batch_destroy", C.c_int, [V]),
    ("bssn_b200_adjoint_create", C.c_int, [PCD, PGD, C.c_int, C.c_int, V, C.POINTER(V)]),
    ("bssn_b200_adjoint_forward", C.c_int, [V, C.POINTER(C.c_double)]),
    ("bssn_b200_adjoint_backward", C.c_int, [V, C.c_double, PR, C.POINTER(C.c_double)]),
    ("bssn_b200_adjoint_functional", C.c_int, [V, PR, C.POINTER(C.c_double)]),
    ("bssn_b200_adjoint_functional_vjp", C.c_int, [V, PR, C.c_double, PR]),
    ("bssn_b200_adjoint_step_vjp", C.c_int, [V, PR, PR]),
    ("bssn_b200_adjoint_id_vjp", C.c_int, [V, PR, C.POINTER(C.c_double)]),
    ("bssn_b200_adjoint_destroy", C.c_int, [V]),
    ("bssn_b200_write_checkpoint", C.c_int, [PCD, REAL, PGD, V]),
    ("bssn_b200_read_checkpoint", C.c_int, [PCD, PR, PGD, V]),
    ("bssn_b200_memcpy", C.c_int, [V, V, C.c_size_t, C.c_int]),
    ("bssn_b200_device_synchronize", C.c_int, []),
]
DATA_SYMBOLS = ["bssn_b200_evol_gf_parity", "gridfunctions_wavespeed", "gridfunctions_f_infinity"]


def load(path=None) -> C.CDLL:
    """Load and bind libbssn_b200.so (raises OSError if it is missing)."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = pathlib.Path(path) if path else _lib_path()
    if not p.exists():
        raise OSError(f"{p.name} not found at {p}; build it with `python -m nrpy_b200.build --fd-order {FD_ORDER}`")
    lib = C.CDLL(str(p))
    for name, res, args in SIGNATURES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if lib.bssn_b200_fd_order() != FD_ORDER:
        raise OSError(f"{p} is built for fd_order {lib.bssn_b200_fd_order()}, this process expects {FD_ORDER} "
                      "(BSSN_B200_FD_ORDER)")
    if path is None:
        _LIB = lib
    return lib


def check(rc: int) -> None:
    if rc != 0:
        msg = load().bssn_b200_last_error().decode(errors="replace")
        raise BssnError(f"libbssn_b200 status {rc}: {msg}")
