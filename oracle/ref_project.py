"""Emit a reference BHaH BSSN project (generated C/OpenMP) for use as the oracle.

Test infrastructure only: this script imports the nrpy package (the reference) and
runs its own code generators. It follows the registration sequence of
nrpy/examples/two_blackholes_collide.py:60-440 with the settings the workloads need:

* Kreiss-Oliger dissipation ON (the example has it off, two_blackholes_collide.py:124),
  CAKO on, strengths 0.3 (rhs_eval.py:48-49);
* CoordSystem Spherical, SinhSpherical or SinhCylindrical; ``--axisym`` sets the
  axisymmetry axis of the coordinate system (symmetry_axes="2", the phi index of the
  Spherical family, two_blackholes_collide.py:141-143; "1" for the cylindrical family,
  blackhole_spectroscopy.py:153), otherwise the grid is full 3-D;
* SinhCylindrical as blackhole_spectroscopy.py:60-160 sets it up: AMPLRHO = AMPLZ =
  grid_physical_size, SINHWRHO = SINHWZ = 0.2, CFL_FACTOR 0.5;
* the BHaHAHA horizon finder off (it is a diagnostic, not the step);
* every coordinate system's CodeParameters registered ("All"), so that one
  params_struct layout serves every project variant;
* ``--checkpoint`` also registers write_checkpoint/read_checkpoint (checkpointing.py:473-490),
  which adds the REAL CodeParameter checkpoint_every to commondata_struct;
* ``--fd-order N`` sets the interior finite-difference order (4 by default; NGHOSTS = N/2 + 1),
  the outer radiation condition staying at radiation_BC_fd_order = 4;
* the reference metrics of Spherical, SinhSpherical, SinhCylindrical and Cylindrical (the
  eigen-coordinates of SinhCylindrical, whose bcstruct set-up instantiates it) are all
  instantiated, so that every variant's params_struct carries the CodeParameters of all four
  and one layout serves every project variant.

Run it with the reference on PYTHONPATH (oracle/gen_ref.py does this).
"""

import argparse
import os
import shutil

import nrpy.helpers.parallel_codegen as pcg
import nrpy.params as par
import nrpy.reference_metric as refmetric
from nrpy.helpers.generic import copy_files
from nrpy.infrastructures import BHaH

ap = argparse.ArgumentParser()
ap.add_argument("--coord", default="Spherical")
ap.add_argument("--axisym", action="store_true")
ap.add_argument("--project-dir", required=True)
ap.add_argument("--cuda", action="store_true")
ap.add_argument("--checkpoint", action="store_true")
ap.add_argument("--fd-order", type=int, default=4)
args = ap.parse_args()

parallelization = "cuda" if args.cuda else "openmp"
par.set_parval_from_str("Infrastructure", "BHaH")
par.set_parval_from_str("parallelization", parallelization)
par.set_parval_from_str("fp_type", "double")

CoordSystem = args.coord
set_of_CoordSystems = {CoordSystem}
grid_physical_size = 7.5 if CoordSystem == "Spherical" else 10.0
Nxx_dict = {"Spherical": [72, 12, 2], "SinhSpherical": [256, 64, 64], "SinhCylindrical": [400, 2, 1200]}
OMP_collapse = 2
if args.axisym:
    par.set_parval_from_str("symmetry_axes", "1" if "Cylindrical" in CoordSystem else "2")

project_dir = args.project_dir
shutil.rmtree(project_dir, ignore_errors=True)
par.set_parval_from_str("enable_parallel_codegen", True)
par.set_parval_from_str("fd_order", args.fd_order)
par.set_parval_from_str("CoordSystem_to_register_CodeParameters", "All")
# Instantiate the four reference metrics so that all register their CodeParameters (RMAX for
# Spherical; AMPL, SINHW for SinhSpherical; AMPLRHO, AMPLZ, SINHWRHO, SINHWZ for
# SinhCylindrical; RHOMAX, ZMIN, ZMAX for Cylindrical): every variant then shares one
# params_struct layout.
for _coord in ("Spherical", "SinhSpherical", "SinhCylindrical", "Cylindrical"):
    _ = refmetric.reference_metric[_coord]

if parallelization == "cuda":
    BHaH.parallelization.cuda_utilities.register_CFunctions_HostDevice__operations()
    BHaH.parallelization.cuda_utilities.register_CFunction_find_global_minimum()
    BHaH.parallelization.cuda_utilities.register_CFunction_find_global_sum()

BHaH.general_relativity.initial_data.register_CFunction_initial_data(
    IDtype="BrillLindquist",
    IDCoordSystem="Cartesian",
    set_of_CoordSystems=set_of_CoordSystems,
    ID_persist_struct_str="",
)
BHaH.numerical_grids_and_timestep.register_CFunctions(
    set_of_CoordSystems=set_of_CoordSystems,
    list_of_grid_physical_sizes=[grid_physical_size],
    Nxx_dict=Nxx_dict,
    enable_rfm_precompute=True,
    enable_CurviBCs=True,
)
BHaH.general_relativity.diagnostic_gfs_set.register_CFunction_diagnostic_gfs_set(
    enable_interp_diagnostics=False, enable_psi4=False
)
BHaH.general_relativity.diagnostics_nearest.register_CFunction_diagnostics_nearest()
BHaH.general_relativity.diagnostics_volume_integration.register_CFunction_diagnostics_volume_integration()
BHaH.rfm_precompute.register_CFunctions_rfm_precompute(
    set_of_CoordSystems=set_of_CoordSystems
)
BHaH.general_relativity.rhs_eval.register_CFunction_rhs_eval(
    CoordSystem=CoordSystem,
    enable_rfm_precompute=True,
    enable_RbarDD_gridfunctions=True,
    enable_T4munu=False,
    enable_intrinsics=True,
    enable_fd_functions=True,
    LapseEvolutionOption="OnePlusLog",
    ShiftEvolutionOption="GammaDriving2ndOrder_Covariant",
    enable_KreissOliger_dissipation=True,
    enable_CAKO=True,
    OMP_collapse=OMP_collapse,
)
BHaH.general_relativity.Ricci_eval.register_CFunction_Ricci_eval(
    CoordSystem=CoordSystem,
    enable_intrinsics=True,
    enable_fd_functions=True,
    OMP_collapse=OMP_collapse,
)
if parallelization == "cuda":
    BHaH.general_relativity.Ricci_eval.register_CFunction_Ricci_eval(
        CoordSystem=CoordSystem,
        enable_intrinsics=True,
        enable_fd_functions=True,
        OMP_collapse=OMP_collapse,
        host_only_version=True,
    )
BHaH.general_relativity.enforce_detgammabar_equals_detgammahat.register_CFunction_enforce_detgammabar_equals_detgammahat(
    CoordSystem=CoordSystem,
    enable_rfm_precompute=True,
    enable_fd_functions=True,
    OMP_collapse=OMP_collapse,
)
BHaH.diagnostics.diagnostics.register_all_diagnostics(
    project_dir=project_dir,
    set_of_CoordSystems=set_of_CoordSystems,
    default_diagnostics_out_every=0.25,
    enable_nearest_diagnostics=True,
    enable_interp_diagnostics=False,
    enable_volume_integration_diagnostics=True,
    enable_rfm_precompute=True,
    enable_RbarDD_gridfunctions=True,
    enable_free_auxevol=False,
    enable_psi4_diagnostics=False,
    enable_bhahaha=False,
    enable_raytracing_data_output=False,
)
BHaH.general_relativity.constraints_eval.register_CFunction_constraints_eval(
    CoordSystem=CoordSystem,
    enable_T4munu=False,
    enable_fd_functions=True,
    OMP_collapse=OMP_collapse,
)

if __name__ == "__main__":
    pcg.do_parallel_codegen()

BHaH.CurviBoundaryConditions.register_all.register_C_functions(
    set_of_CoordSystems=set_of_CoordSystems, radiation_BC_fd_order=4
)
rhs_string = """Ricci_eval(params, rfmstruct, RK_INPUT_GFS, auxevol_gfs);
rhs_eval(commondata, params, rfmstruct, auxevol_gfs, RK_INPUT_GFS, RK_OUTPUT_GFS);
if (strncmp(commondata->outer_bc_type, "radiation", 50) == 0)
  apply_bcs_outerradiation_and_inner(commondata, params, bcstruct, griddata[grid].xx,
                                     gridfunctions_wavespeed,gridfunctions_f_infinity,
                                     RK_INPUT_GFS, RK_OUTPUT_GFS);"""
BHaH.MoLtimestepping.register_all.register_CFunctions(
    MoL_method="RK4",
    rhs_string=rhs_string,
    post_rhs_string="""if (strncmp(commondata->outer_bc_type, "extrapolation", 50) == 0)
  apply_bcs_outerextrap_and_inner(commondata, params, bcstruct, RK_OUTPUT_GFS);
  enforce_detgammabar_equals_detgammahat(params, rfmstruct, RK_OUTPUT_GFS, auxevol_gfs);""",
    enable_rfm_precompute=True,
    enable_curviBCs=True,
    rational_const_alias=("static constexpr" if parallelization == "cuda" else "static const"),
)
BHaH.xx_tofrom_Cart.register_CFunction_Cart_to_xx_and_nearest_i0i1i2_assume_valid(CoordSystem)
BHaH.xx_tofrom_Cart.register_CFunction_xx_to_Cart(CoordSystem)
BHaH.diagnostics.progress_indicator.register_CFunction_progress_indicator()
if args.checkpoint:
    import nrpy.infrastructures.BHaH.checkpointing as checkpointing

    checkpointing.register_CFunctions(default_checkpoint_every=2.0)
BHaH.general_relativity.basis_transforms.register_all.register_CFunctions(
    set_of_CoordSystems=set_of_CoordSystems
)
BHaH.rfm_wrapper_functions.register_CFunctions_CoordSystem_wrapper_funcs()

par.adjust_CodeParam_default("t_final", grid_physical_size)
if CoordSystem == "SinhSpherical":
    par.adjust_CodeParam_default("SINHW", 0.2)
if CoordSystem == "SinhCylindrical":
    par.adjust_CodeParam_default("AMPLRHO", grid_physical_size)
    par.adjust_CodeParam_default("AMPLZ", grid_physical_size)
    par.adjust_CodeParam_default("SINHWRHO", 0.2)
    par.adjust_CodeParam_default("SINHWZ", 0.2)
    par.adjust_CodeParam_default("CFL_FACTOR", 0.5)
par.adjust_CodeParam_default("eta", 1.0)
par.adjust_CodeParam_default("BH1_mass", 0.5)
par.adjust_CodeParam_default("BH2_mass", 0.5)
par.adjust_CodeParam_default("BH1_posn_z", 0.5)
par.adjust_CodeParam_default("BH2_posn_z", -0.5)

BHaH.diagnostics.diagnostic_gfs_h_create.diagnostics_gfs_h_create(project_dir=project_dir)
BHaH.CodeParameters.write_CodeParameters_h_files(project_dir=project_dir)
BHaH.CodeParameters.register_CFunctions_params_commondata_struct_set_to_default()
BHaH.cmdline_input_and_parfiles.generate_default_parfile(
    project_dir=project_dir, project_name="bssn_ref"
)
BHaH.cmdline_input_and_parfiles.register_CFunction_cmdline_input_and_parfile_parser(
    project_name="bssn_ref", cmdline_inputs=["convergence_factor"]
)
BHaH.BHaH_device_defines_h.output_device_headers(project_dir, num_streams=1)
BHaH.BHaH_defines_h.output_BHaH_defines_h(
    project_dir=project_dir,
    enable_rfm_precompute=True,
    fin_NGHOSTS_add_one_for_upwinding_or_KO=True,
    DOUBLE_means="REAL",
    restrict_pointer_type="*" if parallelization == "cuda" else "*restrict",
)
BHaH.main_c.register_CFunction_main_c(
    initial_data_desc="BrillLindquist",
    MoL_method="RK4",
    boundary_conditions_desc="outgoing radiation",
)
BHaH.griddata_commondata.register_CFunction_griddata_free(
    enable_rfm_precompute=True, enable_CurviBCs=True, enable_bhahaha=False
)
intrinsics = ["simd_intrinsics.h"] + (["cuda_intrinsics.h"] if args.cuda else [])
copy_files(
    package="nrpy.helpers",
    filenames_list=intrinsics,
    project_dir=project_dir,
    subdirectory="intrinsics",
)
BHaH.Makefile_helpers.output_CFunctions_function_prototypes_and_construct_Makefile(
    project_dir=project_dir,
    project_name="bssn_ref",
    exec_or_library_name="bssn_ref",
    compiler_opt_option=("nvcc" if args.cuda else "default"),
    CC=("nvcc" if args.cuda else "autodetect"),
    src_code_file_ext=("cu" if args.cuda else "c"),
)
print("generated", project_dir)
