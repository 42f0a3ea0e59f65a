// Oracle harness: a thin C driver around the reference's generated BHaH project.
//
// Test infrastructure only. It is compiled together with the C sources that the
// reference's own generator emits (oracle/gen_ref.py) and exposes flat entry points
// that ctypes can call without mirroring every generated struct. It performs the same
// set-up sequence as the generated main() (nrpy/infrastructures/BHaH/main_c.py:125-343):
// defaults -> numerical_grid_params_Nxx_dxx_xx -> rfm_precompute -> bcstruct_set_up
// -> cfl_limited_timestep -> initial_data -> MoL_malloc_intermediate_stage_gfs,
// with the grid size, resolution and Brill-Lindquist parameters given by the caller.
#include "BHaH_defines.h"
#include "BHaH_function_prototypes.h"
#include "diagnostics/diagnostic_gfs.h"
#include <stddef.h>

typedef struct {
  commondata_struct commondata;
  griddata_struct *griddata;  // malloc'd as in main(); griddata_free() releases it
} ref_sim;

ref_sim *ref_create(const int Nx0, const int Nx1, const int Nx2, const double grid_physical_size, const double sinhw,
                    const double m1, const double z1, const double m2, const double z2, const double cfl,
                    const int outer_bc_extrapolation) {
  ref_sim *s = (ref_sim *)calloc(1, sizeof(ref_sim));
  s->griddata = (griddata_struct *)calloc(MAXNUMGRIDS, sizeof(griddata_struct));
  commondata_struct_set_to_default(&s->commondata);
  s->commondata.BH1_mass = m1;
  s->commondata.BH1_posn_z = z1;
  s->commondata.BH2_mass = m2;
  s->commondata.BH2_posn_z = z2;
  s->commondata.CFL_FACTOR = cfl;
  s->commondata.NUMGRIDS = 1;
  if (outer_bc_extrapolation)
    snprintf(s->commondata.outer_bc_type, 50, "extrapolation");
  params_struct_set_to_default(&s->commondata, s->griddata);
  griddata_struct *g = &s->griddata[0];
  params_struct *params = &g->params;
  params->grid_physical_size = grid_physical_size;
  params->SINHW = sinhw;
  params->SINHWRHO = sinhw;
  params->SINHWZ = sinhw;
  params->grid_idx = 0;
  const int Nx[3] = {Nx0, Nx1, Nx2};
  // CoordSystem hash: each generated project contains exactly one CoordSystem.
#if defined(SINHCYLINDRICAL)
  params->CoordSystem_hash = SINHCYLINDRICAL;
  snprintf(params->gridname, 100, "grid_SinhCylindrical");
#elif defined(SINHSPHERICAL)
  params->CoordSystem_hash = SINHSPHERICAL;
  snprintf(params->gridname, 100, "grid_SinhSpherical");
#else
  params->CoordSystem_hash = SPHERICAL;
  snprintf(params->gridname, 100, "grid_Spherical");
#endif
  numerical_grid_params_Nxx_dxx_xx(&s->commondata, params, g->xx, Nx, true);
  g->rfmstruct = (rfm_struct *)malloc(sizeof(rfm_struct));
  rfm_precompute_malloc(&s->commondata, params, g->rfmstruct);
  rfm_precompute_defines(&s->commondata, params, g->rfmstruct, g->xx);
  bcstruct_set_up(&s->commondata, params, g->xx, &g->bcstruct);
  s->commondata.dt = 1e30;
  cfl_limited_timestep(&s->commondata, params, g->xx);
  s->commondata.nn = 0;
  s->commondata.nn_0 = 0;
  s->commondata.t_0 = 0.0;
  s->commondata.time = 0.0;
  const size_t ntot = (size_t)params->Nxx_plus_2NGHOSTS0 * params->Nxx_plus_2NGHOSTS1 * params->Nxx_plus_2NGHOSTS2;
  g->gridfuncs.y_n_gfs = (REAL *)calloc(ntot * NUM_EVOL_GFS, sizeof(REAL));
  g->gridfuncs.auxevol_gfs = (REAL *)calloc(ntot * NUM_AUXEVOL_GFS, sizeof(REAL));
  initial_data(&s->commondata, s->griddata);
  MoL_malloc_intermediate_stage_gfs(&s->commondata, params, &g->gridfuncs);
  return s;
}

void ref_destroy(ref_sim *s) {
  griddata_free(&s->commondata, s->griddata, true);
  free(s);
}

// ---- sizes, layouts and raw pointers -------------------------------------------------
size_t ref_sizeof_commondata(void) { return sizeof(commondata_struct); }
int ref_nghosts(void) { return NGHOSTS; }
size_t ref_sizeof_params(void) { return sizeof(params_struct); }
size_t ref_sizeof_bc_struct(void) { return sizeof(bc_struct); }
size_t ref_sizeof_griddata(void) { return sizeof(griddata_struct); }
size_t ref_sizeof_innerpt(void) { return sizeof(innerpt_bc_struct); }
size_t ref_sizeof_outerpt(void) { return sizeof(outerpt_bc_struct); }
size_t ref_offsetof_params_Nxx0(void) { return offsetof(params_struct, Nxx0); }
size_t ref_offsetof_params_invdxx0(void) { return offsetof(params_struct, invdxx0); }
size_t ref_offsetof_params_hash(void) { return offsetof(params_struct, CoordSystem_hash); }
size_t ref_offsetof_commondata_eta(void) { return offsetof(commondata_struct, eta); }
size_t ref_offsetof_commondata_dt(void) { return offsetof(commondata_struct, dt); }
size_t ref_offsetof_commondata_bc(void) { return offsetof(commondata_struct, outer_bc_type); }
size_t ref_offsetof_commondata_nn(void) { return offsetof(commondata_struct, nn); }

commondata_struct *ref_commondata(ref_sim *s) { return &s->commondata; }
params_struct *ref_params(ref_sim *s) { return &s->griddata[0].params; }
int ref_N(ref_sim *s, int d) {
  const params_struct *p = &s->griddata[0].params;
  return d == 0 ? p->Nxx_plus_2NGHOSTS0 : (d == 1 ? p->Nxx_plus_2NGHOSTS1 : p->Nxx_plus_2NGHOSTS2);
}
double ref_dt(ref_sim *s) { return s->commondata.dt; }
double ref_time(ref_sim *s) { return s->commondata.time; }
int ref_nn(ref_sim *s) { return s->commondata.nn; }
double ref_param_double(ref_sim *s, int which) {
  const params_struct *p = &s->griddata[0].params;
  switch (which) {
  case 0: return p->dxx0;
  case 1: return p->dxx1;
  case 2: return p->dxx2;
  case 3: return p->invdxx0;
  case 4: return p->invdxx1;
  case 5: return p->invdxx2;
  case 6: return p->xxmin0;
  case 7: return p->xxmin1;
  case 8: return p->xxmin2;
  case 9: return p->xxmax0;
  case 10: return p->xxmax1;
  case 11: return p->xxmax2;
  case 12: return p->AMPL;
  case 13: return p->SINHW;
  case 14: return p->RMAX;
  }
  return 0.0 / 0.0;
}
REAL *ref_y_n(ref_sim *s) { return s->griddata[0].gridfuncs.y_n_gfs; }
REAL *ref_auxevol(ref_sim *s) { return s->griddata[0].gridfuncs.auxevol_gfs; }
REAL *ref_k_odd(ref_sim *s) { return s->griddata[0].gridfuncs.k_odd_gfs; }
REAL *ref_xx(ref_sim *s, int d) { return s->griddata[0].xx[d]; }
// rfm_struct is generated; its fields are a prefix-compatible list of REAL* arrays.
REAL *ref_rfm(ref_sim *s, int which) {
  REAL **fields = (REAL **)s->griddata[0].rfmstruct;
  return fields[which];
}
int ref_rfm_nfields(void) { return (int)(sizeof(rfm_struct) / sizeof(REAL *)); }

int ref_num_inner(ref_sim *s) { return s->griddata[0].bcstruct.bc_info.num_inner_boundary_points; }
innerpt_bc_struct *ref_inner(ref_sim *s) { return s->griddata[0].bcstruct.inner_bc_array; }
int ref_num_pure_outer(ref_sim *s, int gz, int dirn) {
  return s->griddata[0].bcstruct.bc_info.num_pure_outer_boundary_points[gz][dirn];
}
outerpt_bc_struct *ref_pure_outer(ref_sim *s, int gz, int dirn) {
  return s->griddata[0].bcstruct.pure_outer_bc_array[dirn + 3 * gz];
}
const int8_t *ref_evol_gf_parity(void) { return evol_gf_parity; }

// ---- the hot-path operators, on the handle's own grid -----------------------------------
void ref_Ricci(ref_sim *s, const REAL *in, REAL *aux) {
  griddata_struct *g = &s->griddata[0];
  Ricci_eval(&g->params, g->rfmstruct, in, aux);
}
void ref_rhs(ref_sim *s, const REAL *aux, const REAL *in, REAL *rhs) {
  griddata_struct *g = &s->griddata[0];
  rhs_eval(&s->commondata, &g->params, g->rfmstruct, aux, in, rhs);
}
void ref_bc_radiation(ref_sim *s, REAL *gfs, REAL *rhs) {
  griddata_struct *g = &s->griddata[0];
  apply_bcs_outerradiation_and_inner(&s->commondata, &g->params, &g->bcstruct, g->xx, gridfunctions_wavespeed,
                                     gridfunctions_f_infinity, gfs, rhs);
}
void ref_bc_extrap(ref_sim *s, REAL *gfs) {
  griddata_struct *g = &s->griddata[0];
  apply_bcs_outerextrap_and_inner(&s->commondata, &g->params, &g->bcstruct, gfs);
}
void ref_bc_inner(ref_sim *s, REAL *gfs) {
  griddata_struct *g = &s->griddata[0];
  apply_bcs_inner_only(&s->commondata, &g->params, &g->bcstruct, gfs);
}
void ref_enforce(ref_sim *s, REAL *gfs) {
  griddata_struct *g = &s->griddata[0];
  enforce_detgammabar_equals_detgammahat(&g->params, g->rfmstruct, gfs, g->gridfuncs.auxevol_gfs);
}
void ref_step(ref_sim *s, int nsteps) {
  for (int n = 0; n < nsteps; n++)
    MoL_step_forward_in_time(&s->commondata, s->griddata);
}
int ref_num_diag_gfs(void) { return TOTAL_NUM_DIAG_GFS; }
int ref_diag_index(int which) {
  switch (which) {
  case 0: return DIAG_HAMILTONIANGF;
  case 1: return DIAG_MSQUAREDGF;
  case 2: return DIAG_LAMBDA_CONSTRAINTGF;
  }
  return -1;
}
// diag must hold TOTAL_NUM_DIAG_GFS * ntot doubles.
void ref_constraints(ref_sim *s, const REAL *in, const REAL *aux, REAL *diag) {
  griddata_struct *g = &s->griddata[0];
  constraints_eval(&s->commondata, &g->params, g->rfmstruct, in, aux, diag);
}
// Volume element sqrt(detgammahat) d^3xx at one point (diagnostics/sqrt_detgammahat_d3xx_volume_element.c).
double ref_dV(ref_sim *s, int i0, int i1, int i2) {
  griddata_struct *g = &s->griddata[0];
  REAL dV;
  sqrt_detgammahat_d3xx_volume_element(&g->params, g->xx[0][i0], g->xx[1][i1], g->xx[2][i2], &dV);
  return dV;
}
// The generated project's diagnostics() driver at the present state: output cadence, step
// counter and time are set first; files are written to the current directory.
void ref_diagnostics(ref_sim *s, int nn, double time, double output_every) {
  s->commondata.nn = nn;
  s->commondata.time = time;
  s->commondata.diagnostics_output_every = output_every;
  diagnostics(&s->commondata, s->griddata);
}
// The generated initial_data() (Brill-Lindquist -> BSSN, lambda^i, BCs) on this grid.
void ref_initial_data(ref_sim *s) { initial_data(&s->commondata, s->griddata); }
// Clock of the run (the test sets the same step counter and time on both sides).
void ref_set_clock(ref_sim *s, int nn, double time) {
  s->commondata.nn = nn;
  s->commondata.time = time;
}
double ref_t_0(ref_sim *s) { return s->commondata.t_0; }
int ref_nn_0(ref_sim *s) { return s->commondata.nn_0; }
#ifdef REF_HAS_CHECKPOINT
// The generated write_checkpoint()/read_checkpoint() (checkpointing.py:15-470) of a project that
// registers checkpointing; the file checkpoint-conv_factor%.2f.dat is in the current directory.
void ref_write_checkpoint(ref_sim *s, double checkpoint_every) {
  s->commondata.checkpoint_every = checkpoint_every;
  write_checkpoint(&s->commondata, s->griddata);
}
int ref_read_checkpoint(ref_sim *s) { return read_checkpoint(&s->commondata, s->griddata); }
double ref_checkpoint_every(ref_sim *s) { return s->commondata.checkpoint_every; }
size_t ref_offsetof_commondata_checkpoint_every(void) { return offsetof(commondata_struct, checkpoint_every); }
#endif
