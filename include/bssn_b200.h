/*
 * bssn_b200.h -- C ABI of libbssn_b200.so, a B200 (sm_100a) implementation of the
 * BlackHoles@Home single-patch BSSN evolution step.
 *
 * The struct layouts and the void entry points are those of the C project that NRPy's
 * BHaH generator emits for a BSSN evolution (two_blackholes_collide-style, Kreiss-Oliger
 * on, CodeParameters of both Spherical and SinhSpherical registered), so a caller of
 * that project's step functions can link this library instead. Each entry point cites
 * the generator of the function it replaces (paths relative to the nrpy repository).
 *
 * Memory convention (the reference's CUDA build keeps the same split):
 *   - gridfunction arrays (in_gfs, rhs_gfs, auxevol_gfs, y_n_gfs, ..., diagnostic_gfs)
 *     and xx[3] are DEVICE arrays, laid out IDX4(gf,i0,i1,i2) = i0 + N0*(i1 + N1*(i2 + N2*gf));
 *   - params_struct / commondata_struct are HOST structs;
 *   - rfm_struct and bc_struct are HOST structs whose array members point to DEVICE memory
 *     (filled by rfm_precompute_defines() and bcstruct_set_up() of this library).
 * The void entry points launch on the legacy default stream and return when the work
 * is queued; fatal errors print to stderr and exit(1), as the reference does. The
 * bssn_b200_* entry points take an explicit stream and return 0 or a negative status,
 * with the message available from bssn_b200_last_error().
 */
#ifndef BSSN_B200_H
#define BSSN_B200_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>
#include <time.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef REAL
#define REAL double
#endif
/* Interior finite-difference order of this build: 4 (libbssn_b200.so, the default) or 8
 * (libbssn_b200_fd8.so, built with -DBSSN_B200_FD_ORDER=8). NGHOSTS = order/2 + 1, as the
 * generated project's BHaH_defines.h sets it for fd_order with upwinding/KO, so the structs
 * below that depend on it (bc_info_struct, bc_struct) match a project of the same order. */
#ifndef BSSN_B200_FD_ORDER
#define BSSN_B200_FD_ORDER 4
#endif
#define NGHOSTS (BSSN_B200_FD_ORDER / 2 + 1)
#define NUM_EVOL_GFS 24
#define NUM_AUXEVOL_GFS 6
#define MAXNUMGRIDS 15

/* Evolved gridfunction indices (BHaH_defines.h "EVOL VARIABLES"). */
enum {
  ADD00GF, ADD01GF, ADD02GF, ADD11GF, ADD12GF, ADD22GF, ALPHAGF, BETU0GF, BETU1GF, BETU2GF,
  CFGF, HDD00GF, HDD01GF, HDD02GF, HDD11GF, HDD12GF, HDD22GF, LAMBDAU0GF, LAMBDAU1GF,
  LAMBDAU2GF, TRKGF, VETU0GF, VETU1GF, VETU2GF
};
/* Auxiliary evolution gridfunctions: the conformal Ricci tensor. */
enum { RBARDD00GF, RBARDD01GF, RBARDD02GF, RBARDD11GF, RBARDD12GF, RBARDD22GF };
/* Diagnostic gridfunctions written by constraints_eval() (a 3-slot array). */
enum { BSSN_B200_DIAG_HAMILTONIAN, BSSN_B200_DIAG_MSQUARED, BSSN_B200_DIAG_LAMBDA_CONSTRAINT, BSSN_B200_NUM_DIAG_GFS };
/* The generated project's diagnostic gridfunctions (its diagnostics/diagnostic_gfs.h, the
 * DIAG_* enum of two_blackholes_collide): the layout of the diagnostic_gfs arrays that the
 * drop-ins constraints_eval, diagnostic_gfs_set, diagnostics_nearest and
 * diagnostics_volume_integration read and write. */
enum {
  BSSN_B200_DIAG_GRIDINDEXGF, BSSN_B200_DIAG_HAMILTONIANGF, BSSN_B200_DIAG_LAMBDA_CONSTRAINTGF, BSSN_B200_DIAG_LAPSEGF,
  BSSN_B200_DIAG_MSQUAREDGF, BSSN_B200_DIAG_RBARDD00GF, BSSN_B200_DIAG_RBARDD01GF, BSSN_B200_DIAG_RBARDD02GF,
  BSSN_B200_DIAG_RBARDD11GF, BSSN_B200_DIAG_RBARDD12GF, BSSN_B200_DIAG_RBARDD22GF, BSSN_B200_DIAG_WGF,
  BSSN_B200_TOTAL_NUM_DIAG_GFS
};

/* CoordSystem_hash values (BHaH_defines.h). */
#define SPHERICAL 1307621703
#define SINHSPHERICAL 579707936
#define SINHCYLINDRICAL 1325205359

/* commondata_struct: CodeParameters shared by all grids (BHaH_defines_h.py, CodeParameters.py:17-199). */
typedef struct __commondata_struct__ {
  REAL BH1_mass;
  REAL BH1_posn_x;
  REAL BH1_posn_y;
  REAL BH1_posn_z;
  REAL BH2_mass;
  REAL BH2_posn_x;
  REAL BH2_posn_y;
  REAL BH2_posn_z;
  REAL CFL_FACTOR;
  REAL KreissOliger_strength_gauge;
  REAL KreissOliger_strength_nongauge;
  REAL convergence_factor;
  REAL diagnostics_output_every;
  REAL dt;
  REAL eta;
  REAL t_0;
  REAL t_final;
  REAL time;
  struct timespec start_wallclock_time;
  char outer_bc_type[50];
  int NUMGRIDS;
  int nn;
  int nn_0;
  int output_progress_every;
} commondata_struct;

/* params_struct: per-grid CodeParameters (BHaH_defines_h.py; numerical_grids_and_timestep.py). */
typedef struct __params_struct__ {
  REAL AMPL;
  REAL AMPLRHO;
  REAL AMPLZ;
  REAL Cart_originx;
  REAL Cart_originy;
  REAL Cart_originz;
  REAL PI;
  REAL RHOMAX;
  REAL RMAX;
  REAL SINHW;
  REAL SINHWRHO;
  REAL SINHWZ;
  REAL ZMAX;
  REAL ZMIN;
  REAL dxx0;
  REAL dxx1;
  REAL dxx2;
  REAL grid_hole_radius;
  REAL grid_physical_size;
  REAL invdxx0;
  REAL invdxx1;
  REAL invdxx2;
  REAL xmax;
  REAL xmin;
  REAL xxmax0;
  REAL xxmax1;
  REAL xxmax2;
  REAL xxmin0;
  REAL xxmin1;
  REAL xxmin2;
  REAL ymax;
  REAL ymin;
  REAL zmax;
  REAL zmin;
  bool grid_rotates;
  bool is_host;
  char CoordSystemName[100];
  char gridname[100];
  int CoordSystem_hash;
  int Nxx0;
  int Nxx1;
  int Nxx2;
  int Nxx_plus_2NGHOSTS0;
  int Nxx_plus_2NGHOSTS1;
  int Nxx_plus_2NGHOSTS2;
  int grid_idx;
} params_struct;

/* rfm_struct: 1-D reference-metric precompute arrays (rfm_precompute.py:84-565). The
 * SinhSpherical field list is used for the Spherical family (for Spherical the radial
 * derivatives are 1, 0, 0). A SinhCylindrical project's rfm_struct has the same seven
 * pointers with f3_of_xx2, f3_of_xx2__D2, f3_of_xx2__DD22 (functions of xx2, arrays of
 * Nxx_plus_2NGHOSTS2 entries) in the last three places, which the library reads through
 * these names. Array members are device pointers. */
typedef struct __rfmstruct__ {
  REAL *f0_of_xx0;
  REAL *f0_of_xx0__D0;
  REAL *f0_of_xx0__DD00;
  REAL *f0_of_xx0__DDD000;
  REAL *f1_of_xx1;
  REAL *f1_of_xx1__D1;
  REAL *f1_of_xx1__DD11;
} rfm_struct;

/* Curvilinear boundary-condition structures (CurviBoundaryConditions/BHaH_defines.py:41-199). */
typedef struct __innerpt_bc_struct__ {
  int dstpt;
  int srcpt;
  int8_t parity[10];
} innerpt_bc_struct;

typedef struct __outerpt_bc_struct__ {
  short i0, i1, i2;
  int8_t FACEX0, FACEX1, FACEX2;
} outerpt_bc_struct;

typedef struct __bc_info_struct__ {
  int num_inner_boundary_points;
  int num_pure_outer_boundary_points[NGHOSTS][3];
  int bc_loop_bounds[NGHOSTS][6][6];
} bc_info_struct;

typedef struct __bc_struct__ {
  innerpt_bc_struct *inner_bc_array;               /* device */
  outerpt_bc_struct *pure_outer_bc_array[NGHOSTS * 3]; /* device */
  bc_info_struct bc_info;
} bc_struct;

/* Method-of-lines RK4 storage (MoLtimestepping/BHaH_defines.py:18). Device arrays. */
typedef struct __MoL_gridfunctions_struct__ {
  REAL *y_n_gfs;
  REAL *y_nplus1_running_total_gfs;
  REAL *k_odd_gfs;
  REAL *k_even_gfs;
  REAL *auxevol_gfs;
} MoL_gridfunctions_struct;

typedef struct __griddata__ {
  REAL *xx[3]; /* device */
  bc_struct bcstruct;
  MoL_gridfunctions_struct gridfuncs;
  params_struct params;
  rfm_struct *rfmstruct; /* host struct, device arrays */
} griddata_struct;

/* Per-gridfunction parity type, outer-boundary wave speed and asymptotic value
 * (BHaH_defines.h: evol_gf_parity, gridfunctions_wavespeed, gridfunctions_f_infinity). */
extern const int8_t bssn_b200_evol_gf_parity[NUM_EVOL_GFS];
extern const REAL gridfunctions_wavespeed[NUM_EVOL_GFS];
extern const REAL gridfunctions_f_infinity[NUM_EVOL_GFS];

/* ======================= drop-in entry points (void, exit(1) on error) ======================= */

/* Defaults of every CodeParameter (CodeParameters.py: params/commondata_struct_set_to_default). */
void commondata_struct_set_to_default(commondata_struct *commondata);
void params_struct_set_to_default(commondata_struct *commondata, griddata_struct *griddata);

/* numerical_grids_and_timestep.py:31-190 -- Nxx, dxx, invdxx, cell-centred xx[3] (allocated on device).
 * Nxx = Nx when all three entries are set (not -1), else the generated project's default
 * (72, 12, 2) (two_blackholes_collide's Nxx_dict); then the convergence factor is applied. */
void numerical_grid_params_Nxx_dxx_xx(const commondata_struct *commondata, params_struct *params, REAL *xx[3],
                                      const int Nx[3], const bool apply_convergence_factor_and_set_xxminmax_defaults);
/* rfm_precompute.py:84-565 */
void rfm_precompute_malloc(const commondata_struct *commondata, const params_struct *params, rfm_struct *rfmstruct);
void rfm_precompute_defines(const commondata_struct *commondata, const params_struct *params, rfm_struct *rfmstruct,
                            REAL *xx[3]);
void rfm_precompute_free(const commondata_struct *commondata, const params_struct *params, rfm_struct *rfmstruct);
/* CurviBoundaryConditions/bcstruct_set_up.py:442-792 (computed on the host, arrays uploaded). */
void bcstruct_set_up(const commondata_struct *commondata, const params_struct *params, REAL *xx[3], bc_struct *bcstruct);
void bcstruct_free(bc_struct *bcstruct);
/* numerical_grids_and_timestep.py:498-560 -- dt = min(dt, CFL_FACTOR * min ds). */
void cfl_limited_timestep(commondata_struct *commondata, params_struct *params, REAL *xx[3]);
/* general_relativity/initial_data.py:24 with Brill-Lindquist data (InitialData_Cartesian.py:111-141) and the
 * ADM->BSSN converter (ADM_Initial_Data_Reader__BSSN_Converter.py:33-1181). Needs y_n_gfs allocated. */
void initial_data(commondata_struct *commondata, griddata_struct *griddata);
/* MoLtimestepping/register_all.py */
void MoL_malloc_y_n_gfs(const commondata_struct *commondata, const params_struct *params, MoL_gridfunctions_struct *gridfuncs);
void MoL_malloc_intermediate_stage_gfs(const commondata_struct *commondata, const params_struct *params,
                                       MoL_gridfunctions_struct *gridfuncs);
void MoL_free_intermediate_stage_gfs(MoL_gridfunctions_struct *gridfuncs);

/* general_relativity/Ricci_eval.py:27-167 */
void Ricci_eval(const params_struct *params, const rfm_struct *rfmstruct, const REAL *in_gfs, REAL *auxevol_gfs);
/* general_relativity/rhs_eval.py:38-413 */
void rhs_eval(const commondata_struct *commondata, const params_struct *params, const rfm_struct *rfmstruct,
              const REAL *auxevol_gfs, const REAL *in_gfs, REAL *rhs_gfs);
/* CurviBoundaryConditions/apply_bcs_outerradiation_and_inner.py:46-723 */
void apply_bcs_outerradiation_and_inner(const commondata_struct *commondata, const params_struct *params,
                                        const bc_struct *bcstruct, REAL *xx[3], const REAL custom_wavespeed[NUM_EVOL_GFS],
                                        const REAL custom_f_infinity[NUM_EVOL_GFS], REAL *gfs, REAL *rhs_gfs);
/* CurviBoundaryConditions/apply_bcs_outerextrap_and_inner.py:28-398 */
void apply_bcs_outerextrap_and_inner(const commondata_struct *commondata, const params_struct *params,
                                     const bc_struct *bcstruct, REAL *gfs);
/* CurviBoundaryConditions/apply_bcs_inner_only.py:26-199 */
void apply_bcs_inner_only(const commondata_struct *commondata, const params_struct *params, const bc_struct *bcstruct,
                          REAL *gfs);
/* general_relativity/enforce_detgammabar_equals_detgammahat.py:198-342 */
void enforce_detgammabar_equals_detgammahat(const params_struct *params, const rfm_struct *rfmstruct, REAL *in_gfs,
                                            const REAL *auxevol_gfs);
/* MoLtimestepping/MoL_step_forward_in_time.py:39-507 (RK4, radiation or extrapolation outer BCs). */
void MoL_step_forward_in_time(commondata_struct *commondata, griddata_struct *griddata);
/* general_relativity/constraints_eval.py:364-492 -- diagnostic_gfs holds BSSN_B200_TOTAL_NUM_DIAG_GFS
 * gridfunctions on the device (the generated project's layout); H, M^2 and |Lambda constraint| are written at
 * the interior points of BSSN_B200_DIAG_HAMILTONIANGF, _MSQUAREDGF and _LAMBDA_CONSTRAINTGF. */
void constraints_eval(const commondata_struct *commondata, const params_struct *params, const rfm_struct *rfmstruct,
                      const REAL *in_gfs, const REAL *auxevol_gfs, REAL *diagnostic_gfs);

/* ---- diagnostics (diagnostics/diagnostics.py:46-270 and the helpers it registers) ----
 * Diagnostic arrays are DEVICE arrays of BSSN_B200_TOTAL_NUM_DIAG_GFS gridfunctions; samples are
 * gathered on the GPU and only they are copied to the host. Output files (the reference's names and
 * ASCII formats) go to the current directory:
 *   out0d-grid%02d-<Coord>-conv_factor-%.2f.txt            H, M^2 at the point next to the origin
 *   out1d-{y,z}-<Coord>-grid%02d-conv_factor%.2f-t%08.2f.txt  H, M^2 along the lines nearest the y, z axes
 *   out2d-{xy,yz}-<Coord>-grid%02d-conv_factor%.2f-t%08.2f.txt H, M^2 on the planes nearest xy, yz
 *   out3d-integrals-conv_factor%.2f-<recipe>.txt            volume integrals, L2 and RMS of H, M^2, |Lambda|
 *     over recipes "whole_domain" and "sphere_R_gt_8" (r > 8), as two_blackholes_collide defines them. */
/* diagnostics.py:46-270 -- on output steps (|round(t/every)*every - t| < dt/2): diagnostic_gfs_set,
 * diagnostics_nearest, diagnostics_volume_integration; then progress_indicator. */
void diagnostics(commondata_struct *commondata, griddata_struct *griddata);
/* diagnostic_gfs_set: Ricci, constraints, lapse, W, grid index (and Rbar_ij) into each grid's array. */
void diagnostic_gfs_set(const commondata_struct *commondata, const griddata_struct *griddata,
                        REAL *diagnostic_gfs[MAXNUMGRIDS]);
/* diagnostics_nearest.c / diagnostics_nearest_{grid_center,1d_y_and_z_axes,2d_xy_and_yz_planes}. */
void diagnostics_nearest(commondata_struct *commondata, griddata_struct *griddata,
                         const REAL *diagnostic_gfs[MAXNUMGRIDS]);
/* diagnostics_volume_integration.c + diagnostics_volume_integration_helpers.h. */
void diagnostics_volume_integration(commondata_struct *commondata, griddata_struct *griddata,
                                    const REAL *diagnostic_gfs[MAXNUMGRIDS]);
/* progress_indicator.py: one status line on stderr every output_progress_every steps. */
void progress_indicator(commondata_struct *commondata, const griddata_struct *griddata);

/* ======================= status-returning entry points (explicit stream) ======================= */
/* `stream` is a cudaStream_t passed as void* (NULL = legacy default stream). Return 0 on success,
 * a negative BSSN_B200_E* code otherwise; bssn_b200_last_error() describes the last failure. */
enum {
  BSSN_B200_OK = 0,
  BSSN_B200_EINVAL = -1,   /* bad argument (size, pointer, coordinate system, symmetry) */
  BSSN_B200_ECUDA = -2,    /* a CUDA runtime call or kernel launch failed */
  BSSN_B200_ESETUP = -3,   /* boundary set-up failed (a ghost point did not map to the grid) */
  BSSN_B200_ENOMEM = -4
};
const char *bssn_b200_last_error(void);
const char *bssn_b200_version(void);
/* BSSN_B200_FD_ORDER of the loaded library (4 or 8). */
int bssn_b200_fd_order(void);

/* Symmetry axes of the generated algebra: "" (full 3-D, default) or "2" (axisymmetric:
 * derivatives in xx2 vanish, as nrpy's symmetry_axes="2"). Process-wide setting. */
int bssn_b200_set_symmetry_axes(const char *axes);

int bssn_b200_ricci_eval(const params_struct *params, const rfm_struct *rfmstruct, const REAL *in_gfs,
                         REAL *auxevol_gfs, void *stream);
int bssn_b200_rhs_eval(const commondata_struct *commondata, const params_struct *params, const rfm_struct *rfmstruct,
                       const REAL *auxevol_gfs, const REAL *in_gfs, REAL *rhs_gfs, void *stream);
/* rhs_eval with the RHS algebra (not the stencils) in FP32; state and outputs stay FP64. */
int bssn_b200_rhs_eval_mixed(const commondata_struct *commondata, const params_struct *params,
                             const rfm_struct *rfmstruct, const REAL *auxevol_gfs, const REAL *in_gfs, REAL *rhs_gfs,
                             void *stream);
int bssn_b200_apply_bcs_outerradiation_and_inner(const commondata_struct *commondata, const params_struct *params,
                                                 const bc_struct *bcstruct, REAL *xx[3], const REAL *wavespeed,
                                                 const REAL *f_infinity, REAL *gfs, REAL *rhs_gfs, void *stream);
int bssn_b200_apply_bcs_outerextrap_and_inner(const params_struct *params, const bc_struct *bcstruct, REAL *gfs,
                                              void *stream);
int bssn_b200_apply_bcs_inner_only(const params_struct *params, const bc_struct *bcstruct, REAL *gfs, int num_gfs,
                                   const int8_t *gf_parity_types, void *stream);
int bssn_b200_enforce_detgammabar_equals_detgammahat(const params_struct *params, const rfm_struct *rfmstruct,
                                                     REAL *in_gfs, void *stream);
/* Compact layout: diagnostic_gfs holds BSSN_B200_NUM_DIAG_GFS gridfunctions (H, M^2, |Lambda|). */
int bssn_b200_constraints_eval(const commondata_struct *commondata, const params_struct *params,
                               const rfm_struct *rfmstruct, const REAL *in_gfs, const REAL *auxevol_gfs,
                               REAL *diagnostic_gfs, void *stream);
/* Volume integrals over the interior (diagnostics_volume_integration_helpers.h:400-470):
 * out[0..2] = sum_interior f^2 dV for f = H, M^2, |Lambda|; out[3] = sum dV, with
 * dV = sqrt(det gammahat) |dxx0 dxx1 dxx2|. `out` is a HOST array, written after the
 * stream synchronises. The L2 norm of f is sqrt(out[k]); its RMS is sqrt(out[k]/out[3]).
 * Uses a device scratch buffer that the library allocates on first use and keeps. */
int bssn_b200_constraint_integrals(const params_struct *params, const rfm_struct *rfmstruct,
                                   const REAL *diagnostic_gfs, double out[4], void *stream);

/* The same integrals for callers that cannot allocate device memory -- code inside a host
 * framework that owns every allocation through its own pool or arena (a cudaMalloc behind
 * its back escapes its accounting and its memory cap), or embedded hosts that forbid
 * allocation after start-up so that their footprint stays fixed.
 * No counterpart in the reference (whose integrals run on the host). It allocates
 * nothing: its partial sums live in a file-scope __device__ array of 16384*4+4 doubles
 * (512 KiB + 32 B), which every GPU that loads the library holds until the process exits.
 * Limit: grids of at most 33,554,432 interior points; larger grids return BSSN_B200_EINVAL.
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress)
 * with that device current and keeps it; make that first call before any stream capture,
 * and do not use the library across a cudaDeviceReset, which makes the kept address stale.
 * All calls share the one array, so calls that overlap on the GPU (other streams, other
 * host threads) race; every call overwrites the entries it reads, so nothing needs clearing.
 * Synchronises `stream`; `out` is a HOST array of 4 doubles. */
int bssn_b200_constraint_integrals_noalloc(const params_struct *params, const rfm_struct *rfmstruct,
                                           const REAL *diagnostic_gfs, double out[4], void *stream);

/* One RK4 step (all four stages) on one grid. mode: 0 = stage-by-stage as the reference
 * (Ricci, RHS, BCs, RK update, enforce); 1 = fused stages (RK update and detgammabar
 * enforcement in the RHS epilogue). mixed != 0 evaluates the RHS algebra in FP32. */
int bssn_b200_mol_step(commondata_struct *commondata, griddata_struct *griddata, int mode, int mixed, void *stream);

/* A captured CUDA graph of `steps_per_graph` RK4 steps of one grid; replayed by
 * bssn_b200_stepper_run. The graph bakes in dt and the buffer addresses. */
typedef struct bssn_b200_stepper bssn_b200_stepper;
int bssn_b200_stepper_create(commondata_struct *commondata, griddata_struct *griddata, int mode, int mixed,
                             int steps_per_graph, void *stream, bssn_b200_stepper **out);
int bssn_b200_stepper_run(bssn_b200_stepper *st, int graph_launches);
int bssn_b200_stepper_destroy(bssn_b200_stepper *st);
/* Number of kernel nodes in one replay of the stepper's graph. */
int bssn_b200_stepper_kernel_nodes(const bssn_b200_stepper *st, unsigned long long *out);

/* Batched evolutions: `nevo` independent grids (each set up through the entry points above:
 * grid, rfm, bcstruct, storage, initial data; all of one coordinate system, full 3-D,
 * radiation outer BCs; each with its own commondata: masses, dt, ...) advanced together.
 * Each RK4 stage of the whole batch takes a fixed number of launches (one per group kernel
 * for every 120 grids): the Ricci and RHS group kernels run one block per tile over the tiles
 * of all grids; a tile is tile_bx x tile_by = 128 points, or, with tile_bx = tile_by = 0, per
 * grid the 128-point brick (i0 x i1 x i2, i0 extent 16 to 128) that pads that grid's
 * interior least.
 * `steps_per_graph` RK4 steps are captured into a CUDA graph on `stream` (non-default);
 * bssn_b200_batch_run replays it. Creation allocates the per-grid RHS shells and the
 * device work lists; the caller's states are unchanged by it. */
typedef struct bssn_b200_batch bssn_b200_batch;
int bssn_b200_batch_create(int nevo, commondata_struct *const *commondatas, griddata_struct *const *griddatas,
                           int tile_bx, int tile_by, int steps_per_graph, void *stream, bssn_b200_batch **out);
int bssn_b200_batch_run(bssn_b200_batch *batch, int graph_launches);
int bssn_b200_batch_info(const bssn_b200_batch *batch, int *ntiles, int *nouter, int *ninner,
                         unsigned long long *kernel_nodes);
/* Interior points of the batch and the points its tiles cover (interior plus padding of the
 * partial tiles at the grids' edges). */
int bssn_b200_batch_tile_fill(const bssn_b200_batch *batch, long long *interior_points, long long *padded_points);
int bssn_b200_batch_destroy(bssn_b200_batch *batch);

/* Reverse mode (no counterpart in the reference, which has no adjoint). Gradient of
 *   J = sum over interior points of H^2 + alpha(NGHOSTS, N1/2, N2/2)
 * after `nsteps` RK4 steps (radiation outer BCs) with respect to the Brill-Lindquist
 * parameters (BH1_mass, BH1_posn_z, BH2_mass, BH2_posn_z) of the initial data, by the
 * discrete adjoint of the stage-by-stage step (mode 0 of bssn_b200_mol_step). The forward
 * keeps y every `checkpoint_every` steps; the backward recomputes each segment from its
 * checkpoint. Spherical coordinates without symmetry axes; one grid (NUMGRIDS = 1).
 * The handle uses the grid's MoL storage as workspace: after backward, y_n_gfs holds the
 * final state again. `stream` as in the other entry points. */
typedef struct bssn_b200_adjoint bssn_b200_adjoint;
int bssn_b200_adjoint_create(commondata_struct *commondata, griddata_struct *griddata, int nsteps,
                             int checkpoint_every, void *stream, bssn_b200_adjoint **out);
/* Evolve y_n_gfs (the initial data) nsteps steps; out = {J, sum H^2, alpha term} (host). */
int bssn_b200_adjoint_forward(bssn_b200_adjoint *adj, double out[3]);
/* grad (host, 4) = Jbar * dJ/d(BH1_mass, BH1_posn_z, BH2_mass, BH2_posn_z); optionally the
 * adjoint of the initial state y_0 into ybar0 (device, NUM_EVOL_GFS gridfunctions). */
int bssn_b200_adjoint_backward(bssn_b200_adjoint *adj, double Jbar, double *ybar0, double grad[4]);
/* Pieces of the chain on a given device state y (NUM_EVOL_GFS gridfunctions):
 * J(y); ybar = Jbar dJ/dy; ybar <- (dF/dy)^T ybar for one RK4 step F at y_n;
 * grad from the adjoint of y_0 through the initial-data BCs and psi^-2. */
int bssn_b200_adjoint_functional(bssn_b200_adjoint *adj, const double *y, double out[3]);
int bssn_b200_adjoint_functional_vjp(bssn_b200_adjoint *adj, const double *y, double Jbar, double *ybar);
int bssn_b200_adjoint_step_vjp(bssn_b200_adjoint *adj, const double *y_n, double *ybar);
int bssn_b200_adjoint_id_vjp(bssn_b200_adjoint *adj, const double *ybar0, double grad[4]);
int bssn_b200_adjoint_destroy(bssn_b200_adjoint *adj);

/* The diagnostics() driver with a status return and an explicit stream (the diagnostic arrays are
 * kept by the library per grid and reused). */
int bssn_b200_diagnostics(commondata_struct *commondata, griddata_struct *griddata, void *stream);

/* ---- checkpoint / restart (checkpointing.py:15-470) ----
 * The file is checkpoint-conv_factor%.2f.dat (convergence_factor) in the current directory, byte for
 * byte in the format of the generated write_checkpoint/read_checkpoint of a project that registers
 * checkpointing, so either side can resume the other's file:
 *   bssn_b200_checkpoint_commondata (that project's commondata_struct), then per grid:
 *   params_struct, int count, int indices[count], REAL data[count][NUM_EVOL_GFS] (point-major;
 *   every point of the grid, indices 0..ntot-1, as the single-patch writer selects them).
 * Registering checkpointing adds the REAL CodeParameter checkpoint_every to commondata_struct
 * (checkpointing.py:253-255); the generated struct lists REAL fields by name, which puts it after
 * KreissOliger_strength_nongauge. This library's commondata_struct is the layout of a project
 * without it, so the cadence is an argument here and no drop-in named write_checkpoint or
 * read_checkpoint is exported (its commondata argument would have the other layout).
 * The first call on a device allocates staging buffers (two 12.6 MB device chunks and two 12.6 MB
 * pinned host chunks) that the library keeps until the process exits; calls are serialised. */
typedef struct {
  REAL BH1_mass;
  REAL BH1_posn_x;
  REAL BH1_posn_y;
  REAL BH1_posn_z;
  REAL BH2_mass;
  REAL BH2_posn_x;
  REAL BH2_posn_y;
  REAL BH2_posn_z;
  REAL CFL_FACTOR;
  REAL KreissOliger_strength_gauge;
  REAL KreissOliger_strength_nongauge;
  REAL checkpoint_every;
  REAL convergence_factor;
  REAL diagnostics_output_every;
  REAL dt;
  REAL eta;
  REAL t_0;
  REAL t_final;
  REAL time;
  struct timespec start_wallclock_time;
  char outer_bc_type[50];
  int NUMGRIDS;
  int nn;
  int nn_0;
  int output_progress_every;
} bssn_b200_checkpoint_commondata;

/* write_checkpoint (checkpointing.py:246-470). Writes only on checkpoint steps, as the reference:
 * checkpoint_every > 0 and |round(time/checkpoint_every)*checkpoint_every - time| < dt/2. Returns 1
 * when the file was written, 0 when this is not a checkpoint step, a negative code on failure (the
 * reference exits instead). The state is read from each grid's device y_n_gfs; the packing into
 * point-major order runs on the GPU, in chunks, overlapped with the file writes. */
int bssn_b200_write_checkpoint(const commondata_struct *commondata, REAL checkpoint_every,
                               const griddata_struct *griddata, void *stream);
/* read_checkpoint (checkpointing.py:15-243). Returns 0 when the file does not exist, 1 when it was
 * read, a negative code on failure (the reference exits instead). commondata is overwritten with the
 * file's values, then t_0 = time and nn_0 = nn; checkpoint_every (may be NULL) receives the file's
 * cadence. griddata == NULL reads only commondata (to rebuild the grids first). Otherwise griddata
 * must hold the file's NUMGRIDS grids, as for the reference's read_checkpoint, and each grid's
 * saved params must match its Nxx_plus_2NGHOSTS* and CoordSystem_hash, count must lie in [0, ntot] and
 * every index in [0, ntot); y_n_gfs (device, already allocated) is zeroed and the saved points are
 * scattered into it on the GPU. */
int bssn_b200_read_checkpoint(commondata_struct *commondata, REAL *checkpoint_every, griddata_struct *griddata,
                              void *stream);

/* Instrumentation: kernels launched by this library since it was loaded (each graph replay
 * counts its kernel nodes), and a launch of only the interior RHS + RK-update + projection
 * kernel of RK4 stage `stage` (1..4) of grid 0, used to time the dominant kernel alone.
 * The latter overwrites that stage's output buffer. */
unsigned long long bssn_b200_kernel_launches(void);
int bssn_b200_rhs_fused_stage(commondata_struct *commondata, griddata_struct *griddata, int stage, int mixed,
                              void *stream);
/* FP64 FMA throughput of this GPU, as a roofline denominator for the FP64-bound point kernels:
 * a kernel of independent FMA chains (no memory traffic) on every SM, timed with CUDA events,
 * best of `reps` launches. out_tflops = 2 x FMAs / time, in TFLOP/s. Synchronises `stream`. */
int bssn_b200_fp64_fma_rate(int reps, double *out_tflops, void *stream);

/* Synchronous copy for callers without their own CUDA binding:
 * kind 0 = host->device, 1 = device->host, 2 = device->device. */
int bssn_b200_memcpy(void *dst, const void *src, size_t bytes, int kind);
int bssn_b200_device_synchronize(void);

#ifdef __cplusplus
}
#endif
#endif /* BSSN_B200_H */
