// extern "C" entry points of libbssn_b200.so (declared in include/bssn_b200.h).
#include <cstdarg>
#include <cstring>
#include <atomic>
#include <mutex>
#include <vector>

#include "bssn_common.cuh"

namespace bssn {

// ---------------------------------------------------------------- errors
static thread_local char g_err[1024] = "";
void set_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
const char *last_error() { return g_err; }

static std::atomic<unsigned long long> g_launches{0};
void count_launch(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

static int g_sym_mask = 0;
int symmetry_axes_mask() { return g_sym_mask; }

int variant_of(const params_struct *p, Variant *out) {
  if (!p) {
    set_error("params is NULL");
    return BSSN_B200_EINVAL;
  }
  const bool axi = (g_sym_mask & 4) != 0;
  if (p->CoordSystem_hash == SPHERICAL) *out = axi ? SPH_AXI : SPH_3D;
  else if (p->CoordSystem_hash == SINHSPHERICAL) *out = axi ? SINH_AXI : SINH_3D;
  else if (p->CoordSystem_hash == SINHCYLINDRICAL) {
    // SinhCylindrical is built axisymmetric about z (symmetry_axes "1"), as blackhole_spectroscopy runs it.
    if (g_sym_mask != 2) {
      set_error("SinhCylindrical is built with symmetry_axes \"1\" only (set it before the set-up)");
      return BSSN_B200_EINVAL;
    }
    *out = SINHCYL_AXI;
  } else {
    set_error("CoordSystem_hash %d not supported (Spherical=%d, SinhSpherical=%d, SinhCylindrical=%d)",
              p->CoordSystem_hash, SPHERICAL, SINHSPHERICAL, SINHCYLINDRICAL);
    return BSSN_B200_EINVAL;
  }
  return BSSN_B200_OK;
}

// Set-up (setup.cu)
void commondata_defaults(commondata_struct *cd);
void params_defaults(params_struct *p);
int grid_params(const commondata_struct *cd, params_struct *p, REAL *xx[3], const int Nx[3], bool apply_defaults);
int rfm_malloc(const params_struct *p, rfm_struct *r);
int rfm_free(rfm_struct *r);
int rfm_defines(const params_struct *p, rfm_struct *r, REAL *xx[3]);
int bcstruct_setup(const params_struct *p, REAL *xx[3], bc_struct *bc);
int bcstruct_release(bc_struct *bc);
int cfl_dt(commondata_struct *cd, const params_struct *p, REAL *xx[3]);
int bl_initial_data(const commondata_struct *cd, const params_struct *p, REAL *xx[3], const bc_struct *bc,
                    double *y_n, cudaStream_t s);
// Reductions (reductions.cu)
int constraint_integrals(const params_struct *p, const RfmArrays &rfm, const double *diag, double *scratch,
                         double out[4], cudaStream_t s);
size_t constraint_integrals_scratch_doubles();
int constraint_integrals_noalloc(const params_struct *p, const RfmArrays &rfm, const double *diag, double out[4],
                                 cudaStream_t s);
// MoL (mol.cu)
int mol_step(commondata_struct *cd, griddata_struct *gd, int mode, int mixed, cudaStream_t s);
int fused_interior_stage(const commondata_struct *cd, griddata_struct *gd, int grid, int stage, int mixed,
                         cudaStream_t s);
int mol_prepare(const commondata_struct *cd, griddata_struct *gd, int mode);
// Instrumentation (reductions.cu)
int fp64_fma_rate(int reps, double *out_tflops, cudaStream_t s);

static int check_ptr(const void *p, const char *what) {
  if (!p) {
    set_error("%s is NULL", what);
    return BSSN_B200_EINVAL;
  }
  return BSSN_B200_OK;
}

static void die_on(int rc, const char *fn) {
  if (rc != BSSN_B200_OK) {
    fprintf(stderr, "ERROR in %s(): %s\n", fn, last_error());
    exit(1);
  }
}

int initial_data_grid(commondata_struct *cd, griddata_struct *G, cudaStream_t s) {
  BSSN_TRY(check_ptr(G->gridfuncs.y_n_gfs, "y_n_gfs"));
  BSSN_TRY(check_ptr(G->rfmstruct, "rfmstruct"));
  Variant v;
  BSSN_TRY(variant_of(&G->params, &v));
  BSSN_TRY(bl_initial_data(cd, &G->params, G->xx, &G->bcstruct, G->gridfuncs.y_n_gfs, s));
  const GridDims g = grid_dims(&G->params);
  BSSN_TRY(launch_lambda_id(v, g, rfm_arrays(G->rfmstruct), G->gridfuncs.y_n_gfs, s));
  BSSN_TRY(launch_extrap_bcs(g, &G->bcstruct, G->gridfuncs.y_n_gfs, s));
  BSSN_TRY(launch_inner_bcs(g, &G->bcstruct, G->gridfuncs.y_n_gfs, NUM_EVOL_GFS, nullptr, s));
  return BSSN_B200_OK;
}

// ---------------------------------------------------------------- CUDA-graph stepper
}  // namespace bssn

struct bssn_b200_stepper {
  commondata_struct *cd;
  griddata_struct *gd;
  cudaStream_t stream;
  cudaGraph_t graph;
  cudaGraphExec_t exec;
  int steps_per_graph;
  unsigned long long kernel_nodes;
};

using namespace bssn;

extern "C" {

const int8_t bssn_b200_evol_gf_parity[NUM_EVOL_GFS] = {4, 5, 6, 7, 8, 9, 0, 1, 2, 3, 0, 4,
                                                       5, 6, 7, 8, 9, 1, 2, 3, 0, 1, 2, 3};
const REAL gridfunctions_wavespeed[NUM_EVOL_GFS] = {1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.41421356237310, 1.0,
                                                    1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0,
                                                    1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0};
const REAL gridfunctions_f_infinity[NUM_EVOL_GFS] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0, 0.0,
                                                     0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};

const char *bssn_b200_last_error(void) { return last_error(); }
const char *bssn_b200_version(void) { return "bssn_b200 1.0 (sm_100a)"; }

int bssn_b200_fd_order(void) { return BSSN_B200_FD_ORDER; }

int bssn_b200_set_symmetry_axes(const char *axes) {
  int mask = 0;
  if (axes) {
    for (const char *c = axes; *c; c++) {
      if (*c < '0' || *c > '2') {
        set_error("symmetry axes \"%s\": only digits 0-2 allowed", axes);
        return BSSN_B200_EINVAL;
      }
      mask |= 1 << (*c - '0');
    }
  }
  if (mask != 0 && mask != 4 && mask != 2) {
    set_error("symmetry axes \"%s\": only \"\" (3-D), \"2\" (axisymmetric Spherical family) and \"1\" "
              "(axisymmetric SinhCylindrical) are generated", axes ? axes : "");
    return BSSN_B200_EINVAL;
  }
  g_sym_mask = mask;
  return BSSN_B200_OK;
}

// ---------------------------------------------------------------- set-up (void, drop-in)
void commondata_struct_set_to_default(commondata_struct *commondata) { commondata_defaults(commondata); }

void params_struct_set_to_default(commondata_struct *commondata, griddata_struct *griddata) {
  (void)commondata;
  for (int grid = 0; grid < MAXNUMGRIDS; grid++) params_defaults(&griddata[grid].params);
}

void numerical_grid_params_Nxx_dxx_xx(const commondata_struct *commondata, params_struct *params, REAL *xx[3],
                                      const int Nx[3], const bool apply_defaults) {
  die_on(grid_params(commondata, params, xx, Nx, apply_defaults), __func__);
}
void rfm_precompute_malloc(const commondata_struct *, const params_struct *params, rfm_struct *rfmstruct) {
  die_on(rfm_malloc(params, rfmstruct), __func__);
}
void rfm_precompute_defines(const commondata_struct *, const params_struct *params, rfm_struct *rfmstruct,
                            REAL *xx[3]) {
  die_on(rfm_defines(params, rfmstruct, xx), __func__);
}
void rfm_precompute_free(const commondata_struct *, const params_struct *, rfm_struct *rfmstruct) {
  die_on(rfm_free(rfmstruct), __func__);
}
void bcstruct_set_up(const commondata_struct *, const params_struct *params, REAL *xx[3], bc_struct *bcstruct) {
  die_on(bcstruct_setup(params, xx, bcstruct), __func__);
}
void bcstruct_free(bc_struct *bcstruct) { die_on(bcstruct_release(bcstruct), __func__); }
void cfl_limited_timestep(commondata_struct *commondata, params_struct *params, REAL *xx[3]) {
  die_on(cfl_dt(commondata, params, xx), __func__);
}
void initial_data(commondata_struct *commondata, griddata_struct *griddata) {
  for (int grid = 0; grid < commondata->NUMGRIDS; grid++)
    die_on(initial_data_grid(commondata, &griddata[grid], 0), __func__);
  die_on(cudaDeviceSynchronize() == cudaSuccess ? 0 : BSSN_B200_ECUDA, __func__);
}

static int malloc_gfs(double **p, size_t n) {
  if (cudaMalloc(p, n * sizeof(double)) != cudaSuccess) {
    set_error("cudaMalloc of %zu doubles failed", n);
    return BSSN_B200_ENOMEM;
  }
  return BSSN_B200_OK;
}
void MoL_malloc_y_n_gfs(const commondata_struct *, const params_struct *params, MoL_gridfunctions_struct *gridfuncs) {
  const size_t ntot = (size_t)params->Nxx_plus_2NGHOSTS0 * params->Nxx_plus_2NGHOSTS1 * params->Nxx_plus_2NGHOSTS2;
  die_on(malloc_gfs(&gridfuncs->y_n_gfs, ntot * NUM_EVOL_GFS), __func__);
  die_on(malloc_gfs(&gridfuncs->auxevol_gfs, ntot * NUM_AUXEVOL_GFS), __func__);
}
void MoL_malloc_intermediate_stage_gfs(const commondata_struct *, const params_struct *params,
                                       MoL_gridfunctions_struct *gridfuncs) {
  const size_t ntot = (size_t)params->Nxx_plus_2NGHOSTS0 * params->Nxx_plus_2NGHOSTS1 * params->Nxx_plus_2NGHOSTS2;
  die_on(malloc_gfs(&gridfuncs->y_nplus1_running_total_gfs, ntot * NUM_EVOL_GFS), __func__);
  die_on(malloc_gfs(&gridfuncs->k_odd_gfs, ntot * NUM_EVOL_GFS), __func__);
  die_on(malloc_gfs(&gridfuncs->k_even_gfs, ntot * NUM_EVOL_GFS), __func__);
  if (!gridfuncs->auxevol_gfs) die_on(malloc_gfs(&gridfuncs->auxevol_gfs, ntot * NUM_AUXEVOL_GFS), __func__);
}
void MoL_free_intermediate_stage_gfs(MoL_gridfunctions_struct *gridfuncs) {
  cudaFree(gridfuncs->y_nplus1_running_total_gfs);
  cudaFree(gridfuncs->k_odd_gfs);
  cudaFree(gridfuncs->k_even_gfs);
  gridfuncs->y_nplus1_running_total_gfs = gridfuncs->k_odd_gfs = gridfuncs->k_even_gfs = nullptr;
}

// ---------------------------------------------------------------- hot-path operators (status)
int bssn_b200_ricci_eval(const params_struct *params, const rfm_struct *rfmstruct, const REAL *in_gfs,
                         REAL *auxevol_gfs, void *stream) {
  BSSN_TRY(check_ptr(rfmstruct, "rfmstruct"));
  BSSN_TRY(check_ptr(in_gfs, "in_gfs"));
  BSSN_TRY(check_ptr(auxevol_gfs, "auxevol_gfs"));
  Variant v;
  BSSN_TRY(variant_of(params, &v));
  return launch_ricci(v, grid_dims(params), rfm_arrays(rfmstruct), in_gfs, auxevol_gfs, (cudaStream_t)stream);
}

static int rhs_common(const commondata_struct *cd, const params_struct *params, const rfm_struct *rfmstruct,
                      const REAL *aux, const REAL *in, REAL *rhs, bool mixed, void *stream) {
  BSSN_TRY(check_ptr(cd, "commondata"));
  BSSN_TRY(check_ptr(rfmstruct, "rfmstruct"));
  BSSN_TRY(check_ptr(aux, "auxevol_gfs"));
  BSSN_TRY(check_ptr(in, "in_gfs"));
  BSSN_TRY(check_ptr(rhs, "rhs_gfs"));
  Variant v;
  BSSN_TRY(variant_of(params, &v));
  const PhysParams pp{cd->eta, cd->KreissOliger_strength_gauge, cd->KreissOliger_strength_nongauge};
  return launch_rhs(v, mixed, grid_dims(params), rfm_arrays(rfmstruct), pp, aux, in, rhs, (cudaStream_t)stream);
}
int bssn_b200_rhs_eval(const commondata_struct *cd, const params_struct *params, const rfm_struct *rfmstruct,
                       const REAL *aux, const REAL *in, REAL *rhs, void *stream) {
  return rhs_common(cd, params, rfmstruct, aux, in, rhs, false, stream);
}
int bssn_b200_rhs_eval_mixed(const commondata_struct *cd, const params_struct *params, const rfm_struct *rfmstruct,
                             const REAL *aux, const REAL *in, REAL *rhs, void *stream) {
  return rhs_common(cd, params, rfmstruct, aux, in, rhs, true, stream);
}

int bssn_b200_apply_bcs_outerradiation_and_inner(const commondata_struct *, const params_struct *params,
                                                 const bc_struct *bcstruct, REAL *xx[3], const REAL *wavespeed,
                                                 const REAL *f_infinity, REAL *gfs, REAL *rhs_gfs, void *stream) {
  BSSN_TRY(check_ptr(params, "params"));
  BSSN_TRY(check_ptr(bcstruct, "bcstruct"));
  BSSN_TRY(check_ptr(gfs, "gfs"));
  BSSN_TRY(check_ptr(rhs_gfs, "rhs_gfs"));
  const GridDims g = grid_dims(params);
  const double *xxc[3] = {xx[0], xx[1], xx[2]};
  BSSN_TRY(launch_radiation_bcs(g, params, bcstruct, xxc, wavespeed, f_infinity, gfs, rhs_gfs, (cudaStream_t)stream));
  return launch_inner_bcs(g, bcstruct, rhs_gfs, NUM_EVOL_GFS, nullptr, (cudaStream_t)stream);
}
int bssn_b200_apply_bcs_outerextrap_and_inner(const params_struct *params, const bc_struct *bcstruct, REAL *gfs,
                                              void *stream) {
  BSSN_TRY(check_ptr(params, "params"));
  BSSN_TRY(check_ptr(bcstruct, "bcstruct"));
  BSSN_TRY(check_ptr(gfs, "gfs"));
  const GridDims g = grid_dims(params);
  BSSN_TRY(launch_extrap_bcs(g, bcstruct, gfs, (cudaStream_t)stream));
  return launch_inner_bcs(g, bcstruct, gfs, NUM_EVOL_GFS, nullptr, (cudaStream_t)stream);
}
int bssn_b200_apply_bcs_inner_only(const params_struct *params, const bc_struct *bcstruct, REAL *gfs, int num_gfs,
                                   const int8_t *gf_parity_types, void *stream) {
  BSSN_TRY(check_ptr(params, "params"));
  BSSN_TRY(check_ptr(bcstruct, "bcstruct"));
  BSSN_TRY(check_ptr(gfs, "gfs"));
  return launch_inner_bcs(grid_dims(params), bcstruct, gfs, num_gfs, gf_parity_types, (cudaStream_t)stream);
}
int bssn_b200_enforce_detgammabar_equals_detgammahat(const params_struct *params, const rfm_struct *rfmstruct,
                                                     REAL *in_gfs, void *stream) {
  BSSN_TRY(check_ptr(rfmstruct, "rfmstruct"));
  BSSN_TRY(check_ptr(in_gfs, "in_gfs"));
  Variant v;
  BSSN_TRY(variant_of(params, &v));
  return launch_enforce(v, grid_dims(params), rfm_arrays(rfmstruct), in_gfs, (cudaStream_t)stream);
}
int bssn_b200_constraints_eval(const commondata_struct *, const params_struct *params, const rfm_struct *rfmstruct,
                               const REAL *in_gfs, const REAL *auxevol_gfs, REAL *diagnostic_gfs, void *stream) {
  BSSN_TRY(check_ptr(rfmstruct, "rfmstruct"));
  BSSN_TRY(check_ptr(in_gfs, "in_gfs"));
  BSSN_TRY(check_ptr(auxevol_gfs, "auxevol_gfs"));
  BSSN_TRY(check_ptr(diagnostic_gfs, "diagnostic_gfs"));
  Variant v;
  BSSN_TRY(variant_of(params, &v));
  return launch_constraints(v, grid_dims(params), rfm_arrays(rfmstruct), in_gfs, auxevol_gfs, diagnostic_gfs,
                            (cudaStream_t)stream);
}

int bssn_b200_constraint_integrals(const params_struct *params, const rfm_struct *rfmstruct,
                                   const REAL *diagnostic_gfs, double out[4], void *stream) {
  BSSN_TRY(check_ptr(params, "params"));
  BSSN_TRY(check_ptr(rfmstruct, "rfmstruct"));
  BSSN_TRY(check_ptr(diagnostic_gfs, "diagnostic_gfs"));
  BSSN_TRY(check_ptr(out, "out"));
  static std::mutex mu;
  static double *scratch[64] = {nullptr};
  int dev = 0;
  BSSN_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error("device ordinal %d out of range", dev);
    return BSSN_B200_EINVAL;
  }
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!scratch[dev]) BSSN_CUDA_TRY(cudaMalloc(&scratch[dev], sizeof(double) * constraint_integrals_scratch_doubles()));
  }
  return constraint_integrals(params, rfm_arrays(rfmstruct), diagnostic_gfs, scratch[dev], out, (cudaStream_t)stream);
}

int bssn_b200_constraint_integrals_noalloc(const params_struct *params, const rfm_struct *rfmstruct,
                                           const REAL *diagnostic_gfs, double out[4], void *stream) {
  BSSN_TRY(check_ptr(params, "params"));
  BSSN_TRY(check_ptr(rfmstruct, "rfmstruct"));
  BSSN_TRY(check_ptr(diagnostic_gfs, "diagnostic_gfs"));
  BSSN_TRY(check_ptr(out, "out"));
  return constraint_integrals_noalloc(params, rfm_arrays(rfmstruct), diagnostic_gfs, out, (cudaStream_t)stream);
}

int bssn_b200_mol_step(commondata_struct *commondata, griddata_struct *griddata, int mode, int mixed, void *stream) {
  BSSN_TRY(check_ptr(commondata, "commondata"));
  BSSN_TRY(check_ptr(griddata, "griddata"));
  return mol_step(commondata, griddata, mode, mixed, (cudaStream_t)stream);
}

int bssn_b200_stepper_create(commondata_struct *cd, griddata_struct *gd, int mode, int mixed, int steps_per_graph,
                             void *stream, bssn_b200_stepper **out) {
  BSSN_TRY(check_ptr(cd, "commondata"));
  BSSN_TRY(check_ptr(gd, "griddata"));
  BSSN_TRY(check_ptr(out, "out"));
  if (steps_per_graph < 1 || steps_per_graph > 1000) {
    set_error("steps_per_graph=%d not in [1,1000]", steps_per_graph);
    return BSSN_B200_EINVAL;
  }
  cudaStream_t s = (cudaStream_t)stream;
  if (s == nullptr) {
    set_error("stepper: capture needs a non-default stream");
    return BSSN_B200_EINVAL;
  }
  BSSN_TRY(mol_prepare(cd, gd, mode));
  // Capture on a copy of commondata so that time/nn advance only when the graph runs.
  commondata_struct tmp = *cd;
  BSSN_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  int rc = BSSN_B200_OK;
  for (int n = 0; n < steps_per_graph && rc == BSSN_B200_OK; n++) rc = mol_step(&tmp, gd, mode, mixed, s);
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(s, &graph);
  if (rc != BSSN_B200_OK) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e != cudaSuccess) {
    set_error("stream capture failed: %s", cudaGetErrorString(e));
    return BSSN_B200_ECUDA;
  }
  cudaGraphExec_t exec = nullptr;
  e = cudaGraphInstantiate(&exec, graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    set_error("graph instantiate failed: %s", cudaGetErrorString(e));
    return BSSN_B200_ECUDA;
  }
  size_t nnodes = 0;
  BSSN_CUDA_TRY(cudaGraphGetNodes(graph, nullptr, &nnodes));
  std::vector<cudaGraphNode_t> nodes(nnodes);
  unsigned long long nkern = 0;
  if (nnodes) BSSN_CUDA_TRY(cudaGraphGetNodes(graph, nodes.data(), &nnodes));
  for (size_t k = 0; k < nnodes; k++) {
    cudaGraphNodeType t;
    BSSN_CUDA_TRY(cudaGraphNodeGetType(nodes[k], &t));
    if (t == cudaGraphNodeTypeKernel) nkern++;
  }
  bssn_b200_stepper *st = new bssn_b200_stepper{cd, gd, s, graph, exec, steps_per_graph, nkern};
  *out = st;
  return BSSN_B200_OK;
}

int bssn_b200_stepper_run(bssn_b200_stepper *st, int graph_launches) {
  BSSN_TRY(check_ptr(st, "stepper"));
  for (int n = 0; n < graph_launches; n++) {
    BSSN_CUDA_TRY(cudaGraphLaunch(st->exec, st->stream));
    count_launch(st->kernel_nodes);
    for (int k = 0; k < st->steps_per_graph; k++) {
      st->cd->time = st->cd->t_0 + (double)(st->cd->nn - st->cd->nn_0 + 1) * st->cd->dt;
      st->cd->nn++;
    }
  }
  return BSSN_B200_OK;
}

int bssn_b200_stepper_kernel_nodes(const bssn_b200_stepper *st, unsigned long long *out) {
  BSSN_TRY(check_ptr(st, "stepper"));
  BSSN_TRY(check_ptr(out, "out"));
  *out = st->kernel_nodes;
  return BSSN_B200_OK;
}

unsigned long long bssn_b200_kernel_launches(void) { return g_launches.load(); }

int bssn_b200_fp64_fma_rate(int reps, double *out_tflops, void *stream) {
  BSSN_TRY(check_ptr(out_tflops, "out_tflops"));
  if (reps < 1 || reps > 100) {
    set_error("reps=%d not in [1,100]", reps);
    return BSSN_B200_EINVAL;
  }
  return fp64_fma_rate(reps, out_tflops, (cudaStream_t)stream);
}

int bssn_b200_rhs_fused_stage(commondata_struct *cd, griddata_struct *gd, int stage, int mixed, void *stream) {
  BSSN_TRY(check_ptr(cd, "commondata"));
  BSSN_TRY(check_ptr(gd, "griddata"));
  return fused_interior_stage(cd, gd, 0, stage, mixed, (cudaStream_t)stream);
}

int bssn_b200_stepper_destroy(bssn_b200_stepper *st) {
  if (!st) return BSSN_B200_OK;
  if (st->exec) cudaGraphExecDestroy(st->exec);
  if (st->graph) cudaGraphDestroy(st->graph);
  delete st;
  return BSSN_B200_OK;
}

int bssn_b200_memcpy(void *dst, const void *src, size_t bytes, int kind) {
  if (bytes == 0) return BSSN_B200_OK;
  BSSN_TRY(check_ptr(dst, "dst"));
  BSSN_TRY(check_ptr(src, "src"));
  cudaMemcpyKind k;
  switch (kind) {
    case 0: k = cudaMemcpyHostToDevice; break;
    case 1: k = cudaMemcpyDeviceToHost; break;
    case 2: k = cudaMemcpyDeviceToDevice; break;
    default: set_error("memcpy kind %d not in {0,1,2}", kind); return BSSN_B200_EINVAL;
  }
  BSSN_CUDA_TRY(cudaMemcpy(dst, src, bytes, k));
  return BSSN_B200_OK;
}

int bssn_b200_device_synchronize(void) {
  BSSN_CUDA_TRY(cudaDeviceSynchronize());
  return BSSN_B200_OK;
}

// ---------------------------------------------------------------- hot-path operators (void, drop-in)
void Ricci_eval(const params_struct *params, const rfm_struct *rfmstruct, const REAL *in_gfs, REAL *auxevol_gfs) {
  die_on(bssn_b200_ricci_eval(params, rfmstruct, in_gfs, auxevol_gfs, nullptr), __func__);
}
void rhs_eval(const commondata_struct *commondata, const params_struct *params, const rfm_struct *rfmstruct,
              const REAL *auxevol_gfs, const REAL *in_gfs, REAL *rhs_gfs) {
  die_on(bssn_b200_rhs_eval(commondata, params, rfmstruct, auxevol_gfs, in_gfs, rhs_gfs, nullptr), __func__);
}
void apply_bcs_outerradiation_and_inner(const commondata_struct *commondata, const params_struct *params,
                                        const bc_struct *bcstruct, REAL *xx[3], const REAL custom_wavespeed[NUM_EVOL_GFS],
                                        const REAL custom_f_infinity[NUM_EVOL_GFS], REAL *gfs, REAL *rhs_gfs) {
  die_on(bssn_b200_apply_bcs_outerradiation_and_inner(commondata, params, bcstruct, xx, custom_wavespeed,
                                                      custom_f_infinity, gfs, rhs_gfs, nullptr),
         __func__);
}
void apply_bcs_outerextrap_and_inner(const commondata_struct *, const params_struct *params, const bc_struct *bcstruct,
                                     REAL *gfs) {
  die_on(bssn_b200_apply_bcs_outerextrap_and_inner(params, bcstruct, gfs, nullptr), __func__);
}
void apply_bcs_inner_only(const commondata_struct *, const params_struct *params, const bc_struct *bcstruct,
                          REAL *gfs) {
  die_on(bssn_b200_apply_bcs_inner_only(params, bcstruct, gfs, NUM_EVOL_GFS, nullptr, nullptr), __func__);
}
void enforce_detgammabar_equals_detgammahat(const params_struct *params, const rfm_struct *rfmstruct, REAL *in_gfs,
                                            const REAL *) {
  die_on(bssn_b200_enforce_detgammabar_equals_detgammahat(params, rfmstruct, in_gfs, nullptr), __func__);
}
void MoL_step_forward_in_time(commondata_struct *commondata, griddata_struct *griddata) {
  die_on(bssn_b200_mol_step(commondata, griddata, 0, 0, nullptr), __func__);
}
void constraints_eval(const commondata_struct *commondata, const params_struct *params, const rfm_struct *rfmstruct,
                      const REAL *in_gfs, const REAL *auxevol_gfs, REAL *diagnostic_gfs) {
  // The generated project's diagnostic array: BSSN_B200_TOTAL_NUM_DIAG_GFS gridfunctions.
  (void)commondata;
  static const int slots[3] = {BSSN_B200_DIAG_HAMILTONIANGF, BSSN_B200_DIAG_MSQUAREDGF,
                               BSSN_B200_DIAG_LAMBDA_CONSTRAINTGF};
  int rc = check_ptr(rfmstruct, "rfmstruct");
  if (rc == BSSN_B200_OK) rc = check_ptr(in_gfs, "in_gfs");
  if (rc == BSSN_B200_OK) rc = check_ptr(auxevol_gfs, "auxevol_gfs");
  if (rc == BSSN_B200_OK) rc = check_ptr(diagnostic_gfs, "diagnostic_gfs");
  Variant v;
  if (rc == BSSN_B200_OK) rc = variant_of(params, &v);
  if (rc == BSSN_B200_OK)
    rc = launch_constraints(v, grid_dims(params), rfm_arrays(rfmstruct), in_gfs, auxevol_gfs, diagnostic_gfs, nullptr,
                            slots);
  die_on(rc, __func__);
}

}  // extern "C"
