// Oracle harness for the reference's own CUDA build (nrpy --cuda, compiled for sm_100a).
//
// Test and measurement infrastructure only: it is compiled together with the CUDA sources
// that the reference's generator emits (oracle/gen_ref.py, variant sinh3d_cuda) and exposes
// flat entry points for ctypes. It performs the set-up of the generated CUDA main() and
// numerical_grids_and_timestep() (nrpy/infrastructures/BHaH/main_c.py:125-343,
// numerical_grids_and_timestep.py:31-190): stream and __constant__ set-up
// (BHaH_CUDA_global_init.h), defaults, numerical_grid_params_Nxx_dxx_xx with the caller's Nx,
// the device and host rfm_struct, bcstruct_set_up (host + device copies), the CFL time step,
// device y_n / auxevol storage, initial_data and MoL_malloc_intermediate_stage_gfs. Each step
// is the generated MoL_step_forward_in_time(commondata, griddata_device), unchanged.
#include "BHaH_defines.h"
#include "BHaH_function_prototypes.h"
#include "BHaH_global_device_defines.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>

struct refc_sim {
  commondata_struct commondata;
  griddata_struct *gd;  // device-side griddata, as main()'s griddata_device
  griddata_struct *gh;  // host mirror, as main()'s griddata_host
  cudaEvent_t e0, e1;
};

static bool g_refc_init = false;

static void refc_global_init() {
  if (g_refc_init) return;
#include "BHaH_CUDA_global_init.h"
  g_refc_init = true;
}

extern "C" refc_sim *refc_create(const int Nx0, const int Nx1, const int Nx2, const double grid_physical_size,
                                 const double sinhw, const double m1, const double z1, const double m2, const double z2,
                                 const double cfl) {
  refc_global_init();
  refc_sim *s = (refc_sim *)calloc(1, sizeof(refc_sim));
  s->gd = (griddata_struct *)calloc(MAXNUMGRIDS, sizeof(griddata_struct));
  s->gh = (griddata_struct *)calloc(MAXNUMGRIDS, sizeof(griddata_struct));
  commondata_struct *cd = &s->commondata;
  commondata_struct_set_to_default(cd);
  cd->BH1_mass = m1;
  cd->BH1_posn_z = z1;
  cd->BH2_mass = m2;
  cd->BH2_posn_z = z2;
  cd->CFL_FACTOR = cfl;
  params_struct_set_to_default(cd, s->gd);
  for (int grid = 0; grid < MAXNUMGRIDS; grid++) s->gd[grid].params.is_host = false;
  params_struct *params = &s->gd[0].params;
  snprintf(params->gridname, 100, "grid_SinhSpherical");
  params->CoordSystem_hash = SINHSPHERICAL;
  params->grid_physical_size = grid_physical_size;
  params->SINHW = sinhw;
  params->grid_idx = 0;
  const int Nx[3] = {Nx0, Nx1, Nx2};
  numerical_grid_params_Nxx_dxx_xx(cd, params, s->gd[0].xx, Nx, true);
  memcpy(&s->gh[0].params, params, sizeof(params_struct));
  s->gh[0].params.is_host = true;
  cd->NUMGRIDS = 1;
  cpyDevicetoHost__grid(cd, s->gh, s->gd);
  BHAH_DEVICE_SYNC();
  BHAH_MALLOC_DEVICE(s->gd[0].rfmstruct, sizeof(rfm_struct));
  cpyHosttoDevice_params__constant(params, params->grid_idx % NUM_STREAMS);
  rfm_precompute_malloc(cd, params, s->gd[0].rfmstruct);
  rfm_precompute_defines(cd, params, s->gd[0].rfmstruct, s->gd[0].xx);
  BHAH_MALLOC(s->gh[0].rfmstruct, sizeof(rfm_struct));
  rfm_precompute_malloc(cd, &s->gh[0].params, s->gh[0].rfmstruct);
  rfm_precompute_defines(cd, &s->gh[0].params, s->gh[0].rfmstruct, s->gh[0].xx);
  bcstruct_set_up(cd, params, s->gh[0].xx, &s->gh[0].bcstruct, &s->gd[0].bcstruct);
  cd->dt = 1e30;
  cpyHosttoDevice_params__constant(params, params->grid_idx % NUM_STREAMS);
  cfl_limited_timestep(cd, params, s->gd[0].xx);
  cd->nn = 0;
  cd->nn_0 = 0;
  cd->t_0 = 0.0;
  cd->time = 0.0;
  const size_t ntot = (size_t)params->Nxx_plus_2NGHOSTS0 * params->Nxx_plus_2NGHOSTS1 * params->Nxx_plus_2NGHOSTS2;
  BHAH_MALLOC_DEVICE(s->gd[0].gridfuncs.y_n_gfs, sizeof(REAL) * ntot * NUM_EVOL_GFS);
  BHAH_MALLOC_DEVICE(s->gd[0].gridfuncs.auxevol_gfs, sizeof(REAL) * ntot * NUM_AUXEVOL_GFS);
  BHAH_MALLOC(s->gh[0].gridfuncs.auxevol_gfs, sizeof(REAL) * ntot * NUM_AUXEVOL_GFS);
  BHAH_MALLOC_PINNED(s->gh[0].gridfuncs.y_n_gfs, sizeof(REAL) * ntot * NUM_EVOL_GFS);
  initial_data(cd, s->gh, s->gd);
  MoL_malloc_intermediate_stage_gfs(cd, params, &s->gd[0].gridfuncs);
  BHAH_DEVICE_SYNC();
  cudaEventCreate(&s->e0);
  cudaEventCreate(&s->e1);
  return s;
}

extern "C" int refc_N(refc_sim *s, int d) {
  const params_struct *p = &s->gd[0].params;
  return d == 0 ? p->Nxx_plus_2NGHOSTS0 : (d == 1 ? p->Nxx_plus_2NGHOSTS1 : p->Nxx_plus_2NGHOSTS2);
}
extern "C" double refc_dt(refc_sim *s) { return s->commondata.dt; }
extern "C" int refc_nn(refc_sim *s) { return s->commondata.nn; }

static size_t refc_ntot(refc_sim *s) { return (size_t)refc_N(s, 0) * refc_N(s, 1) * refc_N(s, 2); }

// Host <-> device copies of the evolved state y_n_gfs (24 gridfunctions, IDX4 layout).
extern "C" int refc_set_y_n(refc_sim *s, const double *host) {
  cudaError_t e = cudaMemcpy(s->gd[0].gridfuncs.y_n_gfs, host, sizeof(REAL) * refc_ntot(s) * NUM_EVOL_GFS,
                             cudaMemcpyHostToDevice);
  return e == cudaSuccess ? 0 : -1;
}
extern "C" int refc_get_y_n(refc_sim *s, double *host) {
  cudaError_t e = cudaMemcpy(host, s->gd[0].gridfuncs.y_n_gfs, sizeof(REAL) * refc_ntot(s) * NUM_EVOL_GFS,
                             cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? 0 : -1;
}

// n calls of the generated MoL_step_forward_in_time; returns the device time in ms between
// events recorded on the generated code's stream before the first and after the last step.
extern "C" double refc_steps(refc_sim *s, const int n) {
  cudaDeviceSynchronize();
  cudaEventRecord(s->e0, streams[0]);
  for (int k = 0; k < n; k++) MoL_step_forward_in_time(&s->commondata, s->gd);
  cudaEventRecord(s->e1, streams[0]);
  cudaEventSynchronize(s->e1);
  cudaDeviceSynchronize();
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, s->e0, s->e1);
  return cudaGetLastError() == cudaSuccess ? (double)ms : -1.0;
}

extern "C" void refc_destroy(refc_sim *s) {
  BHAH_DEVICE_SYNC();
  cudaEventDestroy(s->e0);
  cudaEventDestroy(s->e1);
  griddata_free_device(&s->commondata, s->gd, true);
  // main() allocates the host auxevol copy with BHAH_MALLOC; release it the same way before
  // griddata_free (which would pass it to cudaFreeHost).
  BHAH_FREE(s->gh[0].gridfuncs.auxevol_gfs);
  griddata_free(&s->commondata, s->gh, true);
  free(s);
}
