// Method-of-lines RK4 time step on the device.
//
// mode 0 follows the reference stage by stage (MoL_step_forward_in_time.py:322-485):
//   Ricci_eval -> rhs_eval -> outer radiation + inner BCs on the RHS -> rk_substep_s over
//   all points -> [extrapolation + inner BCs] -> detgammabar projection over all points.
// mode 1 fuses each stage into three passes: Ricci_eval; RHS + RK update + projection on
//   the interior (the raw RHS kept only on the interior shell); then the outer points
//   (radiation RHS, RK update, projection) and parity copies of the stage output into the
//   inner ghost points. Inner ghost points of the stage output are parity copies of
//   updated interior points instead of RK updates of parity copies; the two agree exactly
//   before the projection, which is evaluated at the source point.
#include <cstring>

#include "bssn_common.cuh"

namespace bssn {

// rk_substep_{1..4} over all points of all 24 gridfunctions (2 doubles per thread).
template <int STAGE>
__global__ void rk_substep_kernel(const size_t n, double *__restrict__ k, double *__restrict__ y,
                                  double *__restrict__ run, const double dt) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double kv = k[i];
  const double yv = y[i];
  if constexpr (STAGE == 1) {
    run[i] = (1.0 / 6.0) * dt * kv;
    k[i] = (1.0 / 2.0) * dt * kv + yv;
  } else if constexpr (STAGE == 2) {
    run[i] = (1.0 / 3.0) * dt * kv + run[i];
    k[i] = (1.0 / 2.0) * dt * kv + yv;
  } else if constexpr (STAGE == 3) {
    run[i] = (1.0 / 3.0) * dt * kv + run[i];
    k[i] = dt * kv + yv;
  } else {
    y[i] = (1.0 / 6.0) * dt * kv + yv + run[i];
  }
}

int launch_rk_substep(int stage, double dt, const GridDims &g, const StageBuffers &b, cudaStream_t s) {
  const size_t n = (size_t)g.ntot * NUM_EVOL_GFS;
  const int threads = 256;
  const unsigned blocks = (unsigned)((n + threads - 1) / threads);
  switch (stage) {
    case 1: rk_substep_kernel<1><<<blocks, threads, 0, s>>>(n, b.kout, b.y, b.run, dt); break;
    case 2: rk_substep_kernel<2><<<blocks, threads, 0, s>>>(n, b.kout, b.y, b.run, dt); break;
    case 3: rk_substep_kernel<3><<<blocks, threads, 0, s>>>(n, b.kout, b.y, b.run, dt); break;
    case 4: rk_substep_kernel<4><<<blocks, threads, 0, s>>>(n, b.kout, b.y, b.run, dt); break;
    default: set_error("RK4 stage %d out of range", stage); return BSSN_B200_EINVAL;
  }
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

// Per-grid scratch for mode 1: raw RHS on the interior shell and the outer ghost points.
struct GridScratch {
  double *krhs = nullptr;
  size_t bytes = 0;
};
static GridScratch g_scratch[MAXNUMGRIDS];

static int ensure_scratch(int grid, size_t bytes) {
  GridScratch &sc = g_scratch[grid];
  if (sc.bytes >= bytes) return BSSN_B200_OK;
  if (sc.krhs) cudaFree(sc.krhs);
  sc.krhs = nullptr;
  sc.bytes = 0;
  if (cudaMalloc(&sc.krhs, bytes) != cudaSuccess) {
    set_error("cudaMalloc of %zu bytes for the fused-stage RHS shell failed", bytes);
    return BSSN_B200_ENOMEM;
  }
  sc.bytes = bytes;
  return BSSN_B200_OK;
}

static int stage_buffers(const MoL_gridfunctions_struct &gf, int stage, StageBuffers *b) {
  // IN -> K (= OUT for stages 1-3) -> OUT, as the reference's k_odd / k_even rotation.
  b->y = gf.y_n_gfs;
  b->run = gf.y_nplus1_running_total_gfs;
  switch (stage) {
    case 1: b->kin = gf.y_n_gfs; b->kout = gf.k_odd_gfs; break;
    case 2: b->kin = gf.k_odd_gfs; b->kout = gf.k_even_gfs; break;
    case 3: b->kin = gf.k_even_gfs; b->kout = gf.k_odd_gfs; break;
    default: b->kin = gf.k_odd_gfs; b->kout = gf.k_even_gfs; break;
  }
  if (!b->y || !b->run || !b->kin || !b->kout || !gf.auxevol_gfs) {
    set_error("MoL step: gridfunction storage not allocated (call MoL_malloc_intermediate_stage_gfs)");
    return BSSN_B200_EINVAL;
  }
  return BSSN_B200_OK;
}

static bool outer_is(const commondata_struct *cd, const char *what) {
  return strncmp(cd->outer_bc_type, what, 50) == 0;
}

int mol_stage(const commondata_struct *cd, griddata_struct *gd, int grid, int stage, int mode, int mixed,
              cudaStream_t s) {
  griddata_struct &G = gd[grid];
  const params_struct *p = &G.params;
  Variant v;
  BSSN_TRY(variant_of(p, &v));
  const GridDims g = grid_dims(p);
  const RfmArrays rfm = rfm_arrays(G.rfmstruct);
  const PhysParams pp{cd->eta, cd->KreissOliger_strength_gauge, cd->KreissOliger_strength_nongauge};
  StageBuffers b;
  BSSN_TRY(stage_buffers(G.gridfuncs, stage, &b));
  const double dt = cd->dt;
  const bool radiation = outer_is(cd, "radiation");
  const bool extrap = outer_is(cd, "extrapolation");
  // In the stage-4 RK update the reference writes y_n in place; OUT is y_n then.
  BSSN_TRY(launch_ricci(v, g, rfm, b.kin, G.gridfuncs.auxevol_gfs, s, mixed != 0));
  if (mode == 0) {
    BSSN_TRY(launch_rhs(v, mixed != 0, g, rfm, pp, G.gridfuncs.auxevol_gfs, b.kin, b.kout, s));
    if (radiation) {
      BSSN_TRY(launch_radiation_bcs(g, p, &G.bcstruct, G.xx, kWavespeed, kFInfinity, b.kin, b.kout, s));
      BSSN_TRY(launch_inner_bcs(g, &G.bcstruct, b.kout, NUM_EVOL_GFS, nullptr, s));
    }
    BSSN_TRY(launch_rk_substep(stage, dt, g, b, s));
    double *out = (stage == 4) ? b.y : b.kout;
    if (extrap) {
      BSSN_TRY(launch_extrap_bcs(g, &G.bcstruct, out, s));
      BSSN_TRY(launch_inner_bcs(g, &G.bcstruct, out, NUM_EVOL_GFS, nullptr, s));
    }
    return launch_enforce(v, g, rfm, out, s);
  }
  // mode 1 (fused)
  if (!radiation) {
    set_error("fused MoL stages support outer_bc_type \"radiation\" only");
    return BSSN_B200_EINVAL;
  }
  BSSN_TRY(ensure_scratch(grid, (size_t)g.ntot * NUM_EVOL_GFS * sizeof(double)));
  StageBuffers bo = b;
  if (stage == 4) bo.kout = b.y;  // stage 4 writes y_n
  BSSN_TRY(launch_rhs_fused_stage(v, mixed != 0, stage, dt, g, rfm, pp, G.gridfuncs.auxevol_gfs, bo,
                                  g_scratch[grid].krhs, s));
  return launch_radiation_rk_bcs(v, g, p, &G.bcstruct, G.xx, rfm, stage, dt, bo, g_scratch[grid].krhs, s);
}

// Allocate the per-grid scratch outside any stream capture.
int mol_prepare(const commondata_struct *cd, griddata_struct *gd, int mode) {
  if (mode != 1) return BSSN_B200_OK;
  for (int grid = 0; grid < cd->NUMGRIDS; grid++) {
    const GridDims g = grid_dims(&gd[grid].params);
    BSSN_TRY(ensure_scratch(grid, (size_t)g.ntot * NUM_EVOL_GFS * sizeof(double)));
  }
  return BSSN_B200_OK;
}

// Only the interior kernel of a fused stage (for timing the dominant kernel in isolation).
int fused_interior_stage(const commondata_struct *cd, griddata_struct *gd, int grid, int stage, int mixed,
                         cudaStream_t s) {
  griddata_struct &G = gd[grid];
  Variant v;
  BSSN_TRY(variant_of(&G.params, &v));
  const GridDims g = grid_dims(&G.params);
  StageBuffers b;
  BSSN_TRY(stage_buffers(G.gridfuncs, stage, &b));
  if (stage == 4) b.kout = b.y;
  BSSN_TRY(ensure_scratch(grid, (size_t)g.ntot * NUM_EVOL_GFS * sizeof(double)));
  const PhysParams pp{cd->eta, cd->KreissOliger_strength_gauge, cd->KreissOliger_strength_nongauge};
  return launch_rhs_fused_stage(v, mixed != 0, stage, cd->dt, g, rfm_arrays(G.rfmstruct), pp, G.gridfuncs.auxevol_gfs,
                                b, g_scratch[grid].krhs, s);
}

int mol_step(commondata_struct *cd, griddata_struct *gd, int mode, int mixed, cudaStream_t s) {
  if (mode != 0 && mode != 1) {
    set_error("MoL step: mode %d not in {0,1}", mode);
    return BSSN_B200_EINVAL;
  }
  if (cd->NUMGRIDS < 1 || cd->NUMGRIDS > MAXNUMGRIDS) {
    set_error("MoL step: NUMGRIDS=%d out of range", cd->NUMGRIDS);
    return BSSN_B200_EINVAL;
  }
  const double time_start = cd->time;
  static const double stage_time[4] = {0.0, 0.5, 0.5, 1.0};
  for (int stage = 1; stage <= 4; stage++) {
    for (int grid = 0; grid < cd->NUMGRIDS; grid++) {
      cd->time = time_start + stage_time[stage - 1] * cd->dt;
      BSSN_TRY(mol_stage(cd, gd, grid, stage, mode, mixed, s));
    }
  }
  cd->time = cd->t_0 + (double)(cd->nn - cd->nn_0 + 1) * cd->dt;
  cd->nn++;
  return BSSN_B200_OK;
}

}  // namespace bssn
