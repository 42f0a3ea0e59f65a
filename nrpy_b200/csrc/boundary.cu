// Curvilinear boundary conditions on the device.
//
// * inner (parity) BCs: gf[dst] = +/- gf[src], apply_bcs_inner_only.py:26-199. The sign
//   is applied by flipping the IEEE sign bit (the reference's apply_parity_branchless), so
//   the copy is exact. Source points are interior or pure-outer points, never other inner
//   points, so all copies are independent.
// * outer radiation BCs on the RHS: apply_bcs_outerradiation_and_inner.py:46-723, one
//   launch per (ghost layer, face direction) in the reference's order because a layer's
//   points read the RHS of the layer inside it.
// * outer extrapolation BCs: f0 = 3 f1 - 3 f2 + f3 along the face normal,
//   apply_bcs_outerextrap_and_inner.py:28-157.
#include "bssn_common.cuh"

namespace bssn {

const int8_t kEvolParity[NUM_EVOL_GFS] = {4, 5, 6, 7, 8, 9, 0, 1, 2, 3, 0, 4, 5, 6, 7, 8, 9, 1, 2, 3, 0, 1, 2, 3};
const double kWavespeed[NUM_EVOL_GFS] = {1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.41421356237310, 1.0, 1.0, 1.0, 1.0, 1.0,
                                         1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0};
const double kFInfinity[NUM_EVOL_GFS] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 1.0, 0.0,
                                         0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};

struct GfTable {
  int8_t parity[NUM_EVOL_GFS];
  double wavespeed[NUM_EVOL_GFS];
  double finf[NUM_EVOL_GFS];
};

__device__ __forceinline__ double flip_sign(double v, int8_t p) {
  unsigned long long bits = __double_as_longlong(v);
  bits ^= (unsigned long long)(p < 0) << 63;
  return __longlong_as_double(bits);
}

// One thread per (inner point, gridfunction); the point index runs fastest so that the
// parity records of a warp are contiguous.
__global__ void inner_bcs_kernel(const int ntot, const innerpt_bc_struct *__restrict__ pts, const int npts,
                                 double *__restrict__ gfs, const int num_gfs, const GfTable tab) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * num_gfs) return;
  const int gf = t / npts;
  const int pt = t - gf * npts;
  const innerpt_bc_struct bc = pts[pt];
  double *g = gfs + (size_t)gf * ntot;
  g[bc.dstpt] = flip_sign(g[bc.srcpt], bc.parity[tab.parity[gf]]);
}

int launch_inner_bcs(const GridDims &g, const bc_struct *bc, double *gfs, int num_gfs, const int8_t *parity_types,
                     cudaStream_t s) {
  const int npts = bc->bc_info.num_inner_boundary_points;
  if (npts <= 0 || num_gfs <= 0) return BSSN_B200_OK;
  if (num_gfs > NUM_EVOL_GFS) {
    set_error("inner BCs: num_gfs=%d exceeds %d", num_gfs, NUM_EVOL_GFS);
    return BSSN_B200_EINVAL;
  }
  GfTable tab{};
  for (int k = 0; k < num_gfs; k++) {
    const int8_t p = parity_types ? parity_types[k] : kEvolParity[k];
    if (p < 0 || p > 9) {
      set_error("inner BCs: parity type %d of gridfunction %d not in 0..9", (int)p, k);
      return BSSN_B200_EINVAL;
    }
    tab.parity[k] = p;
  }
  const long long work = (long long)npts * num_gfs;
  const int threads = 256;
  inner_bcs_kernel<<<(unsigned)((work + threads - 1) / threads), threads, 0, s>>>(g.ntot, bc->inner_bc_array, npts,
                                                                                   gfs, num_gfs, tab);
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

// ---------------------------------------------------------------- radiation
// 4th-order first derivative along i0 on a 5-point stencil shifted by `offset` (-2..2),
// FD1_arbitrary_upwind_x0_dirn of the reference (radiation_BC_fd_order = 4).
__device__ __forceinline__ double fd1_x0(const double *__restrict__ f, int idx, int offset, double invdx) {
  switch (offset) {
    case 0:
      return ((1.0 / 12.0) * f[idx - 2] - (2.0 / 3.0) * f[idx - 1] + (2.0 / 3.0) * f[idx + 1] -
              (1.0 / 12.0) * f[idx + 2]) * invdx;
    case 1:
      return (-(1.0 / 4.0) * f[idx - 1] - (5.0 / 6.0) * f[idx] + (3.0 / 2.0) * f[idx + 1] - (1.0 / 2.0) * f[idx + 2] +
              (1.0 / 12.0) * f[idx + 3]) * invdx;
    case -1:
      return (-(1.0 / 12.0) * f[idx - 3] + (1.0 / 2.0) * f[idx - 2] - (3.0 / 2.0) * f[idx - 1] + (5.0 / 6.0) * f[idx] +
              (1.0 / 4.0) * f[idx + 1]) * invdx;
    case 2:
      return (-(25.0 / 12.0) * f[idx] + 4.0 * f[idx + 1] - 3.0 * f[idx + 2] + (4.0 / 3.0) * f[idx + 3] -
              (1.0 / 4.0) * f[idx + 4]) * invdx;
    default:  // -2
      return ((1.0 / 4.0) * f[idx - 4] - (4.0 / 3.0) * f[idx - 3] + 3.0 * f[idx - 2] - 4.0 * f[idx - 1] +
              (25.0 / 12.0) * f[idx]) * invdx;
  }
}

__device__ __forceinline__ int fd1_offset(int dest_i0, int face, int N0) {
  const int R = 2;  // stencil radius for 4th order
  int off = face;
  if (dest_i0 < R) off = R - dest_i0;
  else if (dest_i0 > N0 - R - 1) off = (N0 - R - 1) - dest_i0;
  return off;
}

// One thread per (outer point, gridfunction) of one (layer, direction) list.
__global__ void radiation_kernel(const GridDims g, const RadialMap rm, const double *__restrict__ xx0,
                                 const outerpt_bc_struct *__restrict__ pts, const int npts,
                                 const double *__restrict__ gfs, double *__restrict__ rhs, const GfTable tab) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * NUM_EVOL_GFS) return;
  const int gf = t / npts;
  const int pt = t - gf * npts;
  const outerpt_bc_struct p = pts[pt];
  const int i0 = p.i0, i1 = p.i1, i2 = p.i2;
  const int j0 = i0 + p.FACEX0, j1 = i1 + p.FACEX1, j2 = i2 + p.FACEX2;
  double r, dx0dr, r_int, dx0dr_int;
  rm.eval(xx0[i0], r, dx0dr);
  rm.eval(xx0[j0], r_int, dx0dr_int);
  const double *f = gfs + (size_t)gf * g.ntot;
  const int idx = i0 + g.s1 * i1 + g.s2 * i2;
  const int idx_int = j0 + g.s1 * j1 + g.s2 * j2;
  const double dfdr = dx0dr * fd1_x0(f, idx, fd1_offset(i0, p.FACEX0, g.N0), g.invdxx0);
  const double dfdr_int = dx0dr_int * fd1_x0(f, idx_int, fd1_offset(j0, p.FACEX0, g.N0), g.invdxx0);
  const double c = tab.wavespeed[gf], finf = tab.finf[gf];
  const double dtf_int = rhs[idx_int + (size_t)gf * g.ntot];
  const double fv = f[idx], fv_int = f[idx_int];
  const double out_int = -c * (dfdr_int + (fv_int - finf) / r_int);
  const double k = r_int * r_int * r_int * (dtf_int - out_int);
  const double rinv = 1.0 / r;
  const double out_here = -c * (dfdr + (fv - finf) * rinv);
  rhs[idx + (size_t)gf * g.ntot] = out_here + k * rinv * rinv * rinv;
}

// The same 4th-order first derivative along a direction of index stride `st` (i2: s2).
__device__ __forceinline__ double fd1_dir(const double *__restrict__ f, int idx, int st, int offset, double invdx) {
  switch (offset) {
    case 0:
      return ((1.0 / 12.0) * f[idx - 2 * st] - (2.0 / 3.0) * f[idx - st] + (2.0 / 3.0) * f[idx + st] -
              (1.0 / 12.0) * f[idx + 2 * st]) * invdx;
    case 1:
      return (-(1.0 / 4.0) * f[idx - st] - (5.0 / 6.0) * f[idx] + (3.0 / 2.0) * f[idx + st] -
              (1.0 / 2.0) * f[idx + 2 * st] + (1.0 / 12.0) * f[idx + 3 * st]) * invdx;
    case -1:
      return (-(1.0 / 12.0) * f[idx - 3 * st] + (1.0 / 2.0) * f[idx - 2 * st] - (3.0 / 2.0) * f[idx - st] +
              (5.0 / 6.0) * f[idx] + (1.0 / 4.0) * f[idx + st]) * invdx;
    case 2:
      return (-(25.0 / 12.0) * f[idx] + 4.0 * f[idx + st] - 3.0 * f[idx + 2 * st] + (4.0 / 3.0) * f[idx + 3 * st] -
              (1.0 / 4.0) * f[idx + 4 * st]) * invdx;
    default:  // -2
      return ((1.0 / 4.0) * f[idx - 4 * st] - (4.0 / 3.0) * f[idx - 3 * st] + 3.0 * f[idx - 2 * st] -
              4.0 * f[idx - st] + (25.0 / 12.0) * f[idx]) * invdx;
  }
}

// SinhCylindrical: r = sqrt(rho^2 + z^2) has partial derivatives along xx0 and xx2, so
// partial_r f = (dx0/dr) d_x0 f + (dx2/dr) d_x2 f, each one-sided FD shifted away from the
// face and from the grid's edges as in the reference's compute_partial_r_f.
__global__ void radiation_cyl_kernel(const GridDims g, const CylMap cm, const double *__restrict__ xx0,
                                     const double *__restrict__ xx2, const outerpt_bc_struct *__restrict__ pts,
                                     const int npts, const double *__restrict__ gfs, double *__restrict__ rhs,
                                     const GfTable tab) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * NUM_EVOL_GFS) return;
  const int gf = t / npts;
  const int pt = t - gf * npts;
  const outerpt_bc_struct p = pts[pt];
  const int i0 = p.i0, i1 = p.i1, i2 = p.i2;
  const int j0 = i0 + p.FACEX0, j1 = i1 + p.FACEX1, j2 = i2 + p.FACEX2;
  double r, dx0dr, dx2dr, r_int, dx0dr_int, dx2dr_int;
  cm.radial(xx0[i0], xx2[i2], r, dx0dr, dx2dr);
  cm.radial(xx0[j0], xx2[j2], r_int, dx0dr_int, dx2dr_int);
  const double *f = gfs + (size_t)gf * g.ntot;
  const int idx = i0 + g.s1 * i1 + g.s2 * i2;
  const int idx_int = j0 + g.s1 * j1 + g.s2 * j2;
  const double dfdr = dx0dr * fd1_dir(f, idx, 1, fd1_offset(i0, p.FACEX0, g.N0), g.invdxx0) +
                      dx2dr * fd1_dir(f, idx, g.s2, fd1_offset(i2, p.FACEX2, g.N2), g.invdxx2);
  const double dfdr_int = dx0dr_int * fd1_dir(f, idx_int, 1, fd1_offset(j0, p.FACEX0, g.N0), g.invdxx0) +
                          dx2dr_int * fd1_dir(f, idx_int, g.s2, fd1_offset(j2, p.FACEX2, g.N2), g.invdxx2);
  const double c = tab.wavespeed[gf], finf = tab.finf[gf];
  const double dtf_int = rhs[idx_int + (size_t)gf * g.ntot];
  const double fv = f[idx], fv_int = f[idx_int];
  const double out_int = -c * (dfdr_int + (fv_int - finf) / r_int);
  const double k = r_int * r_int * r_int * (dtf_int - out_int);
  const double rinv = 1.0 / r;
  const double out_here = -c * (dfdr + (fv - finf) * rinv);
  rhs[idx + (size_t)gf * g.ntot] = out_here + k * rinv * rinv * rinv;
}

int radial_map(const params_struct *p, RadialMap *rm) {
  if (p->CoordSystem_hash == SPHERICAL) {
    *rm = RadialMap{0, 0.0, 0.0};
  } else if (p->CoordSystem_hash == SINHSPHERICAL) {
    *rm = RadialMap{1, p->AMPL, p->SINHW};
  } else {
    set_error("radiation BCs: CoordSystem_hash %d not supported", p->CoordSystem_hash);
    return BSSN_B200_EINVAL;
  }
  return BSSN_B200_OK;
}

int launch_radiation_bcs(const GridDims &g, const params_struct *p, const bc_struct *bc, const double *const xx[3],
                         const double *wavespeed, const double *f_inf, const double *gfs, double *rhs,
                         cudaStream_t s) {
  GfTable tab{};
  for (int k = 0; k < NUM_EVOL_GFS; k++) {
    tab.wavespeed[k] = wavespeed ? wavespeed[k] : kWavespeed[k];
    tab.finf[k] = f_inf ? f_inf[k] : kFInfinity[k];
  }
  if (p->CoordSystem_hash == SINHCYLINDRICAL) {
    // layer by layer and face direction by face direction, as the reference orders them
    const CylMap cm = cyl_map(p);
    for (int gz = 0; gz < NGHOSTS; gz++)
      for (int dirn = 0; dirn < 3; dirn++) {
        const int n = bc->bc_info.num_pure_outer_boundary_points[gz][dirn];
        if (n <= 0) continue;
        const int threads = 256;
        const long long work = (long long)n * NUM_EVOL_GFS;
        radiation_cyl_kernel<<<(unsigned)((work + threads - 1) / threads), threads, 0, s>>>(
            g, cm, xx[0], xx[2], bc->pure_outer_bc_array[dirn + 3 * gz], n, gfs, rhs, tab);
        BSSN_LAUNCH_CHECK();
      }
    return BSSN_B200_OK;
  }
  RadialMap rm;
  BSSN_TRY(radial_map(p, &rm));
  for (int gz = 0; gz < NGHOSTS; gz++) {
    for (int dirn = 0; dirn < 3; dirn++) {
      const int n = bc->bc_info.num_pure_outer_boundary_points[gz][dirn];
      if (n <= 0) continue;
      if (dirn != 0) {
        set_error("radiation BCs: outer points on face direction %d are not supported for Spherical-family grids",
                  dirn);
        return BSSN_B200_EINVAL;
      }
      const int threads = 256;
      const long long work = (long long)n * NUM_EVOL_GFS;
      radiation_kernel<<<(unsigned)((work + threads - 1) / threads), threads, 0, s>>>(
          g, rm, xx[0], bc->pure_outer_bc_array[dirn + 3 * gz], n, gfs, rhs, tab);
      BSSN_LAUNCH_CHECK();
    }
  }
  return BSSN_B200_OK;
}

// ---------------------------------------------------------------- extrapolation
__global__ void extrap_kernel(const GridDims g, const outerpt_bc_struct *__restrict__ pts, const int npts,
                              double *__restrict__ gfs) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * NUM_EVOL_GFS) return;
  const int gf = t / npts;
  const int pt = t - gf * npts;
  const outerpt_bc_struct p = pts[pt];
  const int d = p.FACEX0 + g.s1 * p.FACEX1 + g.s2 * p.FACEX2;
  const int idx = p.i0 + g.s1 * p.i1 + g.s2 * p.i2;
  double *f = gfs + (size_t)gf * g.ntot;
  f[idx] = +3.0 * f[idx + d] - 3.0 * f[idx + 2 * d] + 1.0 * f[idx + 3 * d];
}

int launch_extrap_bcs(const GridDims &g, const bc_struct *bc, double *gfs, cudaStream_t s) {
  for (int gz = 0; gz < NGHOSTS; gz++) {
    for (int dirn = 0; dirn < 3; dirn++) {
      const int n = bc->bc_info.num_pure_outer_boundary_points[gz][dirn];
      if (n <= 0) continue;
      const int threads = 256;
      const long long work = (long long)n * NUM_EVOL_GFS;
      extrap_kernel<<<(unsigned)((work + threads - 1) / threads), threads, 0, s>>>(
          g, bc->pure_outer_bc_array[dirn + 3 * gz], n, gfs);
      BSSN_LAUNCH_CHECK();
    }
  }
  return BSSN_B200_OK;
}

// ---------------------------------------------------------------- fused-stage boundary pass
int launch_radiation_rk_bcs(Variant v, const GridDims &g, const params_struct *p, const bc_struct *bc,
                            const double *const xx[3], const RfmArrays &rfm, int stage, double dt,
                            const StageBuffers &b, double *krhs, cudaStream_t s) {
  // 1. radiation RHS of every pure outer point, layer by layer (reads the stage input and krhs).
  BSSN_TRY(launch_radiation_bcs(g, p, bc, xx, nullptr, nullptr, b.kin, krhs, s));
  // 2. RK update + detgammabar projection of those points.
  for (int gz = 0; gz < NGHOSTS; gz++)
    for (int dirn = 0; dirn < 3; dirn++) {
      const int n = bc->bc_info.num_pure_outer_boundary_points[gz][dirn];
      if (n > 0) BSSN_TRY(launch_rk_points(v, stage, dt, g, rfm, b, bc->pure_outer_bc_array[dirn + 3 * gz], n, krhs, s));
    }
  // 3. parity copies of the stage output into every inner ghost point.
  return launch_inner_bcs(g, bc, b.kout, NUM_EVOL_GFS, nullptr, s);
}

// ---------------------------------------------------------------- batched evolutions
// Radiation RHS of one ghost layer's pure outer points of every evolution (one thread per
// point and gridfunction); reads the stage input and the RHS one layer in, writes krhs.
__global__ void radiation_batched_kernel(const EvoDesc *__restrict__ descs, const BatchOuterPt *__restrict__ pts,
                                         const int npts, const int stage) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * NUM_EVOL_GFS) return;
  const int gf = t / npts;
  const BatchOuterPt q = pts[t - gf * npts];
  const EvoDesc &d = descs[q.evo];
  double *kin, *kout;
  stage_io(d, stage, kin, kout);
  const RadialMap rm{d.radial_sinh, d.AMPL, d.SINHW};
  const GridDims &g = d.g;
  const outerpt_bc_struct p = q.p;
  const int i0 = p.i0, i1 = p.i1, i2 = p.i2;
  const int j0 = i0 + p.FACEX0, j1 = i1 + p.FACEX1, j2 = i2 + p.FACEX2;
  double r, dx0dr, r_int, dx0dr_int;
  rm.eval(d.xx0[i0], r, dx0dr);
  rm.eval(d.xx0[j0], r_int, dx0dr_int);
  const double *f = kin + (size_t)gf * g.ntot;
  const int idx = i0 + g.s1 * i1 + g.s2 * i2;
  const int idx_int = j0 + g.s1 * j1 + g.s2 * j2;
  const double dfdr = dx0dr * fd1_x0(f, idx, fd1_offset(i0, p.FACEX0, g.N0), g.invdxx0);
  const double dfdr_int = dx0dr_int * fd1_x0(f, idx_int, fd1_offset(j0, p.FACEX0, g.N0), g.invdxx0);
  const double c = (gf == ALPHAGF) ? 1.41421356237310 : 1.0;
  const double finf = (gf == ALPHAGF || gf == CFGF) ? 1.0 : 0.0;
  double *rhs = d.krhs + (size_t)gf * g.ntot;
  const double dtf_int = rhs[idx_int];
  const double fv = f[idx], fv_int = f[idx_int];
  const double out_int = -c * (dfdr_int + (fv_int - finf) / r_int);
  const double k = r_int * r_int * r_int * (dtf_int - out_int);
  const double rinv = 1.0 / r;
  rhs[idx] = -c * (dfdr + (fv - finf) * rinv) + k * rinv * rinv * rinv;
}

int launch_radiation_batched(int stage, const EvoDesc *descs, const BatchOuterPt *pts, int npts, cudaStream_t s) {
  if (npts <= 0) return BSSN_B200_OK;
  const int threads = 256;
  const long long work = (long long)npts * NUM_EVOL_GFS;
  radiation_batched_kernel<<<(unsigned)((work + threads - 1) / threads), threads, 0, s>>>(descs, pts, npts, stage);
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

// Parity copies into every inner ghost point of every evolution's stage output. One thread
// per inner point copies all 24 gridfunctions: the point's record and its evolution's
// descriptor are read once, and a warp's 32 consecutive records (mostly consecutive dstpt
// and srcpt along i0) make each gridfunction's loads and stores contiguous.
__global__ void inner_batched_kernel(const EvoDesc *__restrict__ descs, const BatchInnerPt *__restrict__ pts,
                                     const int npts, const int stage) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts) return;
  const BatchInnerPt q = pts[t];
  const EvoDesc &d = descs[q.evo];
  double *kin, *kout;
  stage_io(d, stage, kin, kout);
  const size_t ntot = (size_t)d.g.ntot;
  constexpr int8_t parity[NUM_EVOL_GFS] = {4, 5, 6, 7, 8, 9, 0, 1, 2, 3, 0, 4, 5, 6, 7, 8, 9, 1, 2, 3, 0, 1, 2, 3};
  double v[NUM_EVOL_GFS];
#pragma unroll
  for (int gf = 0; gf < NUM_EVOL_GFS; gf++) v[gf] = kout[q.b.srcpt + gf * ntot];
#pragma unroll
  for (int gf = 0; gf < NUM_EVOL_GFS; gf++) kout[q.b.dstpt + gf * ntot] = flip_sign(v[gf], q.b.parity[parity[gf]]);
}

int launch_inner_batched(int stage, const EvoDesc *descs, const BatchInnerPt *pts, int npts, cudaStream_t s) {
  if (npts <= 0) return BSSN_B200_OK;
  const int threads = 128;
  inner_batched_kernel<<<(unsigned)((npts + threads - 1) / threads), threads, 0, s>>>(descs, pts, npts, stage);
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

}  // namespace bssn
