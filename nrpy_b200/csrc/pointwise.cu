// Pointwise BSSN operators: conformal Ricci tensor, RHS (upwinded advection, KO
// dissipation), constraints, the detgammabar projection and the initial-data lambda^i.
// The algebra is the generated code in gen/*.cuh; this file supplies the stencil-load
// contexts and the launch geometry.
//
// Layout: gf-major IDX4(gf,i0,i1,i2) = i0 + N0*(i1 + N1*(i2 + N2*gf)). One thread per
// interior point; a warp spans 32 consecutive i0, so each stencil load of a warp touches
// one or two contiguous 256-byte segments that neighbouring warps reuse from L1/L2.
#include <type_traits>

#include "bssn_common.cuh"

namespace bssn {

// Interior block geometry: 32 points along i0 x 4 along i1, one i2 plane per blockIdx.z.
constexpr int BX = 32, BY = 4;

template <typename T>
__device__ __forceinline__ T ipow(T x, int n) {
  T r = x;
  for (int k = 1; k < n; k++) r *= x;
  return r;
}

// Stencil loads from global memory around one point.
struct PointCtx {
  const double *__restrict__ in;   // in_gfs + IDX3(i0,i1,i2)
  const double *__restrict__ aux;  // auxevol_gfs + IDX3(i0,i1,i2)
  int s1, s2, ntot;
  int i0, i1, i2;
  double invdxx0, invdxx1, invdxx2;
  RfmArrays rfm;
  double eta, KreissOliger_strength_gauge, KreissOliger_strength_nongauge;
  __device__ __forceinline__ double ld(int gf, int a, int b, int c) const {
    return __ldg(in + (gf * ntot + (a + b * s1 + c * s2)));
  }
  __device__ __forceinline__ double ldaux(int k) const { return __ldg(aux + k * ntot); }
  // L1 prefetch of the line holding stencil point (0, b, c) of gridfunction gf.
  __device__ __forceinline__ void prefetch_row(int gf, int b, int c) const {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(in + (gf * ntot + (b * s1 + c * s2))));
  }
  __device__ __forceinline__ void prefetch_row_l2(int gf, int b, int c) const {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(in + (gf * ntot + (b * s1 + c * s2))));
  }
};

// Point values held in registers (pointwise operators without stencils).
struct RegCtx {
  const double *v;  // NUM_EVOL_GFS values of this point
  int i0, i1, i2;
  RfmArrays rfm;
  __device__ __forceinline__ double ld(int gf, int, int, int) const { return v[gf]; }
};

#define LD(gf, a, b, c) ctx.ld(gf, a, b, c)
#define LDAUX(k) ctx.ldaux(k)
#define PREFETCH_ROW(gf, b, c) ctx.prefetch_row(gf, b, c)
#define PREFETCH_ROW_L2(gf, b, c) ctx.prefetch_row_l2(gf, b, c)
#define RFM(arr, d) __ldg(ctx.rfm.arr + ctx.i##d)
#define rfm_f0 f0
#define rfm_f0_D0 f0_D0
#define rfm_f0_DD00 f0_DD00
#define rfm_f0_DDD000 f0_DDD000
#define rfm_f1 f1
#define rfm_f1_D1 f1_D1
#define rfm_f1_DD11 f1_DD11
#define PARAM(name) ctx.name
// Per-thread shared-memory slot k (the kernel passes `sm` already offset by its thread).
// NT is the slot stride: the template parameter of the generated function (threads per block).
#define SMEM(k) sm[(k) * NT]
#define invdxx0 ctx.invdxx0
#define invdxx1 ctx.invdxx1
#define invdxx2 ctx.invdxx2
#if BSSN_B200_FD_ORDER == 4
#include "gen/bssn_sinh_3d.cuh"
#include "gen/bssn_sinh_axi.cuh"
#include "gen/bssn_sph_3d.cuh"
#include "gen/bssn_sph_axi.cuh"
#include "gen/bssn_sinhcyl_axi.cuh"
#elif BSSN_B200_FD_ORDER == 8
#include "gen/bssn_sinh_3d_fd8.cuh"
#include "gen/bssn_sinh_axi_fd8.cuh"
#include "gen/bssn_sph_3d_fd8.cuh"
#include "gen/bssn_sph_axi_fd8.cuh"
#include "gen/bssn_sinhcyl_axi_fd8.cuh"
#else
#error "BSSN_B200_FD_ORDER: generated algebra exists for 4 and 8"
#endif
#undef invdxx0
#undef invdxx1
#undef invdxx2

// Output-group traits of the generated variants: RicciGroup<V,G> / RhsGroup<V,G> expose
// N (outputs), GF[] (their gridfunction indices), SLOTS / SLOTS_F32 (per-thread shared-memory
// slots of the spilled values in the FP64 and in the FP32 evaluation, which may have
// allocations of their own) and eval().
template <Variant V, int G>
using RicciG = std::conditional_t<
    V == SPH_3D, RicciGroup_sph_3d<G>,
    std::conditional_t<
        V == SPH_AXI, RicciGroup_sph_axi<G>,
        std::conditional_t<V == SINH_3D, RicciGroup_sinh_3d<G>,
                           std::conditional_t<V == SINH_AXI, RicciGroup_sinh_axi<G>, RicciGroup_sinhcyl_axi<G>>>>>;
template <Variant V, int G>
using RhsG = std::conditional_t<
    V == SPH_3D, RhsGroup_sph_3d<G>,
    std::conditional_t<
        V == SPH_AXI, RhsGroup_sph_axi<G>,
        std::conditional_t<V == SINH_3D, RhsGroup_sinh_3d<G>,
                           std::conditional_t<V == SINH_AXI, RhsGroup_sinh_axi<G>, RhsGroup_sinhcyl_axi<G>>>>>;
constexpr int kRicciGroups = ricci_group_count_sph_3d, kRhsGroups = rhs_group_count_sph_3d;
static_assert(ricci_group_count_sph_axi == kRicciGroups && ricci_group_count_sinh_3d == kRicciGroups &&
                  ricci_group_count_sinh_axi == kRicciGroups && ricci_group_count_sinhcyl_axi == kRicciGroups &&
                  rhs_group_count_sph_axi == kRhsGroups && rhs_group_count_sinh_3d == kRhsGroups &&
                  rhs_group_count_sinh_axi == kRhsGroups && rhs_group_count_sinhcyl_axi == kRhsGroups,
              "every variant has the same output groups");

// Calls f(std::integral_constant<int, G>) for G = G0 .. NG-1, stopping at the first error.
template <int G0, int NG, typename F>
static int for_each_group(F &&f) {
  if constexpr (G0 < NG) {
    BSSN_TRY(f(std::integral_constant<int, G0>{}));
    return for_each_group<G0 + 1, NG>(f);
  } else {
    return BSSN_B200_OK;
  }
}

// Point functions without shared-memory slots get a typed null slot pointer.
#define NOSLOTS(T) static_cast<volatile T *>(nullptr)
#define DISPATCH_POINT(NAME, V, T, TF, CTX, OUT)                                  \
  do {                                                                            \
    if constexpr (V == SPH_3D) NAME##_sph_3d<T, TF>(CTX, OUT, NOSLOTS(T));        \
    else if constexpr (V == SPH_AXI) NAME##_sph_axi<T, TF>(CTX, OUT, NOSLOTS(T)); \
    else if constexpr (V == SINH_3D) NAME##_sinh_3d<T, TF>(CTX, OUT, NOSLOTS(T)); \
    else if constexpr (V == SINH_AXI) NAME##_sinh_axi<T, TF>(CTX, OUT, NOSLOTS(T)); \
    else NAME##_sinhcyl_axi<T, TF>(CTX, OUT, NOSLOTS(T));                         \
  } while (0)

__device__ __forceinline__ PointCtx make_ctx(const GridDims &g, const RfmArrays &rfm, const double *in,
                                             const double *aux, int i0, int i1, int i2) {
  PointCtx c;
  const int idx = i0 + g.s1 * i1 + g.s2 * i2;
  c.in = in + idx;
  c.aux = aux ? aux + idx : nullptr;
  c.s1 = g.s1;
  c.s2 = g.s2;
  c.ntot = g.ntot;
  c.i0 = i0;
  c.i1 = i1;
  c.i2 = i2;
  c.invdxx0 = g.invdxx0;
  c.invdxx1 = g.invdxx1;
  c.invdxx2 = g.invdxx2;
  c.rfm = rfm;
  c.eta = 0.0;
  c.KreissOliger_strength_gauge = 0.0;
  c.KreissOliger_strength_nongauge = 0.0;
  return c;
}

static dim3 interior_grid(const GridDims &g, int by = BY) {
  const int n0 = g.N0 - 2 * NGHOSTS, n1 = g.N1 - 2 * NGHOSTS, n2 = g.N2 - 2 * NGHOSTS;
  return dim3((n0 + BX - 1) / BX, (n1 + by - 1) / by, n2);
}

#define INTERIOR_INDEX_OR_RETURN(g)                       \
  const int i0 = NGHOSTS + blockIdx.x * BX + threadIdx.x; \
  const int i1 = NGHOSTS + blockIdx.y * blockDim.y + threadIdx.y; \
  const int i2 = NGHOSTS + blockIdx.z;                    \
  if (i0 >= g.N0 - NGHOSTS || i1 >= g.N1 - NGHOSTS) return;

// Group-kernel block geometry: TX points along i0, NT / (TX * TZ) along i1 and TZ along i2.
#ifndef BSSN_TILE_X
#define BSSN_TILE_X 32
#endif
#ifndef BSSN_TILE_Z
#define BSSN_TILE_Z 1
#endif
constexpr int TX = BSSN_TILE_X, TZ = BSSN_TILE_Z;

// A grid with fewer than NT / TX interior points along i1 (the axisymmetric SinhCylindrical
// grid has 2 phi points) would leave block rows idle; there the block takes the remaining
// threads along i2 instead (32 x 2 x 2 for 128 threads and 2 phi points).
static dim3 group_block(const GridDims &g, int nt) {
  const int n1 = g.N1 - 2 * NGHOSTS;
  int ty = nt / (TX * TZ), tz = TZ;
  while (ty > 1 && ty / 2 >= n1) {
    ty /= 2;
    tz *= 2;
  }
  return dim3(TX, ty, tz);
}

static dim3 group_grid(const GridDims &g, const dim3 &blk) {
  const int n0 = g.N0 - 2 * NGHOSTS, n1 = g.N1 - 2 * NGHOSTS, n2 = g.N2 - 2 * NGHOSTS;
  return dim3((n0 + blk.x - 1) / blk.x, (n1 + blk.y - 1) / blk.y, (n2 + blk.z - 1) / blk.z);
}

#define GROUP_INDEX_OR_RETURN(g)                                        \
  const int i0 = NGHOSTS + blockIdx.x * blockDim.x + threadIdx.x;       \
  const int i1 = NGHOSTS + blockIdx.y * blockDim.y + threadIdx.y;       \
  const int i2 = NGHOSTS + blockIdx.z * blockDim.z + threadIdx.z;       \
  if (i0 >= g.N0 - NGHOSTS || i1 >= g.N1 - NGHOSTS || i2 >= g.N2 - NGHOSTS) return;

template <typename T>
__device__ __forceinline__ volatile T *thread_slots() {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  return reinterpret_cast<volatile T *>(smem_raw) + (threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z));
}

// S: the slot element type, volatile T or plain T (see the group's eval).
template <Variant V, int G, typename T, int NTB, typename S>
__device__ __forceinline__ void ricci_body(const GridDims &g, const RfmArrays &rfm, const double *in, double *aux,
                                           int i0, int i1, int i2, S *sm) {
  using Grp = RicciG<V, G>;
  const PointCtx ctx = make_ctx(g, rfm, in, nullptr, i0, i1, i2);
  T out[Grp::N];
  Grp::template eval<T, double, NTB>(ctx, out, sm);
  const int idx = i0 + g.s1 * i1 + g.s2 * i2;
#pragma unroll
  for (int k = 0; k < Grp::N; k++) aux[idx + Grp::GF(k) * g.ntot] = double(out[k]);
}

template <Variant V, int G, typename T>
__global__ void __launch_bounds__(RicciG<V, G>::NT, 1) ricci_kernel(const GridDims g, const RfmArrays rfm,
                                                          const double *__restrict__ in, double *__restrict__ aux) {
  volatile T *sm = thread_slots<T>();
  GROUP_INDEX_OR_RETURN(g);
  ricci_body<V, G, T, RicciG<V, G>::NT>(g, rfm, in, aux, i0, i1, i2, sm);
}

template <Variant V, typename T, int G>
__global__ void __launch_bounds__(RhsG<V, G>::NT, 1) rhs_kernel(const GridDims g, const RfmArrays rfm, const PhysParams pp,
                                                        const double *__restrict__ aux, const double *__restrict__ in,
                                                        double *__restrict__ rhs) {
  using Grp = RhsG<V, G>;
  volatile T *sm = thread_slots<T>();
  GROUP_INDEX_OR_RETURN(g);
  PointCtx ctx = make_ctx(g, rfm, in, aux, i0, i1, i2);
  ctx.eta = pp.eta;
  ctx.KreissOliger_strength_gauge = pp.ko_gauge;
  ctx.KreissOliger_strength_nongauge = pp.ko_nongauge;
  T out[Grp::N];
  Grp::template eval<T, double, Grp::NT>(ctx, out, sm);
  const int idx = i0 + g.s1 * i1 + g.s2 * i2;
#pragma unroll
  for (int k = 0; k < Grp::N; k++) rhs[idx + Grp::GF(k) * g.ntot] = double(out[k]);
}

template <Variant V>
__global__ void __launch_bounds__(BX *BY, 1) constraints_kernel(const GridDims g, const RfmArrays rfm,
                                                             const double *__restrict__ in,
                                                             const double *__restrict__ aux,
                                                             double *__restrict__ diag, const int3 slot) {
  INTERIOR_INDEX_OR_RETURN(g);
  const PointCtx ctx = make_ctx(g, rfm, in, aux, i0, i1, i2);
  double out[3];
  DISPATCH_POINT(constraints_point, V, double, double, ctx, out);
  const size_t idx = (size_t)i0 + (size_t)g.s1 * i1 + (size_t)g.s2 * i2;
  diag[idx + (size_t)slot.x * g.ntot] = out[0];
  diag[idx + (size_t)slot.y * g.ntot] = out[1];
  diag[idx + (size_t)slot.z * g.ntot] = out[2];
}

// lambda^i = Lambdabar^i / ReU[i] from centred derivatives of hDD (initial data;
// ADM_Initial_Data_Reader__BSSN_Converter.py:462-580). Writes LAMBDAU0..2 of the interior.
template <Variant V>
__global__ void __launch_bounds__(BX *BY) lambda_id_kernel(const GridDims g, const RfmArrays rfm,
                                                           double *__restrict__ gfs) {
  INTERIOR_INDEX_OR_RETURN(g);
  const PointCtx ctx = make_ctx(g, rfm, gfs, nullptr, i0, i1, i2);
  double out[3];
  DISPATCH_POINT(lambda_point, V, double, double, ctx, out);
  const int idx = i0 + g.s1 * i1 + g.s2 * i2;
#pragma unroll
  for (int k = 0; k < 3; k++) gfs[idx + (LAMBDAU0GF + k) * g.ntot] = out[k];
}

// detgammabar = detgammahat projection of hDD at ALL points (ghost zones included).
template <Variant V>
__global__ void enforce_kernel(const GridDims g, const RfmArrays rfm, double *__restrict__ gfs) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= g.ntot) return;
  const int i2 = idx / g.s2;
  const int rem = idx - i2 * g.s2;
  const int i1 = rem / g.s1;
  const int i0 = rem - i1 * g.s1;
  const PointCtx ctx = make_ctx(g, rfm, gfs, nullptr, i0, i1, i2);
  double out[6];
  DISPATCH_POINT(enforce_point, V, double, double, ctx, out);
#pragma unroll
  for (int k = 0; k < 6; k++) gfs[idx + (HDD00GF + k) * g.ntot] = out[k];
}

// ---------------------------------------------------------------- fused RK stage
// Same association as the reference's rk_substep_{1..4} (MoL_step_forward_in_time.py:346-470).
template <int STAGE>
__device__ __forceinline__ void rk_update(const double k, const double y, double &run, double &out, const double dt) {
  if constexpr (STAGE == 1) {
    run = (1.0 / 6.0) * dt * k;
    out = (1.0 / 2.0) * dt * k + y;
  } else if constexpr (STAGE == 2) {
    run = (1.0 / 3.0) * dt * k + run;
    out = (1.0 / 2.0) * dt * k + y;
  } else if constexpr (STAGE == 3) {
    run = (1.0 / 3.0) * dt * k + run;
    out = dt * k + y;
  } else {
    out = (1.0 / 6.0) * dt * k + y + run;
  }
}

template <Variant V, int STAGE>
__device__ __forceinline__ void rk_and_project_point(const GridDims &g, const RfmArrays &rfm, const StageBuffers &b,
                                                     const int idx, const int i0, const int i1, const int i2,
                                                     const double *kk,
                                                     const double dt) {
  double o[NUM_EVOL_GFS];
#pragma unroll
  for (int k = 0; k < NUM_EVOL_GFS; k++) {
    const size_t a = idx + (size_t)k * g.ntot;
    double run = (STAGE == 1) ? 0.0 : b.run[a];
    rk_update<STAGE>(kk[k], b.y[a], run, o[k], dt);
    if (STAGE != 4) b.run[a] = run;
  }
  RegCtx rc{o, i0, i1, i2, rfm};
  double h[6];
  DISPATCH_POINT(enforce_point, V, double, double, rc, h);
#pragma unroll
  for (int k = 0; k < 6; k++) o[HDD00GF + k] = h[k];
#pragma unroll
  for (int k = 0; k < NUM_EVOL_GFS; k++) b.kout[idx + (size_t)k * g.ntot] = o[k];
}

// One output group of the RHS at an interior point, then in registers the RK4 stage update
// of that group's gridfunctions; the group holding hDD also applies the detgammabar
// projection to the new hDD. The raw RHS is also stored to `krhs` on the interior shell
// (the layer next to each face), where the outer radiation condition reads it.
template <Variant V, typename T, int STAGE, int G, int NTB, typename S>
__device__ __forceinline__ void fused_body(const GridDims &g, const RfmArrays &rfm, const PhysParams &pp,
                                           const double *aux, const StageBuffers &b, double *krhs, const double dt,
                                           int i0, int i1, int i2, S *sm) {
  using Grp = RhsG<V, G>;
#if BSSN_B200_FD_ORDER == 4
  {
    // The RK update at the end reads y (and the running total) of this point's outputs; ask
    // for their lines in L2 now, so that they arrive while the algebra runs instead of
    // stalling the update. No registers are held. (Measured: +0.9% FP64 and +2.6% mixed at
    // 4th order; at 8th order it lost 1.9%, so it is left out there.)
    const size_t idx0 = (size_t)i0 + (size_t)g.s1 * i1 + (size_t)g.s2 * i2;
#pragma unroll
    for (int k = 0; k < Grp::N; k++) {
      const size_t a = idx0 + (size_t)Grp::GF(k) * g.ntot;
      asm volatile("prefetch.global.L2 [%0];" ::"l"(b.y + a));
      if (STAGE != 1) asm volatile("prefetch.global.L2 [%0];" ::"l"(b.run + a));
    }
  }
#endif
  PointCtx ctx = make_ctx(g, rfm, b.kin, aux, i0, i1, i2);
  ctx.eta = pp.eta;
  ctx.KreissOliger_strength_gauge = pp.ko_gauge;
  ctx.KreissOliger_strength_nongauge = pp.ko_nongauge;
  T kt[Grp::N];
  Grp::template eval<T, double, NTB>(ctx, kt, sm);
  const int idx = i0 + g.s1 * i1 + g.s2 * i2;
  const bool shell = (i0 == NGHOSTS) | (i0 == g.N0 - NGHOSTS - 1) | (i1 == NGHOSTS) | (i1 == g.N1 - NGHOSTS - 1) |
                     (i2 == NGHOSTS) | (i2 == g.N2 - NGHOSTS - 1);
  double o[NUM_EVOL_GFS];  // indexed by gridfunction; only this group's entries are used
  constexpr bool has_h = [] {
    int n = 0;
    for (int k = 0; k < Grp::N; k++) n += (Grp::GF(k) >= HDD00GF && Grp::GF(k) <= HDD22GF);
    return n == 6;
  }();
#pragma unroll
  for (int k = 0; k < Grp::N; k++) {
    const double kv = double(kt[k]);
    const size_t a = idx + (size_t)Grp::GF(k) * g.ntot;
    if (shell) krhs[a] = kv;
    double run = (STAGE == 1) ? 0.0 : b.run[a];
    rk_update<STAGE>(kv, b.y[a], run, o[Grp::GF(k)], dt);
    if (STAGE != 4) b.run[a] = run;
  }
  if constexpr (has_h) {
    RegCtx rc{o, i0, i1, i2, rfm};
    double h[6];
    DISPATCH_POINT(enforce_point, V, double, double, rc, h);
#pragma unroll
    for (int k = 0; k < 6; k++) o[HDD00GF + k] = h[k];
  }
#pragma unroll
  for (int k = 0; k < Grp::N; k++) b.kout[idx + (size_t)Grp::GF(k) * g.ntot] = o[Grp::GF(k)];
}

// One output group of the RHS at an interior point, then in registers the RK4 stage update
// of that group's gridfunctions; the group holding hDD also applies the detgammabar
// projection to the new hDD. The raw RHS is also stored to `krhs` on the interior shell
// (the layer next to each face), where the outer radiation condition reads it.
template <Variant V, typename T, int STAGE, int G>
__global__ void __launch_bounds__(RhsG<V, G>::NT, 1) rhs_fused_kernel(const GridDims g, const RfmArrays rfm, const PhysParams pp,
                                                              const double *__restrict__ aux, const StageBuffers b,
                                                              double *__restrict__ krhs, const double dt) {
  volatile T *sm = thread_slots<T>();
  GROUP_INDEX_OR_RETURN(g);
  fused_body<V, T, STAGE, G, RhsG<V, G>::NT>(g, rfm, pp, aux, b, krhs, dt, i0, i1, i2, sm);
}

// RK update plus projection of listed boundary points whose RHS is already in krhs.
template <Variant V, int STAGE>
__global__ void rk_points_kernel(const GridDims g, const RfmArrays rfm, const StageBuffers b,
                                 const outerpt_bc_struct *__restrict__ pts, const int npts,
                                 const double *__restrict__ krhs, const double dt) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts) return;
  const outerpt_bc_struct p = pts[t];
  const int idx = p.i0 + g.s1 * p.i1 + g.s2 * p.i2;
  double kk[NUM_EVOL_GFS];
#pragma unroll
  for (int k = 0; k < NUM_EVOL_GFS; k++) kk[k] = krhs[idx + (size_t)k * g.ntot];
  rk_and_project_point<V, STAGE>(g, rfm, b, idx, p.i0, p.i1, p.i2, kk, dt);
}

// ---------------------------------------------------------------- launchers
#define VARIANT_SWITCH(v, CALL)                 \
  switch (v) {                                  \
    case SPH_3D: { constexpr Variant VV = SPH_3D; CALL; } break;   \
    case SPH_AXI: { constexpr Variant VV = SPH_AXI; CALL; } break; \
    case SINH_3D: { constexpr Variant VV = SINH_3D; CALL; } break; \
    case SINH_AXI: { constexpr Variant VV = SINH_AXI; CALL; } break; \
    case SINHCYL_AXI: { constexpr Variant VV = SINHCYL_AXI; CALL; } break; \
    default: set_error("unknown algebra variant %d", (int)v); return BSSN_B200_EINVAL; \
  }

static bool empty_interior(const GridDims &g) {
  return g.N0 <= 2 * NGHOSTS || g.N1 <= 2 * NGHOSTS || g.N2 <= 2 * NGHOSTS;
}

// Dynamic shared memory of a group kernel: SLOTS values of type T for each of its NT threads.
template <typename Grp, typename T>
constexpr size_t slot_bytes() {
  return (size_t)(std::is_same<T, float>::value ? Grp::SLOTS_F32 : Grp::SLOTS) * Grp::NT * sizeof(T);
}

template <typename KernelPtr>
static int set_smem(KernelPtr k, size_t bytes) {
  if (bytes > 48 * 1024) BSSN_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return BSSN_B200_OK;
}

template <Variant V, int G, typename T>
static int launch_ricci_group(const GridDims &g, const RfmArrays &rfm, const double *in, double *aux, cudaStream_t s) {
  using Grp = RicciG<V, G>;
  constexpr size_t sb = slot_bytes<Grp, T>();
  BSSN_TRY(set_smem(ricci_kernel<V, G, T>, sb));
  const dim3 blk = group_block(g, Grp::NT);
  ricci_kernel<V, G, T><<<group_grid(g, blk), blk, sb, s>>>(g, rfm, in, aux);
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

template <Variant V, typename T>
static int launch_ricci_v(const GridDims &g, const RfmArrays &rfm, const double *in, double *aux, cudaStream_t s) {
  return for_each_group<0, kRicciGroups>(
      [&](auto gc) { return launch_ricci_group<V, decltype(gc)::value, T>(g, rfm, in, aux, s); });
}

int launch_ricci(Variant v, const GridDims &g, const RfmArrays &rfm, const double *in, double *aux, cudaStream_t s,
                 bool mixed) {
  if (empty_interior(g)) return BSSN_B200_OK;
  if (mixed) {
    VARIANT_SWITCH(v, return (launch_ricci_v<VV, float>(g, rfm, in, aux, s)));
  } else {
    VARIANT_SWITCH(v, return (launch_ricci_v<VV, double>(g, rfm, in, aux, s)));
  }
  return BSSN_B200_OK;
}

template <Variant V, typename T, int G>
static int launch_rhs_group(const GridDims &g, const RfmArrays &rfm, const PhysParams &pp, const double *aux,
                            const double *in, double *rhs, cudaStream_t s) {
  using Grp = RhsG<V, G>;
  constexpr size_t sb = slot_bytes<Grp, T>();
  BSSN_TRY(set_smem(rhs_kernel<V, T, G>, sb));
  const dim3 blk = group_block(g, Grp::NT);
  rhs_kernel<V, T, G><<<group_grid(g, blk), blk, sb, s>>>(g, rfm, pp, aux, in, rhs);
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

template <Variant V, typename T>
static int launch_rhs_v(const GridDims &g, const RfmArrays &rfm, const PhysParams &pp, const double *aux,
                        const double *in, double *rhs, cudaStream_t s) {
  return for_each_group<0, kRhsGroups>(
      [&](auto gc) { return launch_rhs_group<V, T, decltype(gc)::value>(g, rfm, pp, aux, in, rhs, s); });
}

int launch_rhs(Variant v, bool mixed, const GridDims &g, const RfmArrays &rfm, const PhysParams &pp,
               const double *aux, const double *in, double *rhs, cudaStream_t s) {
  if (empty_interior(g)) return BSSN_B200_OK;
  if (mixed) {
    VARIANT_SWITCH(v, return (launch_rhs_v<VV, float>(g, rfm, pp, aux, in, rhs, s)));
  } else {
    VARIANT_SWITCH(v, return (launch_rhs_v<VV, double>(g, rfm, pp, aux, in, rhs, s)));
  }
  return BSSN_B200_OK;
}

int launch_constraints(Variant v, const GridDims &g, const RfmArrays &rfm, const double *in, const double *aux,
                       double *diag, cudaStream_t s, const int *slots) {
  if (empty_interior(g)) return BSSN_B200_OK;
  const int3 sl = slots ? make_int3(slots[0], slots[1], slots[2]) : make_int3(0, 1, 2);
  VARIANT_SWITCH(v, (constraints_kernel<VV><<<interior_grid(g), dim3(BX, BY), 0, s>>>(g, rfm, in, aux, diag, sl)));
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

int launch_lambda_id(Variant v, const GridDims &g, const RfmArrays &rfm, double *gfs, cudaStream_t s) {
  if (empty_interior(g)) return BSSN_B200_OK;
  VARIANT_SWITCH(v, (lambda_id_kernel<VV><<<interior_grid(g), dim3(BX, BY), 0, s>>>(g, rfm, gfs)));
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

int launch_enforce(Variant v, const GridDims &g, const RfmArrays &rfm, double *gfs, cudaStream_t s) {
  const int threads = 128;
  const int blocks = (g.ntot + threads - 1) / threads;
  VARIANT_SWITCH(v, (enforce_kernel<VV><<<blocks, threads, 0, s>>>(g, rfm, gfs)));
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

template <Variant V, typename T, int STAGE, int G>
static int launch_fused_group(const GridDims &g, const RfmArrays &rfm, const PhysParams &pp, const double *aux,
                              const StageBuffers &b, double *krhs, double dt, cudaStream_t s) {
  using Grp = RhsG<V, G>;
  constexpr size_t sb = slot_bytes<Grp, T>();
  BSSN_TRY(set_smem(rhs_fused_kernel<V, T, STAGE, G>, sb));
  const dim3 blk = group_block(g, Grp::NT);
  rhs_fused_kernel<V, T, STAGE, G><<<group_grid(g, blk), blk, sb, s>>>(g, rfm, pp, aux, b,
                                                                                              krhs, dt);
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

template <Variant V, typename T, int STAGE>
static int launch_fused_stage_groups(const GridDims &g, const RfmArrays &rfm, const PhysParams &pp, const double *aux,
                                     const StageBuffers &b, double *krhs, double dt, cudaStream_t s) {
  return for_each_group<0, kRhsGroups>(
      [&](auto gc) { return launch_fused_group<V, T, STAGE, decltype(gc)::value>(g, rfm, pp, aux, b, krhs, dt, s); });
}

template <Variant V, typename T>
static int launch_fused_typed(int stage, const GridDims &g, const RfmArrays &rfm, const PhysParams &pp,
                              const double *aux, const StageBuffers &b, double *krhs, double dt, cudaStream_t s) {
  switch (stage) {
    case 1: return launch_fused_stage_groups<V, T, 1>(g, rfm, pp, aux, b, krhs, dt, s);
    case 2: return launch_fused_stage_groups<V, T, 2>(g, rfm, pp, aux, b, krhs, dt, s);
    case 3: return launch_fused_stage_groups<V, T, 3>(g, rfm, pp, aux, b, krhs, dt, s);
    default: return launch_fused_stage_groups<V, T, 4>(g, rfm, pp, aux, b, krhs, dt, s);
  }
}

int launch_rhs_fused_stage(Variant v, bool mixed, int stage, double dt, const GridDims &g, const RfmArrays &rfm,
                           const PhysParams &pp, const double *aux, const StageBuffers &b, double *krhs,
                           cudaStream_t s) {
  if (stage < 1 || stage > 4) {
    set_error("RK4 stage %d out of range", stage);
    return BSSN_B200_EINVAL;
  }
  if (empty_interior(g)) return BSSN_B200_OK;
  if (mixed) {
    VARIANT_SWITCH(v, return (launch_fused_typed<VV, float>(stage, g, rfm, pp, aux, b, krhs, dt, s)));
  } else {
    VARIANT_SWITCH(v, return (launch_fused_typed<VV, double>(stage, g, rfm, pp, aux, b, krhs, dt, s)));
  }
  return BSSN_B200_OK;
}

template <Variant V>
static void launch_rk_points_typed(int stage, const GridDims &g, const RfmArrays &rfm, const StageBuffers &b,
                                   const outerpt_bc_struct *pts, int npts, const double *krhs, double dt,
                                   cudaStream_t s) {
  const int threads = 128, blocks = (npts + threads - 1) / threads;
  switch (stage) {
    case 1: rk_points_kernel<V, 1><<<blocks, threads, 0, s>>>(g, rfm, b, pts, npts, krhs, dt); break;
    case 2: rk_points_kernel<V, 2><<<blocks, threads, 0, s>>>(g, rfm, b, pts, npts, krhs, dt); break;
    case 3: rk_points_kernel<V, 3><<<blocks, threads, 0, s>>>(g, rfm, b, pts, npts, krhs, dt); break;
    default: rk_points_kernel<V, 4><<<blocks, threads, 0, s>>>(g, rfm, b, pts, npts, krhs, dt); break;
  }
}

int launch_rk_points(Variant v, int stage, double dt, const GridDims &g, const RfmArrays &rfm, const StageBuffers &b,
                     const outerpt_bc_struct *pts, int npts, const double *krhs, cudaStream_t s) {
  if (npts <= 0) return BSSN_B200_OK;
  VARIANT_SWITCH(v, (launch_rk_points_typed<VV>(stage, g, rfm, b, pts, npts, krhs, dt, s)));
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

// ---------------------------------------------------------------- batched evolutions
// Ricci and fused RHS group kernels over a chunk of evolutions: block b takes tile
// b / (128 / NT) of the chunk (a group with NT < 128 threads covers a tile in 128 / NT
// blocks). The tile's evolution is found by a binary search over the chunk's tile_begin
// table; its local index runs over (tiles_x, tiles_y, tiles_z) tiles of that evolution's
// shape tile_bx x tile_by x tile_bz = 128 interior points (i0 fastest).
__device__ __forceinline__ bool tile_point(const EvoDesc &d, int t_local, int lin, int &i0, int &i1, int &i2) {
  const int tx = t_local % d.tiles_x;
  const int r = t_local / d.tiles_x;
  const int ty = r % d.tiles_y;
  const int tz = r / d.tiles_y;
  const int lx = lin % d.tile_bx, q = lin / d.tile_bx;
  i0 = NGHOSTS + tx * d.tile_bx + lx;
  i1 = NGHOSTS + ty * d.tile_by + q % d.tile_by;
  i2 = NGHOSTS + tz * d.tile_bz + q / d.tile_by;
  return i0 < d.g.N0 - NGHOSTS && i1 < d.g.N1 - NGHOSTS && i2 < d.g.N2 - NGHOSTS;
}

// Evolution of chunk-local tile t: the last e with tile_begin[e] <= t.
__device__ __forceinline__ int chunk_evo(const BatchChunk &c, int t) {
  int lo = 0, hi = c.nevo;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (c.tile_begin[mid] <= t) lo = mid;
    else hi = mid;
  }
  return lo;
}

template <Variant V, int G>
__global__ void __launch_bounds__(RicciG<V, G>::NT, 1) ricci_batched_kernel(const __grid_constant__ BatchChunk c,
                                                                          const int stage) {
  constexpr int NT = RicciG<V, G>::NT, PER = (BX * BY) / NT;
  const int t = blockIdx.x / PER;
  const int e = chunk_evo(c, t);
  const EvoDesc &d = c.evo[e];
  int i0, i1, i2;
  if (!tile_point(d, t - c.tile_begin[e], (blockIdx.x % PER) * NT + threadIdx.x, i0, i1, i2)) return;
  double *kin, *kout;
  stage_io(d, stage, kin, kout);
  volatile double *sm = thread_slots<double>();
  ricci_body<V, G, double, NT>(d.g, d.rfm, kin, d.aux, i0, i1, i2, sm);
}

template <Variant V, int STAGE, int G>
__global__ void __launch_bounds__(RhsG<V, G>::NT, 1) rhs_fused_batched_kernel(const __grid_constant__ BatchChunk c) {
  constexpr int NT = RhsG<V, G>::NT, PER = (BX * BY) / NT;
  const int t = blockIdx.x / PER;
  const int e = chunk_evo(c, t);
  const EvoDesc &d = c.evo[e];
  int i0, i1, i2;
  if (!tile_point(d, t - c.tile_begin[e], (blockIdx.x % PER) * NT + threadIdx.x, i0, i1, i2)) return;
  StageBuffers b;
  b.y = d.y;
  b.run = d.run;
  stage_io(d, STAGE, b.kin, b.kout);
  // Plain slots: the batched RHS groups ran faster with them.
  double *sm = const_cast<double *>(thread_slots<double>());
  fused_body<V, double, STAGE, G, NT>(d.g, d.rfm, d.pp, d.aux, b, d.krhs, d.dt, i0, i1, i2, sm);
}

template <Variant V, int STAGE>
__global__ void rk_points_batched_kernel(const EvoDesc *__restrict__ descs, const BatchOuterPt *__restrict__ pts,
                                         const int npts) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts) return;
  const BatchOuterPt q = pts[t];
  const EvoDesc &d = descs[q.evo];
  StageBuffers b;
  b.y = d.y;
  b.run = d.run;
  stage_io(d, STAGE, b.kin, b.kout);
  const int idx = q.p.i0 + d.g.s1 * q.p.i1 + d.g.s2 * q.p.i2;
  double kk[NUM_EVOL_GFS];
#pragma unroll
  for (int k = 0; k < NUM_EVOL_GFS; k++) kk[k] = d.krhs[idx + (size_t)k * d.g.ntot];
  rk_and_project_point<V, STAGE>(d.g, d.rfm, b, idx, q.p.i0, q.p.i1, q.p.i2, kk, d.dt);
}

template <Variant V, int G>
static int launch_ricci_batched_group(int stage, const BatchChunk &c, cudaStream_t s) {
  using Grp = RicciG<V, G>;
  constexpr size_t sb = slot_bytes<Grp, double>();
  BSSN_TRY(set_smem(ricci_batched_kernel<V, G>, sb));
  ricci_batched_kernel<V, G><<<c.ntiles * (BX * BY / Grp::NT), Grp::NT, sb, s>>>(c, stage);
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

template <Variant V, int STAGE, int G>
static int launch_fused_batched_group(const BatchChunk &c, cudaStream_t s) {
  using Grp = RhsG<V, G>;
  constexpr size_t sb = slot_bytes<Grp, double>();
  BSSN_TRY(set_smem(rhs_fused_batched_kernel<V, STAGE, G>, sb));
  rhs_fused_batched_kernel<V, STAGE, G><<<c.ntiles * (BX * BY / Grp::NT), Grp::NT, sb, s>>>(c);
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

template <Variant V, int STAGE>
static int launch_fused_batched_stage(const BatchChunk &c, cudaStream_t s) {
  return for_each_group<0, kRhsGroups>(
      [&](auto gc) { return launch_fused_batched_group<V, STAGE, decltype(gc)::value>(c, s); });
}

int launch_ricci_batched(Variant v, int stage, const BatchChunk &c, cudaStream_t s) {
  if (c.ntiles <= 0) return BSSN_B200_OK;
  if (v != SPH_3D && v != SINH_3D) {
    set_error("batched evolutions: only full 3-D variants are instantiated");
    return BSSN_B200_EINVAL;
  }
  if (v == SPH_3D) {
    return for_each_group<0, kRicciGroups>(
        [&](auto gc) { return launch_ricci_batched_group<SPH_3D, decltype(gc)::value>(stage, c, s); });
  }
  return for_each_group<0, kRicciGroups>(
      [&](auto gc) { return launch_ricci_batched_group<SINH_3D, decltype(gc)::value>(stage, c, s); });
}

template <Variant V>
static int launch_fused_batched_v(int stage, const BatchChunk &c, cudaStream_t s) {
  switch (stage) {
    case 1: return launch_fused_batched_stage<V, 1>(c, s);
    case 2: return launch_fused_batched_stage<V, 2>(c, s);
    case 3: return launch_fused_batched_stage<V, 3>(c, s);
    default: return launch_fused_batched_stage<V, 4>(c, s);
  }
}

int launch_rhs_fused_batched(Variant v, int stage, const BatchChunk &c, cudaStream_t s) {
  if (c.ntiles <= 0) return BSSN_B200_OK;
  if (v == SPH_3D) return launch_fused_batched_v<SPH_3D>(stage, c, s);
  if (v == SINH_3D) return launch_fused_batched_v<SINH_3D>(stage, c, s);
  set_error("batched evolutions: only full 3-D variants are instantiated");
  return BSSN_B200_EINVAL;
}

template <Variant V>
static void launch_rk_points_batched_v(int stage, const EvoDesc *descs, const BatchOuterPt *pts, int npts,
                                       cudaStream_t s) {
  const int threads = 128, blocks = (npts + threads - 1) / threads;
  switch (stage) {
    case 1: rk_points_batched_kernel<V, 1><<<blocks, threads, 0, s>>>(descs, pts, npts); break;
    case 2: rk_points_batched_kernel<V, 2><<<blocks, threads, 0, s>>>(descs, pts, npts); break;
    case 3: rk_points_batched_kernel<V, 3><<<blocks, threads, 0, s>>>(descs, pts, npts); break;
    default: rk_points_batched_kernel<V, 4><<<blocks, threads, 0, s>>>(descs, pts, npts); break;
  }
}

int launch_rk_points_batched(Variant v, int stage, const EvoDesc *descs, const BatchOuterPt *pts, int npts,
                             cudaStream_t s) {
  if (npts <= 0) return BSSN_B200_OK;
  if (v == SPH_3D) launch_rk_points_batched_v<SPH_3D>(stage, descs, pts, npts, s);
  else if (v == SINH_3D) launch_rk_points_batched_v<SINH_3D>(stage, descs, pts, npts, s);
  else {
    set_error("batched evolutions: only full 3-D variants are instantiated");
    return BSSN_B200_EINVAL;
  }
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

}  // namespace bssn
