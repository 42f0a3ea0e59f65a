// Internal definitions shared by the libbssn_b200 translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>

#include "bssn_b200.h"

namespace bssn {

// ---------------------------------------------------------------- errors
void set_error(const char *fmt, ...);
const char *last_error();
void count_launch(unsigned long long n);

#define BSSN_CUDA_TRY(call)                                                                                  \
  do {                                                                                                       \
    cudaError_t err_ = (call);                                                                               \
    if (err_ != cudaSuccess) {                                                                               \
      ::bssn::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(err_));                \
      return BSSN_B200_ECUDA;                                                                                \
    }                                                                                                        \
  } while (0)

// Every kernel launch site is followed by this check; it also counts the launch.
#define BSSN_LAUNCH_CHECK()                                                                                  \
  do {                                                                                                       \
    cudaError_t err_ = cudaGetLastError();                                                                   \
    if (err_ != cudaSuccess) {                                                                               \
      ::bssn::set_error("%s:%d: kernel launch: %s", __FILE__, __LINE__, cudaGetErrorString(err_));            \
      return BSSN_B200_ECUDA;                                                                                \
    }                                                                                                        \
    ::bssn::count_launch(1);                                                                                 \
  } while (0)

#define BSSN_TRY(call)                                                                                       \
  do {                                                                                                       \
    int rc_ = (call);                                                                                        \
    if (rc_ != BSSN_B200_OK) return rc_;                                                                     \
  } while (0)

// ---------------------------------------------------------------- variants
// Generated algebra variants: CoordSystem x symmetry axes.
enum Variant { SPH_3D = 0, SPH_AXI = 1, SINH_3D = 2, SINH_AXI = 3, SINHCYL_AXI = 4, NUM_VARIANTS = 5 };
int symmetry_axes_mask();  // bit d set: derivatives in direction d vanish
int variant_of(const params_struct *params, Variant *out);

// ---------------------------------------------------------------- grid geometry passed to kernels
struct GridDims {
  int N0, N1, N2;      // Nxx_plus_2NGHOSTS*
  int s1, s2;          // strides of i1, i2
  int ntot;            // points per gridfunction
  double invdxx0, invdxx1, invdxx2;
};
inline GridDims grid_dims(const params_struct *p) {
  GridDims g;
  g.N0 = p->Nxx_plus_2NGHOSTS0;
  g.N1 = p->Nxx_plus_2NGHOSTS1;
  g.N2 = p->Nxx_plus_2NGHOSTS2;
  g.s1 = g.N0;
  g.s2 = g.N0 * g.N1;
  g.ntot = g.N0 * g.N1 * g.N2;
  g.invdxx0 = p->invdxx0;
  g.invdxx1 = p->invdxx1;
  g.invdxx2 = p->invdxx2;
  return g;
}

struct RfmArrays {
  const double *f0, *f0_D0, *f0_DD00, *f0_DDD000, *f1, *f1_D1, *f1_DD11;
};
inline RfmArrays rfm_arrays(const rfm_struct *r) {
  return RfmArrays{r->f0_of_xx0, r->f0_of_xx0__D0, r->f0_of_xx0__DD00, r->f0_of_xx0__DDD000,
                   r->f1_of_xx1, r->f1_of_xx1__D1, r->f1_of_xx1__DD11};
}

struct PhysParams {
  double eta, ko_gauge, ko_nongauge;
};

// Pointwise operators implemented in pointwise.cu.
// mixed = true evaluates the algebra in FP32 (stencils, inputs and outputs stay FP64).
int launch_ricci(Variant v, const GridDims &g, const RfmArrays &rfm, const double *in, double *aux, cudaStream_t s,
                 bool mixed = false);
int launch_rhs(Variant v, bool mixed, const GridDims &g, const RfmArrays &rfm, const PhysParams &pp,
               const double *aux, const double *in, double *rhs, cudaStream_t s);
// H, M^2, |Lambda| at interior points into diag gridfunctions slots[0..2] (default 0, 1, 2).
int launch_constraints(Variant v, const GridDims &g, const RfmArrays &rfm, const double *in, const double *aux,
                       double *diag, cudaStream_t s, const int *slots = nullptr);
int launch_enforce(Variant v, const GridDims &g, const RfmArrays &rfm, double *gfs, cudaStream_t s);
int launch_lambda_id(Variant v, const GridDims &g, const RfmArrays &rfm, double *gfs, cudaStream_t s);

// RK4 stage coefficients of the low-storage form used by the reference
// (MoLtimestepping/MoL_step_forward_in_time.py:322-485): per stage s,
//   s=1: run  = dt/6 K;        OUT = y + dt/2 K   (OUT = K buffer)
//   s=2: run += dt/3 K;        OUT = y + dt/2 K
//   s=3: run += dt/3 K;        OUT = y + dt K
//   s=4: y    = y + run + dt/6 K
struct StageBuffers {
  double *y;     // y_n_gfs
  double *run;   // y_nplus1_running_total_gfs
  double *kin;   // stage input
  double *kout;  // RHS / stage output buffer
};
int launch_rhs_fused_stage(Variant v, bool mixed, int stage, double dt, const GridDims &g, const RfmArrays &rfm,
                           const PhysParams &pp, const double *aux, const StageBuffers &b, double *krhs,
                           cudaStream_t s);
int launch_rk_points(Variant v, int stage, double dt, const GridDims &g, const RfmArrays &rfm, const StageBuffers &b,
                     const outerpt_bc_struct *pts, int npts, const double *krhs, cudaStream_t s);
int launch_rk_substep(int stage, double dt, const GridDims &g, const StageBuffers &b, cudaStream_t s);

// r(xx0) and d(xx0)/dr for the Spherical family (the only nonzero partial x^i / partial r).
struct RadialMap {
  int sinh;  // 0: r = xx0 ; 1: r = AMPL sinh(xx0/SINHW)/sinh(1/SINHW)
  double AMPL, SINHW;
  __device__ __forceinline__ void eval(double xx0, double &r, double &dx0dr) const {
    if (!sinh) {
      r = xx0;
      dx0dr = 1.0;
      return;
    }
    // Same expression tree as the reference's r_and_partial_xi_partial_r_derivs (SinhSpherical).
    const double tmp0 = 1.0 / SINHW;
    const double tmp1 = exp(tmp0) - exp(-tmp0);
    const double tmp3 = exp(tmp0 * xx0);
    const double tmp4 = exp(-tmp0 * xx0);
    r = AMPL * (tmp3 - tmp4) / tmp1;
    dx0dr = tmp1 / (AMPL * (tmp0 * tmp3 + tmp0 * tmp4));
  }
};

int radial_map(const params_struct *p, RadialMap *rm);

// SinhCylindrical (reference_metric.py:1593-1630): rho = AMPLRHO sinh(xx0/SINHWRHO)/sinh(1/SINHWRHO),
// phi = xx1, z = AMPLZ sinh(xx2/SINHWZ)/sinh(1/SINHWZ), in the expression trees of the
// generated rfm_precompute_defines.
struct CylMap {
  double AMPLRHO, SINHWRHO, AMPLZ, SINHWZ;
  __host__ __device__ static double sinhv(double x, double A, double w) {
    return A * (exp(x / w) - exp(-x / w)) / (exp((1.0 / (w))) - exp(-1 / w));
  }
  __host__ __device__ static double dsinhv(double x, double A, double w) {
    return A * (exp(x / w) / w + exp(-x / w) / w) / (exp((1.0 / (w))) - exp(-1 / w));
  }
  __host__ __device__ double rho(double xx0) const { return sinhv(xx0, AMPLRHO, SINHWRHO); }
  __host__ __device__ double drho(double xx0) const { return dsinhv(xx0, AMPLRHO, SINHWRHO); }
  __host__ __device__ double z(double xx2) const { return sinhv(xx2, AMPLZ, SINHWZ); }
  __host__ __device__ double dz(double xx2) const { return dsinhv(xx2, AMPLZ, SINHWZ); }
  // r = sqrt(rho^2 + z^2) and partial x^i / partial r at fixed spherical angles (the
  // reference's r_and_partial_xi_partial_r_derivs, apply_bcs_outerradiation_and_inner.py:46-120):
  // dx0/dr = (rho/r)/rho'(xx0), dx1/dr = 0, dx2/dr = (z/r)/z'(xx2).
  __host__ __device__ void radial(double xx0, double xx2, double &r, double &dx0dr, double &dx2dr) const {
    const double rh = rho(xx0), zz = z(xx2);
    r = sqrt(rh * rh + zz * zz);
    dx0dr = rh / (r * drho(xx0));
    dx2dr = zz / (r * dz(xx2));
  }
};
inline CylMap cyl_map(const params_struct *p) { return CylMap{p->AMPLRHO, p->SINHWRHO, p->AMPLZ, p->SINHWZ}; }

// Boundary conditions implemented in boundary.cu.
int launch_inner_bcs(const GridDims &g, const bc_struct *bc, double *gfs, int num_gfs, const int8_t *parity_types,
                     cudaStream_t s);
int launch_radiation_bcs(const GridDims &g, const params_struct *p, const bc_struct *bc, const double *const xx[3],
                         const double *wavespeed, const double *f_inf, const double *gfs, double *rhs,
                         cudaStream_t s);
int launch_extrap_bcs(const GridDims &g, const bc_struct *bc, double *gfs, cudaStream_t s);
// Fused-stage boundary update: radiation RHS at pure outer points followed by the RK update
// of those points and the detgammabar projection; then parity copies of every inner point.
int launch_radiation_rk_bcs(Variant v, const GridDims &g, const params_struct *p, const bc_struct *bc,
                            const double *const xx[3], const RfmArrays &rfm, int stage, double dt,
                            const StageBuffers &b, double *krhs_scratch, cudaStream_t s);

// ---------------------------------------------------------------- batched evolutions
// One independent evolution of a batch, as the device sees it. Stage buffers rotate as in
// a single-grid RK4 step: stage 1 reads y and writes k_odd, 2: k_odd -> k_even,
// 3: k_even -> k_odd, 4: k_odd -> y.
struct EvoDesc {
  GridDims g;
  RfmArrays rfm;
  PhysParams pp;
  double dt;
  double *y, *run, *kodd, *keven, *aux, *krhs;
  const double *xx0;
  int radial_sinh;  // 0: r = xx0 ; 1: SinhSpherical r(xx0)
  double AMPL, SINHW;
  int tiles_x, tiles_y;               // this evolution's tiles along i0 and i1
  int tile_bx, tile_by, tile_bz;     // its tile shape: tile_bx * tile_by * tile_bz = 128 points
};
struct BatchOuterPt {
  int evo;
  outerpt_bc_struct p;
};
struct BatchInnerPt {
  int evo;
  innerpt_bc_struct b;
};
__host__ __device__ inline void stage_io(const EvoDesc &d, int stage, double *&kin, double *&kout) {
  switch (stage) {
    case 1: kin = d.y; kout = d.kodd; break;
    case 2: kin = d.kodd; kout = d.keven; break;
    case 3: kin = d.keven; kout = d.kodd; break;
    default: kin = d.kodd; kout = d.y; break;
  }
}
// Up to kChunkEvos evolutions as one launch of a Ricci or RHS group kernel sees them. The
// chunk is passed BY VALUE as the kernel parameter (it lands in the constant bank): every
// block reads its evolution's descriptor there with a block-uniform index, so the fields the
// point algebra uses throughout (strides, grid spacings, rfm and buffer pointers) stay
// uniform operands instead of taking per-thread registers. With the descriptors in global
// memory the same kernels spilled 300-600 bytes more per thread.
constexpr int kChunkEvos = 120;
struct BatchChunk {
  int nevo;                         // evolutions in this chunk
  int ntiles;                       // tiles of this chunk
  int tile_begin[kChunkEvos + 1];   // first chunk-local tile of each evolution; [nevo] = ntiles
  EvoDesc evo[kChunkEvos];
};
static_assert(sizeof(BatchChunk) + 16 <= 32764, "a BatchChunk must fit the 32764-byte kernel parameter space");
// Batched launchers (pointwise.cu, boundary.cu). The Ricci and RHS group kernels run one
// block per 128-point tile of a chunk; the boundary kernels cover every evolution in one
// launch, reading the descriptor array in device memory.
int launch_ricci_batched(Variant v, int stage, const BatchChunk &c, cudaStream_t s);
int launch_rhs_fused_batched(Variant v, int stage, const BatchChunk &c, cudaStream_t s);
int launch_radiation_batched(int stage, const EvoDesc *descs, const BatchOuterPt *pts, int npts, cudaStream_t s);
int launch_rk_points_batched(Variant v, int stage, const EvoDesc *descs, const BatchOuterPt *pts, int npts,
                             cudaStream_t s);
int launch_inner_batched(int stage, const EvoDesc *descs, const BatchInnerPt *pts, int npts, cudaStream_t s);

// Device constants (wave speeds, asymptotic values, parity types).
extern const int8_t kEvolParity[NUM_EVOL_GFS];
extern const double kWavespeed[NUM_EVOL_GFS];
extern const double kFInfinity[NUM_EVOL_GFS];

}  // namespace bssn
