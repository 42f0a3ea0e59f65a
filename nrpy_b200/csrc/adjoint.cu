// Reverse mode (discrete adjoint) of the RK4 BSSN step, for gradients of a scalar
// functional of the evolved state with respect to the Brill-Lindquist parameters.
//
// The differentiated forward model is the stage-by-stage RK4 step (the reference's stage
// order, MoL_step_forward_in_time.py:322-485) with radiation outer BCs:
//   stage s:  R = Ricci(Y_s); K = RHS(Y_s, R) on the interior; K = radiation(Y_s, K) on the
//             pure outer points (ghost layer by layer); K = parity(K) on the inner points;
//             Z_s = y_n + c_s dt K (+ run for s = 4); OUT_s = enforce(Z_s) on every point.
// Its adjoint, per stage in reverse: the projection's VJP at Z_s and the RK coefficients
// give Kbar; the inner-BC transpose moves Kbar from each inner point to its source; the
// radiation transpose (ghost layers outermost first) moves it inward and adds the radial
// stencil terms to Ybar; on the interior the RHS and Ricci VJPs (generated reverse-mode
// point functions, gen/bssn_adj_*.cuh) give the adjoint of every finite-difference leaf at
// every point, and the stencil-transpose kernel gathers those into Ybar.
//
// Gradients: J(y_N) -> ybar_N (Hamiltonian-constraint VJP + point seed), N steps back with
// checkpoints of y every `every` steps; each segment is recomputed forward from its
// checkpoint and each step once more while its adjoint runs (stage inputs and pre-
// projection hDD are stored for that step). The initial-data transpose (inner parity, then
// extrapolation, in reverse) leaves the adjoint of the interior alpha and W = cf, whose
// Brill-Lindquist derivatives d psi^-2 / d(m_i, z_i) give the gradient.
#include <algorithm>
#include <cstring>

#include "bssn_common.cuh"

// The reverse-mode algebra and stencil transposes are generated for the 4th-order build only.
#if BSSN_B200_FD_ORDER == 4

namespace bssn {
namespace {

template <typename T>
__device__ __forceinline__ T ipow(T x, int n) {
  T r = x;
  for (int k = 1; k < n; k++) r *= x;
  return r;
}

// Adds on assignment: the generated code writes each leaf adjoint once per function as
// `OUT(row) = value;`, and several functions contribute to one row.
struct AccRef {
  double *p;
  __device__ __forceinline__ void operator=(double v) const { *p += v; }
};

constexpr int ABX = 32, ABY = 2;  // VJP kernels: 64 threads, per-thread shared-memory slots

// Stencil loads, rfm values and parameters around one interior point, plus the adjoint
// seeds (read through Seeds::SEED(j)) and the leaf-adjoint outputs of that point.
struct VjpCtxBase {
  const double *__restrict__ in;   // stage input + idx
  const double *__restrict__ aux;  // Rbar_ij + idx
  int s1, s2, ntot;
  int i0, i1;
  double invdxx0, invdxx1, invdxx2;
  RfmArrays rfm;
  double eta, KreissOliger_strength_gauge, KreissOliger_strength_nongauge;
  const double *seed;  // + idx
  double seed_scale;
  double *la;      // leaf-adjoint rows + idx
  double *auxbar;  // Rbar adjoint + idx
  __device__ __forceinline__ double ld(int gf, int a, int b, int c) const {
    return __ldg(in + ((size_t)gf * ntot + (a + b * s1 + c * s2)));
  }
  __device__ __forceinline__ double ldaux(int k) const { return __ldg(aux + (size_t)k * ntot); }
  __device__ __forceinline__ AccRef out(int r) const { return AccRef{la + (size_t)r * ntot}; }
  __device__ __forceinline__ AccRef outr(int k) const { return AccRef{auxbar + (size_t)k * ntot}; }
};
template <class Seeds>
struct VjpCtx : VjpCtxBase {
  __device__ __forceinline__ double adjin(int j) const {
    return seed_scale * __ldg(seed + (size_t)Seeds::SEED(j) * ntot);
  }
};

// Pointwise context of the projection's VJP: hDD before the projection (6 gridfunctions)
// and the adjoint of its output; leaf adjoints go to a local array.
struct EnforceCtx {
  const double *zh;    // pre-projection hDD + idx
  const double *obar;  // adjoint of the stage output + idx
  double *zb;          // 6 local values
  int ntot, i0, i1;
  RfmArrays rfm;
  __device__ __forceinline__ double ld(int gf, int, int, int) const { return zh[(size_t)(gf - HDD00GF) * ntot]; }
  __device__ __forceinline__ double adjin(int j) const { return obar[(size_t)(HDD00GF + j) * ntot]; }
  __device__ __forceinline__ AccRef out(int r) const { return AccRef{zb + (r - HDD00GF)}; }
};

}  // namespace

#define LD(gf, a, b, c) ctx.ld(gf, a, b, c)
#define LDAUX(k) ctx.ldaux(k)
#define RFM(arr, d) __ldg(ctx.rfm.arr + ctx.i##d)
#define rfm_f0 f0
#define rfm_f0_D0 f0_D0
#define rfm_f0_DD00 f0_DD00
#define rfm_f0_DDD000 f0_DDD000
#define rfm_f1 f1
#define rfm_f1_D1 f1_D1
#define rfm_f1_DD11 f1_DD11
#define PARAM(name) ctx.name
#define SMEM(k) sm[(k) * (ABX * ABY)]
#define ADJIN(j) ctx.adjin(j)
#define OUT(r) ctx.out(r)
#define OUTR(k) ctx.outr(k)
#define invdxx0 ctx.invdxx0
#define invdxx1 ctx.invdxx1
#define invdxx2 ctx.invdxx2
#include "gen/bssn_adj_sph_3d.cuh"
#undef invdxx0
#undef invdxx1
#undef invdxx2

namespace {

constexpr int NROWS = adj_nrows_sph_3d;

struct HVjp {
  static constexpr int N = 1;
  static constexpr int SLOTS = h_vjp_sph_3d_SMEM_SLOTS;
  __host__ __device__ static constexpr int SEED(int) { return 0; }
  template <typename T, typename TF, typename Ctx>
  __device__ __forceinline__ static void eval(const Ctx &ctx, volatile T *sm) {
    h_vjp_sph_3d<T, TF>(ctx, sm);
  }
};

__constant__ signed char c_rows[NROWS][4];
__constant__ int c_row_begin[NUM_EVOL_GFS + 1];  // derivative rows of gridfunction g
__constant__ double c_w[4][7];                   // dD, dDD, dupD, dKOD at offsets -3..3
__constant__ double c_wfd1[5][9];                // radiation FD1, shift -2..2, offsets -4..4
// Parity type of each evolved gridfunction (the reference's evol_gf_parity).
__constant__ int8_t c_parity[NUM_EVOL_GFS] = {4, 5, 6, 7, 8, 9, 0, 1, 2, 3, 0, 4, 5, 6, 7, 8, 9, 1, 2, 3, 0, 1, 2, 3};

__device__ __forceinline__ void fill_ctx(VjpCtxBase &c, const GridDims &g, const RfmArrays &rfm, const PhysParams &pp,
                                         const double *in, const double *aux, int i0, int i1, int i2) {
  const size_t idx = (size_t)i0 + (size_t)g.s1 * i1 + (size_t)g.s2 * i2;
  c.in = in + idx;
  c.aux = aux ? aux + idx : nullptr;
  c.s1 = g.s1;
  c.s2 = g.s2;
  c.ntot = g.ntot;
  c.i0 = i0;
  c.i1 = i1;
  c.invdxx0 = g.invdxx0;
  c.invdxx1 = g.invdxx1;
  c.invdxx2 = g.invdxx2;
  c.rfm = rfm;
  c.eta = pp.eta;
  c.KreissOliger_strength_gauge = pp.ko_gauge;
  c.KreissOliger_strength_nongauge = pp.ko_nongauge;
}

// One thread per interior point: the VJP of one output group at that point.
template <class Grp>
__global__ void __launch_bounds__(ABX *ABY) vjp_kernel(const GridDims g, const RfmArrays rfm, const PhysParams pp,
                                                       const double *__restrict__ in, const double *__restrict__ aux,
                                                       const double *__restrict__ seed, const double seed_scale,
                                                       double *__restrict__ la, double *__restrict__ auxbar) {
  const int i0 = NGHOSTS + blockIdx.x * ABX + threadIdx.x;
  const int i1 = NGHOSTS + blockIdx.y * ABY + threadIdx.y;
  const int i2 = NGHOSTS + blockIdx.z;
  if (i0 >= g.N0 - NGHOSTS || i1 >= g.N1 - NGHOSTS) return;
  extern __shared__ double slots[];
  volatile double *sm = slots + threadIdx.x + ABX * threadIdx.y;
  VjpCtx<Grp> ctx;
  fill_ctx(ctx, g, rfm, pp, in, aux, i0, i1, i2);
  const size_t idx = (size_t)i0 + (size_t)g.s1 * i1 + (size_t)g.s2 * i2;
  ctx.seed = seed + idx;
  ctx.seed_scale = seed_scale;
  ctx.la = la + idx;
  ctx.auxbar = auxbar + idx;
  Grp::template eval<double, double>(ctx, sm);
}

__global__ void upwind_bits_kernel(const GridDims g, const RfmArrays rfm, const double *__restrict__ in,
                                   uint8_t *__restrict__ bits) {
  const int i0 = NGHOSTS + blockIdx.x * 32 + threadIdx.x;
  const int i1 = NGHOSTS + blockIdx.y * 4 + threadIdx.y;
  const int i2 = NGHOSTS + blockIdx.z;
  if (i0 >= g.N0 - NGHOSTS || i1 >= g.N1 - NGHOSTS) return;
  VjpCtxBase ctx;
  fill_ctx(ctx, g, rfm, PhysParams{0.0, 0.0, 0.0}, in, nullptr, i0, i1, i2);
  bits[(size_t)i0 + (size_t)g.s1 * i1 + (size_t)g.s2 * i2] = (uint8_t)upwind_bits_sph_3d<double, double>(ctx);
}

// Transpose of every finite-difference leaf: Ybar_g(q) += sum over the rows of
// gridfunction g and their stencil offsets s of w(s) * la_row(q - s). Leaf adjoints are
// zero outside the interior, so only the stencil direction needs a bounds check. For
// upwinded rows the stencil side is the one the forward chose at the source point.
__global__ void stencil_transpose_kernel(const GridDims g, const double *__restrict__ la,
                                         const uint8_t *__restrict__ upw, double *__restrict__ ybar) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)g.ntot * NUM_EVOL_GFS) return;
  const int gf = (int)(t / g.ntot);
  const int q = (int)(t - (long long)gf * g.ntot);
  const int i2 = q / g.s2;
  const int rem = q - i2 * g.s2;
  const int i1 = rem / g.s1;
  const int i0 = rem - i1 * g.s1;
  const int ii[3] = {i0, i1, i2};
  const int nn[3] = {g.N0, g.N1, g.N2};
  const int st[3] = {1, g.s1, g.s2};
  const double inv[3] = {g.invdxx0, g.invdxx1, g.invdxx2};
  const size_t nt = (size_t)g.ntot;
  double acc = la[(size_t)gf * nt + q];
  for (int r = c_row_begin[gf]; r < c_row_begin[gf + 1]; r++) {
    const int kind = c_rows[r][1], d1 = c_rows[r][2], d2 = c_rows[r][3];
    const double *L = la + (size_t)r * nt;
    if (kind == 2 && d1 != d2) {  // mixed second derivative: product of centred first derivatives
      const double f = inv[d1] * inv[d2];
      for (int s = -2; s <= 2; s++) {
        const int a = ii[d1] - s;
        if (s == 0 || a < 0 || a >= nn[d1]) continue;
        for (int u = -2; u <= 2; u++) {
          const int b = ii[d2] - u;
          if (u == 0 || b < 0 || b >= nn[d2]) continue;
          acc += c_w[0][s + 3] * c_w[0][u + 3] * f * L[q - s * st[d1] - u * st[d2]];
        }
      }
      continue;
    }
    const double f = (kind == 2) ? inv[d1] * inv[d1] : inv[d1];
    for (int s = -3; s <= 3; s++) {
      const int a = ii[d1] - s;
      if (a < 0 || a >= nn[d1]) continue;
      const int p = q - s * st[d1];
      double w;
      if (kind == 3) {  // upwinded: forward read U ? f(p+t) : -f(p-t) with weight up[t]
        const bool U = (upw[p] >> d1) & 1;
        w = U ? c_w[2][s + 3] : -c_w[2][3 - s];
      } else {
        w = c_w[kind == 1 ? 0 : (kind == 2 ? 1 : 3)][s + 3];
      }
      if (w != 0.0) acc += w * f * L[p];
    }
  }
  ybar[t] += acc;
}

// Transpose of the inner (parity) BCs: gbar[src] += sign * gbar[dst]; gbar[dst] = 0.
// Sources are never inner points; several inner points may share a source.
__global__ void inner_adjoint_kernel(const int ntot, const innerpt_bc_struct *__restrict__ pts, const int npts,
                                     double *__restrict__ gbar) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * NUM_EVOL_GFS) return;
  const int gf = t / npts;
  const innerpt_bc_struct bc = pts[t - gf * npts];
  double *gb = gbar + (size_t)gf * ntot;
  const double v = gb[bc.dstpt];
  gb[bc.dstpt] = 0.0;
  if (v != 0.0) atomicAdd(gb + bc.srcpt, bc.parity[c_parity[gf]] < 0 ? -v : v);
}

__device__ __forceinline__ int fd1_shift(int dest_i0, int face, int N0) {
  const int R = 2;
  int off = face;
  if (dest_i0 < R) off = R - dest_i0;
  else if (dest_i0 > N0 - R - 1) off = (N0 - R - 1) - dest_i0;
  return off;
}

// Transpose of one ghost layer of the radiation BC (one thread per outer point and
// gridfunction). Forward: K(q) = -c (dr f(q) + (f(q) - finf)/r) + (r_int/r)^3 (K(q_int) +
// c (dr f(q_int) + (f(q_int) - finf)/r_int)), dr f = dxx0/dr * FD1 along i0.
__global__ void radiation_adjoint_kernel(const GridDims g, const RadialMap rm, const double *__restrict__ xx0,
                                         const outerpt_bc_struct *__restrict__ pts, const int npts,
                                         double *__restrict__ kbar, double *__restrict__ ybar) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * NUM_EVOL_GFS) return;
  const int gf = t / npts;
  const outerpt_bc_struct p = pts[t - gf * npts];
  const int i0 = p.i0, j0 = i0 + p.FACEX0;
  const size_t nt = (size_t)g.ntot;
  const size_t idx = (size_t)i0 + (size_t)g.s1 * p.i1 + (size_t)g.s2 * p.i2;
  const size_t idx_int = (size_t)j0 + (size_t)g.s1 * (p.i1 + p.FACEX1) + (size_t)g.s2 * (p.i2 + p.FACEX2);
  double *kb = kbar + (size_t)gf * nt;
  double *fb = ybar + (size_t)gf * nt;
  const double v = kb[idx];
  kb[idx] = 0.0;
  double r, dx0dr, r_int, dx0dr_int;
  rm.eval(__ldg(xx0 + i0), r, dx0dr);
  rm.eval(__ldg(xx0 + j0), r_int, dx0dr_int);
  const double c = (gf == ALPHAGF) ? 1.41421356237310 : 1.0;
  const double rinv = 1.0 / r;
  const double ratio3 = (r_int * r_int * r_int) * (rinv * rinv * rinv);
  kb[idx_int] += ratio3 * v;
  const int sh = fd1_shift(i0, p.FACEX0, g.N0) + 2;
  const int sh_int = fd1_shift(j0, p.FACEX0, g.N0) + 2;
  const double a = -c * dx0dr * g.invdxx0 * v;
  const double b = ratio3 * c * dx0dr_int * g.invdxx0 * v;
  for (int s = -4; s <= 4; s++) {
    const double w = c_wfd1[sh][s + 4];
    if (w != 0.0) fb[idx + s] += a * w;
    const double wi = c_wfd1[sh_int][s + 4];
    if (wi != 0.0) fb[idx_int + s] += b * wi;
  }
  fb[idx] += -c * rinv * v;
  fb[idx_int] += ratio3 * c / r_int * v;
}

// Transpose of one ghost layer of the extrapolation BC f(q) = 3 f(q+n) - 3 f(q+2n) + f(q+3n).
__global__ void extrap_adjoint_kernel(const GridDims g, const outerpt_bc_struct *__restrict__ pts, const int npts,
                                      double *__restrict__ gbar) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * NUM_EVOL_GFS) return;
  const int gf = t / npts;
  const outerpt_bc_struct p = pts[t - gf * npts];
  const long long d = p.FACEX0 + (long long)g.s1 * p.FACEX1 + (long long)g.s2 * p.FACEX2;
  const long long idx = p.i0 + (long long)g.s1 * p.i1 + (long long)g.s2 * p.i2;
  double *f = gbar + (size_t)gf * g.ntot;
  const double v = f[idx];
  f[idx] = 0.0;
  f[idx + d] += 3.0 * v;
  f[idx + 2 * d] -= 3.0 * v;
  f[idx + 3 * d] += v;
}

// Stage s of the RK update and projection, in reverse, at every point: Zbar = projection
// VJP (hDD) or Obar (other gridfunctions); Kbar = c_s dt Zbar + d_s dt runbar; ybar += Zbar.
template <int STAGE>
__global__ void rk_enforce_adjoint_kernel(const GridDims g, const RfmArrays rfm, const double *__restrict__ zh,
                                          const double *__restrict__ obar, double *__restrict__ kbar,
                                          double *__restrict__ runbar, double *__restrict__ ybar, const double dt) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= g.ntot) return;
  const int i2 = idx / g.s2;
  const int rem = idx - i2 * g.s2;
  const int i1 = rem / g.s1;
  const int i0 = rem - i1 * g.s1;
  double zb[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  EnforceCtx ctx{zh + idx, obar + idx, zb, g.ntot, i0, i1, rfm};
  enforce_vjp_sph_3d<double, double>(ctx, nullptr);
  const size_t nt = (size_t)g.ntot;
#pragma unroll
  for (int gf = 0; gf < NUM_EVOL_GFS; gf++) {
    const size_t i = (size_t)gf * nt + idx;
    const double z = (gf >= HDD00GF && gf < HDD00GF + 6) ? zb[gf - HDD00GF] : obar[i];
    if constexpr (STAGE == 4) {
      runbar[i] = z;
      ybar[i] = z;
      kbar[i] = (1.0 / 6.0) * dt * z;
    } else {
      const double cz = (STAGE == 3) ? 1.0 : 0.5;
      const double cr = (STAGE == 1) ? (1.0 / 6.0) : (1.0 / 3.0);
      kbar[i] = cz * dt * z + cr * dt * runbar[i];
      ybar[i] += z;
    }
  }
}

__global__ void axpy_kernel(const size_t n, const double *__restrict__ x, double *__restrict__ y) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] += x[i];
}

__global__ void add_point_kernel(double *p, const double v) { *p += v; }

// Deterministic block sums: warp shuffles, then one value per warp in shared memory.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double *out) {
  __shared__ double red[K][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; k++) {
    double x = v[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) red[k][warp] = x;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) {
      double x = lane < (int)(blockDim.x >> 5) ? red[k][lane] : 0.0;
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (lane == 0) out[k] = x;
    }
  }
}

constexpr int RED_BLOCKS = 296, RED_THREADS = 256;

// Partial sums over interior points of H^2 (K = 1) or of the Brill-Lindquist parameter
// derivatives weighted by the initial-data adjoint (K = 4).
__global__ void sum_h2_kernel(const GridDims g, const double *__restrict__ h, double *__restrict__ partials) {
  const int n0 = g.N0 - 2 * NGHOSTS, n1 = g.N1 - 2 * NGHOSTS, n2 = g.N2 - 2 * NGHOSTS;
  const long long n = (long long)n0 * n1 * n2;
  double v[1] = {0.0};
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(t % n0);
    const long long r = t / n0;
    const int b = (int)(r % n1), c = (int)(r / n1);
    const double x = h[(size_t)(a + NGHOSTS) + (size_t)g.s1 * (b + NGHOSTS) + (size_t)g.s2 * (c + NGHOSTS)];
    v[0] += x * x;
  }
  block_sum<1>(v, partials + blockIdx.x);
}

struct BLParams {
  double m1, x1, y1, z1, m2, x2, y2, z2;
};

// d/d(m1, z1, m2, z2) of alpha = W = psi^-2, psi = 1 + m1/(2 d1) + m2/(2 d2), contracted
// with the adjoint of the interior initial-data alpha and cf.
__global__ void bl_id_vjp_kernel(const GridDims g, const RadialMap rm, const double *__restrict__ xx0,
                                 const double *__restrict__ xx1, const double *__restrict__ xx2, const BLParams bl,
                                 const double *__restrict__ ybar, double *__restrict__ partials) {
  const int n0 = g.N0 - 2 * NGHOSTS, n1 = g.N1 - 2 * NGHOSTS, n2 = g.N2 - 2 * NGHOSTS;
  const long long n = (long long)n0 * n1 * n2;
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i0 = (int)(t % n0) + NGHOSTS;
    const long long r = t / n0;
    const int i1 = (int)(r % n1) + NGHOSTS, i2 = (int)(r / n1) + NGHOSTS;
    const size_t idx = (size_t)i0 + (size_t)g.s1 * i1 + (size_t)g.s2 * i2;
    const double wbar = ybar[(size_t)ALPHAGF * g.ntot + idx] + ybar[(size_t)CFGF * g.ntot + idx];
    if (wbar == 0.0) continue;
    double rr, dummy;
    rm.eval(xx0[i0], rr, dummy);
    const double tmp = rr * sin(xx1[i1]);
    const double X = tmp * cos(xx2[i2]), Y = tmp * sin(xx2[i2]), Z = rr * cos(xx1[i1]);
    const double d1 = sqrt((X - bl.x1) * (X - bl.x1) + (Y - bl.y1) * (Y - bl.y1) + (Z - bl.z1) * (Z - bl.z1));
    const double d2 = sqrt((X - bl.x2) * (X - bl.x2) + (Y - bl.y2) * (Y - bl.y2) + (Z - bl.z2) * (Z - bl.z2));
    const double psi = 1.0 + 0.5 * bl.m1 / d1 + 0.5 * bl.m2 / d2;
    const double dpsi = -2.0 / (psi * psi * psi) * wbar;  // d(psi^-2)/d psi times the adjoint
    v[0] += dpsi * (0.5 / d1);
    v[1] += dpsi * (0.5 * bl.m1 * (Z - bl.z1) / (d1 * d1 * d1));
    v[2] += dpsi * (0.5 / d2);
    v[3] += dpsi * (0.5 * bl.m2 * (Z - bl.z2) / (d2 * d2 * d2));
  }
  block_sum<4>(v, partials + 4 * blockIdx.x);
}

template <int K>
__global__ void finish_sum_kernel(const double *__restrict__ partials, const int nblocks, double *__restrict__ out) {
  double v[K];
#pragma unroll
  for (int k = 0; k < K; k++) v[k] = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < K; k++) v[k] += partials[K * b + k];
  block_sum<K>(v, out);
}

template <class K>
int set_slots(K kernel, size_t bytes) {
  if (bytes > 48 * 1024) BSSN_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return BSSN_B200_OK;
}

template <class Grp>
int launch_vjp(const GridDims &g, const RfmArrays &rfm, const PhysParams &pp, const double *in, const double *aux,
               const double *seed, double scale, double *la, double *auxbar, cudaStream_t s) {
  const size_t bytes = (size_t)Grp::SLOTS * ABX * ABY * sizeof(double);
  BSSN_TRY(set_slots(vjp_kernel<Grp>, bytes));
  const dim3 grid((g.N0 - 2 * NGHOSTS + ABX - 1) / ABX, (g.N1 - 2 * NGHOSTS + ABY - 1) / ABY, g.N2 - 2 * NGHOSTS);
  vjp_kernel<Grp><<<grid, dim3(ABX, ABY), bytes, s>>>(g, rfm, pp, in, aux, seed, scale, la, auxbar);
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

unsigned blocks_for(long long work, int threads) { return (unsigned)((work + threads - 1) / threads); }

}  // namespace

}  // namespace bssn

using namespace bssn;

struct bssn_b200_adjoint {
  commondata_struct *cd;
  griddata_struct *gd;
  int nsteps, every, nseg;
  cudaStream_t s;
  GridDims g;
  RfmArrays rfm;
  PhysParams pp;
  RadialMap rm;
  size_t nt;
  double *ckpt = nullptr;    // (nseg + 1) states: y at steps 0, every, 2 every, ...; the last is y_N
  double *segy = nullptr;    // `every` states of the segment being reversed
  double *stY = nullptr;     // 4 stage inputs of the step being reversed
  double *stZh = nullptr;    // 4 x 6 pre-projection hDD of that step
  double *obar = nullptr, *kbar = nullptr, *runbar = nullptr, *ybar = nullptr;
  double *la = nullptr;      // NROWS leaf-adjoint rows
  double *auxbar = nullptr;  // 6 Rbar adjoints
  double *diag = nullptr;    // H, M^2, |Lambda|
  uint8_t *upw = nullptr;
  double *partials = nullptr;
  double *dout = nullptr;
  size_t idx_alpha = 0;
  bool forward_done = false;
};

namespace bssn {
int mol_step(commondata_struct *cd, griddata_struct *gd, int mode, int mixed, cudaStream_t s);
namespace {

int adj_alloc(double **p, size_t n) {
  if (cudaMalloc(p, n * sizeof(double)) != cudaSuccess) {
    set_error("adjoint: cudaMalloc of %zu doubles failed", n);
    return BSSN_B200_ENOMEM;
  }
  return BSSN_B200_OK;
}

void adj_free(bssn_b200_adjoint *a) {
  double *bufs[] = {a->ckpt, a->segy, a->stY,  a->stZh,   a->obar, a->kbar,     a->runbar,
                    a->ybar, a->la,   a->auxbar, a->diag, a->partials, a->dout};
  for (double *b : bufs)
    if (b) cudaFree(b);
  if (a->upw) cudaFree(a->upw);
}

int copy_d2d(double *dst, const double *src, size_t n, cudaStream_t s) {
  BSSN_CUDA_TRY(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
  return BSSN_B200_OK;
}
int zero(double *p, size_t n, cudaStream_t s) {
  BSSN_CUDA_TRY(cudaMemsetAsync(p, 0, n * sizeof(double), s));
  return BSSN_B200_OK;
}

int upload_tables() {
  int begin[NUM_EVOL_GFS + 1];
  int r = NUM_EVOL_GFS;
  for (int gf = 0; gf < NUM_EVOL_GFS; gf++) {
    begin[gf] = r;
    while (r < NROWS && adj_rows_sph_3d[r][0] == gf) r++;
  }
  begin[NUM_EVOL_GFS] = r;
  if (r != NROWS) {
    set_error("adjoint: leaf table is not sorted by gridfunction");
    return BSSN_B200_EINVAL;
  }
  double w[4][7], wf[5][9];
  for (int s = 0; s < 7; s++) {
    w[0][s] = adj_wD_sph_3d[s];
    w[1][s] = adj_wDD_sph_3d[s];
    w[2][s] = adj_wUP_sph_3d[s];
    w[3][s] = adj_wKO_sph_3d[s];
  }
  for (int a = 0; a < 5; a++)
    for (int s = 0; s < 9; s++) wf[a][s] = adj_wFD1_sph_3d[a][s];
  BSSN_CUDA_TRY(cudaMemcpyToSymbol(c_rows, adj_rows_sph_3d, sizeof(adj_rows_sph_3d)));
  BSSN_CUDA_TRY(cudaMemcpyToSymbol(c_row_begin, begin, sizeof(begin)));
  BSSN_CUDA_TRY(cudaMemcpyToSymbol(c_w, w, sizeof(w)));
  BSSN_CUDA_TRY(cudaMemcpyToSymbol(c_wfd1, wf, sizeof(wf)));
  return BSSN_B200_OK;
}

int launch_sum(const bssn_b200_adjoint *a, const double *h, double *host_out) {
  sum_h2_kernel<<<RED_BLOCKS, RED_THREADS, 0, a->s>>>(a->g, h, a->partials);
  BSSN_LAUNCH_CHECK();
  finish_sum_kernel<1><<<1, RED_THREADS, 0, a->s>>>(a->partials, RED_BLOCKS, a->dout);
  BSSN_LAUNCH_CHECK();
  BSSN_CUDA_TRY(cudaMemcpyAsync(host_out, a->dout, sizeof(double), cudaMemcpyDeviceToHost, a->s));
  BSSN_CUDA_TRY(cudaStreamSynchronize(a->s));
  return BSSN_B200_OK;
}

// Leaf adjoints of the Ricci groups from the Rbar adjoint (seeds in auxbar).
int ricci_vjps(const bssn_b200_adjoint *a, const double *Y) {
  BSSN_TRY((launch_vjp<RicciVjp_sph_3d<0>>(a->g, a->rfm, a->pp, Y, nullptr, a->auxbar, 1.0, a->la, a->auxbar, a->s)));
  BSSN_TRY((launch_vjp<RicciVjp_sph_3d<1>>(a->g, a->rfm, a->pp, Y, nullptr, a->auxbar, 1.0, a->la, a->auxbar, a->s)));
  return launch_vjp<RicciVjp_sph_3d<2>>(a->g, a->rfm, a->pp, Y, nullptr, a->auxbar, 1.0, a->la, a->auxbar, a->s);
}

int transpose(const bssn_b200_adjoint *a, double *ybar) {
  const long long work = (long long)a->nt * NUM_EVOL_GFS;
  stencil_transpose_kernel<<<blocks_for(work, 256), 256, 0, a->s>>>(a->g, a->la, a->upw, ybar);
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

int inner_adjoint(const bssn_b200_adjoint *a, double *gbar) {
  const bc_struct &bc = a->gd[0].bcstruct;
  const int n = bc.bc_info.num_inner_boundary_points;
  if (n <= 0) return BSSN_B200_OK;
  inner_adjoint_kernel<<<blocks_for((long long)n * NUM_EVOL_GFS, 256), 256, 0, a->s>>>(a->g.ntot, bc.inner_bc_array, n,
                                                                                     gbar);
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

// Adjoint of G(Y) = inner(radiation(RHS(Y, Ricci(Y)))): kbar (all points) -> ybar_out.
int g_adjoint(bssn_b200_adjoint *a, const double *Y, double *ybar_out) {
  const griddata_struct &G = a->gd[0];
  const bc_struct &bc = G.bcstruct;
  BSSN_TRY(inner_adjoint(a, a->kbar));
  BSSN_TRY(zero(ybar_out, a->nt * NUM_EVOL_GFS, a->s));
  for (int gz = NGHOSTS - 1; gz >= 0; gz--)
    for (int dirn = 2; dirn >= 0; dirn--) {
      const int n = bc.bc_info.num_pure_outer_boundary_points[gz][dirn];
      if (n <= 0) continue;
      if (dirn != 0) {
        set_error("adjoint: outer points on face direction %d are not supported", dirn);
        return BSSN_B200_EINVAL;
      }
      radiation_adjoint_kernel<<<blocks_for((long long)n * NUM_EVOL_GFS, 256), 256, 0, a->s>>>(
          a->g, a->rm, G.xx[0], bc.pure_outer_bc_array[dirn + 3 * gz], n, a->kbar, ybar_out);
      BSSN_LAUNCH_CHECK();
    }
  double *aux = G.gridfuncs.auxevol_gfs;
  BSSN_TRY(launch_ricci(SPH_3D, a->g, a->rfm, Y, aux, a->s));
  {
    const dim3 grid((a->g.N0 - 2 * NGHOSTS + 31) / 32, (a->g.N1 - 2 * NGHOSTS + 3) / 4, a->g.N2 - 2 * NGHOSTS);
    upwind_bits_kernel<<<grid, dim3(32, 4), 0, a->s>>>(a->g, a->rfm, Y, a->upw);
    BSSN_LAUNCH_CHECK();
  }
  BSSN_TRY(zero(a->la, a->nt * NROWS, a->s));
  BSSN_TRY(zero(a->auxbar, a->nt * NUM_AUXEVOL_GFS, a->s));
  BSSN_TRY((launch_vjp<RhsVjp_sph_3d<0>>(a->g, a->rfm, a->pp, Y, aux, a->kbar, 1.0, a->la, a->auxbar, a->s)));
  BSSN_TRY((launch_vjp<RhsVjp_sph_3d<1>>(a->g, a->rfm, a->pp, Y, aux, a->kbar, 1.0, a->la, a->auxbar, a->s)));
  BSSN_TRY((launch_vjp<RhsVjp_sph_3d<2>>(a->g, a->rfm, a->pp, Y, aux, a->kbar, 1.0, a->la, a->auxbar, a->s)));
  BSSN_TRY(ricci_vjps(a, Y));
  return transpose(a, ybar_out);
}

// One RK4 step from the state in y_n, stage by stage, keeping each stage input and the
// hDD of each stage output before the projection.
int forward_step_record(bssn_b200_adjoint *a) {
  griddata_struct &G = a->gd[0];
  MoL_gridfunctions_struct &gf = G.gridfuncs;
  const double dt = a->cd->dt;
  for (int stage = 1; stage <= 4; stage++) {
    StageBuffers b;
    b.y = gf.y_n_gfs;
    b.run = gf.y_nplus1_running_total_gfs;
    switch (stage) {
      case 1: b.kin = gf.y_n_gfs; b.kout = gf.k_odd_gfs; break;
      case 2: b.kin = gf.k_odd_gfs; b.kout = gf.k_even_gfs; break;
      case 3: b.kin = gf.k_even_gfs; b.kout = gf.k_odd_gfs; break;
      default: b.kin = gf.k_odd_gfs; b.kout = gf.k_even_gfs; break;
    }
    BSSN_TRY(copy_d2d(a->stY + (size_t)(stage - 1) * NUM_EVOL_GFS * a->nt, b.kin, a->nt * NUM_EVOL_GFS, a->s));
    BSSN_TRY(launch_ricci(SPH_3D, a->g, a->rfm, b.kin, gf.auxevol_gfs, a->s));
    BSSN_TRY(launch_rhs(SPH_3D, false, a->g, a->rfm, a->pp, gf.auxevol_gfs, b.kin, b.kout, a->s));
    BSSN_TRY(launch_radiation_bcs(a->g, &G.params, &G.bcstruct, G.xx, kWavespeed, kFInfinity, b.kin, b.kout, a->s));
    BSSN_TRY(launch_inner_bcs(a->g, &G.bcstruct, b.kout, NUM_EVOL_GFS, nullptr, a->s));
    BSSN_TRY(launch_rk_substep(stage, dt, a->g, b, a->s));
    double *out = (stage == 4) ? b.y : b.kout;
    BSSN_TRY(copy_d2d(a->stZh + (size_t)(stage - 1) * 6 * a->nt, out + (size_t)HDD00GF * a->nt, 6 * a->nt, a->s));
    BSSN_TRY(launch_enforce(SPH_3D, a->g, a->rfm, out, a->s));
  }
  return BSSN_B200_OK;
}

template <int STAGE>
int rk_enforce_adjoint(bssn_b200_adjoint *a) {
  rk_enforce_adjoint_kernel<STAGE><<<blocks_for(a->g.ntot, 128), 128, 0, a->s>>>(
      a->g, a->rfm, a->stZh + (size_t)(STAGE - 1) * 6 * a->nt, a->obar, a->kbar, a->runbar, a->ybar, a->cd->dt);
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

// obar: adjoint of y_{n+1} on entry, of y_n on exit; y_n_in is the state at step n.
int step_adjoint(bssn_b200_adjoint *a, const double *y_n_in) {
  griddata_struct &G = a->gd[0];
  const size_t n = a->nt * NUM_EVOL_GFS;
  if (y_n_in != G.gridfuncs.y_n_gfs) BSSN_TRY(copy_d2d(G.gridfuncs.y_n_gfs, y_n_in, n, a->s));
  BSSN_TRY(forward_step_record(a));
  BSSN_TRY(rk_enforce_adjoint<4>(a));
  BSSN_TRY(g_adjoint(a, a->stY + 3 * n, a->obar));
  BSSN_TRY(rk_enforce_adjoint<3>(a));
  BSSN_TRY(g_adjoint(a, a->stY + 2 * n, a->obar));
  BSSN_TRY(rk_enforce_adjoint<2>(a));
  BSSN_TRY(g_adjoint(a, a->stY + 1 * n, a->obar));
  BSSN_TRY(rk_enforce_adjoint<1>(a));
  BSSN_TRY(g_adjoint(a, a->stY, a->obar));
  axpy_kernel<<<blocks_for((long long)n, 256), 256, 0, a->s>>>(n, a->ybar, a->obar);
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

// J(y) = sum over the interior of H^2 + alpha at the point next to the origin.
int functional(bssn_b200_adjoint *a, const double *y, double out[3]) {
  griddata_struct &G = a->gd[0];
  double *aux = G.gridfuncs.auxevol_gfs;
  BSSN_TRY(launch_ricci(SPH_3D, a->g, a->rfm, y, aux, a->s));
  BSSN_TRY(launch_constraints(SPH_3D, a->g, a->rfm, y, aux, a->diag, a->s));
  double h2 = 0.0, alpha = 0.0;
  BSSN_TRY(launch_sum(a, a->diag, &h2));
  BSSN_CUDA_TRY(cudaMemcpyAsync(&alpha, y + (size_t)ALPHAGF * a->nt + a->idx_alpha, sizeof(double),
                                cudaMemcpyDeviceToHost, a->s));
  BSSN_CUDA_TRY(cudaStreamSynchronize(a->s));
  out[0] = h2 + alpha;
  out[1] = h2;
  out[2] = alpha;
  return BSSN_B200_OK;
}

// ybar = Jbar * dJ/dy at y.
int functional_vjp(bssn_b200_adjoint *a, const double *y, double Jbar, double *ybar) {
  griddata_struct &G = a->gd[0];
  double *aux = G.gridfuncs.auxevol_gfs;
  BSSN_TRY(launch_ricci(SPH_3D, a->g, a->rfm, y, aux, a->s));
  BSSN_TRY(launch_constraints(SPH_3D, a->g, a->rfm, y, aux, a->diag, a->s));
  BSSN_TRY(zero(a->la, a->nt * NROWS, a->s));
  BSSN_TRY(zero(a->auxbar, a->nt * NUM_AUXEVOL_GFS, a->s));
  BSSN_TRY(zero(ybar, a->nt * NUM_EVOL_GFS, a->s));
  BSSN_CUDA_TRY(cudaMemsetAsync(a->upw, 0, a->nt, a->s));
  BSSN_TRY(launch_vjp<HVjp>(a->g, a->rfm, a->pp, y, aux, a->diag, 2.0 * Jbar, a->la, a->auxbar, a->s));
  BSSN_TRY(ricci_vjps(a, y));
  BSSN_TRY(transpose(a, ybar));
  add_point_kernel<<<1, 1, 0, a->s>>>(ybar + (size_t)ALPHAGF * a->nt + a->idx_alpha, Jbar);
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

// Gradient of sum_p ybar0(p) . y0(p) with y0 = inner(extrap(BL(theta))):
// grad = (d/dm1, d/dz1, d/dm2, d/dz2). ybar0 is consumed.
int id_adjoint(bssn_b200_adjoint *a, double *ybar0, double grad[4]) {
  griddata_struct &G = a->gd[0];
  const bc_struct &bc = G.bcstruct;
  BSSN_TRY(inner_adjoint(a, ybar0));
  for (int gz = NGHOSTS - 1; gz >= 0; gz--)
    for (int dirn = 2; dirn >= 0; dirn--) {
      const int n = bc.bc_info.num_pure_outer_boundary_points[gz][dirn];
      if (n <= 0) continue;
      extrap_adjoint_kernel<<<blocks_for((long long)n * NUM_EVOL_GFS, 256), 256, 0, a->s>>>(
          a->g, bc.pure_outer_bc_array[dirn + 3 * gz], n, ybar0);
      BSSN_LAUNCH_CHECK();
    }
  const commondata_struct *cd = a->cd;
  const BLParams bl{cd->BH1_mass, cd->BH1_posn_x, cd->BH1_posn_y, cd->BH1_posn_z,
                    cd->BH2_mass, cd->BH2_posn_x, cd->BH2_posn_y, cd->BH2_posn_z};
  bl_id_vjp_kernel<<<RED_BLOCKS, RED_THREADS, 0, a->s>>>(a->g, a->rm, G.xx[0], G.xx[1], G.xx[2], bl, ybar0,
                                                         a->partials);
  BSSN_LAUNCH_CHECK();
  finish_sum_kernel<4><<<1, RED_THREADS, 0, a->s>>>(a->partials, RED_BLOCKS, a->dout);
  BSSN_LAUNCH_CHECK();
  BSSN_CUDA_TRY(cudaMemcpyAsync(grad, a->dout, 4 * sizeof(double), cudaMemcpyDeviceToHost, a->s));
  BSSN_CUDA_TRY(cudaStreamSynchronize(a->s));
  return BSSN_B200_OK;
}

int check_adjoint(const bssn_b200_adjoint *a) {
  if (!a) {
    set_error("adjoint: NULL handle");
    return BSSN_B200_EINVAL;
  }
  return BSSN_B200_OK;
}

}  // namespace
}  // namespace bssn

extern "C" {

int bssn_b200_adjoint_create(commondata_struct *cd, griddata_struct *gd, int nsteps, int checkpoint_every,
                             void *stream, bssn_b200_adjoint **out) {
  if (!cd || !gd || !out) {
    set_error("adjoint_create: NULL argument");
    return BSSN_B200_EINVAL;
  }
  *out = nullptr;
  if (cd->NUMGRIDS != 1) {
    set_error("adjoint_create: one grid only (NUMGRIDS=%d)", cd->NUMGRIDS);
    return BSSN_B200_EINVAL;
  }
  if (nsteps < 1 || checkpoint_every < 1) {
    set_error("adjoint_create: nsteps=%d and checkpoint_every=%d must be positive", nsteps, checkpoint_every);
    return BSSN_B200_EINVAL;
  }
  Variant v;
  BSSN_TRY(variant_of(&gd[0].params, &v));
  if (v != SPH_3D) {
    set_error("adjoint_create: reverse-mode kernels exist for Spherical coordinates without symmetry axes only");
    return BSSN_B200_EINVAL;
  }
  if (strncmp(cd->outer_bc_type, "radiation", 50) != 0) {
    set_error("adjoint_create: outer_bc_type must be \"radiation\"");
    return BSSN_B200_EINVAL;
  }
  const MoL_gridfunctions_struct &gf = gd[0].gridfuncs;
  if (!gf.y_n_gfs || !gf.y_nplus1_running_total_gfs || !gf.k_odd_gfs || !gf.k_even_gfs || !gf.auxevol_gfs) {
    set_error("adjoint_create: gridfunction storage not allocated (call MoL_malloc_intermediate_stage_gfs)");
    return BSSN_B200_EINVAL;
  }
  BSSN_TRY(upload_tables());
  auto *a = new bssn_b200_adjoint();
  a->cd = cd;
  a->gd = gd;
  a->nsteps = nsteps;
  a->every = checkpoint_every;
  a->nseg = (nsteps + checkpoint_every - 1) / checkpoint_every;
  a->s = (cudaStream_t)stream;
  a->g = grid_dims(&gd[0].params);
  a->rfm = rfm_arrays(gd[0].rfmstruct);
  a->pp = PhysParams{cd->eta, cd->KreissOliger_strength_gauge, cd->KreissOliger_strength_nongauge};
  int rc = radial_map(&gd[0].params, &a->rm);
  a->nt = (size_t)a->g.ntot;
  a->idx_alpha = (size_t)NGHOSTS + (size_t)a->g.s1 * (a->g.N1 / 2) + (size_t)a->g.s2 * (a->g.N2 / 2);
  const size_t n = a->nt * NUM_EVOL_GFS;
  const int every = std::min(checkpoint_every, nsteps);
  if (rc == BSSN_B200_OK) rc = adj_alloc(&a->ckpt, n * (a->nseg + 1));
  if (rc == BSSN_B200_OK) rc = adj_alloc(&a->segy, n * every);
  if (rc == BSSN_B200_OK) rc = adj_alloc(&a->stY, n * 4);
  if (rc == BSSN_B200_OK) rc = adj_alloc(&a->stZh, a->nt * 6 * 4);
  if (rc == BSSN_B200_OK) rc = adj_alloc(&a->obar, n);
  if (rc == BSSN_B200_OK) rc = adj_alloc(&a->kbar, n);
  if (rc == BSSN_B200_OK) rc = adj_alloc(&a->runbar, n);
  if (rc == BSSN_B200_OK) rc = adj_alloc(&a->ybar, n);
  if (rc == BSSN_B200_OK) rc = adj_alloc(&a->la, a->nt * NROWS);
  if (rc == BSSN_B200_OK) rc = adj_alloc(&a->auxbar, a->nt * NUM_AUXEVOL_GFS);
  if (rc == BSSN_B200_OK) rc = adj_alloc(&a->diag, a->nt * BSSN_B200_NUM_DIAG_GFS);
  if (rc == BSSN_B200_OK) rc = adj_alloc(&a->partials, 4 * RED_BLOCKS);
  if (rc == BSSN_B200_OK) rc = adj_alloc(&a->dout, 4);
  if (rc == BSSN_B200_OK && cudaMalloc(&a->upw, a->nt) != cudaSuccess) {
    set_error("adjoint: cudaMalloc of the upwind bits failed");
    rc = BSSN_B200_ENOMEM;
  }
  if (rc == BSSN_B200_OK && cudaMemsetAsync(a->upw, 0, a->nt, a->s) != cudaSuccess) {
    set_error("adjoint: cudaMemsetAsync failed");
    rc = BSSN_B200_ECUDA;
  }
  if (rc != BSSN_B200_OK) {
    adj_free(a);
    delete a;
    return rc;
  }
  *out = a;
  return BSSN_B200_OK;
}

int bssn_b200_adjoint_forward(bssn_b200_adjoint *a, double out[3]) {
  BSSN_TRY(check_adjoint(a));
  if (!out) {
    set_error("adjoint_forward: NULL output");
    return BSSN_B200_EINVAL;
  }
  griddata_struct &G = a->gd[0];
  const size_t n = a->nt * NUM_EVOL_GFS;
  a->forward_done = false;
  for (int step = 0; step < a->nsteps; step++) {
    if (step % a->every == 0) BSSN_TRY(copy_d2d(a->ckpt + (size_t)(step / a->every) * n, G.gridfuncs.y_n_gfs, n, a->s));
    BSSN_TRY(mol_step(a->cd, a->gd, 1, 0, a->s));
  }
  BSSN_TRY(copy_d2d(a->ckpt + (size_t)a->nseg * n, G.gridfuncs.y_n_gfs, n, a->s));
  BSSN_TRY(functional(a, G.gridfuncs.y_n_gfs, out));
  a->forward_done = true;
  return BSSN_B200_OK;
}

int bssn_b200_adjoint_backward(bssn_b200_adjoint *a, double Jbar, double *ybar0, double grad[4]) {
  BSSN_TRY(check_adjoint(a));
  if (!grad) {
    set_error("adjoint_backward: NULL gradient output");
    return BSSN_B200_EINVAL;
  }
  if (!a->forward_done) {
    set_error("adjoint_backward: run bssn_b200_adjoint_forward first");
    return BSSN_B200_EINVAL;
  }
  griddata_struct &G = a->gd[0];
  double *y = G.gridfuncs.y_n_gfs;
  const size_t n = a->nt * NUM_EVOL_GFS;
  const double time = a->cd->time;
  const int nn = a->cd->nn;
  BSSN_TRY(functional_vjp(a, a->ckpt + (size_t)a->nseg * n, Jbar, a->obar));
  for (int seg = a->nseg - 1; seg >= 0; seg--) {
    const int nst = std::min(a->every, a->nsteps - seg * a->every);
    BSSN_TRY(copy_d2d(y, a->ckpt + (size_t)seg * n, n, a->s));
    for (int j = 0; j < nst; j++) {
      BSSN_TRY(copy_d2d(a->segy + (size_t)j * n, y, n, a->s));
      if (j + 1 < nst) BSSN_TRY(mol_step(a->cd, a->gd, 0, 0, a->s));
    }
    for (int j = nst - 1; j >= 0; j--) BSSN_TRY(step_adjoint(a, a->segy + (size_t)j * n));
  }
  if (ybar0) BSSN_TRY(copy_d2d(ybar0, a->obar, n, a->s));
  BSSN_TRY(id_adjoint(a, a->obar, grad));
  BSSN_TRY(copy_d2d(y, a->ckpt + (size_t)a->nseg * n, n, a->s));
  BSSN_CUDA_TRY(cudaStreamSynchronize(a->s));
  a->cd->time = time;
  a->cd->nn = nn;
  return BSSN_B200_OK;
}

int bssn_b200_adjoint_functional(bssn_b200_adjoint *a, const double *y, double out[3]) {
  BSSN_TRY(check_adjoint(a));
  if (!y || !out) {
    set_error("adjoint_functional: NULL argument");
    return BSSN_B200_EINVAL;
  }
  return functional(a, y, out);
}

int bssn_b200_adjoint_functional_vjp(bssn_b200_adjoint *a, const double *y, double Jbar, double *ybar) {
  BSSN_TRY(check_adjoint(a));
  if (!y || !ybar) {
    set_error("adjoint_functional_vjp: NULL argument");
    return BSSN_B200_EINVAL;
  }
  BSSN_TRY(functional_vjp(a, y, Jbar, ybar));
  BSSN_CUDA_TRY(cudaStreamSynchronize(a->s));
  return BSSN_B200_OK;
}

int bssn_b200_adjoint_step_vjp(bssn_b200_adjoint *a, const double *y_n, double *ybar) {
  BSSN_TRY(check_adjoint(a));
  if (!y_n || !ybar) {
    set_error("adjoint_step_vjp: NULL argument");
    return BSSN_B200_EINVAL;
  }
  const size_t n = a->nt * NUM_EVOL_GFS;
  BSSN_TRY(copy_d2d(a->segy, y_n, n, a->s));
  BSSN_TRY(copy_d2d(a->obar, ybar, n, a->s));
  BSSN_TRY(step_adjoint(a, a->segy));
  BSSN_TRY(copy_d2d(ybar, a->obar, n, a->s));
  BSSN_CUDA_TRY(cudaStreamSynchronize(a->s));
  return BSSN_B200_OK;
}

int bssn_b200_adjoint_id_vjp(bssn_b200_adjoint *a, const double *ybar0, double grad[4]) {
  BSSN_TRY(check_adjoint(a));
  if (!ybar0 || !grad) {
    set_error("adjoint_id_vjp: NULL argument");
    return BSSN_B200_EINVAL;
  }
  BSSN_TRY(copy_d2d(a->obar, ybar0, a->nt * NUM_EVOL_GFS, a->s));
  return id_adjoint(a, a->obar, grad);
}

int bssn_b200_adjoint_destroy(bssn_b200_adjoint *a) {
  if (!a) return BSSN_B200_OK;
  cudaStreamSynchronize(a->s);
  adj_free(a);
  delete a;
  return BSSN_B200_OK;
}

}  // extern "C"

#else  // BSSN_B200_FD_ORDER != 4: the entry points exist and refuse

namespace {
int adjoint_unavailable() {
  bssn::set_error("the adjoint is built for 4th-order finite differences only (this library: order %d)",
                  BSSN_B200_FD_ORDER);
  return BSSN_B200_EINVAL;
}
}  // namespace

extern "C" {
int bssn_b200_adjoint_create(commondata_struct *, griddata_struct *, int, int, void *, bssn_b200_adjoint **out) {
  if (out) *out = nullptr;
  return adjoint_unavailable();
}
int bssn_b200_adjoint_forward(bssn_b200_adjoint *, double *) { return adjoint_unavailable(); }
int bssn_b200_adjoint_backward(bssn_b200_adjoint *, double, double *, double *) { return adjoint_unavailable(); }
int bssn_b200_adjoint_functional(bssn_b200_adjoint *, const double *, double *) { return adjoint_unavailable(); }
int bssn_b200_adjoint_functional_vjp(bssn_b200_adjoint *, const double *, double, double *) {
  return adjoint_unavailable();
}
int bssn_b200_adjoint_step_vjp(bssn_b200_adjoint *, const double *, double *) { return adjoint_unavailable(); }
int bssn_b200_adjoint_id_vjp(bssn_b200_adjoint *, const double *, double *) { return adjoint_unavailable(); }
int bssn_b200_adjoint_destroy(bssn_b200_adjoint *) { return BSSN_B200_OK; }
}  // extern "C"

#endif  // BSSN_B200_FD_ORDER
