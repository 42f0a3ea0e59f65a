// Diagnostics on the device: the generated project's diagnostics() family
// (infrastructures/BHaH/diagnostics/diagnostics.py:46-270 and the helpers it registers).
//
// The diagnostic gridfunctions stay on the GPU. Ricci, the constraints, lapse, W and the
// grid index are set there (diagnostic_gfs_set). The nearest-point samples (grid centre;
// lines nearest the y and z axes; planes nearest xy and yz) are gathered by one kernel into
// a compact buffer, and only that buffer crosses to the host. The volume integrals of each
// recipe are reduced on the GPU (deterministic block sums). The host writes the reference's
// file names and ASCII formats, so the output files can be compared line by line.
// What is sampled and integrated follows the generated two_blackholes_collide project:
// H and M^2 at the nearest points; H^2, M^2^2 and |Lambda|^2 over "whole_domain" and
// "sphere_R_gt_8" (points with r > 8).
#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <mutex>
#include <string>
#include <vector>

#include "bssn_common.cuh"

namespace bssn {
namespace {

constexpr int NDIAG = BSSN_B200_TOTAL_NUM_DIAG_GFS;
// Names of the diagnostic gridfunctions (the generated diagnostic_gf_names table).
const char *const kDiagNames[NDIAG] = {"DIAG_GRIDINDEX",
                                       "DIAG_HAMILTONIAN",
                                       "Covariant_conformal_connection_constraint_magnitude",
                                       "DIAG_LAPSE",
                                       "DIAG_MSQUARED",
                                       "Ricci_tensor_component_RbarDD_DIAG_RBARDD00",
                                       "Ricci_tensor_component_RbarDD_DIAG_RBARDD01",
                                       "Ricci_tensor_component_RbarDD_DIAG_RBARDD02",
                                       "Ricci_tensor_component_RbarDD_DIAG_RBARDD11",
                                       "Ricci_tensor_component_RbarDD_DIAG_RBARDD12",
                                       "Ricci_tensor_component_RbarDD_DIAG_RBARDD22",
                                       "DIAG_W"};
// Sampled at the nearest points (diagnostics_nearest.c).
constexpr int kNearestNum = 2;
const int kNearestGfs[kNearestNum] = {BSSN_B200_DIAG_HAMILTONIANGF, BSSN_B200_DIAG_MSQUAREDGF};

// Volume-integration recipes (diagnostics_volume_integration.c): spherical exclusion rules
// and squared integrands.
constexpr int kMaxRecipes = 2, kMaxRules = 1, kNumIntegrands = 3;
struct Recipes {
  int n;
  int nrules[kMaxRecipes];
  double cx[kMaxRecipes][kMaxRules], cy[kMaxRecipes][kMaxRules], cz[kMaxRecipes][kMaxRules];
  double radius[kMaxRecipes][kMaxRules];
  int exclude_inside[kMaxRecipes][kMaxRules];
  int gf[kNumIntegrands];
};
const char *const kRecipeNames[kMaxRecipes] = {"whole_domain", "sphere_R_gt_8"};
Recipes default_recipes() {
  Recipes r{};
  r.n = 2;
  r.nrules[0] = 0;
  r.nrules[1] = 1;
  r.cx[1][0] = r.cy[1][0] = r.cz[1][0] = 0.0;
  r.radius[1][0] = 8.0;
  r.exclude_inside[1][0] = 1;
  r.gf[0] = BSSN_B200_DIAG_HAMILTONIANGF;
  r.gf[1] = BSSN_B200_DIAG_MSQUAREDGF;
  r.gf[2] = BSSN_B200_DIAG_LAMBDA_CONSTRAINTGF;
  return r;
}

// Cartesian position and proper volume element of a cell (xx_to_Cart, sqrt_detgammahat_d3xx_volume_element),
// with the expression trees of the generated functions so that coordinates agree to the last bit.
enum CoordKind { KIND_SPHERICAL = 0, KIND_SINHSPHERICAL = 1, KIND_SINHCYLINDRICAL = 2 };
struct CoordMap {
  int kind;
  double AMPL, SINHW, ox, oy, oz, dxx0, dxx1, dxx2;
  double AMPLRHO, SINHWRHO, AMPLZ, SINHWZ;
  __host__ __device__ void to_cart(double xx0, double xx1, double xx2, double out[3]) const {
    if (kind == KIND_SINHCYLINDRICAL) {
      const double t0 = 1.0 / SINHWRHO, t3 = 1.0 / SINHWZ;
      const double rho = AMPLRHO * (exp(t0 * xx0) - exp(-t0 * xx0)) / (exp(t0) - exp(-t0));
      out[0] = ox + rho * cos(xx1);
      out[1] = oy + rho * sin(xx1);
      out[2] = AMPLZ * (exp(t3 * xx2) - exp(-t3 * xx2)) / (exp(t3) - exp(-t3)) + oz;
      return;
    }
    const int sinh = kind == KIND_SINHSPHERICAL;
    double rr;
    if (sinh) {
      const double t0 = 1.0 / SINHW;
      rr = AMPL * (exp(t0 * xx0) - exp(-t0 * xx0)) / (exp(t0) - exp(-t0));
    } else {
      rr = xx0;
    }
    const double t = rr * sin(xx1);
    out[0] = ox + t * cos(xx2);
    out[1] = oy + t * sin(xx2);
    out[2] = oz + rr * cos(xx1);
  }
  __device__ double dV(double xx0, double xx1, double xx2) const {
    const double d3 = fabs(dxx0 * dxx1 * dxx2);
    if (kind == KIND_SINHCYLINDRICAL) {
      // |rho'(xx0) rho(xx0) z'(xx2)| written as the generated square root of its square
      const double t0 = 2.0 / SINHWRHO, t2 = 1.0 / SINHWZ;
      const double t1 = exp(t0 * xx0);
      const double a = 1.0 - t1, b = t1 + 1.0, e2 = exp(2.0 * t2 * xx2) + 1.0;
      const double c0 = 1.0 - exp(t0), c2 = 1.0 - exp(2.0 * t2);
      return AMPLRHO * AMPLRHO *
             sqrt(a * a * (b * b) * (e2 * e2) *
                  exp(t0 * t2 * (-SINHWRHO * xx2 + SINHWRHO - 2.0 * SINHWZ * xx0 + 2.0 * SINHWZ)) /
                  (SINHWRHO * SINHWRHO * (SINHWZ * SINHWZ) * (c0 * c0 * c0 * c0) * (c2 * c2))) *
             fabs(AMPLZ) * d3;
    }
    const double s1 = sin(xx1);
    if (kind == KIND_SPHERICAL) return sqrt(xx0 * xx0 * xx0 * xx0 * (s1 * s1)) * d3;
    const double t0 = 1.0 / SINHW;
    const double t2 = exp(2.0 * t0 * xx0);
    const double a = 1.0 - t2, b = t2 + 1.0, c = 1.0 - exp(2.0 * t0);
    const double c6 = c * c * c * c * c * c;
    return AMPL * AMPL * sqrt(a * a * a * a * (b * b) * exp(6.0 * t0 * (1.0 - xx0)) * (s1 * s1) / (SINHW * SINHW * c6)) *
           fabs(AMPL) * d3;
  }
};

int coord_map(const params_struct *p, CoordMap *m) {
  int kind;
  if (p->CoordSystem_hash == SPHERICAL) kind = KIND_SPHERICAL;
  else if (p->CoordSystem_hash == SINHSPHERICAL) kind = KIND_SINHSPHERICAL;
  else if (p->CoordSystem_hash == SINHCYLINDRICAL) kind = KIND_SINHCYLINDRICAL;
  else {
    set_error("diagnostics: CoordSystem_hash %d not supported", p->CoordSystem_hash);
    return BSSN_B200_EINVAL;
  }
  *m = CoordMap{kind,           p->AMPL,         p->SINHW,      p->Cart_originx, p->Cart_originy,
                p->Cart_originz, p->dxx0,        p->dxx1,       p->dxx2,         p->AMPLRHO,
                p->SINHWRHO,     p->AMPLZ,       p->SINHWZ};
  return BSSN_B200_OK;
}

// lapse, W, grid index and Rbar_ij into the diagnostic array (every point).
__global__ void diag_fill_kernel(const int ntot, const double *__restrict__ y, const double *__restrict__ aux,
                                 double *__restrict__ diag, const double grid) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ntot) return;
  const size_t n = (size_t)ntot;
  diag[BSSN_B200_DIAG_LAPSEGF * n + i] = y[ALPHAGF * n + i];
  diag[BSSN_B200_DIAG_WGF * n + i] = y[CFGF * n + i];
  diag[BSSN_B200_DIAG_GRIDINDEXGF * n + i] = grid;
#pragma unroll
  for (int k = 0; k < 6; k++) diag[(BSSN_B200_DIAG_RBARDD00GF + k) * n + i] = aux[k * n + i];
}

// out[j * n + i] = diag[gf_j][idx[i]] for the sampled gridfunctions gf_0 = gfs.x, gf_1 = gfs.y.
__global__ void gather_kernel(const double *__restrict__ diag, const size_t ntot, const int *__restrict__ idx,
                              const int n, const int2 gfs, double *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t p = (size_t)idx[i];
  out[i] = diag[(size_t)gfs.x * ntot + p];
  out[(size_t)n + i] = diag[(size_t)gfs.y * ntot + p];
}

constexpr int RED_BLOCKS = 296, RED_THREADS = 256;
constexpr int NACC = kMaxRecipes * (1 + kNumIntegrands);

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

// Per block: for each recipe, the kept proper volume and the integrals of f^2 dV.
__global__ void integrate_kernel(const GridDims g, const CoordMap cm, const double *__restrict__ xx0,
                                 const double *__restrict__ xx1, const double *__restrict__ xx2,
                                 const double *__restrict__ diag, const Recipes rc, double *__restrict__ partials) {
  const int n0 = g.N0 - 2 * NGHOSTS, n1 = g.N1 - 2 * NGHOSTS, n2 = g.N2 - 2 * NGHOSTS;
  const long long n = (long long)n0 * n1 * n2;
  double acc[NACC];
#pragma unroll
  for (int k = 0; k < NACC; k++) acc[k] = 0.0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i0 = (int)(t % n0) + NGHOSTS;
    const long long r = t / n0;
    const int i1 = (int)(r % n1) + NGHOSTS, i2 = (int)(r / n1) + NGHOSTS;
    const double a0 = xx0[i0], a1 = xx1[i1], a2 = xx2[i2];
    const double dV = cm.dV(a0, a1, a2);
    if (dV == 0.0) continue;
    double X[3];
    cm.to_cart(a0, a1, a2, X);
    const size_t idx = (size_t)i0 + (size_t)g.s1 * i1 + (size_t)g.s2 * i2;
    double f2[kNumIntegrands];
#pragma unroll
    for (int k = 0; k < kNumIntegrands; k++) {
      const double f = diag[(size_t)rc.gf[k] * g.ntot + idx];
      f2[k] = f * f;
    }
#pragma unroll
    for (int q = 0; q < kMaxRecipes; q++) {
      if (q >= rc.n) break;
      bool excluded = false;
      for (int u = 0; u < rc.nrules[q]; u++) {
        const double dx = X[0] - rc.cx[q][u], dy = X[1] - rc.cy[q][u], dz = X[2] - rc.cz[q][u];
        const double rr = sqrt(dx * dx + dy * dy + dz * dz);
        excluded |= rc.exclude_inside[q][u] ? (rr <= rc.radius[q][u]) : (rr > rc.radius[q][u]);
      }
      if (excluded) continue;
      acc[q * (1 + kNumIntegrands)] += dV;
#pragma unroll
      for (int k = 0; k < kNumIntegrands; k++) acc[q * (1 + kNumIntegrands) + 1 + k] += f2[k] * dV;
    }
  }
  block_sum<NACC>(acc, partials + (size_t)NACC * blockIdx.x);
}

__global__ void finish_kernel(const double *__restrict__ partials, const int nblocks, double *__restrict__ out) {
  double v[NACC];
#pragma unroll
  for (int k = 0; k < NACC; k++) v[k] = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
    for (int k = 0; k < NACC; k++) v[k] += partials[NACC * b + k];
  block_sum<NACC>(v, out);
}

// Library-held device buffers (grow-only): gather indices and samples, reduction partials,
// and one diagnostic array per grid for the diagnostics() driver.
struct Scratch {
  int *idx = nullptr;
  double *samples = nullptr;
  size_t cap = 0;
  double *partials = nullptr;
  double *diag[MAXNUMGRIDS] = {nullptr};
  size_t diag_n[MAXNUMGRIDS] = {0};
};
std::mutex g_mu;
Scratch g_scratch;

int ensure_samples(size_t n) {
  if (g_scratch.cap >= n) return BSSN_B200_OK;
  cudaFree(g_scratch.idx);
  cudaFree(g_scratch.samples);
  g_scratch.idx = nullptr;
  g_scratch.samples = nullptr;
  g_scratch.cap = 0;
  BSSN_CUDA_TRY(cudaMalloc(&g_scratch.idx, n * sizeof(int)));
  BSSN_CUDA_TRY(cudaMalloc(&g_scratch.samples, n * kNearestNum * sizeof(double)));
  g_scratch.cap = n;
  return BSSN_B200_OK;
}

int host_xx(const params_struct *p, REAL *const xx[3], std::vector<double> h[3]) {
  const int N[3] = {p->Nxx_plus_2NGHOSTS0, p->Nxx_plus_2NGHOSTS1, p->Nxx_plus_2NGHOSTS2};
  for (int d = 0; d < 3; d++) {
    if (!xx[d]) {
      set_error("diagnostics: xx[%d] is NULL", d);
      return BSSN_B200_EINVAL;
    }
    h[d].resize(N[d]);
    BSSN_CUDA_TRY(cudaMemcpy(h[d].data(), xx[d], N[d] * sizeof(double), cudaMemcpyDeviceToHost));
  }
  return BSSN_B200_OK;
}

// ---------------------------------------------------------------- the reference's text formats
FILE *open_out(const char *prefix, const char *coordsys, const commondata_struct *cd, bool with_time) {
  char name[256];
  if (with_time)
    snprintf(name, sizeof name, "%s-%s-conv_factor%.2f-t%08.2f.txt", prefix, coordsys, cd->convergence_factor,
             cd->time);
  else
    snprintf(name, sizeof name, "%s-%s-conv_factor-%.2f.txt", prefix, coordsys, cd->convergence_factor);
  FILE *f = fopen(name, cd->nn == 0 ? "w" : "a");
  if (!f) set_error("diagnostics: cannot open %s for writing", name);
  return f;
}

void write_header(FILE *f, const char *coord_names) {
  int spaces = 0;
  for (const char *c = coord_names; *c; ++c) spaces += (*c == ' ');
  fprintf(f, "# %s", coord_names);
  for (int k = 0; k < kNearestNum; k++) fprintf(f, " %s(%d)", kDiagNames[kNearestGfs[k]], k + spaces + 2);
  fprintf(f, "\n");
}

// One row "%.15e %.15e ...\n" appended to a buffer (std::to_chars gives the same digits as
// printf's %.15e, correctly rounded, and runs several times faster).
void append_row(std::string &buf, int ncols, const double *v) {
  char tmp[40];
  for (int k = 0; k < ncols; k++) {
    if (k) buf.push_back(' ');
    const auto r = std::to_chars(tmp, tmp + sizeof tmp, v[k], std::chars_format::scientific, 15);
    buf.append(tmp, r.ptr);
  }
  buf.push_back('\n');
}

void write_row(FILE *f, int ncols, const double *v) {
  std::string b;
  append_row(b, ncols, v);
  fwrite(b.data(), 1, b.size(), f);
}

std::string rule_name(const Recipes &rc, int q, int u) {
  char b[256];
  snprintf(b, sizeof b, rc.exclude_inside[q][u] ? "KeepOutside_r>%.17g_at(%.17g,%.17g,%.17g)"
                                                : "KeepInside_r<=%.17g_at(%.17g,%.17g,%.17g)",
           rc.radius[q][u], rc.cx[q][u], rc.cy[q][u], rc.cz[q][u]);
  return b;
}

void write_integration_header(FILE *f, const Recipes &rc, int q) {
  fprintf(f, "# diagnostics_integration: column mapping & rule documentation\n");
  fprintf(f, "# recipe_index : %d\n", q);
  fprintf(f, "# recipe_name  : %s\n", kRecipeNames[q]);
  fprintf(f, "# row semantics: only the *full* rules-applied row is emitted (k = num_rules)\n");
  if (rc.nrules[q] > 0) {
    for (int u = 0; u < rc.nrules[q]; u++)
      fprintf(f, "#   rule[%d] name=\"%s\" : center=(%.17g, %.17g, %.17g), radius=%.17g, action=%s\n", u,
              rule_name(rc, q, u).c_str(), rc.cx[q][u], rc.cy[q][u], rc.cz[q][u], rc.radius[q][u],
              rc.exclude_inside[q][u] ? "exclude INSIDE (keep OUTSIDE: r > radius)"
                                      : "exclude OUTSIDE (keep INSIDE: r <= radius)");
  } else {
    fprintf(f, "#   (no rules; the entire computational domain is used)\n");
  }
  int col = 1;
  fprintf(f, "#   %3d: time                    (current simulation time; commondata->time)\n", col++);
  fprintf(f, "#   %3d: remaining_volume        (proper volume after applying the prefix rules)\n", col++);
  std::string compact = "# COLUMNS: time remaining_volume", legacy = "# time remaining_volume";
  for (int k = 0; k < kNumIntegrands; k++) {
    const char *nm = kDiagNames[rc.gf[k]];
    fprintf(f, "#   %3d: INT[prefix:%s^2]      (integral of (%s)^2 dV)\n", col++, nm, nm);
    compact += std::string(" INT[prefix:") + nm + "^2]";
    legacy += std::string(" INT[prefix:") + nm + "^2]";
    fprintf(f, "#   %3d: L2[prefix:%s]         (sqrt( max( INT[prefix:%s^2], 0 ) ))\n", col++, nm, nm);
    fprintf(f,
            "#   %3d: RMS[prefix:%s]        ((remaining_volume>0) ? sqrt( max( INT[prefix:%s^2], 0 ) / "
            "remaining_volume ) : 0)\n",
            col++, nm, nm);
    const std::string l2rms = std::string(" L2[prefix:") + nm + "] RMS[prefix:" + nm + "]";
    compact += l2rms;
    legacy += l2rms;
  }
  fprintf(f, "# --- Prefix mapping (how to interpret \"prefix:\" per row) ----------------------\n");
  fprintf(f, "#   For a row with rules_applied = k, substitute:\n");
  fprintf(f, "#     k = 0 : prefix = p0\n");
  for (int k0 = 1; k0 <= rc.nrules[q]; k0++)
    fprintf(f, "#     k = %d : prefix = p%d|rule[%d]:%s\n", k0, k0, k0 - 1, rule_name(rc, q, k0 - 1).c_str());
  fprintf(f, "%s\n", compact.c_str());
  fprintf(f, "%s\n", legacy.c_str());
}

struct Sample {
  double c0, c1;  // coordinates written before the values
  int idx;
};

// ---------------------------------------------------------------- the three drop-ins
int diag_set(const commondata_struct *cd, const griddata_struct *gd, REAL *const diags[], cudaStream_t s) {
  for (int grid = 0; grid < cd->NUMGRIDS; grid++) {
    const griddata_struct &G = gd[grid];
    const params_struct *p = &G.params;
    if (!diags[grid] || !G.gridfuncs.y_n_gfs || !G.gridfuncs.auxevol_gfs || !G.rfmstruct) {
      set_error("diagnostic_gfs_set: grid %d: NULL diagnostic array, state or rfm", grid);
      return BSSN_B200_EINVAL;
    }
    Variant v;
    BSSN_TRY(variant_of(p, &v));
    const GridDims g = grid_dims(p);
    const RfmArrays rfm = rfm_arrays(G.rfmstruct);
    static const int slots[3] = {BSSN_B200_DIAG_HAMILTONIANGF, BSSN_B200_DIAG_MSQUAREDGF,
                                 BSSN_B200_DIAG_LAMBDA_CONSTRAINTGF};
    BSSN_TRY(launch_ricci(v, g, rfm, G.gridfuncs.y_n_gfs, G.gridfuncs.auxevol_gfs, s));
    BSSN_TRY(launch_constraints(v, g, rfm, G.gridfuncs.y_n_gfs, G.gridfuncs.auxevol_gfs, diags[grid], s, slots));
    diag_fill_kernel<<<(g.ntot + 255) / 256, 256, 0, s>>>(g.ntot, G.gridfuncs.y_n_gfs, G.gridfuncs.auxevol_gfs,
                                                         diags[grid], (double)grid);
    BSSN_LAUNCH_CHECK();
  }
  return BSSN_B200_OK;
}

int nearest(const commondata_struct *cd, const griddata_struct *gd, const REAL *const diags[], cudaStream_t s) {
  for (int grid = 0; grid < cd->NUMGRIDS; grid++) {
    const griddata_struct &G = gd[grid];
    const params_struct *p = &G.params;
    if (!diags[grid]) {
      set_error("diagnostics_nearest: grid %d: NULL diagnostic array", grid);
      return BSSN_B200_EINVAL;
    }
    CoordMap cm;
    BSSN_TRY(coord_map(p, &cm));
    std::vector<double> hx[3];
    BSSN_TRY(host_xx(p, G.xx, hx));
    const int N0 = p->Nxx_plus_2NGHOSTS0, N1 = p->Nxx_plus_2NGHOSTS1, N2 = p->Nxx_plus_2NGHOSTS2;
    const int N0int = N0 - 2 * NGHOSTS, N1int = N1 - 2 * NGHOSTS, N2int = N2 - 2 * NGHOSTS;
    auto IDX = [&](int i0, int i1, int i2) { return i0 + N0 * (i1 + N1 * i2); };
    const int i1_mid = N1 / 2, i2_mid = N2 / 2;
    const int i1_max = N1 - NGHOSTS - 1;
    const int i2_q1 = (int)(NGHOSTS + 0.25 * (double)N2int - 0.5), i2_q3 = (int)(NGHOSTS + 0.75 * (double)N2int - 0.5);
    const int i1_q1 = (int)(NGHOSTS + 0.25 * (double)N1int - 0.5), i1_q3 = (int)(NGHOSTS + 0.75 * (double)N1int - 0.5);
    auto cart = [&](int i0, int i1, int i2, double X[3]) { cm.to_cart(hx[0][i0], hx[1][i1], hx[2][i2], X); };
    // Sample lists in the reference's order (lines sorted by their coordinate). Spherical
    // family: y lines at the equator and phi ~ +-pi/2, z lines at the two poles, the xy plane
    // at the equator, the yz plane at phi ~ +-pi/2. Cylindrical family: y lines at phi ~ +-pi/2
    // in the z mid-plane, the z line along the axis (innermost rho), the xy plane at mid z, the
    // yz plane at phi ~ +-pi/2 (diagnostics_nearest_1d_y_and_z_axes.py:76-200,
    // diagnostics_nearest_2d_xy_and_yz_planes.py:67-140).
    std::vector<Sample> ys, zs, xy, yz;
    double X[3];
    const bool cylf = cm.kind == KIND_SINHCYLINDRICAL;
    if (cylf) {
      for (int i1 : {i1_q1, i1_q3})
        for (int i0 = NGHOSTS; i0 < N0 - NGHOSTS; i0++) {
          cart(i0, i1, i2_mid, X);
          ys.push_back({X[1], 0.0, IDX(i0, i1, i2_mid)});
        }
      for (int i2 = NGHOSTS; i2 < N2 - NGHOSTS; i2++) {
        cart(NGHOSTS, NGHOSTS, i2, X);
        zs.push_back({X[2], 0.0, IDX(NGHOSTS, NGHOSTS, i2)});
      }
    } else {
      for (int i2 : {i2_q1, i2_q3})
        for (int i0 = NGHOSTS; i0 < N0 - NGHOSTS; i0++) {
          cart(i0, i1_mid, i2, X);
          ys.push_back({X[1], 0.0, IDX(i0, i1_mid, i2)});
        }
      for (int i1 : {NGHOSTS, i1_max})
        for (int i0 = NGHOSTS; i0 < N0 - NGHOSTS; i0++) {
          cart(i0, i1, NGHOSTS, X);
          zs.push_back({X[2], 0.0, IDX(i0, i1, NGHOSTS)});
        }
    }
    auto by_coord = [](const Sample &a, const Sample &b) { return a.c0 < b.c0; };
    std::stable_sort(ys.begin(), ys.end(), by_coord);
    std::stable_sort(zs.begin(), zs.end(), by_coord);
    if (cylf) {
      for (int i1 = NGHOSTS; i1 < N1 - NGHOSTS; i1++)
        for (int i0 = NGHOSTS; i0 < N0 - NGHOSTS; i0++) {
          cart(i0, i1, i2_mid, X);
          xy.push_back({X[0], X[1], IDX(i0, i1, i2_mid)});
        }
      for (int i1 : {i1_q1, i1_q3})
        for (int i2 = NGHOSTS; i2 < N2 - NGHOSTS; i2++)
          for (int i0 = NGHOSTS; i0 < N0 - NGHOSTS; i0++) {
            cart(i0, i1, i2, X);
            yz.push_back({X[1], X[2], IDX(i0, i1, i2)});
          }
    } else {
      for (int i2 = NGHOSTS; i2 < N2 - NGHOSTS; i2++)
        for (int i0 = NGHOSTS; i0 < N0 - NGHOSTS; i0++) {
          cart(i0, i1_mid, i2, X);
          xy.push_back({X[0], X[1], IDX(i0, i1_mid, i2)});
        }
      for (int i2 : {i2_q1, i2_q3})
        for (int i1 = NGHOSTS; i1 < N1 - NGHOSTS; i1++)
          for (int i0 = NGHOSTS; i0 < N0 - NGHOSTS; i0++) {
            cart(i0, i1, i2, X);
            yz.push_back({X[1], X[2], IDX(i0, i1, i2)});
          }
    }
    (void)N0int;
    // one gather of every sample
    std::vector<int> idx;
    idx.push_back(IDX(NGHOSTS, i1_mid, i2_mid));
    for (auto *v : {&ys, &zs, &xy, &yz})
      for (const Sample &q : *v) idx.push_back(q.idx);
    const int n = (int)idx.size();
    std::vector<double> vals((size_t)n * kNearestNum);
    {
      std::lock_guard<std::mutex> lk(g_mu);
      BSSN_TRY(ensure_samples(n));
      BSSN_CUDA_TRY(cudaMemcpyAsync(g_scratch.idx, idx.data(), n * sizeof(int), cudaMemcpyHostToDevice, s));
      static_assert(kNearestNum == 2, "two sampled gridfunctions");
      gather_kernel<<<(n + 255) / 256, 256, 0, s>>>(diags[grid], (size_t)N0 * N1 * N2, g_scratch.idx, n,
                                                    make_int2(kNearestGfs[0], kNearestGfs[1]), g_scratch.samples);
      BSSN_LAUNCH_CHECK();
      BSSN_CUDA_TRY(cudaMemcpyAsync(vals.data(), g_scratch.samples, vals.size() * sizeof(double),
                                    cudaMemcpyDeviceToHost, s));
      BSSN_CUDA_TRY(cudaStreamSynchronize(s));
    }
    auto val = [&](int i, int j) { return vals[(size_t)j * n + i]; };
    // 0-D: appended row per output step
    char cs[160];
    snprintf(cs, sizeof cs, "grid%02d-%s", grid, p->CoordSystemName);
    FILE *f = open_out("out0d", cs, cd, false);
    if (!f) return BSSN_B200_EINVAL;
    if (cd->nn == 0) {
      fprintf(f, "# %s", "time");
      for (int k = 0; k < kNearestNum; k++) fprintf(f, " %s(%d)", kDiagNames[kNearestGfs[k]], k + 2);
      fprintf(f, "\n");
    }
    {
      const double row[3] = {cd->time, val(0, 0), val(0, 1)};
      write_row(f, 1 + kNearestNum, row);
    }
    fclose(f);
    // 1-D and 2-D: one file per output time
    snprintf(cs, sizeof cs, "%s-grid%02d", p->CoordSystemName, grid);
    int at = 1;
    for (int line = 0; line < 2; line++) {
      const std::vector<Sample> &v = line == 0 ? ys : zs;
      FILE *o = open_out(line == 0 ? "out1d-y" : "out1d-z", cs, cd, true);
      if (!o) return BSSN_B200_EINVAL;
      fprintf(o, "# [time] = %.15e\n", cd->time);
      write_header(o, line == 0 ? "y" : "z");
      std::string buf;
      buf.reserve(v.size() * 72);
      for (size_t q = 0; q < v.size(); q++, at++) {
        const double row[3] = {v[q].c0, val(at, 0), val(at, 1)};
        append_row(buf, 1 + kNearestNum, row);
      }
      fwrite(buf.data(), 1, buf.size(), o);
      fclose(o);
    }
    for (int plane = 0; plane < 2; plane++) {
      const std::vector<Sample> &v = plane == 0 ? xy : yz;
      FILE *o = open_out(plane == 0 ? "out2d-xy" : "out2d-yz", cs, cd, true);
      if (!o) return BSSN_B200_EINVAL;
      fprintf(o, "# [time] = %.15e\n", cd->time);
      write_header(o, plane == 0 ? "x y" : "y z");
      std::string buf;
      buf.reserve(v.size() * 96);
      for (size_t q = 0; q < v.size(); q++, at++) {
        const double row[4] = {v[q].c0, v[q].c1, val(at, 0), val(at, 1)};
        append_row(buf, 2 + kNearestNum, row);
      }
      fwrite(buf.data(), 1, buf.size(), o);
      fclose(o);
    }
  }
  return BSSN_B200_OK;
}

int volume_integration(const commondata_struct *cd, const griddata_struct *gd, const REAL *const diags[],
                       cudaStream_t s) {
  const Recipes rc = default_recipes();
  double tot[NACC] = {0.0};
  for (int grid = 0; grid < cd->NUMGRIDS; grid++) {
    const griddata_struct &G = gd[grid];
    const params_struct *p = &G.params;
    if (!diags[grid]) {
      set_error("diagnostics_volume_integration: grid %d: NULL diagnostic array", grid);
      return BSSN_B200_EINVAL;
    }
    CoordMap cm;
    BSSN_TRY(coord_map(p, &cm));
    double out[NACC];
    {
      std::lock_guard<std::mutex> lk(g_mu);
      if (!g_scratch.partials)
        BSSN_CUDA_TRY(cudaMalloc(&g_scratch.partials, (size_t)(RED_BLOCKS + 1) * NACC * sizeof(double)));
      double *fin = g_scratch.partials + (size_t)RED_BLOCKS * NACC;
      integrate_kernel<<<RED_BLOCKS, RED_THREADS, 0, s>>>(grid_dims(p), cm, G.xx[0], G.xx[1], G.xx[2], diags[grid],
                                                          rc, g_scratch.partials);
      BSSN_LAUNCH_CHECK();
      finish_kernel<<<1, RED_THREADS, 0, s>>>(g_scratch.partials, RED_BLOCKS, fin);
      BSSN_LAUNCH_CHECK();
      BSSN_CUDA_TRY(cudaMemcpyAsync(out, fin, sizeof out, cudaMemcpyDeviceToHost, s));
      BSSN_CUDA_TRY(cudaStreamSynchronize(s));
    }
    for (int k = 0; k < NACC; k++) tot[k] += out[k];
  }
  for (int q = 0; q < rc.n; q++) {
    char name[256];
    snprintf(name, sizeof name, "out3d-integrals-conv_factor%.2f-%s.txt", cd->convergence_factor, kRecipeNames[q]);
    FILE *f = fopen(name, cd->nn == 0 ? "w" : "a");
    if (!f) {
      set_error("diagnostics_volume_integration: cannot open %s", name);
      return BSSN_B200_EINVAL;
    }
    if (cd->nn == 0) write_integration_header(f, rc, q);
    const double vol = tot[q * (1 + kNumIntegrands)];
    fprintf(f, "%.15e %.15e", cd->time, vol);
    for (int k = 0; k < kNumIntegrands; k++) {
      const double I = tot[q * (1 + kNumIntegrands) + 1 + k];
      fprintf(f, " %.15e", I);
      fprintf(f, " %.15e %.15e", sqrt(fmax(I, 0.0)), vol > 0.0 ? sqrt(fmax(I, 0.0) / vol) : 0.0);
    }
    fprintf(f, "\n");
    fclose(f);
  }
  return BSSN_B200_OK;
}

void progress(commondata_struct *cd) {
  if (cd->nn == cd->nn_0) clock_gettime(CLOCK_REALTIME, &cd->start_wallclock_time);
  if (!(cd->output_progress_every > 0 && cd->nn % cd->output_progress_every == 0)) return;
  struct timespec now;
  clock_gettime(CLOCK_REALTIME, &now);
  const double ns = (double)(1000000000L * (now.tv_sec - cd->start_wallclock_time.tv_sec) + now.tv_nsec -
                             cd->start_wallclock_time.tv_nsec);
  const double per_sec = (cd->time - cd->t_0) / (ns / 1e9);
  const double remaining = (int)((cd->t_final - cd->time) / per_sec);
  int hrs = (int)(remaining / 3600.0), mins = (int)(remaining / 60.0) % 60;
  int secs = (int)remaining - mins * 60 - hrs * 3600;
  if (cd->nn == 0) hrs = mins = secs = 0;
  fprintf(stderr, "%c[2K", 27);
  fprintf(stderr, "It: %d t=%.3f / %.1f = %.2f%% dt=1/%.1f | t/h=%.2f ETA %dh%02dm%02ds\r", cd->nn, cd->time,
          cd->t_final, 100.0 * cd->time / cd->t_final, 1.0 / cd->dt, per_sec * 3600.0, hrs, mins, secs);
  fflush(stderr);
  if (cd->time + cd->dt > cd->t_final) fprintf(stderr, "\n");
}

int run_diagnostics(commondata_struct *cd, griddata_struct *gd, cudaStream_t s) {
  if (!cd || !gd) {
    set_error("diagnostics: NULL argument");
    return BSSN_B200_EINVAL;
  }
  if (cd->NUMGRIDS < 1 || cd->NUMGRIDS > MAXNUMGRIDS) {
    set_error("diagnostics: NUMGRIDS=%d out of range", cd->NUMGRIDS);
    return BSSN_B200_EINVAL;
  }
  const double t = cd->time, dt = cd->dt, every = cd->diagnostics_output_every;
  if (every > 0.0 && fabs(round(t / every) * every - t) < 0.5 * dt) {
    REAL *diags[MAXNUMGRIDS] = {nullptr};
    {
      std::lock_guard<std::mutex> lk(g_mu);
      for (int grid = 0; grid < cd->NUMGRIDS; grid++) {
        const params_struct *p = &gd[grid].params;
        const size_t n = (size_t)NDIAG * p->Nxx_plus_2NGHOSTS0 * p->Nxx_plus_2NGHOSTS1 * p->Nxx_plus_2NGHOSTS2;
        if (g_scratch.diag_n[grid] < n) {
          cudaFree(g_scratch.diag[grid]);
          g_scratch.diag[grid] = nullptr;
          g_scratch.diag_n[grid] = 0;
          BSSN_CUDA_TRY(cudaMalloc(&g_scratch.diag[grid], n * sizeof(double)));
          g_scratch.diag_n[grid] = n;
        }
        diags[grid] = g_scratch.diag[grid];
      }
    }
    BSSN_TRY(diag_set(cd, gd, diags, s));
    BSSN_TRY(nearest(cd, gd, diags, s));
    BSSN_TRY(volume_integration(cd, gd, diags, s));
  }
  progress(cd);
  return BSSN_B200_OK;
}

int null_args(const char *fn) {
  set_error("%s: NULL argument", fn);
  return BSSN_B200_EINVAL;
}

void die_if(int rc, const char *fn) {
  if (rc != BSSN_B200_OK) {
    fprintf(stderr, "%s: %s\n", fn, last_error());
    exit(1);
  }
}

}  // namespace
}  // namespace bssn

using namespace bssn;

extern "C" {

void diagnostics(commondata_struct *commondata, griddata_struct *griddata) {
  die_if(run_diagnostics(commondata, griddata, nullptr), __func__);
}

void diagnostic_gfs_set(const commondata_struct *commondata, const griddata_struct *griddata,
                        REAL *diagnostic_gfs[MAXNUMGRIDS]) {
  if (!commondata || !griddata || !diagnostic_gfs) die_if(null_args(__func__), __func__);
  die_if(diag_set(commondata, griddata, diagnostic_gfs, nullptr), __func__);
}

void diagnostics_nearest(commondata_struct *commondata, griddata_struct *griddata,
                         const REAL *diagnostic_gfs[MAXNUMGRIDS]) {
  if (!commondata || !griddata || !diagnostic_gfs) die_if(null_args(__func__), __func__);
  die_if(nearest(commondata, griddata, diagnostic_gfs, nullptr), __func__);
}

void diagnostics_volume_integration(commondata_struct *commondata, griddata_struct *griddata,
                                    const REAL *diagnostic_gfs[MAXNUMGRIDS]) {
  if (!commondata || !griddata || !diagnostic_gfs) die_if(null_args(__func__), __func__);
  die_if(volume_integration(commondata, griddata, diagnostic_gfs, nullptr), __func__);
}

void progress_indicator(commondata_struct *commondata, const griddata_struct *griddata) {
  (void)griddata;
  if (commondata) progress(commondata);
}

int bssn_b200_diagnostics(commondata_struct *commondata, griddata_struct *griddata, void *stream) {
  return run_diagnostics(commondata, griddata, (cudaStream_t)stream);
}

}  // extern "C"
