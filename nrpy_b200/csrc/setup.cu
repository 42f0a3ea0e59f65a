// Grid, reference-metric, boundary-structure, timestep and initial-data set-up.
//
// Set-up runs once per grid, on the host, in FP64 with the same closed-form expressions
// as the reference's generated set-up code, and uploads its results. The hot path never
// calls into this file.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "bssn_common.cuh"

namespace bssn {

static const double kPI = 3.14159265358979323846264338327950288;

// ---------------------------------------------------------------- defaults
// CodeParameters.py: commondata/params_struct_set_to_default (values of the generated project).
void commondata_defaults(commondata_struct *cd) {
  memset(cd, 0, sizeof(*cd));
  cd->BH1_mass = 0.5;
  cd->BH1_posn_x = 0.0;
  cd->BH1_posn_y = 0.0;
  cd->BH1_posn_z = 0.5;
  cd->BH2_mass = 0.5;
  cd->BH2_posn_x = 0.0;
  cd->BH2_posn_y = 0.0;
  cd->BH2_posn_z = -0.5;
  cd->CFL_FACTOR = 0.5;
  cd->KreissOliger_strength_gauge = 0.3;
  cd->KreissOliger_strength_nongauge = 0.3;
  cd->NUMGRIDS = 1;
  cd->convergence_factor = 1.0;
  cd->diagnostics_output_every = 0.25;
  cd->eta = 1.0;
  cd->output_progress_every = 1;
  cd->t_final = 10.0;
  snprintf(cd->outer_bc_type, 50, "radiation");
}

void params_defaults(params_struct *p) {
  memset(p, 0, sizeof(*p));
  p->AMPL = 10.0;
  p->AMPLRHO = 10.0;
  p->AMPLZ = 10.0;
  p->Cart_originx = p->Cart_originy = p->Cart_originz = 0.0;
  p->Nxx0 = p->Nxx1 = p->Nxx2 = 64;
  p->PI = kPI;
  p->RHOMAX = 10.0;
  p->RMAX = 10.0;
  p->SINHW = 0.2;
  p->SINHWRHO = 0.2;
  p->SINHWZ = 0.2;
  p->ZMAX = 10.0;
  p->ZMIN = -10.0;
  p->grid_hole_radius = 2.0;
  p->grid_idx = 0;
  p->grid_physical_size = 10.0;
  p->grid_rotates = false;
  p->is_host = true;
  p->xmax = 10.0;
  p->xmin = -10.0;
  p->xxmax0 = p->xxmax1 = p->xxmax2 = 10.0;
  p->xxmin0 = p->xxmin1 = p->xxmin2 = -10.0;
  p->ymax = 10.0;
  p->ymin = -10.0;
  p->zmax = 10.0;
  p->zmin = -10.0;
}

// ---------------------------------------------------------------- coordinates
// xx -> Cartesian. Spherical family: r(xx0) from reference_metric.py:1195-1330;
// SinhCylindrical: rho(xx0), phi = xx1, z(xx2) from reference_metric.py:1593-1630.
enum CoordKind { COORD_SPHERICAL = 0, COORD_SINHSPHERICAL = 1, COORD_SINHCYLINDRICAL = 2 };
struct Coord {
  int kind;
  double AMPL, SINHW;  // SinhSpherical
  CylMap cyl;          // SinhCylindrical
  __host__ __device__ bool cylindrical() const { return kind == COORD_SINHCYLINDRICAL; }
  __host__ __device__ double r(double xx0) const {
    if (kind == COORD_SPHERICAL) return xx0;
    const double tmp0 = 1.0 / SINHW;
    return AMPL * (exp(tmp0 * xx0) - exp(-tmp0 * xx0)) / (exp(tmp0) - exp(-tmp0));
  }
  __host__ __device__ double drdx0(double xx0) const {
    if (kind == COORD_SPHERICAL) return 1.0;
    const double tmp0 = 1.0 / SINHW;
    return AMPL * (exp(tmp0 * xx0) * tmp0 + exp(-tmp0 * xx0) * tmp0) / (exp(tmp0) - exp(-tmp0));
  }
  __host__ __device__ void to_cart(double xx0, double xx1, double xx2, double out[3]) const {
    if (cylindrical()) {
      // the generated xx_to_Cart (SinhCylindrical)
      const double tmp0 = (1.0 / (cyl.SINHWRHO));
      const double tmp3 = (1.0 / (cyl.SINHWZ));
      const double tmp2 = cyl.AMPLRHO * (exp(tmp0 * xx0) - exp(-tmp0 * xx0)) / (exp(tmp0) - exp(-tmp0));
      out[0] = tmp2 * cos(xx1);
      out[1] = tmp2 * sin(xx1);
      out[2] = cyl.AMPLZ * (exp(tmp3 * xx2) - exp(-tmp3 * xx2)) / (exp(tmp3) - exp(-tmp3));
      return;
    }
    const double rr = r(xx0);
    const double tmp = rr * sin(xx1);
    out[0] = tmp * cos(xx2);
    out[1] = tmp * sin(xx2);
    out[2] = rr * cos(xx1);
  }
};

static int coord_of(const params_struct *p, Coord *c) {
  *c = Coord{};
  if (p->CoordSystem_hash == SPHERICAL) c->kind = COORD_SPHERICAL;
  else if (p->CoordSystem_hash == SINHSPHERICAL) *c = Coord{COORD_SINHSPHERICAL, p->AMPL, p->SINHW, CylMap{}};
  else if (p->CoordSystem_hash == SINHCYLINDRICAL) *c = Coord{COORD_SINHCYLINDRICAL, 0.0, 0.0, cyl_map(p)};
  else {
    set_error("CoordSystem_hash %d: only Spherical (%d), SinhSpherical (%d) and SinhCylindrical (%d) are supported",
              p->CoordSystem_hash, SPHERICAL, SINHSPHERICAL, SINHCYLINDRICAL);
    return BSSN_B200_EINVAL;
  }
  return BSSN_B200_OK;
}

static int host_xx(const params_struct *p, REAL *const xx[3], std::vector<double> h[3]) {
  const int N[3] = {p->Nxx_plus_2NGHOSTS0, p->Nxx_plus_2NGHOSTS1, p->Nxx_plus_2NGHOSTS2};
  for (int d = 0; d < 3; d++) {
    h[d].resize(N[d]);
    BSSN_CUDA_TRY(cudaMemcpy(h[d].data(), xx[d], sizeof(double) * N[d], cudaMemcpyDeviceToHost));
  }
  return BSSN_B200_OK;
}

// numerical_grids_and_timestep.py:31-190.
int grid_params(const commondata_struct *cd, params_struct *p, REAL *xx[3], const int Nx[3], bool apply_defaults) {
  Coord c;
  BSSN_TRY(coord_of(p, &c));
  // Default resolution of the generated project (two_blackholes_collide's Nxx_dict for
  // Spherical and SinhSpherical, blackhole_spectroscopy's for SinhCylindrical), replaced by
  // Nx when all three entries are set.
  p->Nxx0 = c.cylindrical() ? 400 : 72;
  p->Nxx1 = c.cylindrical() ? 2 : 12;
  p->Nxx2 = c.cylindrical() ? 1200 : 2;
  if (Nx != nullptr && Nx[0] != -1 && Nx[1] != -1 && Nx[2] != -1) {
    p->Nxx0 = Nx[0];
    p->Nxx1 = Nx[1];
    p->Nxx2 = Nx[2];
  }
  snprintf(p->CoordSystemName, 100, "%s",
           c.kind == COORD_SPHERICAL ? "Spherical" : (c.cylindrical() ? "SinhCylindrical" : "SinhSpherical"));
  if (apply_defaults) {
    if (p->Nxx0 != 2) p->Nxx0 *= cd->convergence_factor;
    if (p->Nxx1 != 2) p->Nxx1 *= cd->convergence_factor;
    if (p->Nxx2 != 2) p->Nxx2 *= cd->convergence_factor;
  }
  if (p->Nxx0 < 1 || p->Nxx1 < 1 || p->Nxx2 < 1) {
    set_error("grid: Nxx = (%d,%d,%d) must be positive", p->Nxx0, p->Nxx1, p->Nxx2);
    return BSSN_B200_EINVAL;
  }
  p->Nxx_plus_2NGHOSTS0 = p->Nxx0 + 2 * NGHOSTS;
  p->Nxx_plus_2NGHOSTS1 = p->Nxx1 + 2 * NGHOSTS;
  p->Nxx_plus_2NGHOSTS2 = p->Nxx2 + 2 * NGHOSTS;
  const long long ntot = (long long)p->Nxx_plus_2NGHOSTS0 * p->Nxx_plus_2NGHOSTS1 * p->Nxx_plus_2NGHOSTS2;
  if (ntot * NUM_EVOL_GFS >= (1LL << 31) || p->Nxx_plus_2NGHOSTS0 > 32767 || p->Nxx_plus_2NGHOSTS1 > 32767 ||
      p->Nxx_plus_2NGHOSTS2 > 32767) {
    set_error("grid: %lld points x %d gridfunctions exceeds 32-bit indexing", ntot, NUM_EVOL_GFS);
    return BSSN_B200_EINVAL;
  }
  if (c.cylindrical()) {
    p->AMPLRHO = p->grid_physical_size;
    p->AMPLZ = p->grid_physical_size;
    if (apply_defaults) {
      p->xxmin0 = 0;
      p->xxmin1 = -p->PI;
      p->xxmin2 = -1;
      p->xxmax0 = 1;
      p->xxmax1 = p->PI;
      p->xxmax2 = 1;
    }
  } else {
    if (c.kind == COORD_SINHSPHERICAL) p->AMPL = p->grid_physical_size;
    else p->RMAX = p->grid_physical_size;
    if (apply_defaults) {
      p->xxmin0 = 0;
      p->xxmin1 = 0;
      p->xxmin2 = -p->PI;
      p->xxmax0 = c.kind == COORD_SINHSPHERICAL ? 1 : p->RMAX;
      p->xxmax1 = p->PI;
      p->xxmax2 = p->PI;
    }
  }
  p->dxx0 = (p->xxmax0 - p->xxmin0) / ((REAL)p->Nxx0);
  p->dxx1 = (p->xxmax1 - p->xxmin1) / ((REAL)p->Nxx1);
  p->dxx2 = (p->xxmax2 - p->xxmin2) / ((REAL)p->Nxx2);
  p->invdxx0 = ((REAL)p->Nxx0) / (p->xxmax0 - p->xxmin0);
  p->invdxx1 = ((REAL)p->Nxx1) / (p->xxmax1 - p->xxmin1);
  p->invdxx2 = ((REAL)p->Nxx2) / (p->xxmax2 - p->xxmin2);
  const int N[3] = {p->Nxx_plus_2NGHOSTS0, p->Nxx_plus_2NGHOSTS1, p->Nxx_plus_2NGHOSTS2};
  const double xmin[3] = {p->xxmin0, p->xxmin1, p->xxmin2}, dx[3] = {p->dxx0, p->dxx1, p->dxx2};
  for (int d = 0; d < 3; d++) {
    std::vector<double> h(N[d]);
    // xx_j = xxmin + (j - NGHOSTS + 1/2) dxx, rounded once (a fused multiply-add), as the
    // reference's cell-centred-grid macro compiles on FMA-capable hosts.
    for (int j = 0; j < N[d]; j++) h[j] = fma((REAL)(j - NGHOSTS) + (1.0 / 2.0), dx[d], xmin[d]);
    BSSN_CUDA_TRY(cudaMalloc(&xx[d], sizeof(double) * N[d]));
    BSSN_CUDA_TRY(cudaMemcpy(xx[d], h.data(), sizeof(double) * N[d], cudaMemcpyHostToDevice));
  }
  return BSSN_B200_OK;
}

// ---------------------------------------------------------------- rfm precompute (rfm_precompute.py:84-565)
int rfm_malloc(const params_struct *p, rfm_struct *r) {
  // The second function of the reference metric is f1(xx1) in the Spherical family and
  // f3(xx2) for SinhCylindrical (same rfm_struct slots).
  const size_t n0 = p->Nxx_plus_2NGHOSTS0,
               n1 = p->CoordSystem_hash == SINHCYLINDRICAL ? p->Nxx_plus_2NGHOSTS2 : p->Nxx_plus_2NGHOSTS1;
  BSSN_CUDA_TRY(cudaMalloc(&r->f0_of_xx0, sizeof(double) * n0));
  BSSN_CUDA_TRY(cudaMalloc(&r->f0_of_xx0__D0, sizeof(double) * n0));
  BSSN_CUDA_TRY(cudaMalloc(&r->f0_of_xx0__DD00, sizeof(double) * n0));
  BSSN_CUDA_TRY(cudaMalloc(&r->f0_of_xx0__DDD000, sizeof(double) * n0));
  BSSN_CUDA_TRY(cudaMalloc(&r->f1_of_xx1, sizeof(double) * n1));
  BSSN_CUDA_TRY(cudaMalloc(&r->f1_of_xx1__D1, sizeof(double) * n1));
  BSSN_CUDA_TRY(cudaMalloc(&r->f1_of_xx1__DD11, sizeof(double) * n1));
  return BSSN_B200_OK;
}

int rfm_free(rfm_struct *r) {
  double **f = &r->f0_of_xx0;
  for (int k = 0; k < 7; k++) {
    if (f[k]) cudaFree(f[k]);
    f[k] = nullptr;
  }
  return BSSN_B200_OK;
}

int rfm_defines(const params_struct *p, rfm_struct *r, REAL *xx[3]) {
  Coord c;
  BSSN_TRY(coord_of(p, &c));
  std::vector<double> hx[3];
  BSSN_TRY(host_xx(p, xx, hx));
  const int n0 = p->Nxx_plus_2NGHOSTS0, n1 = c.cylindrical() ? p->Nxx_plus_2NGHOSTS2 : p->Nxx_plus_2NGHOSTS1;
  std::vector<double> f0(n0), f0d(n0), f0dd(n0), f0ddd(n0), f1(n1), f1d(n1), f1dd(n1);
  for (int i = 0; i < n0; i++) {
    const double xx0 = hx[0][i];
    if (c.cylindrical()) {
      const double AMPLRHO = c.cyl.AMPLRHO, SINHWRHO = c.cyl.SINHWRHO;
      // Expression trees of the generated rfm_precompute_defines (SinhCylindrical).
      f0[i] = AMPLRHO * (exp(xx0 / SINHWRHO) - exp(-xx0 / SINHWRHO)) / (exp((1.0 / (SINHWRHO))) - exp(-1 / SINHWRHO));
      f0d[i] = AMPLRHO * (exp(xx0 / SINHWRHO) / SINHWRHO + exp(-xx0 / SINHWRHO) / SINHWRHO) /
               (exp((1.0 / (SINHWRHO))) - exp(-1 / SINHWRHO));
      f0dd[i] = AMPLRHO * (exp(xx0 / SINHWRHO) / ((SINHWRHO) * (SINHWRHO)) - exp(-xx0 / SINHWRHO) / ((SINHWRHO) * (SINHWRHO))) /
                (exp((1.0 / (SINHWRHO))) - exp(-1 / SINHWRHO));
      f0ddd[i] = AMPLRHO *
                 (exp(xx0 / SINHWRHO) / ((SINHWRHO) * (SINHWRHO) * (SINHWRHO)) +
                  exp(-xx0 / SINHWRHO) / ((SINHWRHO) * (SINHWRHO) * (SINHWRHO))) /
                 (exp((1.0 / (SINHWRHO))) - exp(-1 / SINHWRHO));
    } else if (c.kind == COORD_SINHSPHERICAL) {
      const double AMPL = c.AMPL, SINHW = c.SINHW;
      // Expression trees of the generated rfm_precompute_defines (SinhSpherical).
      f0[i] = AMPL * (exp(xx0 / SINHW) - exp(-xx0 / SINHW)) / (exp((1.0 / (SINHW))) - exp(-1 / SINHW));
      f0d[i] = AMPL * (exp(xx0 / SINHW) / SINHW + exp(-xx0 / SINHW) / SINHW) / (exp((1.0 / (SINHW))) - exp(-1 / SINHW));
      f0dd[i] = AMPL * (exp(xx0 / SINHW) / ((SINHW) * (SINHW)) - exp(-xx0 / SINHW) / ((SINHW) * (SINHW))) /
                (exp((1.0 / (SINHW))) - exp(-1 / SINHW));
      f0ddd[i] = AMPL * (exp(xx0 / SINHW) / ((SINHW) * (SINHW) * (SINHW)) + exp(-xx0 / SINHW) / ((SINHW) * (SINHW) * (SINHW))) /
                 (exp((1.0 / (SINHW))) - exp(-1 / SINHW));
    } else {
      f0[i] = xx0;
      f0d[i] = 1.0;
      f0dd[i] = 0.0;
      f0ddd[i] = 0.0;
    }
  }
  for (int i = 0; i < n1; i++) {
    if (c.cylindrical()) {
      // f3_of_xx2 = dz/dxx2 and its two derivatives (the rescaled metric needs z', not z).
      const double xx2 = hx[2][i], AMPLZ = c.cyl.AMPLZ, SINHWZ = c.cyl.SINHWZ;
      f1[i] = AMPLZ * (exp(xx2 / SINHWZ) / SINHWZ + exp(-xx2 / SINHWZ) / SINHWZ) /
              (exp((1.0 / (SINHWZ))) - exp(-1 / SINHWZ));
      f1d[i] = AMPLZ * (exp(xx2 / SINHWZ) / ((SINHWZ) * (SINHWZ)) - exp(-xx2 / SINHWZ) / ((SINHWZ) * (SINHWZ))) /
               (exp((1.0 / (SINHWZ))) - exp(-1 / SINHWZ));
      f1dd[i] = AMPLZ *
                (exp(xx2 / SINHWZ) / ((SINHWZ) * (SINHWZ) * (SINHWZ)) +
                 exp(-xx2 / SINHWZ) / ((SINHWZ) * (SINHWZ) * (SINHWZ))) /
                (exp((1.0 / (SINHWZ))) - exp(-1 / SINHWZ));
      continue;
    }
    const double xx1 = hx[1][i];
    f1[i] = sin(xx1);
    f1d[i] = cos(xx1);
    f1dd[i] = -sin(xx1);
  }
  BSSN_CUDA_TRY(cudaMemcpy(r->f0_of_xx0, f0.data(), sizeof(double) * n0, cudaMemcpyHostToDevice));
  BSSN_CUDA_TRY(cudaMemcpy(r->f0_of_xx0__D0, f0d.data(), sizeof(double) * n0, cudaMemcpyHostToDevice));
  BSSN_CUDA_TRY(cudaMemcpy(r->f0_of_xx0__DD00, f0dd.data(), sizeof(double) * n0, cudaMemcpyHostToDevice));
  BSSN_CUDA_TRY(cudaMemcpy(r->f0_of_xx0__DDD000, f0ddd.data(), sizeof(double) * n0, cudaMemcpyHostToDevice));
  BSSN_CUDA_TRY(cudaMemcpy(r->f1_of_xx1, f1.data(), sizeof(double) * n1, cudaMemcpyHostToDevice));
  BSSN_CUDA_TRY(cudaMemcpy(r->f1_of_xx1__D1, f1d.data(), sizeof(double) * n1, cudaMemcpyHostToDevice));
  BSSN_CUDA_TRY(cudaMemcpy(r->f1_of_xx1__DD11, f1dd.data(), sizeof(double) * n1, cudaMemcpyHostToDevice));
  return BSSN_B200_OK;
}

// ---------------------------------------------------------------- bcstruct (bcstruct_set_up.py:442-792)
// Eigen-coordinate map of a ghost point (EigenCoord_set_x0x1x2_inbounds__i0i1i2_inbounds_single_pt):
// (x0,x1,x2) -> Cartesian in the eigen-coordinate system (Spherical for the Spherical family,
// Cylindrical for SinhCylindrical) -> (x0,x1,x2)' -> nearest index.
static int eigen_map(const params_struct *p, const Coord &c, const std::vector<double> hx[3], int i0, int i1,
                     int i2, double xin[3], int iin[3]) {
  const double xx0 = hx[0][i0], xx1 = hx[1][i1], xx2 = hx[2][i2];
  double Cartx, Carty, Cartz, x0in, x1in, x2in;
  if (c.cylindrical()) {
    Cartx = xx0 * cos(xx1);
    Carty = xx0 * sin(xx1);
    Cartz = xx2;
    x0in = sqrt(((Cartx) * (Cartx)) + ((Carty) * (Carty)));
    x1in = atan2(Carty, Cartx);
    x2in = Cartz;
  } else {
    const double tmp0 = xx0 * sin(xx1);
    Cartx = tmp0 * cos(xx2);
    Carty = tmp0 * sin(xx2);
    Cartz = xx0 * cos(xx1);
    const double tmp1 = sqrt(((Cartx) * (Cartx)) + ((Carty) * (Carty)) + ((Cartz) * (Cartz)));
    x0in = tmp1;
    x1in = acos(Cartz / tmp1);
    x2in = atan2(Carty, Cartx);
  }
  const double dxx[3] = {p->dxx0, p->dxx1, p->dxx2};
  const double xxmin[3] = {hx[0][0] - ((double)(0 - NGHOSTS) + (1.0 / 2.0)) * dxx[0],
                           hx[1][0] - ((double)(0 - NGHOSTS) + (1.0 / 2.0)) * dxx[1],
                           hx[2][0] - ((double)(0 - NGHOSTS) + (1.0 / 2.0)) * dxx[2]};
  const double xinb[3] = {x0in, x1in, x2in};
  const int N[3] = {p->Nxx_plus_2NGHOSTS0, p->Nxx_plus_2NGHOSTS1, p->Nxx_plus_2NGHOSTS2};
  for (int d = 0; d < 3; d++) {
    iin[d] = (int)((xinb[d] - xxmin[d] - (1.0 / 2.0) * dxx[d] + ((double)NGHOSTS) * dxx[d]) / dxx[d] + 0.5);
    if (iin[d] < 0 || iin[d] >= N[d]) {
      set_error("bcstruct: ghost point (%d,%d,%d) maps to index %d outside [0,%d) in direction %d", i0, i1, i2, iin[d],
                N[d], d);
      return BSSN_B200_ESETUP;
    }
  }
  // Sanity check in the actual coordinate system: both points must be the same Cartesian point.
  double a[3], b[3];
  c.to_cart(xx0, xx1, xx2, a);
  c.to_cart(hx[0][iin[0]], hx[1][iin[1]], hx[2][iin[2]], b);
  const double EPS_REL = 1e-8;
  const double norm = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]) + 1e-15;
  if (fabs(a[0] - b[0]) > EPS_REL * norm || fabs(a[1] - b[1]) > EPS_REL * norm || fabs(a[2] - b[2]) > EPS_REL * norm) {
    set_error("bcstruct: inner boundary point (%d,%d,%d) does not map to a grid point", i0, i1, i2);
    return BSSN_B200_ESETUP;
  }
  for (int d = 0; d < 3; d++) xin[d] = hx[d][iin[d]];
  return BSSN_B200_OK;
}

// Unit-vector dot products of the 10 parity types (set_parity_for_inner_boundary_single_pt):
// rank-0, the three vector components and the six rank-2 components in the rfm basis.
static int check_parity(const double par[10], int8_t parity[10]) {
  const double EPS_REL = 1e-8;
  for (int k = 0; k < 10; k++) {
    if (fabs(par[k]) < 1 - EPS_REL || fabs(par[k]) > 1 + EPS_REL) {
      set_error("bcstruct: parity type %d evaluated to %e, not +/-1", k, par[k]);
      return BSSN_B200_ESETUP;
    }
    parity[k] = par[k] < 0 ? -1 : 1;
  }
  return BSSN_B200_OK;
}

// Cylindrical eigen-coordinates: rho-hat and phi-hat rotate by the phi difference, z-hat is fixed.
static int parity_signs_cyl(double xx1, const double xin[3], int8_t parity[10]) {
  const double xx1_inbounds = xin[1];
  const double tmp0 = sin(xx1) * sin(xx1_inbounds) + cos(xx1) * cos(xx1_inbounds);
  const double tmp1 = ((tmp0) * (tmp0));
  const double par[10] = {1, tmp0, tmp0, 1, tmp1, tmp1, tmp0, tmp1, tmp0, 1};
  return check_parity(par, parity);
}

static int parity_signs(double xx1, double xx2, const double xin[3], int8_t parity[10]) {
  const double xx1_inbounds = xin[1], xx2_inbounds = xin[2];
  const double tmp0 = cos(xx1) * cos(xx1_inbounds);
  const double tmp1 = sin(xx1) * sin(xx1_inbounds);
  const double tmp2 = sin(xx2) * sin(xx2_inbounds);
  const double tmp3 = cos(xx2) * cos(xx2_inbounds);
  const double tmp4 = tmp0 + tmp1 * tmp2 + tmp1 * tmp3;
  const double tmp5 = tmp0 * tmp2 + tmp0 * tmp3 + tmp1;
  const double tmp6 = tmp2 + tmp3;
  const double par[10] = {1, tmp4, tmp5, tmp6, tmp4 * tmp4, tmp4 * tmp5, tmp4 * tmp6, tmp5 * tmp5, tmp5 * tmp6, tmp6 * tmp6};
  return check_parity(par, parity);
}

struct HostBc {
  std::vector<innerpt_bc_struct> inner;
  std::vector<outerpt_bc_struct> outer[NGHOSTS * 3];
  bc_info_struct info;
};

int bcstruct_host(const params_struct *p, const std::vector<double> hx[3], HostBc *out) {
  Coord c;
  BSSN_TRY(coord_of(p, &c));
  const int N0 = p->Nxx_plus_2NGHOSTS0, N1 = p->Nxx_plus_2NGHOSTS1, N2 = p->Nxx_plus_2NGHOSTS2;
  memset(&out->info, 0, sizeof(out->info));
  out->inner.clear();
  // Step 1: inner boundary points, in i2-i1-i0 loop order.
  for (int i2 = 0; i2 < N2; i2++)
    for (int i1 = 0; i1 < N1; i1++)
      for (int i0 = 0; i0 < N0; i0++) {
        const bool interior = i0 >= NGHOSTS && i0 < N0 - NGHOSTS && i1 >= NGHOSTS && i1 < N1 - NGHOSTS &&
                              i2 >= NGHOSTS && i2 < N2 - NGHOSTS;
        if (interior) continue;
        double xin[3];
        int iin[3];
        BSSN_TRY(eigen_map(p, c, hx, i0, i1, i2, xin, iin));
        if (i0 == iin[0] && i1 == iin[1] && i2 == iin[2]) continue;  // pure outer point
        innerpt_bc_struct bc;
        memset(&bc, 0, sizeof(bc));
        bc.dstpt = i0 + N0 * (i1 + N1 * i2);
        bc.srcpt = iin[0] + N0 * (iin[1] + N1 * iin[2]);
        if (c.cylindrical()) BSSN_TRY(parity_signs_cyl(hx[1][i1], xin, bc.parity));
        else BSSN_TRY(parity_signs(hx[1][i1], hx[2][i2], xin, bc.parity));
        out->inner.push_back(bc);
      }
  out->info.num_inner_boundary_points = (int)out->inner.size();
  // Step 2: pure outer points, layer by layer from the inside out, faces x0, x1, x2.
  int imin[3] = {NGHOSTS, NGHOSTS, NGHOSTS};
  int imax[3] = {N0 - NGHOSTS, N1 - NGHOSTS, N2 - NGHOSTS};
  for (int gz = 0; gz < NGHOSTS; gz++) {
    int r[6][6];
    const int x0min[6] = {imin[0] - 1, imin[0], imin[1], imax[1], imin[2], imax[2]};
    imin[0]--;
    const int x0max[6] = {imax[0], imax[0] + 1, imin[1], imax[1], imin[2], imax[2]};
    imax[0]++;
    const int x1min[6] = {imin[0], imax[0], imin[1] - 1, imin[1], imin[2], imax[2]};
    imin[1]--;
    const int x1max[6] = {imin[0], imax[0], imax[1], imax[1] + 1, imin[2], imax[2]};
    imax[1]++;
    const int x2min[6] = {imin[0], imax[0], imin[1], imax[1], imin[2] - 1, imin[2]};
    imin[2]--;
    const int x2max[6] = {imin[0], imax[0], imin[1], imax[1], imax[2], imax[2] + 1};
    imax[2]++;
    memcpy(r[0], x0min, sizeof(x0min));
    memcpy(r[1], x0max, sizeof(x0max));
    memcpy(r[2], x1min, sizeof(x1min));
    memcpy(r[3], x1max, sizeof(x1max));
    memcpy(r[4], x2min, sizeof(x2min));
    memcpy(r[5], x2max, sizeof(x2max));
    for (int f = 0; f < 6; f++)
      for (int k = 0; k < 6; k++) out->info.bc_loop_bounds[gz][f][k] = r[f][k];
  }
  for (int gz = 0; gz < NGHOSTS; gz++) {
    for (int dirn = 0; dirn < 3; dirn++) {
      std::vector<outerpt_bc_struct> &list = out->outer[dirn + 3 * gz];
      list.clear();
      for (int face = 2 * dirn; face <= 2 * dirn + 1; face++) {
        const int FACEX0 = (face == 0) - (face == 1);
        const int FACEX1 = (face == 2) - (face == 3);
        const int FACEX2 = (face == 4) - (face == 5);
        const int *b = out->info.bc_loop_bounds[gz][face];
        for (int i2 = b[4]; i2 < b[5]; i2++)
          for (int i1 = b[2]; i1 < b[3]; i1++)
            for (int i0 = b[0]; i0 < b[1]; i0++) {
              double xin[3];
              int iin[3];
              BSSN_TRY(eigen_map(p, c, hx, i0, i1, i2, xin, iin));
              if (i0 == iin[0] && i1 == iin[1] && i2 == iin[2]) {
                outerpt_bc_struct o;
                memset(&o, 0, sizeof(o));
                o.i0 = (short)i0;
                o.i1 = (short)i1;
                o.i2 = (short)i2;
                o.FACEX0 = (int8_t)FACEX0;
                o.FACEX1 = (int8_t)FACEX1;
                o.FACEX2 = (int8_t)FACEX2;
                list.push_back(o);
              }
            }
      }
      out->info.num_pure_outer_boundary_points[gz][dirn] = (int)list.size();
    }
  }
  return BSSN_B200_OK;
}

int bcstruct_setup(const params_struct *p, REAL *xx[3], bc_struct *bc) {
  std::vector<double> hx[3];
  BSSN_TRY(host_xx(p, xx, hx));
  HostBc h;
  BSSN_TRY(bcstruct_host(p, hx, &h));
  memset(bc, 0, sizeof(*bc));
  bc->bc_info = h.info;
  const size_t ni = std::max<size_t>(1, h.inner.size());
  BSSN_CUDA_TRY(cudaMalloc(&bc->inner_bc_array, sizeof(innerpt_bc_struct) * ni));
  if (!h.inner.empty())
    BSSN_CUDA_TRY(cudaMemcpy(bc->inner_bc_array, h.inner.data(), sizeof(innerpt_bc_struct) * h.inner.size(),
                             cudaMemcpyHostToDevice));
  for (int k = 0; k < NGHOSTS * 3; k++) {
    const size_t n = std::max<size_t>(1, h.outer[k].size());
    BSSN_CUDA_TRY(cudaMalloc(&bc->pure_outer_bc_array[k], sizeof(outerpt_bc_struct) * n));
    if (!h.outer[k].empty())
      BSSN_CUDA_TRY(cudaMemcpy(bc->pure_outer_bc_array[k], h.outer[k].data(),
                               sizeof(outerpt_bc_struct) * h.outer[k].size(), cudaMemcpyHostToDevice));
  }
  return BSSN_B200_OK;
}

int bcstruct_release(bc_struct *bc) {
  if (bc->inner_bc_array) cudaFree(bc->inner_bc_array);
  bc->inner_bc_array = nullptr;
  for (int k = 0; k < NGHOSTS * 3; k++) {
    if (bc->pure_outer_bc_array[k]) cudaFree(bc->pure_outer_bc_array[k]);
    bc->pure_outer_bc_array[k] = nullptr;
  }
  return BSSN_B200_OK;
}

// ---------------------------------------------------------------- timestep (cfl_limited_timestep)
int cfl_dt(commondata_struct *cd, const params_struct *p, REAL *xx[3]) {
  Coord c;
  BSSN_TRY(coord_of(p, &c));
  std::vector<double> hx[3];
  BSSN_TRY(host_xx(p, xx, hx));
  double ds_min = 1e38;
  for (int i2 = 0; i2 < p->Nxx_plus_2NGHOSTS2; i2++)
    for (int i1 = 0; i1 < p->Nxx_plus_2NGHOSTS1; i1++)
      for (int i0 = 0; i0 < p->Nxx_plus_2NGHOSTS0; i0++) {
        const double xx0 = hx[0][i0], xx1 = hx[1][i1], xx2 = hx[2][i2];
        double ds0, ds1, ds2;
        // The sums of two products are fused as gcc fuses them in the generated C when FMA
        // instructions are available (-march=native in the generated Makefile): the first
        // product goes into the fma. dt then equals that build's bit for bit.
        if (c.cylindrical()) {
          // ds_min_single_pt (SinhCylindrical): dxx0 rho', dxx1 rho, dxx2 z'.
          const double tmp0 = (1.0 / (c.cyl.SINHWRHO));
          const double tmp5 = (1.0 / (c.cyl.SINHWZ));
          const double tmp4 = c.cyl.AMPLRHO / (exp(tmp0) - exp(-tmp0));
          const double tmp2 = exp(tmp0 * xx0);
          const double tmp3 = exp(-tmp0 * xx0);
          ds0 = fabs(p->dxx0 * tmp4 * fma(tmp0, tmp2, tmp0 * tmp3));
          ds1 = fabs(p->dxx1 * tmp4 * (tmp2 - tmp3));
          ds2 = fabs(c.cyl.AMPLZ * p->dxx2 * fma(tmp5, exp(tmp5 * xx2), tmp5 * exp(-tmp5 * xx2)) /
                     (exp(tmp5) - exp(-tmp5)));
        } else if (c.kind == COORD_SINHSPHERICAL) {
          const double tmp0 = (1.0 / (c.SINHW));
          const double tmp4 = c.AMPL / (exp(tmp0) - exp(-tmp0));
          const double tmp2 = exp(tmp0 * xx0);
          const double tmp3 = exp(-tmp0 * xx0);
          const double tmp5 = tmp4 * (tmp2 - tmp3);
          ds0 = fabs(p->dxx0 * tmp4 * fma(tmp0, tmp2, tmp0 * tmp3));
          ds1 = fabs(p->dxx1 * tmp5);
          ds2 = fabs(p->dxx2 * tmp5 * sin(xx1));
        } else {
          ds0 = fabs(p->dxx0);
          ds1 = fabs(p->dxx1 * xx0);
          ds2 = fabs(p->dxx2 * xx0 * sin(xx1));
        }
        const double l = std::min(ds0, std::min(ds1, ds2));
        ds_min = std::min(ds_min, l);
      }
  cd->dt = std::min(cd->dt, ds_min * cd->CFL_FACTOR);
  return BSSN_B200_OK;
}

// ---------------------------------------------------------------- Brill-Lindquist initial data
// InitialData_Cartesian.py:111-141 (psi = 1 + sum m/(2|x-x_i|), gamma = psi^4 delta, K = 0,
// alpha = psi^-2), ADM -> BSSN in the Cartesian basis, then the basis change to the
// reference-metric basis and rescaling (ADM_Initial_Data_Reader__BSSN_Converter.py:33-460),
// lambda^i from centred FD of hDD on the interior, then extrapolation and inner BCs.
struct BLData {
  double m1, x1, y1, z1, m2, x2, y2, z2;
};

// Brill-Lindquist data at every point (InitialData_Cartesian.py:111-141) converted to the
// rescaled BSSN variables (ADM_Initial_Data_Reader__BSSN_Converter.py:33-1181): ADM in
// Cartesian gamma_ij = psi^4 delta_ij, K_ij = 0, alpha = psi^-2; gammabar_ij = (det
// gamma)^(-1/3) gamma_ij transformed to the reference basis, h_ij = (gammabar_ij -
// ghat_ij) / ReDD_ij, W = cf = (det gamma)^(-1/6). Every other gridfunction is zero
// (lambda^i is set afterwards from finite differences of h_ij on the interior).
__global__ void bl_initial_data_kernel(const GridDims g, const Coord c, const double *__restrict__ xx0,
                                       const double *__restrict__ xx1, const double *__restrict__ xx2,
                                       const BLData bl, double *__restrict__ y) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= g.ntot) return;
  const int i2 = idx / g.s2;
  const int rem = idx - i2 * g.s2;
  const int i1 = rem / g.s1;
  const int i0 = rem - i1 * g.s1;
  const double a0 = xx0[i0], a1 = xx1[i1], a2 = xx2[i2];
  double X[3];
  c.to_cart(a0, a1, a2, X);
  const double d1 = sqrt((X[0] - bl.x1) * (X[0] - bl.x1) + (X[1] - bl.y1) * (X[1] - bl.y1) +
                         (X[2] - bl.z1) * (X[2] - bl.z1));
  const double d2 = sqrt((X[0] - bl.x2) * (X[0] - bl.x2) + (X[1] - bl.y2) * (X[1] - bl.y2) +
                         (X[2] - bl.z2) * (X[2] - bl.z2));
  const double psi = (1.0 / 2.0) * bl.m1 / d1 + (1.0 / 2.0) * bl.m2 / d2 + 1;
  const double psi4 = psi * psi * psi * psi;
  const double detg = psi4 * psi4 * psi4;
  const double alpha = 1.0 / sqrt(cbrt(detg));
  const double gbar = psi4 * cbrt(1.0 / detg);  // diagonal of gammabar_ij (= 1 up to rounding)
  const double cf = 1.0 / sqrt(cbrt(detg));
  // Jacobian d Cart^a / d xx^i of the reference basis and its scale factors (ReDD_ij = sf_i sf_j,
  // ghat_ii = sf_i^2).
  double J[3][3], sf[3], ghat[3];
  if (c.cylindrical()) {
    const double rho = c.cyl.rho(a0), drho = c.cyl.drho(a0), dz = c.cyl.dz(a2);
    const double sp_ = sin(a1), cp = cos(a1);
    const double Jc[3][3] = {{drho * cp, -rho * sp_, 0.0}, {drho * sp_, rho * cp, 0.0}, {0.0, 0.0, dz}};
    memcpy(J, Jc, sizeof(J));
    sf[0] = drho;
    sf[1] = rho;
    sf[2] = dz;
    ghat[0] = drho * drho;
    ghat[1] = rho * rho;
    ghat[2] = dz * dz;
  } else {
    const double rr = c.r(a0), dr = c.drdx0(a0);
    const double st = sin(a1), ct = cos(a1), sp_ = sin(a2), cp = cos(a2);
    const double Js[3][3] = {{dr * st * cp, rr * ct * cp, -rr * st * sp_},
                             {dr * st * sp_, rr * ct * sp_, rr * st * cp},
                             {dr * ct, -rr * st, 0.0}};
    memcpy(J, Js, sizeof(J));
    sf[0] = dr;
    sf[1] = rr;
    sf[2] = rr * st;
    ghat[0] = dr * dr;
    ghat[1] = rr * rr;
    ghat[2] = rr * rr * st * st;
  }
  const size_t n = (size_t)g.ntot;
#pragma unroll
  for (int gf = 0; gf < NUM_EVOL_GFS; gf++) y[gf * n + idx] = 0.0;
  int k = 0;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = i; j < 3; j++, k++) {
      double gg = 0.0;
#pragma unroll
      for (int a = 0; a < 3; a++) gg += J[a][i] * J[a][j] * gbar;
      const double gh = (i == j) ? ghat[i] : 0.0;
      y[(HDD00GF + k) * n + idx] = (gg - gh) / (sf[i] * sf[j]);
    }
  y[ALPHAGF * n + idx] = alpha;
  y[CFGF * n + idx] = cf;
}

int bl_initial_data(const commondata_struct *cd, const params_struct *p, REAL *xx[3], const bc_struct *bc,
                    double *y_n, cudaStream_t s) {
  (void)bc;
  Coord c;
  BSSN_TRY(coord_of(p, &c));
  for (int d = 0; d < 3; d++)
    if (!xx[d]) {
      set_error("initial data: xx[%d] is NULL", d);
      return BSSN_B200_EINVAL;
    }
  const GridDims g = grid_dims(p);
  const BLData bl{cd->BH1_mass, cd->BH1_posn_x, cd->BH1_posn_y, cd->BH1_posn_z,
                  cd->BH2_mass, cd->BH2_posn_x, cd->BH2_posn_y, cd->BH2_posn_z};
  bl_initial_data_kernel<<<(g.ntot + 127) / 128, 128, 0, s>>>(g, c, xx[0], xx[1], xx[2], bl, y_n);
  BSSN_LAUNCH_CHECK();
  return BSSN_B200_OK;
}

}  // namespace bssn
