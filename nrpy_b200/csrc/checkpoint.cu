// Checkpoint / restart in the file format of the generated write_checkpoint / read_checkpoint
// (infrastructures/BHaH/checkpointing.py:15-470).
//
// File: the commondata_struct of a project that registers checkpointing, then per grid the
// params_struct, an int count, count int point indices and count x NUM_EVOL_GFS REALs in
// point-major order (all gridfunctions of one point together). The single-patch writer selects
// every point (its mask test `maskval >= 0` always holds), so count = ntot and the indices are
// 0..ntot-1.
//
// The state stays on the GPU: a transpose kernel packs the gf-major y_n_gfs into point-major
// chunks in device memory, each chunk is copied to pinned host memory and written while the next
// one is packed and copied. Reading runs the same pipeline the other way: file chunks are copied
// up and scattered into y_n_gfs by the saved indices.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "bssn_common.cuh"

namespace bssn {
namespace {

constexpr int CK_TILE = 32;                 // points per transpose tile
constexpr int CK_THREADS = 256;
constexpr size_t CK_CHUNK = size_t(1) << 16;  // points per pipeline chunk (12.6 MB of REALs)

// out[(p - p0) * NUM_EVOL_GFS + gf] = y[gf * ntot + p] for p in [p0, p0 + n).
__global__ void __launch_bounds__(CK_THREADS) pack_points_kernel(const double *__restrict__ y, const size_t ntot,
                                                                const size_t p0, const int n,
                                                                double *__restrict__ out) {
  __shared__ double tile[NUM_EVOL_GFS][CK_TILE + 1];
  const int t0 = blockIdx.x * CK_TILE;
  const int m = min(CK_TILE, n - t0);
  for (int k = threadIdx.x; k < NUM_EVOL_GFS * CK_TILE; k += blockDim.x) {
    const int gf = k / CK_TILE, i = k % CK_TILE;
    if (i < m) tile[gf][i] = y[(size_t)gf * ntot + p0 + t0 + i];
  }
  __syncthreads();
  double *dst = out + (size_t)t0 * NUM_EVOL_GFS;
  for (int k = threadIdx.x; k < m * NUM_EVOL_GFS; k += blockDim.x) {
    const int i = k / NUM_EVOL_GFS, gf = k % NUM_EVOL_GFS;
    dst[k] = tile[gf][i];
  }
}

// y[gf * ntot + idx[i]] = data[i * NUM_EVOL_GFS + gf] for i in [0, n). Every idx[i] lies in
// [0, ntot): the host checks the indices before they are uploaded.
__global__ void __launch_bounds__(CK_THREADS) scatter_points_kernel(const double *__restrict__ data,
                                                                   const int *__restrict__ idx, const int n,
                                                                   const size_t ntot, double *__restrict__ y) {
  __shared__ double tile[CK_TILE][NUM_EVOL_GFS + 1];
  const int t0 = blockIdx.x * CK_TILE;
  const int m = min(CK_TILE, n - t0);
  const double *src = data + (size_t)t0 * NUM_EVOL_GFS;
  for (int k = threadIdx.x; k < m * NUM_EVOL_GFS; k += blockDim.x) tile[k / NUM_EVOL_GFS][k % NUM_EVOL_GFS] = src[k];
  __syncthreads();
  for (int k = threadIdx.x; k < NUM_EVOL_GFS * CK_TILE; k += blockDim.x) {
    const int gf = k / CK_TILE, i = k % CK_TILE;
    if (i < m) y[(size_t)gf * ntot + idx[t0 + i]] = tile[i][gf];
  }
}

// Staging buffers of one device: two device chunks, two pinned host chunks and their events.
// Allocated on the first checkpoint call on that device and kept until the process exits
// (2 x 12.6 MB of device memory and 2 x 12.6 MB of pinned host memory), so repeated checkpoints
// pay no allocation. Calls are serialised by the mutex.
struct Staging {
  double *dev[2] = {nullptr, nullptr};
  double *host[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
};
std::mutex g_staging_mu;
Staging g_staging[64];

int staging_for_current_device(Staging **out) {
  int d = 0;
  BSSN_CUDA_TRY(cudaGetDevice(&d));
  if (d < 0 || d >= 64) {
    set_error("checkpoint: device ordinal %d not supported", d);
    return BSSN_B200_EINVAL;
  }
  Staging &st = g_staging[d];
  for (int b = 0; b < 2; b++) {
    if (!st.dev[b]) BSSN_CUDA_TRY(cudaMalloc(&st.dev[b], CK_CHUNK * NUM_EVOL_GFS * sizeof(double)));
    if (!st.host[b]) BSSN_CUDA_TRY(cudaMallocHost(&st.host[b], CK_CHUNK * NUM_EVOL_GFS * sizeof(double)));
    if (!st.ev[b]) BSSN_CUDA_TRY(cudaEventCreateWithFlags(&st.ev[b], cudaEventDisableTiming));
  }
  *out = &st;
  return BSSN_B200_OK;
}

// One call's view of the staging buffers, plus what it owns itself (the file, the device copy
// of the read indices); on every return path it waits for its copies and closes the file.
struct Pipeline {
  std::lock_guard<std::mutex> lock{g_staging_mu};
  double *dev[2] = {nullptr, nullptr};
  double *host[2] = {nullptr, nullptr};
  int *dev_idx = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  FILE *f = nullptr;
  ~Pipeline() {
    for (int b = 0; b < 2; b++) {
      if (ev[b]) cudaEventSynchronize(ev[b]);
    }
    if (dev_idx) cudaFree(dev_idx);
    if (f) fclose(f);
  }
  int attach() {
    Staging *st = nullptr;
    BSSN_TRY(staging_for_current_device(&st));
    for (int b = 0; b < 2; b++) {
      dev[b] = st->dev[b];
      host[b] = st->host[b];
      ev[b] = st->ev[b];
    }
    return BSSN_B200_OK;
  }
};

void checkpoint_filename(const double convergence_factor, char out[256]) {
  snprintf(out, 256, "checkpoint-conv_factor%.2f.dat", convergence_factor);
}

void to_checkpoint_layout(const commondata_struct &c, const double checkpoint_every,
                          bssn_b200_checkpoint_commondata *o) {
  memset(o, 0, sizeof(*o));
  o->BH1_mass = c.BH1_mass;
  o->BH1_posn_x = c.BH1_posn_x;
  o->BH1_posn_y = c.BH1_posn_y;
  o->BH1_posn_z = c.BH1_posn_z;
  o->BH2_mass = c.BH2_mass;
  o->BH2_posn_x = c.BH2_posn_x;
  o->BH2_posn_y = c.BH2_posn_y;
  o->BH2_posn_z = c.BH2_posn_z;
  o->CFL_FACTOR = c.CFL_FACTOR;
  o->KreissOliger_strength_gauge = c.KreissOliger_strength_gauge;
  o->KreissOliger_strength_nongauge = c.KreissOliger_strength_nongauge;
  o->checkpoint_every = checkpoint_every;
  o->convergence_factor = c.convergence_factor;
  o->diagnostics_output_every = c.diagnostics_output_every;
  o->dt = c.dt;
  o->eta = c.eta;
  o->t_0 = c.t_0;
  o->t_final = c.t_final;
  o->time = c.time;
  o->start_wallclock_time = c.start_wallclock_time;
  memcpy(o->outer_bc_type, c.outer_bc_type, sizeof(o->outer_bc_type));
  o->NUMGRIDS = c.NUMGRIDS;
  o->nn = c.nn;
  o->nn_0 = c.nn_0;
  o->output_progress_every = c.output_progress_every;
}

void from_checkpoint_layout(const bssn_b200_checkpoint_commondata &o, commondata_struct *c) {
  c->BH1_mass = o.BH1_mass;
  c->BH1_posn_x = o.BH1_posn_x;
  c->BH1_posn_y = o.BH1_posn_y;
  c->BH1_posn_z = o.BH1_posn_z;
  c->BH2_mass = o.BH2_mass;
  c->BH2_posn_x = o.BH2_posn_x;
  c->BH2_posn_y = o.BH2_posn_y;
  c->BH2_posn_z = o.BH2_posn_z;
  c->CFL_FACTOR = o.CFL_FACTOR;
  c->KreissOliger_strength_gauge = o.KreissOliger_strength_gauge;
  c->KreissOliger_strength_nongauge = o.KreissOliger_strength_nongauge;
  c->convergence_factor = o.convergence_factor;
  c->diagnostics_output_every = o.diagnostics_output_every;
  c->dt = o.dt;
  c->eta = o.eta;
  c->t_0 = o.t_0;
  c->t_final = o.t_final;
  c->time = o.time;
  c->start_wallclock_time = o.start_wallclock_time;
  memcpy(c->outer_bc_type, o.outer_bc_type, sizeof(c->outer_bc_type));
  c->NUMGRIDS = o.NUMGRIDS;
  c->nn = o.nn;
  c->nn_0 = o.nn_0;
  c->output_progress_every = o.output_progress_every;
}

int write_all(FILE *f, const void *p, size_t size, size_t n, const char *what, const char *fname) {
  if (n && fwrite(p, size, n, f) != n) {
    set_error("write_checkpoint: writing %s to %s failed: %s", what, fname, strerror(errno));
    return BSSN_B200_EINVAL;
  }
  return BSSN_B200_OK;
}

int read_all(FILE *f, void *p, size_t size, size_t n, const char *what, const char *fname) {
  if (n && fread(p, size, n, f) != n) {
    set_error("read_checkpoint: reading %s from %s: expected %zu items, got fewer", what, fname, n);
    return BSSN_B200_EINVAL;
  }
  return BSSN_B200_OK;
}

size_t grid_points(const params_struct &p) {
  return (size_t)p.Nxx_plus_2NGHOSTS0 * p.Nxx_plus_2NGHOSTS1 * p.Nxx_plus_2NGHOSTS2;
}

int check_numgrids(int n, const char *who) {
  if (n < 1 || n > MAXNUMGRIDS) {
    set_error("%s: NUMGRIDS = %d outside [1, %d]", who, n, MAXNUMGRIDS);
    return BSSN_B200_EINVAL;
  }
  return BSSN_B200_OK;
}

// Pack each chunk of one grid's points on the GPU, copy it down and write it while the next one
// is packed.
int write_grid_payload(Pipeline &pl, const griddata_struct &g, const char *fname, cudaStream_t s) {
  const size_t ntot = grid_points(g.params);
  const size_t nchunks = (ntot + CK_CHUNK - 1) / CK_CHUNK;
  auto enqueue = [&](size_t c) -> int {
    const int b = (int)(c & 1);
    const size_t p0 = c * CK_CHUNK;
    const int n = (int)std::min(CK_CHUNK, ntot - p0);
    pack_points_kernel<<<(n + CK_TILE - 1) / CK_TILE, CK_THREADS, 0, s>>>(g.gridfuncs.y_n_gfs, ntot, p0, n,
                                                                          pl.dev[b]);
    BSSN_LAUNCH_CHECK();
    BSSN_CUDA_TRY(cudaMemcpyAsync(pl.host[b], pl.dev[b], (size_t)n * NUM_EVOL_GFS * sizeof(double),
                                  cudaMemcpyDeviceToHost, s));
    BSSN_CUDA_TRY(cudaEventRecord(pl.ev[b], s));
    return BSSN_B200_OK;
  };
  if (nchunks) BSSN_TRY(enqueue(0));
  // The indices 0..ntot-1 are written while the first chunk is packed.
  std::vector<int> idx(std::min(CK_CHUNK, ntot));
  for (size_t p0 = 0; p0 < ntot; p0 += CK_CHUNK) {
    const size_t n = std::min(CK_CHUNK, ntot - p0);
    for (size_t i = 0; i < n; i++) idx[i] = (int)(p0 + i);
    BSSN_TRY(write_all(pl.f, idx.data(), sizeof(int), n, "out_data_indices", fname));
  }
  for (size_t c = 0; c < nchunks; c++) {
    if (c + 1 < nchunks) BSSN_TRY(enqueue(c + 1));
    const int b = (int)(c & 1);
    BSSN_CUDA_TRY(cudaEventSynchronize(pl.ev[b]));
    const size_t n = std::min(CK_CHUNK, ntot - c * CK_CHUNK);
    BSSN_TRY(write_all(pl.f, pl.host[b], sizeof(double), n * NUM_EVOL_GFS, "compact_out_data", fname));
  }
  return BSSN_B200_OK;
}

int write_checkpoint_impl(const commondata_struct *cd, const double checkpoint_every, const griddata_struct *gd,
                          cudaStream_t s) {
  if (!cd || !gd) {
    set_error("write_checkpoint: NULL argument");
    return BSSN_B200_EINVAL;
  }
  // Checkpoint steps only (checkpointing.py:318-326).
  if (checkpoint_every <= 0.0) return 0;
  if (!(std::fabs(std::round(cd->time / checkpoint_every) * checkpoint_every - cd->time) < 0.5 * cd->dt)) return 0;
  BSSN_TRY(check_numgrids(cd->NUMGRIDS, "write_checkpoint"));
  for (int grid = 0; grid < cd->NUMGRIDS; grid++) {
    if (!gd[grid].gridfuncs.y_n_gfs) {
      set_error("write_checkpoint: grid %d has no y_n_gfs", grid);
      return BSSN_B200_EINVAL;
    }
    if (grid_points(gd[grid].params) > (size_t)INT32_MAX) {
      set_error("write_checkpoint: grid %d has more points than an int index can hold", grid);
      return BSSN_B200_EINVAL;
    }
  }
  char fname[256];
  checkpoint_filename(cd->convergence_factor, fname);
  Pipeline pl;
  BSSN_TRY(pl.attach());
  pl.f = fopen(fname, "wb");
  if (!pl.f) {
    set_error("write_checkpoint: could not open %s for writing: %s", fname, strerror(errno));
    return BSSN_B200_EINVAL;
  }
  bssn_b200_checkpoint_commondata ck;
  to_checkpoint_layout(*cd, checkpoint_every, &ck);
  BSSN_TRY(write_all(pl.f, &ck, sizeof(ck), 1, "commondata", fname));
  for (int grid = 0; grid < cd->NUMGRIDS; grid++) {
    const griddata_struct &g = gd[grid];
    BSSN_TRY(write_all(pl.f, &g.params, sizeof(params_struct), 1, "params_struct", fname));
    const int count = (int)grid_points(g.params);
    BSSN_TRY(write_all(pl.f, &count, sizeof(int), 1, "gridpoint_count", fname));
    BSSN_TRY(write_grid_payload(pl, g, fname, s));
  }
  const int rc = fclose(pl.f);
  pl.f = nullptr;
  if (rc != 0) {
    set_error("write_checkpoint: closing %s failed: %s", fname, strerror(errno));
    return BSSN_B200_EINVAL;
  }
  return 1;
}

// Read one grid's saved points in chunks, copy each up and scatter it into y_n_gfs.
int read_grid_payload(Pipeline &pl, griddata_struct &g, const int count, const char *fname, cudaStream_t s) {
  const size_t ntot = grid_points(g.params);
  std::vector<int> idx((size_t)count);
  BSSN_TRY(read_all(pl.f, idx.data(), sizeof(int), (size_t)count, "out_data_indices", fname));
  for (int i = 0; i < count; i++) {
    if (idx[i] < 0 || (size_t)idx[i] >= ntot) {
      set_error("read_checkpoint: index %d of entry %d outside the grid's %zu points in %s", idx[i], i, ntot, fname);
      return BSSN_B200_EINVAL;
    }
  }
  BSSN_CUDA_TRY(cudaMemsetAsync(g.gridfuncs.y_n_gfs, 0, ntot * NUM_EVOL_GFS * sizeof(double), s));
  if (count == 0) return BSSN_B200_OK;
  if (pl.dev_idx) {
    BSSN_CUDA_TRY(cudaStreamSynchronize(s));
    BSSN_CUDA_TRY(cudaFree(pl.dev_idx));
    pl.dev_idx = nullptr;
  }
  BSSN_CUDA_TRY(cudaMalloc(&pl.dev_idx, (size_t)count * sizeof(int)));
  BSSN_CUDA_TRY(cudaMemcpyAsync(pl.dev_idx, idx.data(), (size_t)count * sizeof(int), cudaMemcpyHostToDevice, s));
  const size_t nchunks = ((size_t)count + CK_CHUNK - 1) / CK_CHUNK;
  for (size_t c = 0; c < nchunks; c++) {
    const int b = (int)(c & 1);
    // The pinned buffer b was last used by the upload of chunk c - 2.
    BSSN_CUDA_TRY(cudaEventSynchronize(pl.ev[b]));
    const size_t p0 = c * CK_CHUNK;
    const int n = (int)std::min(CK_CHUNK, (size_t)count - p0);
    BSSN_TRY(read_all(pl.f, pl.host[b], sizeof(double), (size_t)n * NUM_EVOL_GFS, "compact_out_data", fname));
    BSSN_CUDA_TRY(cudaMemcpyAsync(pl.dev[b], pl.host[b], (size_t)n * NUM_EVOL_GFS * sizeof(double),
                                  cudaMemcpyHostToDevice, s));
    BSSN_CUDA_TRY(cudaEventRecord(pl.ev[b], s));
    scatter_points_kernel<<<(n + CK_TILE - 1) / CK_TILE, CK_THREADS, 0, s>>>(pl.dev[b], pl.dev_idx + p0, n, ntot,
                                                                             g.gridfuncs.y_n_gfs);
    BSSN_LAUNCH_CHECK();
  }
  // The indices stay in use until the last scatter has run.
  BSSN_CUDA_TRY(cudaStreamSynchronize(s));
  return BSSN_B200_OK;
}

int read_checkpoint_impl(commondata_struct *cd, double *checkpoint_every, griddata_struct *gd, cudaStream_t s) {
  if (!cd) {
    set_error("read_checkpoint: commondata is NULL");
    return BSSN_B200_EINVAL;
  }
  char fname[256];
  checkpoint_filename(cd->convergence_factor, fname);
  Pipeline pl;
  pl.f = fopen(fname, "rb");
  if (!pl.f) {
    if (errno == ENOENT) return 0;  // no checkpoint: a fresh start
    set_error("read_checkpoint: could not open %s for reading: %s", fname, strerror(errno));
    return BSSN_B200_EINVAL;
  }
  bssn_b200_checkpoint_commondata ck;
  BSSN_TRY(read_all(pl.f, &ck, sizeof(ck), 1, "commondata_struct", fname));
  if (!gd) {
    from_checkpoint_layout(ck, cd);
    if (checkpoint_every) *checkpoint_every = ck.checkpoint_every;
    return 1;
  }
  BSSN_TRY(check_numgrids(ck.NUMGRIDS, "read_checkpoint"));
  BSSN_TRY(pl.attach());
  for (int grid = 0; grid < ck.NUMGRIDS; grid++) {
    griddata_struct &g = gd[grid];
    params_struct saved;
    BSSN_TRY(read_all(pl.f, &saved, sizeof(params_struct), 1, "griddata[grid].params", fname));
    int count = 0;
    BSSN_TRY(read_all(pl.f, &count, sizeof(int), 1, "count", fname));
    const params_struct &p = g.params;
    if (saved.Nxx_plus_2NGHOSTS0 != p.Nxx_plus_2NGHOSTS0 || saved.Nxx_plus_2NGHOSTS1 != p.Nxx_plus_2NGHOSTS1 ||
        saved.Nxx_plus_2NGHOSTS2 != p.Nxx_plus_2NGHOSTS2 || saved.CoordSystem_hash != p.CoordSystem_hash) {
      set_error("read_checkpoint: checkpoint/grid mismatch on grid %d: checkpoint dims=(%d,%d,%d) hash=%d, grid "
                "dims=(%d,%d,%d) hash=%d",
                grid, saved.Nxx_plus_2NGHOSTS0, saved.Nxx_plus_2NGHOSTS1, saved.Nxx_plus_2NGHOSTS2,
                saved.CoordSystem_hash, p.Nxx_plus_2NGHOSTS0, p.Nxx_plus_2NGHOSTS1, p.Nxx_plus_2NGHOSTS2,
                p.CoordSystem_hash);
      return BSSN_B200_EINVAL;
    }
    const size_t ntot = grid_points(p);
    if (count < 0 || (size_t)count > ntot) {
      set_error("read_checkpoint: invalid count=%d for grid=%d (ntot_grid=%zu) in %s", count, grid, ntot, fname);
      return BSSN_B200_EINVAL;
    }
    if (!g.gridfuncs.y_n_gfs) {
      set_error("read_checkpoint: grid %d has no y_n_gfs", grid);
      return BSSN_B200_EINVAL;
    }
    BSSN_TRY(read_grid_payload(pl, g, count, fname, s));
  }
  from_checkpoint_layout(ck, cd);
  if (checkpoint_every) *checkpoint_every = ck.checkpoint_every;
  // The restart time becomes the new origin of the run (checkpointing.py:213-215).
  cd->t_0 = cd->time;
  cd->nn_0 = cd->nn;
  return 1;
}

}  // namespace
}  // namespace bssn

extern "C" {

int bssn_b200_write_checkpoint(const commondata_struct *commondata, REAL checkpoint_every,
                               const griddata_struct *griddata, void *stream) {
  return bssn::write_checkpoint_impl(commondata, checkpoint_every, griddata, (cudaStream_t)stream);
}

int bssn_b200_read_checkpoint(commondata_struct *commondata, REAL *checkpoint_every, griddata_struct *griddata,
                              void *stream) {
  return bssn::read_checkpoint_impl(commondata, checkpoint_every, griddata, (cudaStream_t)stream);
}

}  // extern "C"
