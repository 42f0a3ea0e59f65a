// Many independent BSSN evolutions (uneven grid sizes) advanced together.
//
// Every RK4 stage of every evolution runs in a fixed number of launches that each cover
// the whole batch (up to kChunkEvos evolutions per launch of a Ricci or RHS group kernel):
// those kernels run one block per 128-point tile over the tiles of all their evolutions,
// and concatenated point lists serve the outer radiation layers, the RK update of outer
// points and the inner parity copies. The per-evolution geometry, buffers, timestep and
// physical parameters are EvoDesc descriptors: by value in the group kernels' parameters
// (BatchChunk), and as a device array for the boundary kernels. `steps_per_graph` RK4
// steps are captured once into a CUDA graph and replayed; the tile shape comes from the
// caller (nrpy_b200.batch autotunes it).
#include <algorithm>
#include <cstring>
#include <vector>

#include "bssn_common.cuh"

using namespace bssn;

struct bssn_b200_batch {
  int nevo = 0;
  Variant v = SPH_3D;
  std::vector<commondata_struct *> cds;
  std::vector<griddata_struct *> gds;
  EvoDesc *d_descs = nullptr;
  std::vector<BatchChunk> chunks;  // the Ricci / RHS launches' parameters
  int ntiles = 0;
  BatchOuterPt *d_outer_layer[NGHOSTS] = {nullptr, nullptr, nullptr};
  int nouter_layer[NGHOSTS] = {0, 0, 0};
  BatchOuterPt *d_outer_all = nullptr;
  int nouter_all = 0;
  BatchInnerPt *d_inner = nullptr;
  int ninner = 0;
  std::vector<double *> krhs;
  int bx = 32, by = 4, steps_per_graph = 1;  // bx = by = 0: a tile shape per evolution
  long long padded_points = 0, interior_points = 0;          // tile capacity and interior points covered
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  unsigned long long kernel_nodes = 0;
};

namespace bssn {

static int batch_stage(bssn_b200_batch *b, int stage, cudaStream_t s) {
  for (const BatchChunk &c : b->chunks) BSSN_TRY(launch_ricci_batched(b->v, stage, c, s));
  for (const BatchChunk &c : b->chunks) BSSN_TRY(launch_rhs_fused_batched(b->v, stage, c, s));
  for (int gz = 0; gz < NGHOSTS; gz++)
    BSSN_TRY(launch_radiation_batched(stage, b->d_descs, b->d_outer_layer[gz], b->nouter_layer[gz], s));
  BSSN_TRY(launch_rk_points_batched(b->v, stage, b->d_descs, b->d_outer_all, b->nouter_all, s));
  return launch_inner_batched(stage, b->d_descs, b->d_inner, b->ninner, s);
}

static int batch_step(bssn_b200_batch *b, cudaStream_t s) {
  for (int stage = 1; stage <= 4; stage++) BSSN_TRY(batch_stage(b, stage, s));
  return BSSN_B200_OK;
}

// Tile shapes (points along i0, i1, i2; 128 points) among which a batch built with per-grid
// shapes picks, for each evolution, the one that pads its interior least (ties: the wider
// along i0, for coalescing).
struct Brick {
  int bx, by, bz;
};
static const Brick kBricks[] = {{128, 1, 1}, {64, 2, 1}, {64, 1, 2}, {32, 4, 1}, {32, 2, 2}, {32, 1, 4},
                                {16, 8, 1},  {16, 4, 2}, {16, 2, 4}, {16, 1, 8}};

static long long padded_points(int n0, int n1, int n2, const Brick &k) {
  return (long long)((n0 + k.bx - 1) / k.bx) * k.bx * ((n1 + k.by - 1) / k.by) * k.by * ((n2 + k.bz - 1) / k.bz) *
         k.bz;
}

static Brick best_brick(int n0, int n1, int n2) {
  Brick best = kBricks[0];
  for (const Brick &k : kBricks)
    if (padded_points(n0, n1, n2, k) < padded_points(n0, n1, n2, best)) best = k;
  return best;
}

template <typename Tp>
static int upload(Tp **dst, const std::vector<Tp> &v) {
  const size_t n = std::max<size_t>(1, v.size());
  BSSN_CUDA_TRY(cudaMalloc(dst, sizeof(Tp) * n));
  if (!v.empty()) BSSN_CUDA_TRY(cudaMemcpy(*dst, v.data(), sizeof(Tp) * v.size(), cudaMemcpyHostToDevice));
  return BSSN_B200_OK;
}

static void batch_free(bssn_b200_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  cudaFree(b->d_descs);
  for (int gz = 0; gz < NGHOSTS; gz++) cudaFree(b->d_outer_layer[gz]);
  cudaFree(b->d_outer_all);
  cudaFree(b->d_inner);
  for (double *k : b->krhs) cudaFree(k);
}

static int batch_build(bssn_b200_batch *b) {
  std::vector<EvoDesc> descs(b->nevo);
  long long ntiles = 0;
  std::vector<BatchOuterPt> layer[NGHOSTS], all_outer;
  std::vector<BatchInnerPt> inner;
  for (int e = 0; e < b->nevo; e++) {
    const commondata_struct *cd = b->cds[e];
    griddata_struct &G = *b->gds[e];
    Variant v;
    BSSN_TRY(variant_of(&G.params, &v));
    if (e == 0) b->v = v;
    if (v != b->v) {
      set_error("batch: evolution %d uses another coordinate system or symmetry than evolution 0", e);
      return BSSN_B200_EINVAL;
    }
    if (strncmp(cd->outer_bc_type, "radiation", 50) != 0) {
      set_error("batch: evolution %d: only radiation outer boundary conditions are batched", e);
      return BSSN_B200_EINVAL;
    }
    const MoL_gridfunctions_struct &gf = G.gridfuncs;
    if (!gf.y_n_gfs || !gf.y_nplus1_running_total_gfs || !gf.k_odd_gfs || !gf.k_even_gfs || !gf.auxevol_gfs ||
        !G.rfmstruct) {
      set_error("batch: evolution %d has unallocated storage", e);
      return BSSN_B200_EINVAL;
    }
    EvoDesc &d = descs[e];
    memset(&d, 0, sizeof(d));
    d.g = grid_dims(&G.params);
    d.rfm = rfm_arrays(G.rfmstruct);
    d.pp = PhysParams{cd->eta, cd->KreissOliger_strength_gauge, cd->KreissOliger_strength_nongauge};
    d.dt = cd->dt;
    d.y = gf.y_n_gfs;
    d.run = gf.y_nplus1_running_total_gfs;
    d.kodd = gf.k_odd_gfs;
    d.keven = gf.k_even_gfs;
    d.aux = gf.auxevol_gfs;
    double *krhs = nullptr;
    BSSN_CUDA_TRY(cudaMalloc(&krhs, sizeof(double) * (size_t)d.g.ntot * NUM_EVOL_GFS));
    b->krhs.push_back(krhs);
    d.krhs = krhs;
    d.xx0 = G.xx[0];
    d.radial_sinh = G.params.CoordSystem_hash == SINHSPHERICAL ? 1 : 0;
    d.AMPL = G.params.AMPL;
    d.SINHW = G.params.SINHW;
    const int n0 = d.g.N0 - 2 * NGHOSTS, n1 = d.g.N1 - 2 * NGHOSTS, n2 = d.g.N2 - 2 * NGHOSTS;
    const Brick k = b->bx == 0 ? best_brick(n0, n1, n2) : Brick{b->bx, b->by, 1};
    d.tile_bx = k.bx;
    d.tile_by = k.by;
    d.tile_bz = k.bz;
    d.tiles_x = (n0 + k.bx - 1) / k.bx;
    d.tiles_y = (n1 + k.by - 1) / k.by;
    const long long nt = (long long)d.tiles_x * d.tiles_y * ((std::max(n2, 0) + k.bz - 1) / k.bz);
    b->padded_points += padded_points(n0, n1, std::max(n2, 0), k);
    b->interior_points += (long long)n0 * n1 * std::max(n2, 0);
    // chunks of up to kChunkEvos evolutions; a chunk's launch has one block per tile (x2 for
    // 64-thread groups), which must stay below the grid limit
    if (b->chunks.empty() || b->chunks.back().nevo == kChunkEvos) {
      b->chunks.emplace_back();
      memset(&b->chunks.back(), 0, sizeof(BatchChunk));
    }
    BatchChunk &c = b->chunks.back();
    if ((long long)c.ntiles + nt > (1LL << 29)) {
      set_error("batch: too many tiles in one chunk of evolutions");
      return BSSN_B200_EINVAL;
    }
    c.tile_begin[c.nevo] = c.ntiles;
    c.evo[c.nevo] = d;
    c.nevo++;
    c.ntiles += (int)nt;
    c.tile_begin[c.nevo] = c.ntiles;
    ntiles += nt;
    // boundary lists (host copies of this evolution's bcstruct)
    const bc_info_struct &bi = G.bcstruct.bc_info;
    for (int gz = 0; gz < NGHOSTS; gz++)
      for (int dirn = 0; dirn < 3; dirn++) {
        const int n = bi.num_pure_outer_boundary_points[gz][dirn];
        if (n <= 0) continue;
        if (dirn != 0) {
          set_error("batch: outer points off the x0 face are not supported");
          return BSSN_B200_EINVAL;
        }
        std::vector<outerpt_bc_struct> h(n);
        BSSN_CUDA_TRY(cudaMemcpy(h.data(), G.bcstruct.pure_outer_bc_array[dirn + 3 * gz],
                                 sizeof(outerpt_bc_struct) * n, cudaMemcpyDeviceToHost));
        for (const auto &p : h) {
          layer[gz].push_back(BatchOuterPt{e, p});
          all_outer.push_back(BatchOuterPt{e, p});
        }
      }
    const int ni = bi.num_inner_boundary_points;
    if (ni > 0) {
      std::vector<innerpt_bc_struct> h(ni);
      BSSN_CUDA_TRY(
          cudaMemcpy(h.data(), G.bcstruct.inner_bc_array, sizeof(innerpt_bc_struct) * ni, cudaMemcpyDeviceToHost));
      for (const auto &q : h) inner.push_back(BatchInnerPt{e, q});
    }
  }
  if (ntiles > (1LL << 30)) {
    set_error("batch: %lld tiles in all, more than 2^30", ntiles);
    return BSSN_B200_EINVAL;
  }
  b->ntiles = (int)ntiles;
  BSSN_TRY(upload(&b->d_descs, descs));
  for (int gz = 0; gz < NGHOSTS; gz++) {
    b->nouter_layer[gz] = (int)layer[gz].size();
    BSSN_TRY(upload(&b->d_outer_layer[gz], layer[gz]));
  }
  b->nouter_all = (int)all_outer.size();
  BSSN_TRY(upload(&b->d_outer_all, all_outer));
  b->ninner = (int)inner.size();
  BSSN_TRY(upload(&b->d_inner, inner));
  return BSSN_B200_OK;
}

}  // namespace bssn

extern "C" {

int bssn_b200_batch_create(int nevo, commondata_struct *const *cds, griddata_struct *const *gds, int tile_bx,
                           int tile_by, int steps_per_graph, void *stream, bssn_b200_batch **out) {
  if (nevo < 1 || !cds || !gds || !out) {
    set_error("batch: need nevo >= 1 and non-NULL arrays");
    return BSSN_B200_EINVAL;
  }
  const bool per_grid = tile_bx == 0 && tile_by == 0;
  if ((!per_grid && (tile_bx * tile_by != 128 || tile_bx < 1 || tile_by < 1)) || steps_per_graph < 1 ||
      steps_per_graph > 1000) {
    set_error("batch: tile %dx%d must have 128 points (or 0x0: a shape per evolution); "
              "1 <= steps_per_graph <= 1000", tile_bx, tile_by);
    return BSSN_B200_EINVAL;
  }
  if (!stream) {
    set_error("batch: graph capture needs a non-default stream");
    return BSSN_B200_EINVAL;
  }
  bssn_b200_batch *b = new bssn_b200_batch;
  b->nevo = nevo;
  b->cds.assign(cds, cds + nevo);
  b->gds.assign(gds, gds + nevo);
  b->bx = tile_bx;
  b->by = tile_by;
  b->steps_per_graph = steps_per_graph;
  b->stream = (cudaStream_t)stream;
  int rc = batch_build(b);
  if (rc == BSSN_B200_OK) {
    // One eager step outside the capture sets the kernels' shared-memory attributes; the
    // evolutions' states are saved before it and restored after it.
    std::vector<double *> saved(nevo, nullptr);
    for (int e = 0; e < nevo && rc == BSSN_B200_OK; e++) {
      const params_struct &p = b->gds[e]->params;
      const size_t bytes = sizeof(double) * NUM_EVOL_GFS * (size_t)p.Nxx_plus_2NGHOSTS0 * p.Nxx_plus_2NGHOSTS1 *
                           p.Nxx_plus_2NGHOSTS2;
      if (cudaMalloc(&saved[e], bytes) != cudaSuccess ||
          cudaMemcpyAsync(saved[e], b->gds[e]->gridfuncs.y_n_gfs, bytes, cudaMemcpyDeviceToDevice, b->stream) !=
              cudaSuccess) {
        set_error("batch: saving the state of evolution %d failed", e);
        rc = BSSN_B200_ENOMEM;
      }
    }
    if (rc == BSSN_B200_OK) rc = batch_step(b, b->stream);
    for (int e = 0; e < nevo; e++) {
      if (!saved[e]) continue;
      const params_struct &p = b->gds[e]->params;
      const size_t bytes = sizeof(double) * NUM_EVOL_GFS * (size_t)p.Nxx_plus_2NGHOSTS0 * p.Nxx_plus_2NGHOSTS1 *
                           p.Nxx_plus_2NGHOSTS2;
      if (rc == BSSN_B200_OK &&
          cudaMemcpyAsync(b->gds[e]->gridfuncs.y_n_gfs, saved[e], bytes, cudaMemcpyDeviceToDevice, b->stream) !=
              cudaSuccess)
        rc = BSSN_B200_ECUDA;
    }
    if (cudaStreamSynchronize(b->stream) != cudaSuccess && rc == BSSN_B200_OK) rc = BSSN_B200_ECUDA;
    for (double *p : saved) cudaFree(p);
  }
  if (rc == BSSN_B200_OK) {
    if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      set_error("batch: cudaStreamBeginCapture failed");
      rc = BSSN_B200_ECUDA;
    } else {
      for (int n = 0; n < steps_per_graph && rc == BSSN_B200_OK; n++) rc = batch_step(b, b->stream);
      cudaGraph_t graph = nullptr;
      cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
      b->graph = graph;
      if (rc == BSSN_B200_OK && e != cudaSuccess) {
        set_error("batch: stream capture failed: %s", cudaGetErrorString(e));
        rc = BSSN_B200_ECUDA;
      }
      if (rc == BSSN_B200_OK && cudaGraphInstantiate(&b->exec, b->graph, 0) != cudaSuccess) {
        set_error("batch: graph instantiate failed");
        rc = BSSN_B200_ECUDA;
      }
      if (rc == BSSN_B200_OK) {
        size_t nn = 0;
        cudaGraphGetNodes(b->graph, nullptr, &nn);
        std::vector<cudaGraphNode_t> nodes(nn);
        if (nn) cudaGraphGetNodes(b->graph, nodes.data(), &nn);
        for (auto nd : nodes) {
          cudaGraphNodeType t;
          cudaGraphNodeGetType(nd, &t);
          if (t == cudaGraphNodeTypeKernel) b->kernel_nodes++;
        }
      }
    }
  }
  if (rc != BSSN_B200_OK) {
    batch_free(b);
    delete b;
    return rc;
  }
  *out = b;
  return BSSN_B200_OK;
}

int bssn_b200_batch_run(bssn_b200_batch *b, int graph_launches) {
  if (!b || graph_launches < 0) {
    set_error("batch_run: bad arguments");
    return BSSN_B200_EINVAL;
  }
  for (int n = 0; n < graph_launches; n++) {
    BSSN_CUDA_TRY(cudaGraphLaunch(b->exec, b->stream));
    count_launch(b->kernel_nodes);
    for (int e = 0; e < b->nevo; e++) {
      commondata_struct *cd = b->cds[e];
      for (int k = 0; k < b->steps_per_graph; k++) {
        cd->time = cd->t_0 + (double)(cd->nn - cd->nn_0 + 1) * cd->dt;
        cd->nn++;
      }
    }
  }
  return BSSN_B200_OK;
}

int bssn_b200_batch_tile_fill(const bssn_b200_batch *b, long long *interior_points, long long *padded_points) {
  if (!b) {
    set_error("batch_tile_fill: NULL batch");
    return BSSN_B200_EINVAL;
  }
  if (interior_points) *interior_points = b->interior_points;
  if (padded_points) *padded_points = b->padded_points;
  return BSSN_B200_OK;
}

int bssn_b200_batch_info(const bssn_b200_batch *b, int *ntiles, int *nouter, int *ninner,
                         unsigned long long *kernel_nodes) {
  if (!b) {
    set_error("batch_info: NULL batch");
    return BSSN_B200_EINVAL;
  }
  if (ntiles) *ntiles = b->ntiles;
  if (nouter) *nouter = b->nouter_all;
  if (ninner) *ninner = b->ninner;
  if (kernel_nodes) *kernel_nodes = b->kernel_nodes;
  return BSSN_B200_OK;
}

int bssn_b200_batch_destroy(bssn_b200_batch *b) {
  if (!b) return BSSN_B200_OK;
  batch_free(b);
  delete b;
  return BSSN_B200_OK;
}

}  // extern "C"
