// Volume integrals of the constraint diagnostics over the grid interior, FP64, deterministic.
//
// Reference: diagnostics_volume_integration_helpers.h:400-470 -- sum over interior points of
// f^2 dV with dV = sqrt(det gammahat) |dxx0 dxx1 dxx2|, evaluated from the rfm precompute
// arrays (volume_element). Each block reduces a fixed slice of the interior with warp shuffles
// into a partial; a single block then adds the partials in a fixed order, so the result
// does not depend on scheduling.
#include <mutex>

#include "bssn_common.cuh"

namespace bssn {

constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 296;  // 2 x 148 SMs
constexpr int kRedVals = 4;      // H^2 dV, (M^2)^2 dV, |Lambda|^2 dV, dV

// sqrt(det gammahat) |dxx0 dxx1 dxx2| at an interior point: |f0' f0^2 f1| for the Spherical
// family (f0 = r, f1 = sin(xx1)); |rho' rho z'| for SinhCylindrical (f0 = rho; the second
// rfm function holds z'(xx2)).
__device__ __forceinline__ double volume_element(const RfmArrays &rfm, const int cyl, const int i0, const int i1,
                                                 const int i2, const double dvol) {
  const double f0 = rfm.f0[i0];
  if (cyl) return fabs(rfm.f0_D0[i0] * f0 * rfm.f1[i2]) * dvol;
  return fabs(rfm.f0_D0[i0] * f0 * f0 * rfm.f1[i1]) * dvol;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(kRedThreads) constraint_partials_kernel(const GridDims g, const RfmArrays rfm,
                                                                          const int cyl, const double dvol,
                                                                          const double *__restrict__ diag,
                                                                          double *__restrict__ partials) {
  const int n0 = g.N0 - 2 * NGHOSTS, n1 = g.N1 - 2 * NGHOSTS, n2 = g.N2 - 2 * NGHOSTS;
  const long long n = (long long)n0 * n1 * n2;
  double acc[kRedVals] = {0.0, 0.0, 0.0, 0.0};
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i0 = NGHOSTS + (int)(t % n0);
    const long long q = t / n0;
    const int i1 = NGHOSTS + (int)(q % n1);
    const int i2 = NGHOSTS + (int)(q / n1);
    const int idx = i0 + g.s1 * i1 + g.s2 * i2;
    const double dV = volume_element(rfm, cyl, i0, i1, i2, dvol);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const double f = diag[idx + (size_t)k * g.ntot];
      acc[k] += f * f * dV;
    }
    acc[3] += dV;
  }
  __shared__ double sh[kRedVals][kRedThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kRedVals; k++) {
    const double w = warp_sum(acc[k]);
    if (lane == 0) sh[k][warp] = w;
  }
  __syncthreads();
  if (threadIdx.x < kRedVals) {
    double s = 0.0;
    for (int w = 0; w < kRedThreads / 32; w++) s += sh[threadIdx.x][w];
    partials[blockIdx.x * kRedVals + threadIdx.x] = s;
  }
}

__global__ void sum_partials_kernel(const double *__restrict__ partials, const int nblocks,
                                    double *__restrict__ out) {
  // One warp per value; lanes stride the partials, then a fixed-order shuffle tree.
  const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (k >= kRedVals) return;
  double s = 0.0;
  for (int b = lane; b < nblocks; b += 32) s += partials[b * kRedVals + k];
  s = warp_sum(s);
  if (lane == 0) out[k] = s;
}

// scratch: kRedBlocks * kRedVals + kRedVals doubles of device memory.
int constraint_integrals(const params_struct *p, const RfmArrays &rfm, const double *diag, double *scratch,
                         double out[4], cudaStream_t s) {
  const GridDims g = grid_dims(p);
  if (g.N0 <= 2 * NGHOSTS || g.N1 <= 2 * NGHOSTS || g.N2 <= 2 * NGHOSTS) {
    for (int k = 0; k < 4; k++) out[k] = 0.0;
    return BSSN_B200_OK;
  }
  const double dvol = fabs(p->dxx0 * p->dxx1 * p->dxx2);
  const int cyl = p->CoordSystem_hash == SINHCYLINDRICAL;
  constraint_partials_kernel<<<kRedBlocks, kRedThreads, 0, s>>>(g, rfm, cyl, dvol, diag, scratch);
  BSSN_LAUNCH_CHECK();
  double *res = scratch + kRedBlocks * kRedVals;
  sum_partials_kernel<<<1, 32 * kRedVals, 0, s>>>(scratch, kRedBlocks, res);
  BSSN_LAUNCH_CHECK();
  BSSN_CUDA_TRY(cudaMemcpyAsync(out, res, sizeof(double) * kRedVals, cudaMemcpyDeviceToHost, s));
  BSSN_CUDA_TRY(cudaStreamSynchronize(s));
  return BSSN_B200_OK;
}

size_t constraint_integrals_scratch_doubles() { return (size_t)kRedBlocks * kRedVals + kRedVals; }

// ---------------------------------------------------------------- allocation-free variant
// Same integrals, for callers that must not allocate device memory: code running inside
// a host framework that owns every allocation (a memory pool or arena that a foreign
// cudaMalloc would bypass, breaking its accounting and its memory cap), or embedded hosts
// that forbid allocation after start-up so that the footprint stays fixed. The call itself
// allocates nothing. The partial sums live in a file-scope
// __device__ array instead: one partial per block of kNoAllocPtsPerBlock interior points,
// at most kNoAllocMaxBlocks blocks, i.e. grids of up to
// kNoAllocMaxBlocks * kNoAllocPtsPerBlock = 33,554,432 interior points (512 KiB + 32 B of
// device memory, held by every GPU that loads the library until the process exits).
constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocPtsPerThread = 8;
constexpr int kNoAllocPtsPerBlock = kNoAllocThreads * kNoAllocPtsPerThread;
constexpr int kNoAllocMaxBlocks = 16384;
static __device__ __align__(256) double g_noalloc_scratch[(size_t)kNoAllocMaxBlocks * kRedVals + kRedVals];

// Block b sums interior points [b*kNoAllocPtsPerBlock, (b+1)*kNoAllocPtsPerBlock) in a fixed
// order and writes its own partial; nothing accumulates across blocks or calls, so no entry
// has to start at zero.
__global__ void __launch_bounds__(kNoAllocThreads) constraint_partials_blocked_kernel(
    const GridDims g, const RfmArrays rfm, const int cyl, const double dvol, const double *__restrict__ diag,
    double *__restrict__ partials) {
  const int n0 = g.N0 - 2 * NGHOSTS, n1 = g.N1 - 2 * NGHOSTS, n2 = g.N2 - 2 * NGHOSTS;
  const long long n = (long long)n0 * n1 * n2;
  double acc[kRedVals] = {0.0, 0.0, 0.0, 0.0};
  const long long base = (long long)blockIdx.x * kNoAllocPtsPerBlock;
  for (int j = 0; j < kNoAllocPtsPerThread; j++) {
    const long long t = base + (long long)j * kNoAllocThreads + threadIdx.x;
    if (t >= n) break;
    const int i0 = NGHOSTS + (int)(t % n0);
    const long long q = t / n0;
    const int i1 = NGHOSTS + (int)(q % n1);
    const int i2 = NGHOSTS + (int)(q / n1);
    const int idx = i0 + g.s1 * i1 + g.s2 * i2;
    const double dV = volume_element(rfm, cyl, i0, i1, i2, dvol);
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const double f = diag[idx + (size_t)k * g.ntot];
      acc[k] += f * f * dV;
    }
    acc[3] += dV;
  }
  __shared__ double sh[kRedVals][kNoAllocThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kRedVals; k++) {
    const double w = warp_sum(acc[k]);
    if (lane == 0) sh[k][warp] = w;
  }
  __syncthreads();
  if (threadIdx.x < kRedVals) {
    double sum = 0.0;
    for (int w = 0; w < kNoAllocThreads / 32; w++) sum += sh[threadIdx.x][w];
    partials[blockIdx.x * kRedVals + threadIdx.x] = sum;
  }
}

long long constraint_integrals_noalloc_max_points() { return (long long)kNoAllocMaxBlocks * kNoAllocPtsPerBlock; }

// Device address of g_noalloc_scratch, looked up once per device with that device current
// and kept for the life of the process: after a cudaDeviceReset (or any other teardown of
// the device's primary context) the kept address is stale, so the library must not be used
// across one.
static double *noalloc_scratch_address(int *rc) {
  static std::mutex mu;
  static double *addr[64] = {nullptr};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) {
    set_error("no-alloc integrals: cudaGetDevice failed (%s)", cudaGetErrorString(e));
    *rc = BSSN_B200_ECUDA;
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(mu);
  if (!addr[dev]) {
    double *p = nullptr;
    e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_error("no-alloc integrals: cudaGetSymbolAddress failed on device %d (%s)", dev, cudaGetErrorString(e));
      *rc = BSSN_B200_ECUDA;
      return nullptr;
    }
    addr[dev] = p;
  }
  *rc = BSSN_B200_OK;
  return addr[dev];
}

int constraint_integrals_noalloc(const params_struct *p, const RfmArrays &rfm, const double *diag, double out[4],
                                 cudaStream_t s) {
  const GridDims g = grid_dims(p);
  if (g.N0 <= 2 * NGHOSTS || g.N1 <= 2 * NGHOSTS || g.N2 <= 2 * NGHOSTS) {
    for (int k = 0; k < 4; k++) out[k] = 0.0;
    return BSSN_B200_OK;
  }
  const long long n = (long long)(g.N0 - 2 * NGHOSTS) * (g.N1 - 2 * NGHOSTS) * (g.N2 - 2 * NGHOSTS);
  if (n > constraint_integrals_noalloc_max_points()) {
    set_error("no-alloc integrals: %lld interior points exceed the static scratch limit of %lld points", n,
              constraint_integrals_noalloc_max_points());
    return BSSN_B200_EINVAL;
  }
  int rc = BSSN_B200_OK;
  double *scratch = noalloc_scratch_address(&rc);
  if (rc != BSSN_B200_OK) return rc;
  const int nblocks = (int)((n + kNoAllocPtsPerBlock - 1) / kNoAllocPtsPerBlock);
  const double dvol = fabs(p->dxx0 * p->dxx1 * p->dxx2);
  const int cyl = p->CoordSystem_hash == SINHCYLINDRICAL;
  constraint_partials_blocked_kernel<<<nblocks, kNoAllocThreads, 0, s>>>(g, rfm, cyl, dvol, diag, scratch);
  BSSN_LAUNCH_CHECK();
  double *res = scratch + (size_t)kNoAllocMaxBlocks * kRedVals;
  sum_partials_kernel<<<1, 32 * kRedVals, 0, s>>>(scratch, nblocks, res);
  BSSN_LAUNCH_CHECK();
  BSSN_CUDA_TRY(cudaMemcpyAsync(out, res, sizeof(double) * kRedVals, cudaMemcpyDeviceToHost, s));
  BSSN_CUDA_TRY(cudaStreamSynchronize(s));
  return BSSN_B200_OK;
}


// ---------------------------------------------------------------- FP64 FMA throughput
// Eight independent FMA chains per thread keep every FP64 lane busy without memory traffic;
// x <- x*a + b with |a| < 1 stays bounded. One double per block is stored so that the chains
// are not removed.
constexpr int FMA_THREADS = 256, FMA_CHAINS = 8, FMA_ITERS = 4096;

__global__ void __launch_bounds__(FMA_THREADS) fma_chain_kernel(double *__restrict__ out, const double a,
                                                                const double b) {
  double x[FMA_CHAINS];
#pragma unroll
  for (int c = 0; c < FMA_CHAINS; c++) x[c] = 1e-3 * (threadIdx.x + c);
  for (int i = 0; i < FMA_ITERS; i++) {
#pragma unroll
    for (int c = 0; c < FMA_CHAINS; c++) x[c] = fma(x[c], a, b);
  }
  double sum = 0.0;
#pragma unroll
  for (int c = 0; c < FMA_CHAINS; c++) sum += x[c];
  if (threadIdx.x == 0) out[blockIdx.x] = sum;
}

int fp64_fma_rate(int reps, double *out_tflops, cudaStream_t s) {
  int dev = 0, sms = 0;
  BSSN_CUDA_TRY(cudaGetDevice(&dev));
  BSSN_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int blocks = sms * 16;
  double *out = nullptr;
  BSSN_CUDA_TRY(cudaMalloc(&out, sizeof(double) * blocks));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = BSSN_B200_OK;
  float best = 0.0f;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    set_error("fp64_fma_rate: event creation failed");
    rc = BSSN_B200_ECUDA;
  }
  for (int r = -1; r < reps && rc == BSSN_B200_OK; r++) {  // r = -1: warm-up
    cudaEventRecord(e0, s);
    fma_chain_kernel<<<blocks, FMA_THREADS, 0, s>>>(out, 0.999999, 1e-7);
    cudaEventRecord(e1, s);
    if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
      set_error("fp64_fma_rate: kernel failed");
      rc = BSSN_B200_ECUDA;
      break;
    }
    count_launch(1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r >= 0 && (best == 0.0f || ms < best)) best = ms;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(out);
  if (rc != BSSN_B200_OK) return rc;
  const double flop = 2.0 * FMA_CHAINS * (double)FMA_ITERS * FMA_THREADS * blocks;
  *out_tflops = flop / (best * 1e-3) / 1e12;
  return BSSN_B200_OK;
}

}  // namespace bssn
