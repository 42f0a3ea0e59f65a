// Volume integrals of the constraint diagnostics over the grid interior, FP64, deterministic.
//
// Reference: diagnostics_volume_integration_helpers.h:400-470 -- sum over interior points of
// f^2 dV with dV = sqrt(det gammahat) |dxx0 dxx1 dxx2|. For the Spherical family
// sqrt(det gammahat) = |f0' f0^2 f1| (f0 = r(xx0), f1 = sin(xx1)), evaluated from the rfm
// precompute arrays. Each block reduces a fixed slice of the interior with warp shuffles
// into a partial; a single block then adds the partials in a fixed order, so the result
// does not depend on scheduling.
#include "bssn_common.cuh"

namespace bssn {

constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 296;  // 2 x 148 SMs
constexpr int kRedVals = 4;      // H^2 dV, (M^2)^2 dV, |Lambda|^2 dV, dV

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(kRedThreads) constraint_partials_kernel(const GridDims g, const RfmArrays rfm,
                                                                          const double dvol,
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
    const double f0 = rfm.f0[i0];
    const double dV = fabs(rfm.f0_D0[i0] * f0 * f0 * rfm.f1[i1]) * dvol;
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
  constraint_partials_kernel<<<kRedBlocks, kRedThreads, 0, s>>>(g, rfm, dvol, diag, scratch);
  BSSN_LAUNCH_CHECK();
  double *res = scratch + kRedBlocks * kRedVals;
  sum_partials_kernel<<<1, 32 * kRedVals, 0, s>>>(scratch, kRedBlocks, res);
  BSSN_LAUNCH_CHECK();
  BSSN_CUDA_TRY(cudaMemcpyAsync(out, res, sizeof(double) * kRedVals, cudaMemcpyDeviceToHost, s));
  BSSN_CUDA_TRY(cudaStreamSynchronize(s));
  return BSSN_B200_OK;
}

size_t constraint_integrals_scratch_doubles() { return (size_t)kRedBlocks * kRedVals + kRedVals; }

}  // namespace bssn
