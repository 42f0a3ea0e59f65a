"""Time candidate output groups and value allocations of the point kernels on a GPU.

Code-generation-time tuning tool (the output-group split and the per-group allocation
flags in generate.py come from its measurements). Three steps:

  python -m nrpy_b200.codegen.tune_groups generate   # needs nrpy (equation modules)
  python -m nrpy_b200.codegen.tune_groups generate-orders  # present groups x statement orders
  python -m nrpy_b200.codegen.tune_groups generate-caps    # present groups x register budgets
  python -m nrpy_b200.codegen.tune_groups generate-leaf    # present groups on precomputed FD leaves
  python -m nrpy_b200.codegen.tune_groups generate-staged  # Ricci groups on shared-memory tiles
  python -m nrpy_b200.codegen.tune_groups compile    # nvcc, sm_100a, no GPU needed
  python -m nrpy_b200.codegen.tune_groups run        # on a B200; prints one line per kernel

`generate` emits every candidate group (Ricci: 1x6, 2x3, 3x2 (two pairings), 6x1 outputs;
RHS: gauge/metric/extrinsic-curvature outputs merged or split in two or three parts) of the
SinhSpherical 3-D algebra under three allocations (remat_first, deriv_remat) = (1,1),
(1,0), (0,0) at a 90-value register budget, plus lower budgets with forced occupancy for
the present groups. `compile` builds one timing executable per group into
nrpy_b200/_tune/. `run` times each kernel alone on a 256x64x32 interior grid (+3 ghosts)
of seeded values (median of 5 launches, CUDA events) and reports registers, local
memory, slots and resident warps.
"""

import argparse
import concurrent.futures as cf
import json
import os
import pathlib
import subprocess
import sys

ROOT = pathlib.Path(__file__).resolve().parents[2]
OUT = ROOT / "nrpy_b200" / "_tune"

R = ["RbarDD00", "RbarDD01", "RbarDD02", "RbarDD11", "RbarDD12", "RbarDD22"]
A = ["aDD00", "aDD01", "aDD02", "aDD11", "aDD12", "aDD22"]
G1 = ["alpha", "cf", "hDD00", "hDD01", "hDD02", "hDD11", "hDD12", "hDD22", "trK", "vetU0", "vetU1", "vetU2"]
G2 = ["betU0", "betU1", "betU2", "lambdaU0", "lambdaU1", "lambdaU2"]
CANDIDATES = {
    "ricci_1x6": ("ricci", R),
    "ricci_012": ("ricci", R[:3]), "ricci_345": ("ricci", R[3:]),
    "ricci_0001": ("ricci", R[0:2]), "ricci_0211": ("ricci", R[2:4]), "ricci_1222": ("ricci", R[4:6]),
    "ricci_0011": ("ricci", [R[0], R[3]]), "ricci_0112": ("ricci", [R[1], R[4]]), "ricci_0222": ("ricci", [R[2], R[5]]),
    **{f"ricci_{k}": ("ricci", [k]) for k in R},
    "rhs_a": ("rhs", A), "rhs_a3a": ("rhs", A[:3]), "rhs_a3b": ("rhs", A[3:]),
    "rhs_g1": ("rhs", G1), "rhs_g1_scalar_vet": ("rhs", ["alpha", "cf", "trK", "vetU0", "vetU1", "vetU2"]),
    "rhs_g1_h": ("rhs", G1[2:8]), "rhs_g1_scalar": ("rhs", ["alpha", "cf", "trK"]), "rhs_vet": ("rhs", G1[9:]),
    "rhs_a_g1": ("rhs", A + G1), "rhs_a_scalar": ("rhs", A + ["alpha", "cf", "trK"]),
    "rhs_h_vet": ("rhs", G1[2:8] + G1[9:]),
    "rhs_g2": ("rhs", G2), "rhs_lambda": ("rhs", G2[3:]), "rhs_bet": ("rhs", G2[:3]),
}
ALLOCS = [(90, True, True, 1), (90, True, False, 1), (90, False, False, 1)]
# lower register budgets with forced occupancy (launch_bounds min blocks per SM of 128 threads)
LOW = [(60, True, True, 3), (48, True, True, 4)]
LOW_GROUPS = {"ricci_0001", "ricci_0211", "ricci_1222", "rhs_a", "rhs_g1", "rhs_g2"}

HARNESS_HEAD = r'''
#ifndef TUNE_NG
#define TUNE_NG 3
#endif
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <cuda_runtime.h>
struct RfmArrays { const double *f0, *f0_D0, *f0_DD00, *f0_DDD000, *f1, *f1_D1, *f1_DD11; };
template <typename T> __device__ __forceinline__ T ipow(T x, int n) { T r = x; for (int k = 1; k < n; k++) r *= x; return r; }
struct PointCtx {
  const double *__restrict__ in; const double *__restrict__ aux; int s1, s2, ntot; int i0, i1;
  double invdxx0, invdxx1, invdxx2; RfmArrays rfm; double eta, KreissOliger_strength_gauge, KreissOliger_strength_nongauge;
  __device__ __forceinline__ double ld(int gf, int a, int b, int c) const { return __ldg(in + (gf * ntot + (a + b * s1 + c * s2))); }
  __device__ __forceinline__ double ldaux(int k) const { return __ldg(aux + k * ntot); }
};
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
#define SMEM(k) sm[(k) * NT]
#define invdxx0 ctx.invdxx0
#define invdxx1 ctx.invdxx1
#define invdxx2 ctx.invdxx2
#include "GROUP.cuh"
#undef invdxx0
#undef invdxx1
#undef invdxx2
constexpr int NG = TUNE_NG, N0 = 256 + 2 * NG, N1 = 64 + 2 * NG, N2 = 32 + 2 * NG, NTOT = N0 * N1 * N2, MAXOUT = 18;
template <typename VT, int NT, int MINB, int NOUT, class F>
__global__ void __launch_bounds__(NT, MINB) kern(RfmArrays rfm, const double *in, const double *aux, double *out) {
  const int i0 = NG + blockIdx.x * 32 + threadIdx.x, i1 = NG + blockIdx.y * (NT / 32) + threadIdx.y, i2 = NG + blockIdx.z;
  if (i0 >= N0 - NG || i1 >= N1 - NG) return;
  extern __shared__ double smem[];
  volatile VT *sm = reinterpret_cast<VT *>(smem) + threadIdx.x + 32 * threadIdx.y;
  const int idx = i0 + N0 * i1 + N0 * N1 * i2;
  PointCtx ctx;
  ctx.in = in + idx; ctx.aux = aux + idx; ctx.s1 = N0; ctx.s2 = N0 * N1; ctx.ntot = NTOT; ctx.i0 = i0; ctx.i1 = i1;
  ctx.invdxx0 = 10.0; ctx.invdxx1 = 20.0; ctx.invdxx2 = 5.0; ctx.rfm = rfm; ctx.eta = 1.0;
  ctx.KreissOliger_strength_gauge = 0.3; ctx.KreissOliger_strength_nongauge = 0.3;
  VT o[NOUT];
  F::template eval<NT>(ctx, o, sm);
#pragma unroll
  for (int k = 0; k < NOUT; k++) out[idx + k * NTOT] = (double)o[k];
}
template <typename VT, int NT, int MINB, int NOUT, int SLOTS, class F>
void run(const char *name, RfmArrays rfm, const double *in, const double *aux, double *out) {
  auto K = kern<VT, NT, MINB, NOUT, F>;
  const size_t sb = (size_t)SLOTS * NT * sizeof(VT);
  if (sb > 227 * 1024) { printf("{\"kernel\": \"%s\", \"skip\": \"shared memory\"}\n", name); return; }
  if (cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb) != cudaSuccess) return;
  cudaFuncAttributes at;
  cudaFuncGetAttributes(&at, K);
  int nb = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, K, NT, sb);
  const dim3 grid(8, 64 / (NT / 32), 32);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  for (int w = 0; w < 2; w++) K<<<grid, dim3(32, NT / 32), sb>>>(rfm, in, aux, out);
  std::vector<float> ts;
  for (int r = 0; r < 5; r++) {
    cudaEventRecord(a);
    K<<<grid, dim3(32, NT / 32), sb>>>(rfm, in, aux, out);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms;
    cudaEventElapsedTime(&ms, a, b);
    ts.push_back(ms);
  }
  std::sort(ts.begin(), ts.end());
  const cudaError_t e = cudaGetLastError();
  printf("{\"kernel\": \"%s\", \"threads\": %d, \"min_blocks\": %d, \"regs\": %d, \"local_bytes\": %zu, \"slots\": %d, "
         "\"warps_per_sm\": %d, \"us\": %.1f, \"error\": \"%s\"}\n", name, NT, MINB, at.numRegs, at.localSizeBytes, SLOTS,
         nb * NT / 32, ts[2] * 1e3, e == cudaSuccess ? "" : cudaGetErrorString(e));
}
int main() {
  std::vector<double> h((size_t)NTOT * 24);
  srand(7);
  for (auto &x : h) x = 0.5 + (double)rand() / RAND_MAX;
  double *in, *aux, *out, *r[7];
  cudaMalloc(&in, h.size() * 8);
  cudaMemcpy(in, h.data(), h.size() * 8, cudaMemcpyHostToDevice);
  cudaMalloc(&aux, (size_t)NTOT * 6 * 8);
  cudaMemcpy(aux, h.data(), (size_t)NTOT * 6 * 8, cudaMemcpyHostToDevice);
  cudaMalloc(&out, (size_t)NTOT * MAXOUT * 8);
  for (int k = 0; k < 7; k++) {
    cudaMalloc(&r[k], 300 * 8);
    cudaMemcpy(r[k], h.data() + 1000 * k, 300 * 8, cudaMemcpyHostToDevice);
  }
  RfmArrays rfm{r[0], r[1], r[2], r[3], r[4], r[5], r[6]};
'''


def generate() -> None:
    from nrpy_b200.codegen import bssn_exprs as be
    from nrpy_b200.codegen.emit_cuda import emit_point_function

    be.setup_nrpy("")
    rhs, betaU = be.rhs_exprs("SinhSpherical")
    ricci = be.ricci_exprs("SinhSpherical")
    OUT.mkdir(parents=True, exist_ok=True)
    for gname, (kind, names) in CANDIDATES.items():
        src, uv = (ricci, None) if kind == "ricci" else (rhs, betaU)
        allocs = ALLOCS + (LOW if gname in LOW_GROUPS else [])
        parts, wrappers, calls = ["#pragma once\n"], [], []
        for cap, rf, dr, minb in allocs:
            fname = f"{gname}_c{cap}_r{int(rf)}_d{int(dr)}"
            code, st = emit_point_function(fname, [(f"out[{i}]", src[n]) for i, n in enumerate(names)],
                                           upwind_vec=uv, reg_capacity=cap, remat_first=rf, deriv_remat=dr)
            parts.append(code)
            slots = max(st["smem_slots"], 1)
            wrappers.append(f"struct W_{fname} {{ template <int NT, class C, class VT> __device__ __forceinline__ static void "
                            f"eval(const C &c, VT *o, volatile VT *sm) {{ {fname}<VT, double, NT>(c, o, sm); }} }};")
            nt = 128 if 2 * slots * 8 * 128 <= 227 * 1024 else 64
            launches = [(nt, minb)] if minb == 1 else [(128, minb), (64, 2 * minb)]
            if minb == 1 and nt == 128:
                launches.append((64, 1))
            for t, mb in launches:
                calls.append(f'  run<double, {t}, {mb}, {len(names)}, {slots}, W_{fname}>("{fname}", rfm, in, aux, out);')
        (OUT / f"{gname}.cuh").write_text("\n".join(parts))
        head, main = HARNESS_HEAD.replace("GROUP", gname).split("int main() {")
        body = head + "\n".join(wrappers) + "\nint main() {" + main
        (OUT / f"{gname}.cu").write_text(body + "\n".join(calls) + "\n  return 0;\n}\n")
        print(gname, flush=True)


ORDER_GROUPS = ["ricci_012", "ricci_345", "rhs_a_g1", "rhs_g2"]
ORDERS = ["dfs", "sched", "sched_dfs"]


def generate_orders() -> None:
    """The present groups under each statement order and the two recompute-first allocations."""
    from nrpy_b200.codegen import bssn_exprs as be
    from nrpy_b200.codegen.emit_cuda import emit_point_function

    be.setup_nrpy("")
    rhs, betaU = be.rhs_exprs("SinhSpherical")
    ricci = be.ricci_exprs("SinhSpherical")
    OUT.mkdir(parents=True, exist_ok=True)
    for gname in ORDER_GROUPS:
        kind, names = CANDIDATES[gname]
        src, uv = (ricci, None) if kind == "ricci" else (rhs, betaU)
        parts, wrappers, calls = ["#pragma once\n"], [], []
        for order in ORDERS:
            for rf, dr in ((True, True), (True, False)):
                fname = f"{gname}_{order}_r{int(rf)}_d{int(dr)}"
                code, st = emit_point_function(fname, [(f"out[{i}]", src[n]) for i, n in enumerate(names)],
                                               upwind_vec=uv, reg_capacity=90, remat_first=rf, deriv_remat=dr,
                                               order=order)
                parts.append(code)
                slots = max(st["smem_slots"], 1)
                wrappers.append(f"struct W_{fname} {{ template <int NT, class C, class VT> __device__ __forceinline__ static void "
                                f"eval(const C &c, VT *o, volatile VT *sm) {{ {fname}<VT, double, NT>(c, o, sm); }} }};")
                nt = 128 if 2 * slots * 8 * 128 <= 227 * 1024 else 64
                calls.append(f'  run<double, {nt}, 1, {len(names)}, {slots}, W_{fname}>("{fname}", rfm, in, aux, out);')
        tag = f"order_{gname}"
        (OUT / f"{tag}.cuh").write_text("\n".join(parts))
        head, main = HARNESS_HEAD.replace("GROUP", tag).split("int main() {")
        (OUT / f"{tag}.cu").write_text(head + "\n".join(wrappers) + "\nint main() {" + main + "\n".join(calls)
                                        + "\n  return 0;\n}\n")
        print(tag, flush=True)


def generate_caps(caps, fd_order: int = 4, dtype: str = "double", groups=None) -> None:
    """The present groups with their chosen allocation and order (generate.py) at several
    register budgets, at the given finite-difference order, evaluated in `dtype` (double, or
    float as the mixed-precision kernels run them: FP32 algebra on FP64 finite differences,
    with the slot qualifier generate.py gives FP32 groups). `groups` names other candidate
    groups (CANDIDATES) to time instead of the present ones; they get the allocation of the
    present first group of their kind."""
    from nrpy_b200.codegen import bssn_exprs as be
    from nrpy_b200.codegen import fdcoeffs as fdc
    from nrpy_b200.codegen.emit_cuda import emit_point_function
    from nrpy_b200.codegen.generate import RHS_ALLOC, RHS_PLAIN_SLOTS, RICCI_ALLOC, RICCI_PLAIN_SLOTS

    fdc.set_fd_order(fd_order)
    be.setup_nrpy("", fd_order)
    rhs, betaU = be.rhs_exprs("SinhSpherical")
    ricci = be.ricci_exprs("SinhSpherical")
    OUT.mkdir(parents=True, exist_ok=True)
    chosen = dict(zip(ORDER_GROUPS, list(RICCI_ALLOC) + list(RHS_ALLOC)))
    plain = dict(zip(ORDER_GROUPS, [dtype in t for t in list(RICCI_PLAIN_SLOTS) + list(RHS_PLAIN_SLOTS)]))
    for gname in groups or []:
        kind = CANDIDATES[gname][0]
        chosen.setdefault(gname, RICCI_ALLOC[0] if kind == "ricci" else RHS_ALLOC[0])
        plain.setdefault(gname, dtype in (RICCI_PLAIN_SLOTS[0] if kind == "ricci" else RHS_PLAIN_SLOTS[0]))
    vbytes = 4 if dtype == "float" else 8
    for gname in groups or ORDER_GROUPS:
        kind, names = CANDIDATES[gname]
        src, uv = (ricci, None) if kind == "ricci" else (rhs, betaU)
        rf, dr, order = chosen[gname]
        parts, wrappers, calls = ["#pragma once\n"], [], []
        for cap in caps:
            fname = f"{gname}_c{cap}"
            code, st = emit_point_function(fname, [(f"out[{i}]", src[n]) for i, n in enumerate(names)],
                                           upwind_vec=uv, reg_capacity=cap, remat_first=rf, deriv_remat=dr, order=order)
            parts.append(code)
            slots = max(st["smem_slots"], 1)
            smp = "const_cast<VT *>(sm)" if plain[gname] else "sm"
            wrappers.append(f"struct W_{fname} {{ template <int NT, class C, class VT> __device__ __forceinline__ static void "
                            f"eval(const C &c, VT *o, volatile VT *sm) {{ {fname}<VT, double, NT>(c, o, {smp}); }} }};")
            nt = 128 if 2 * slots * vbytes * 128 <= 227 * 1024 else 64
            calls.append(f'  run<{dtype}, {nt}, 1, {len(names)}, {slots}, W_{fname}>("{fname}", rfm, in, aux, out);')
        tag = (f"caps_{gname}" if fd_order == 4 else f"caps{fd_order}_{gname}") + ("_f32" if dtype == "float" else "")
        (OUT / f"{tag}.cuh").write_text("\n".join(parts))
        head, main = HARNESS_HEAD.replace("GROUP", tag).replace("#define TUNE_NG 3", f"#define TUNE_NG {fdc.NGHOSTS}"
                                                                 ).split("int main() {")
        (OUT / f"{tag}.cu").write_text(head + "\n".join(wrappers) + "\nint main() {" + main + "\n".join(calls)
                                        + "\n  return 0;\n}\n")
        print(tag, flush=True)


LEAF_CAPS = (64, 72, 90, 120, 160)


def generate_leaf() -> None:
    """The present groups reading precomputed finite-difference leaves (one array per leaf,
    LDLEAF) at several register budgets, beside their stencil form, and the kernel that
    computes every leaf from stencils (LEAFOUT): is precomputing the derivatives cheaper
    than evaluating them in each group?"""
    from nrpy_b200.codegen import bssn_exprs as be
    from nrpy_b200.codegen.emit_cuda import emit_leaf_function, emit_point_function, leaf_names
    from nrpy_b200.codegen.generate import RHS_ALLOC, RHS_CAPS, RICCI_ALLOC, RICCI_CAPS

    be.setup_nrpy("")
    rhs, betaU = be.rhs_exprs("SinhSpherical")
    ricci = be.ricci_exprs("SinhSpherical")
    names = leaf_names(list(rhs.values()) + list(ricci.values()))
    index = {n: k for k, n in enumerate(names)}
    OUT.mkdir(parents=True, exist_ok=True)
    head = HARNESS_HEAD
    for a, b in (
        ("double eta, KreissOliger_strength_gauge, KreissOliger_strength_nongauge;",
         "double eta, KreissOliger_strength_gauge, KreissOliger_strength_nongauge; const double *__restrict__ leaf; "
         "double *leafout;"),
        ("#define LDAUX(k) ctx.ldaux(k)", "#define LDAUX(k) ctx.ldaux(k)\n#define LDLEAF(k) __ldg(ctx.leaf + (size_t)(k) * NTOT)"
         "\n#define LEAFOUT(k, v) ctx.leafout[(size_t)(k) * NTOT] = (v)"),
        ("constexpr int NG = TUNE_NG, N0 = 256 + 2 * NG, N1 = 64 + 2 * NG, N2 = 32 + 2 * NG, NTOT = N0 * N1 * N2, "
         "MAXOUT = 18;\n", ""),
        ('#include "GROUP.cuh"', 'constexpr int NG = TUNE_NG, N0 = 256 + 2 * NG, N1 = 64 + 2 * NG, N2 = 32 + 2 * NG, '
         'NTOT = N0 * N1 * N2, MAXOUT = 18;\n#include "GROUP.cuh"'),
        ("ctx.KreissOliger_strength_nongauge = 0.3;",
         "ctx.KreissOliger_strength_nongauge = 0.3; ctx.leaf = g_leaf + idx; ctx.leafout = g_leaf + idx;"),
        ("template <int NT, int MINB, int NOUT, class F>\n__global__",
         "__device__ double *g_leaf;\ntemplate <int NT, int MINB, int NOUT, class F>\n__global__"),
    ):
        assert a in head
        head = head.replace(a, b, 1)
    parts, wrappers, calls = ["#pragma once\n"], [], []
    parts.append(emit_leaf_function("leaf_all", names, upwind_vec=betaU)[0])
    chosen = dict(zip(ORDER_GROUPS, zip(list(RICCI_ALLOC) + list(RHS_ALLOC), list(RICCI_CAPS) + list(RHS_CAPS))))
    for gname in ORDER_GROUPS:
        kind, gn = CANDIDATES[gname]
        src, uv = (ricci, None) if kind == "ricci" else (rhs, betaU)
        (rf, dr, order), cap0 = chosen[gname]
        for tag, cap, li in [("stencil", cap0, None)] + [(f"leaf{c}", c, index) for c in LEAF_CAPS]:
            fname = f"{gname}_{tag}"
            code, st = emit_point_function(fname, [(f"out[{i}]", src[n]) for i, n in enumerate(gn)], upwind_vec=uv,
                                           reg_capacity=cap, remat_first=rf, deriv_remat=dr, order=order, leaf_index=li)
            parts.append(code)
            slots = max(st["smem_slots"], 1)
            wrappers.append(f"struct W_{fname} {{ template <int NT, class C, class VT> __device__ __forceinline__ static void "
                            f"eval(const C &c, VT *o, volatile VT *sm) {{ {fname}<VT, double, NT>(c, o, sm); }} }};")
            nt = 128 if 2 * slots * 8 * 128 <= 227 * 1024 else 64
            calls.append(f'  run<double, {nt}, 1, {len(gn)}, {slots}, W_{fname}>("{fname}", rfm, in, aux, out);')
    wrappers.append("struct W_leaf { template <int NT, class C, class VT> __device__ __forceinline__ static void "
                    "eval(const C &c, VT *o, volatile VT *sm) { leaf_all<double, double>(c); o[0] = 0.0; } };")
    calls.append('  run<double, 128, 1, 1, 1, W_leaf>("leaf_all", rfm, in, aux, out);')
    (OUT / "leaf.cuh").write_text("\n".join(parts))
    h, m = head.replace("GROUP", "leaf").split("int main() {")
    n = len(names)
    m = m.replace("RfmArrays rfm{",
                  f"double *lb; cudaMalloc(&lb, (size_t)NTOT * {n} * 8);\n"
                  f"  for (int k = 0; k < {n}; k++) cudaMemcpy(lb + (size_t)k * NTOT, in + (size_t)(k % 24) * NTOT, "
                  "(size_t)NTOT * 8, cudaMemcpyDeviceToDevice);\n"
                  "  cudaMemcpyToSymbol(g_leaf, &lb, sizeof(lb));\n  RfmArrays rfm{", 1)
    (OUT / "leaf.cu").write_text(h + "\n".join(wrappers) + "\nint main() {" + m + "\n".join(calls) + "\n  return 0;\n}\n")
    print(f"leaf: {n} leaves", flush=True)


STAGED_HARNESS = r'''// Feasibility: Ricci group kernels reading their 9 stencil gridfunctions (hDD, lambdaU) from a
// shared-memory copy of the tile plus a 2-point halo, against the same groups reading global memory.
#define TUNE_NG 3
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <cuda_runtime.h>
struct RfmArrays { const double *f0, *f0_D0, *f0_DD00, *f0_DDD000, *f1, *f1_D1, *f1_DD11; };
template <typename T> __device__ __forceinline__ T ipow(T x, int n) { T r = x; for (int k = 1; k < n; k++) r *= x; return r; }
struct PointCtx {
  const double *__restrict__ in; const double *__restrict__ aux; int s1, s2, ntot; int i0, i1;
  double invdxx0, invdxx1, invdxx2; RfmArrays rfm;
  __device__ __forceinline__ double ld(int gf, int a, int b, int c) const { return __ldg(in + (gf * ntot + (a + b * s1 + c * s2))); }
};
template <int SX, int SY, int SZ>
struct SmemCtx {
  const double *s;  // this thread's centre in the staged box of gridfunction 11
  int i0, i1;
  double invdxx0, invdxx1, invdxx2; RfmArrays rfm;
  __device__ __forceinline__ double ld(int gf, int a, int b, int c) const {
    return s[(gf - 11) * (SX * SY * SZ) + c * (SX * SY) + b * SX + a];
  }
};
#define LD(gf, a, b, c) ctx.ld(gf, a, b, c)
#define RFM(arr, d) __ldg(ctx.rfm.arr + ctx.i##d)
#define rfm_f0 f0
#define rfm_f0_D0 f0_D0
#define rfm_f0_DD00 f0_DD00
#define rfm_f0_DDD000 f0_DDD000
#define rfm_f1 f1
#define rfm_f1_D1 f1_D1
#define rfm_f1_DD11 f1_DD11
#define PARAM(name) ctx.name
#define SMEM(k) sm[(k) * NT]
#define invdxx0 ctx.invdxx0
#define invdxx1 ctx.invdxx1
#define invdxx2 ctx.invdxx2
#include "staged_ricci.cuh"
#undef invdxx0
#undef invdxx1
#undef invdxx2
constexpr int NG = TUNE_NG, N0 = 256 + 2 * NG, N1 = 64 + 2 * NG, N2 = 32 + 2 * NG, NTOT = N0 * N1 * N2;
struct G0 { template <int NT, class C, class S> __device__ __forceinline__ static void eval(const C &c, double *o, S *sm) { @G0FN@<double, double, NT>(c, o, sm); } static constexpr int SLOTS = @G0SLOTS@; };
struct G1 { template <int NT, class C, class S> __device__ __forceinline__ static void eval(const C &c, double *o, S *sm) { @G1FN@<double, double, NT>(c, o, sm); } static constexpr int SLOTS = @G1SLOTS@; };

template <class F>
__global__ void __launch_bounds__(128, 1) kern_global(RfmArrays rfm, const double *in, double *out) {
  const int i0 = NG + blockIdx.x * 32 + threadIdx.x, i1 = NG + blockIdx.y * 4 + threadIdx.y, i2 = NG + blockIdx.z;
  extern __shared__ double smem[];
  volatile double *sm = smem + threadIdx.x + 32 * threadIdx.y;
  const int idx = i0 + N0 * i1 + N0 * N1 * i2;
  PointCtx ctx;
  ctx.in = in + idx; ctx.aux = nullptr; ctx.s1 = N0; ctx.s2 = N0 * N1; ctx.ntot = NTOT; ctx.i0 = i0; ctx.i1 = i1;
  ctx.invdxx0 = 10.0; ctx.invdxx1 = 20.0; ctx.invdxx2 = 5.0; ctx.rfm = rfm;
  double o[3];
  F::template eval<128>(ctx, o, sm);
  for (int k = 0; k < 3; k++) out[idx + k * NTOT] = o[k];
}

template <int TX, int TY, int TZ, class F>
__global__ void __launch_bounds__(TX * TY * TZ, 1) kern_staged(RfmArrays rfm, const double *in, double *out) {
  constexpr int NT = TX * TY * TZ, SX = TX + 4, SY = TY + 4, SZ = TZ + 4, BOX = SX * SY * SZ;
  extern __shared__ double smem[];
  const int tid = threadIdx.x + TX * (threadIdx.y + TY * threadIdx.z);
  const int o0 = NG + blockIdx.x * TX - 2, o1 = NG + blockIdx.y * TY - 2, o2 = NG + blockIdx.z * TZ - 2;
  for (int e = tid; e < 9 * BOX; e += NT) {
    const int g = e / BOX, r = e - g * BOX;
    const int z = r / (SX * SY), r2 = r - z * (SX * SY);
    const int y = r2 / SX, x = r2 - y * SX;
    const int j0 = o0 + x, j1 = o1 + y, j2 = o2 + z;
    smem[e] = (j0 < N0 && j1 < N1 && j2 < N2) ? __ldg(in + (size_t)(11 + g) * NTOT + j0 + N0 * (j1 + N1 * j2)) : 0.0;
  }
  __syncthreads();
  const int i0 = NG + blockIdx.x * TX + threadIdx.x, i1 = NG + blockIdx.y * TY + threadIdx.y, i2 = NG + blockIdx.z * TZ + threadIdx.z;
  volatile double *sm = smem + 9 * BOX + tid;
  SmemCtx<SX, SY, SZ> ctx;
  ctx.s = smem + ((threadIdx.z + 2) * SY + (threadIdx.y + 2)) * SX + (threadIdx.x + 2);
  ctx.i0 = i0; ctx.i1 = i1;
  ctx.invdxx0 = 10.0; ctx.invdxx1 = 20.0; ctx.invdxx2 = 5.0; ctx.rfm = rfm;
  double o[3];
  F::template eval<NT>(ctx, o, sm);
  const int idx = i0 + N0 * i1 + N0 * N1 * i2;
  for (int k = 0; k < 3; k++) out[idx + k * NTOT] = o[k];
}

template <class K>
float time_kernel(K k, dim3 grid, dim3 block, size_t sb, RfmArrays rfm, const double *in, double *out, const char *name) {
  if (sb > 227 * 1024) { printf("{\"kernel\": \"%s\", \"skip\": \"smem %zu\"}\n", name, sb); return -1; }
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb);
  cudaFuncAttributes at; cudaFuncGetAttributes(&at, k);
  int nb = 0; cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, block.x * block.y * block.z, sb);
  cudaEvent_t a, b; cudaEventCreate(&a); cudaEventCreate(&b);
  for (int w = 0; w < 2; w++) k<<<grid, block, sb>>>(rfm, in, out);
  std::vector<float> ts;
  for (int r = 0; r < 7; r++) {
    cudaEventRecord(a); k<<<grid, block, sb>>>(rfm, in, out); cudaEventRecord(b); cudaEventSynchronize(b);
    float ms; cudaEventElapsedTime(&ms, a, b); ts.push_back(ms);
  }
  std::sort(ts.begin(), ts.end());
  const cudaError_t e = cudaGetLastError();
  printf("{\"kernel\": \"%s\", \"regs\": %d, \"local\": %zu, \"smem\": %zu, \"warps_per_sm\": %d, \"us\": %.1f, \"error\": \"%s\"}\n",
         name, at.numRegs, at.localSizeBytes, sb, nb * (int)(block.x * block.y * block.z) / 32, ts[3] * 1e3,
         e == cudaSuccess ? "" : cudaGetErrorString(e));
  return ts[3];
}

template <int TX, int TY, int TZ, class F>
void staged(const char *name, RfmArrays rfm, const double *in, double *out, const std::vector<double> &ref) {
  constexpr int BOX = (TX + 4) * (TY + 4) * (TZ + 4);
  const size_t sb = (size_t)(9 * BOX + F::SLOTS * TX * TY * TZ) * 8;
  cudaMemset(out, 0, (size_t)NTOT * 3 * 8);
  time_kernel(kern_staged<TX, TY, TZ, F>, dim3(256 / TX, 64 / TY, 32 / TZ), dim3(TX, TY, TZ), sb, rfm, in, out, name);
  std::vector<double> h((size_t)NTOT * 3);
  cudaMemcpy(h.data(), out, h.size() * 8, cudaMemcpyDeviceToHost);
  double md = 0, mr = 0;
  for (int i2 = NG; i2 < N2 - NG; i2++) for (int i1 = NG; i1 < N1 - NG; i1++) for (int i0 = NG; i0 < N0 - NG; i0++)
    for (int k = 0; k < 3; k++) { const size_t q = i0 + N0 * (i1 + (size_t)N1 * i2) + (size_t)k * NTOT;
      md = std::max(md, std::abs(h[q] - ref[q])); mr = std::max(mr, std::abs(ref[q])); }
  printf("{\"kernel\": \"%s\", \"max_abs_diff_vs_global\": %.3e, \"max_abs\": %.3e}\n", name, md, mr);
}

template <class F>
void both(const char *gname, RfmArrays rfm, const double *in, double *out) {
  char nm[64];
  snprintf(nm, sizeof nm, "%s_global", gname);
  time_kernel(kern_global<F>, dim3(8, 16, 32), dim3(32, 4, 1), (size_t)F::SLOTS * 128 * 8, rfm, in, out, nm);
  std::vector<double> ref((size_t)NTOT * 3);
  cudaMemcpy(ref.data(), out, ref.size() * 8, cudaMemcpyDeviceToHost);
  snprintf(nm, sizeof nm, "%s_staged_32x4x1", gname); staged<32, 4, 1, F>(nm, rfm, in, out, ref);
  snprintf(nm, sizeof nm, "%s_staged_32x4x2", gname); staged<32, 4, 2, F>(nm, rfm, in, out, ref);
  snprintf(nm, sizeof nm, "%s_staged_16x8x2", gname); staged<16, 8, 2, F>(nm, rfm, in, out, ref);
  snprintf(nm, sizeof nm, "%s_staged_16x4x2", gname); staged<16, 4, 2, F>(nm, rfm, in, out, ref);
  snprintf(nm, sizeof nm, "%s_staged_32x2x2", gname); staged<32, 2, 2, F>(nm, rfm, in, out, ref);
  snprintf(nm, sizeof nm, "%s_staged_16x4x4", gname); staged<16, 4, 4, F>(nm, rfm, in, out, ref);
}

int main() {
  std::vector<double> h((size_t)NTOT * 24);
  srand(7);
  for (auto &x : h) x = 0.5 + (double)rand() / RAND_MAX;
  double *in, *out, *r[7];
  cudaMalloc(&in, h.size() * 8);
  cudaMemcpy(in, h.data(), h.size() * 8, cudaMemcpyHostToDevice);
  cudaMalloc(&out, (size_t)NTOT * 3 * 8);
  for (int k = 0; k < 7; k++) {
    cudaMalloc(&r[k], 300 * 8);
    cudaMemcpy(r[k], h.data() + 1000 * k, 300 * 8, cudaMemcpyHostToDevice);
  }
  RfmArrays rfm{r[0], r[1], r[2], r[3], r[4], r[5], r[6]};
  both<G0>("ricci_g0", rfm, in, out);
  both<G1>("ricci_g1", rfm, in, out);
  return 0;
}
'''


def generate_staged() -> None:
    """The present Ricci groups (allocation and budget of generate.py) reading their nine
    stencil gridfunctions (hDD, lambdaU; radius 2) from a shared-memory copy of the block's
    tile plus a 2-point halo, filled by the block before it evaluates, against the same
    groups reading global memory. Tiles 32x4x1 to 16x4x4 points; the harness checks that
    both forms give the same values."""
    from nrpy_b200.codegen import bssn_exprs as be
    from nrpy_b200.codegen.emit_cuda import emit_point_function
    from nrpy_b200.codegen.generate import RICCI_ALLOC, RICCI_CAPS

    be.setup_nrpy("")
    ricci = be.ricci_exprs("SinhSpherical")
    OUT.mkdir(parents=True, exist_ok=True)
    parts, sub = ["#pragma once\n"], {}
    for g, gname in enumerate(("ricci_012", "ricci_345")):
        names = CANDIDATES[gname][1]
        rf, dr, order = RICCI_ALLOC[g]
        fname = f"{gname}_c{RICCI_CAPS[g]}"
        code, st = emit_point_function(fname, [(f"out[{i}]", ricci[n]) for i, n in enumerate(names)],
                                       reg_capacity=RICCI_CAPS[g], remat_first=rf, deriv_remat=dr, order=order)
        parts.append(code)
        sub[f"@G{g}FN@"] = fname
        sub[f"@G{g}SLOTS@"] = str(max(st["smem_slots"], 1))
    (OUT / "staged_ricci.cuh").write_text("\n".join(parts))
    src = STAGED_HARNESS
    for k, v in sub.items():
        src = src.replace(k, v)
    (OUT / "staged_ricci.cu").write_text(src)
    print("staged_ricci", sub, flush=True)


def compile_all(jobs: int) -> None:
    from nrpy_b200.build import nvcc

    cc = nvcc()

    def one(cu: pathlib.Path) -> str:
        exe = cu.with_suffix("")
        r = subprocess.run([cc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                            "--expt-relaxed-constexpr", "-o", str(exe), str(cu)], capture_output=True, text=True)
        return f"{cu.name}: {'ok' if r.returncode == 0 else 'FAILED ' + r.stderr[-500:]}"

    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for line in ex.map(one, sorted(OUT.glob("*.cu"))):
            print(line, flush=True)


def run_all() -> None:
    for exe in sorted(p for p in OUT.iterdir() if p.is_file() and p.suffix == "" and os.access(p, os.X_OK)):
        r = subprocess.run([str(exe)], capture_output=True, text=True)
        sys.stdout.write(r.stdout)
        if r.returncode != 0:
            raise SystemExit(f"{exe.name} exited {r.returncode}: {r.stderr[-500:]}")


def summarize(path: str) -> None:
    rows = [json.loads(ln) for ln in open(path) if ln.startswith("{") and "us" in ln]
    best = {}
    for r in rows:
        g = r["kernel"].rsplit("_c", 1)[0]
        if g not in best or r["us"] < best[g]["us"]:
            best[g] = r
    for g, r in sorted(best.items()):
        print(f"{g:22s} {r['us']:8.1f} us  {r['kernel']}  threads={r['threads']} regs={r['regs']} "
              f"local={r['local_bytes']} slots={r['slots']} warps/SM={r['warps_per_sm']}")


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("step", choices=["generate", "generate-orders", "generate-caps", "generate-leaf",
                                     "generate-staged", "compile", "run", "summarize"])
    ap.add_argument("--caps", default="72,80,90,100")
    ap.add_argument("--fd-order", type=int, default=4)
    ap.add_argument("--dtype", default="double", choices=["double", "float"], help="value type of generate-caps")
    ap.add_argument("--groups", default="", help="generate-caps: candidate groups to time (default: the present ones)")
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 4)
    ap.add_argument("--log", default=None)
    a = ap.parse_args()
    if a.step == "generate":
        generate()
    elif a.step == "generate-orders":
        generate_orders()
    elif a.step == "generate-caps":
        generate_caps([int(c) for c in a.caps.split(",")], a.fd_order, a.dtype, [g for g in a.groups.split(",") if g])
    elif a.step == "generate-leaf":
        generate_leaf()
    elif a.step == "generate-staged":
        generate_staged()
    elif a.step == "compile":
        compile_all(a.jobs)
    elif a.step == "run":
        run_all()
    else:
        summarize(a.log)
