// Integer issue peaks of the device, the denominators of the integer
// roofline: independent chains of 32-bit XORs (the ALU pipe), of 32-bit
// multiply-adds (the FMA pipe), of both interleaved (the issue limit when
// both pipes are fed), of 32 x 32 -> 64-bit multiply-adds (the extension
// products' inner operation), of dp4a (the weight passes) and of funnel-shift
// rotations (BLAKE2s).  Each thread runs 8 independent chains so that
// the dependent latency is hidden; the grid fills every SM with 4 CTAs of 256
// threads.  The instructions are written as inline PTX so the compiler
// neither folds nor reorders them into other forms.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/parcomm_qafold.h"
#include "capi_internal.h"
#include "gpu_common.cuh"

namespace {

constexpr int kChains = 8;
constexpr int kUnroll = 16;

__device__ __forceinline__ uint32_t op_xor(uint32_t a, uint32_t b) {
  uint32_t d;
  asm volatile("xor.b32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}
__device__ __forceinline__ uint32_t op_mad(uint32_t a, uint32_t b) {
  uint32_t d;
  asm volatile("mad.lo.u32 %0, %1, %2, %1;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}
__device__ __forceinline__ uint64_t op_mad_wide(uint32_t a, uint32_t b, uint64_t c) {
  uint64_t d;
  asm volatile("mad.wide.u32 %0, %1, %2, %3;" : "=l"(d) : "r"(a), "r"(b), "l"(c));
  return d;
}

__device__ __forceinline__ uint32_t op_dp4a(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t d;
  asm volatile("dp4a.s32.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}
__device__ __forceinline__ uint32_t op_shf(uint32_t a, uint32_t n) {
  uint32_t d;
  asm volatile("shf.r.wrap.b32 %0, %1, %1, %2;" : "=r"(d) : "r"(a), "r"(n));
  return d;
}

// KIND 0: XOR only; 1: multiply-add only; 2: alternating; 3: widening
// multiply-add (64-bit accumulators); 4: dp4a; 5: funnel-shift rotations.
template <int KIND>
__global__ void __launch_bounds__(256) k_int_peak(uint32_t* sink, uint32_t iters, uint32_t seed) {
  uint32_t a[kChains];
  uint64_t w[kChains];
  const uint32_t b = seed | 1u;
#pragma unroll
  for (int c = 0; c < kChains; ++c) {
    a[c] = threadIdx.x * 2654435761u + uint32_t(c) * 40503u + blockIdx.x;
    w[c] = a[c];
  }
  for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < kUnroll; ++u)
#pragma unroll
      for (int c = 0; c < kChains; ++c) {
        if (KIND == 0) a[c] = op_xor(a[c], b + uint32_t(u));
        else if (KIND == 1) a[c] = op_mad(a[c], b);
        else if (KIND == 2) a[c] = ((u + c) & 1) ? op_mad(a[c], b) : op_xor(a[c], b + uint32_t(u));
        else if (KIND == 3) w[c] = op_mad_wide(a[c], b + uint32_t(u), w[c]);
        else if (KIND == 4) a[c] = op_dp4a(b + uint32_t(u), b, a[c]);
        else a[c] = op_shf(a[c], 7u + uint32_t(u));
      }
  }
  uint32_t x = 0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) x ^= a[c] ^ uint32_t(w[c]) ^ uint32_t(w[c] >> 32);
  if (x == 0x9e3779b9u) sink[0] = x;  // keeps the chains live
}

template <int KIND>
double measure(uint32_t* sink, int sms) {
  const unsigned grid = unsigned(sms) * 4, block = 256;
  const uint32_t iters = 4096;
  cudaEvent_t e0, e1;
  QF_CK(cudaEventCreate(&e0));
  QF_CK(cudaEventCreate(&e1));
  k_int_peak<KIND><<<grid, block>>>(sink, 64, 3u);  // warm-up
  QF_CK(cudaGetLastError());
  float best = 1e30f;
  for (int rep = 0; rep < 3; ++rep) {
    QF_CK(cudaEventRecord(e0));
    k_int_peak<KIND><<<grid, block>>>(sink, iters, 3u);
    QF_CK(cudaGetLastError());
    QF_CK(cudaEventRecord(e1));
    QF_CK(cudaEventSynchronize(e1));
    float ms = 0;
    QF_CK(cudaEventElapsedTime(&ms, e0, e1));
    best = ms < best ? ms : best;
  }
  QF_CK(cudaEventDestroy(e0));
  QF_CK(cudaEventDestroy(e1));
  const double ops = double(grid) * block * iters * kUnroll * kChains;
  return ops / (best / 1e3);
}

}  // namespace

extern "C" int qf_kernel_int_peaks(double* out) {
  return qfc::guarded([&] {
    if (!out) qf::fail(QF_E_ARGUMENT, "null argument");
    qfc::require_device();
    int dev = 0, sms = 0;
    QF_CK(cudaGetDevice(&dev));
    QF_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    uint32_t* sink = nullptr;
    QF_CK(cudaMalloc(&sink, 16));
    out[0] = measure<0>(sink, sms);
    out[1] = measure<1>(sink, sms);
    out[2] = measure<2>(sink, sms);
    out[3] = measure<3>(sink, sms);
    out[4] = measure<4>(sink, sms);
    out[5] = measure<5>(sink, sms);
    QF_CK(cudaFree(sink));
  });
}
