// Device vector kernels for the top opening round and the top Decide round:
// LiteBullet cross products and folds (qafold_short_pc.rs:1895-1999,
// 2858-2910), axpy, scatter of sampled-row weights, inner products, and the
// block fold of a direct-interleaved witness (qafold_short_decide_carry.rs:182-222).
#pragma once
#include <cstdint>

#include "../device/field_dev.cuh"

namespace QFD_NS {

// a[i] += s * b[i]
__global__ void k_axpy(Fe* __restrict__ a, const Fe* __restrict__ b, uint64_t n, Fe s) {
  const Fr fs = load(&s);
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    store(a + i, add(load(a + i), mul(load(b + i), fs)));
}
// a[i] += b[i]
__global__ void k_add(Fe* __restrict__ a, const Fe* __restrict__ b, uint64_t n) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    store(a + i, add(load(a + i), load(b + i)));
}
// dst[idx[i]] = vals[i]  (indices are distinct)
__global__ void k_scatter_set(Fe* __restrict__ dst, const uint64_t* __restrict__ idx, const Fe* __restrict__ vals, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[idx[i]] = vals[i];
}
// partial sums of sum_i a[i] * b[i]
__global__ void k_dot(const Fe* __restrict__ a, const Fe* __restrict__ b, uint64_t n, Fe* __restrict__ partials) {
  Acc acc = acc_zero();
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
    mul_acc(acc, load(a + i), load(b + i));
  Fr s[1] = {acc_reduce(acc)};
  block_reduce<1>(s);
  finish_reduction<1>(s, partials);
}
// LiteBullet cross pair of (L, R) with half h: sum L[i] R[h+i], sum L[h+i] R[i].
__global__ void k_lb_cross(const Fe* __restrict__ L, const Fe* __restrict__ R, uint64_t n, Fe* __restrict__ partials) {
  const uint64_t h = n / 2;
  Acc acc[2] = {acc_zero(), acc_zero()};
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < h; i += uint64_t(gridDim.x) * blockDim.x) {
    mul_acc(acc[0], load(L + i), load(R + h + i));
    mul_acc(acc[1], load(L + h + i), load(R + i));
  }
  Fr s[2] = {acc_reduce(acc[0]), acc_reduce(acc[1])};
  block_reduce<2>(s);
  finish_reduction<2>(s, partials);
}
// Fold L[i] += L[h+i] * wl, R[i] += R[h+i] * wr (h = n/2), in place, and emit
// the cross pair of the folded length-h vectors.  Thread i < n/4 owns the
// positions {i, i + n/4, i + n/2, i + 3n/4}, so the in-place update is race free.
__global__ void k_lb_fold_cross(Fe* __restrict__ L, Fe* __restrict__ R, uint64_t n, Fe wl, Fe wr, Fe* __restrict__ partials) {
  const Fr fl = load(&wl), fr = load(&wr);
  const uint64_t h = n / 2, q = n / 4;
  Acc acc[2] = {acc_zero(), acc_zero()};
  if (n == 2) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      store(L, add(load(L), mul(load(L + 1), fl)));
      store(R, add(load(R), mul(load(R + 1), fr)));
    }
  } else {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < q; i += uint64_t(gridDim.x) * blockDim.x) {
      Fr l0 = add(load(L + i), mul(load(L + i + h), fl));
      Fr l1 = add(load(L + i + q), mul(load(L + i + q + h), fl));
      Fr r0 = add(load(R + i), mul(load(R + i + h), fr));
      Fr r1 = add(load(R + i + q), mul(load(R + i + q + h), fr));
      store(L + i, l0);
      store(L + i + q, l1);
      store(R + i, r0);
      store(R + i + q, r1);
      mul_acc(acc[0], l0, r1);
      mul_acc(acc[1], l1, r0);
    }
  }
  Fr s[2] = {acc_reduce(acc[0]), acc_reduce(acc[1])};
  block_reduce<2>(s);
  finish_reduction<2>(s, partials);
}
// out[r] = sum_b w[b] * in[b * rows + r]  (block coordinate fold, b < nb)
__global__ void k_block_combine(const Fe* __restrict__ in, uint64_t rows, int nb, const Fe* __restrict__ w, Fe* __restrict__ out) {
  __shared__ Fe ws[64];
  if (threadIdx.x < nb) ws[threadIdx.x] = w[threadIdx.x];
  __syncthreads();
  for (uint64_t r = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < rows; r += uint64_t(gridDim.x) * blockDim.x) {
    Fr s = zero();
    for (int b = 0; b < nb; ++b) s = add(s, mul(load(ws + b), load(in + uint64_t(b) * rows + r)));
    store(out + r, s);
  }
}
// Copies a column-major message (cols x rows) into the message halves of a
// codeword (cols x 2 rows).
__global__ void k_to_message_halves(const Fe* __restrict__ src, uint64_t m, int logR, Fe* __restrict__ cw) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x)
    cw[((i >> logR) << (logR + 1)) | (i & ((uint64_t(1) << logR) - 1))] = src[i];
}

}  // namespace QFD_NS
