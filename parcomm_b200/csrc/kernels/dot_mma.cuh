// Exact sums of extension-field products on the tensor cores: the dot
// products and cross pairs of the EO binary rounds (eo.rs:141-160), the
// degree-2 sumcheck messages (packed.rs:652-696) and the LiteBullet rounds
// (qafold_short_pc.rs:1895-1940).  The same sums as the CUDA-core kernels of
// open.cuh and vec.cuh, and the same canonical results.
//
// An element's 16 storage bytes are its coefficients' limbs (F65521^8: two
// bytes per coefficient, KoalaBear^4: four), so for two vectors x, y the
// sums L[a][b] = sum_i byte_a(x_i) * byte_b(y_i) form the 16 x 16 matrix
// X^T Y with K running over the elements.  One mma.sync.m16n8k32 with u8
// operands adds the contribution of 32 elements to one 8-column half of it,
// exactly, in s32.  The coefficient products follow as
//   sum_i x_i[c1] y_i[c2] = sum over limbs l1, l2 of 2^(8 (l1 + l2)) L[(c1,l1)][(c2,l2)],
// and the extension product as the sum over c1 + c2 = k of those, plus the
// wrap factor (X^8 = 17, X^4 = 3) times the ones with c1 + c2 = k + kC.
//
// A warp stages 32 elements of each operand in shared memory as four word
// planes (word w of element j at plane w, column j), so a lane reads the
// words of four consecutive elements with one 128-bit load and forms its
// fragment registers with byte permutes.  Matrix row m (A) or column m (B)
// stands for storage byte rho(m) = 4 ((m & 7) >> 1) + 2 (m >> 3) + (m & 1):
// rows g and g + 8 of a lane's fragment are then bytes of the same word.
// The elements of a chunk take the K positions in the same order in every
// operand, so any order gives the same sums.
#pragma once
#include <cstdint>

#include "open.cuh"

namespace QFD_NS {

constexpr int kDotThreads = 256;               // 8 warps per CTA
constexpr int kDotStride = 4 * 32 + 16;        // words per staged operand (padded: conflict-free puts)
constexpr int kDotLimbs = 16 / kC;             // bytes per coefficient
constexpr int kDotFlush = 256;                 // chunks between moves of the s32 sums
// Each D entry gains at most two products of 32 byte pairs per chunk
// (2 * 32 * 255^2 < 2^22), so 256 chunks stay below 2^31.
static_assert(kDotFlush * 2 * 32 * 255 * 255 < 2147483647.0, "s32 sums between flushes");
constexpr uint32_t kDotWrap = kC == 8 ? 17u : 3u;  // X^kC

// 2^(8 s) mod p for the limb weights s = l1 + l2.
__device__ __forceinline__ uint32_t dot_limb_weight(int s) {
  if (kC == 8) return s == 0 ? 1u : (s == 1 ? 256u : 15u);  // 2^16 = 15 mod 65521
  constexpr uint32_t w[7] = {1u, 256u, 65536u, 16777216u, 33554430u, 67108348u, 134085624u};
  uint32_t r = w[0];
#pragma unroll
  for (int u = 1; u < 7; ++u)
    if (s == u) r = w[u];
  return r;
}

__device__ __forceinline__ int dot_rho(int m) { return 4 * ((m & 7) >> 1) + 2 * (m >> 3) + (m & 1); }

// Lane j's element of operand x into the warp's staging area.
__device__ __forceinline__ void dot_put(uint32_t* s, int x, int j, uint4 u) {
  uint32_t* p = s + x * kDotStride + j;
  p[0] = u.x;
  p[32] = u.y;
  p[64] = u.z;
  p[96] = u.w;
}

// The A fragment of operand x (rows g and g + 8; K 4t..4t+3 and 16+4t..);
// the same registers are the B fragment of x: r[0], r[2] for columns g
// (first 8-column half), r[1], r[3] for columns g + 8.
struct DotFrag {
  uint32_t r[4];
};
__device__ __forceinline__ DotFrag dot_frag(const uint32_t* s, int x) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const uint32_t* p = s + x * kDotStride + (g >> 1) * 32;
  const uint4 u = *reinterpret_cast<const uint4*>(p + 4 * t);
  const uint4 v = *reinterpret_cast<const uint4*>(p + 16 + 4 * t);
  // Bytes b and b + 2 of each word (b = g & 1): rows g and g + 8.
  const uint32_t sel = (g & 1) ? 0x7351u : 0x6240u;
  const uint32_t u01 = __byte_perm(u.x, u.y, sel), u23 = __byte_perm(u.z, u.w, sel);
  const uint32_t v01 = __byte_perm(v.x, v.y, sel), v23 = __byte_perm(v.z, v.w, sel);
  DotFrag f;
  f.r[0] = __byte_perm(u01, u23, 0x5410u);
  f.r[1] = __byte_perm(u01, u23, 0x7632u);
  f.r[2] = __byte_perm(v01, v23, 0x5410u);
  f.r[3] = __byte_perm(v01, v23, 0x7632u);
  return f;
}

// The s32 sums of one product (both 8-column halves).
struct DotAcc {
  int32_t d[2][4];
};
__device__ __forceinline__ void dot_clear(DotAcc& a) {
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int r = 0; r < 4; ++r) a.d[h][r] = 0;
}
__device__ __forceinline__ void mma_u8_k32(int32_t (&d)[4], const DotFrag& a, uint32_t b0, uint32_t b1) {
  asm("mma.sync.aligned.m16n8k32.row.col.s32.u8.u8.s32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
      : "r"(a.r[0]), "r"(a.r[1]), "r"(a.r[2]), "r"(a.r[3]), "r"(b0), "r"(b1));
}
// acc += sum over the chunk of x_j (x) y_j.
__device__ __forceinline__ void dot_mma(DotAcc& acc, const DotFrag& x, const DotFrag& y) {
  mma_u8_k32(acc.d[0], x, y.r[0], y.r[2]);
  mma_u8_k32(acc.d[1], x, y.r[1], y.r[3]);
}
// Adds the lane's share of the extension sum held in acc to out (canonical)
// and clears acc.  Lane (g, t) holds rows g, g + 8 and columns 2t, 2t + 1
// (+ 8 in the second half); the warp's lanes together hold every entry once.
__device__ __forceinline__ void dot_flush(DotAcc& acc, Fr& out) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int ba = dot_rho(g + 8 * (r >> 1)), bb = dot_rho(2 * t + (r & 1) + 8 * h);
      const int c1 = ba / kDotLimbs, l1 = ba % kDotLimbs, c2 = bb / kDotLimbs, l2 = bb % kDotLimbs;
      uint32_t v = red64(uint64_t(red32(uint32_t(acc.d[h][r]))) * dot_limb_weight(l1 + l2));
      int k = c1 + c2;
      if (k >= kC) {
        k -= kC;
        v = red64(uint64_t(v) * kDotWrap);
      }
#pragma unroll
      for (int kk = 0; kk < kC; ++kk)
        if (k == kk) out.c[kk] = addp(out.c[kk], v);
      acc.d[h][r] = 0;
    }
}

// The warp-chunked loop of the tensor-core kernels.  Chunk c covers indices
// [32c, 32c + 32) and lane j takes index 32c + j.  fetch(i, ok, r) loads the
// NR raw inputs of index i (zero when !ok); make(i, ok, r, x) forms the NX
// staged operands from them and performs the kernel's own stores; step(f)
// issues the chunk's products from the fragments; flush() moves the s32
// sums out every kDotFlush chunks and once at the end.  The next chunk's
// fetch is issued before the current chunk's staging and products, so its
// loads are in flight meanwhile.  Every lane of a warp runs the same chunks
// (mma.sync).
template <int NX, int NR, class Fetch, class Make, class Step, class Flush>
__device__ __forceinline__ void dot_loop(uint32_t* s, uint64_t count, Fetch fetch, Make make, Step step, Flush flush) {
  const int lane = threadIdx.x & 31;
  const uint64_t nw = (uint64_t(gridDim.x) * blockDim.x) >> 5;
  uint64_t c = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  uint4 r[NR];
  if (c * 32 < count) {
    const uint64_t i = c * 32 + uint64_t(lane);
    fetch(i, i < count, r);
  }
  int since = 0;
  for (; c * 32 < count; c += nw) {
    const uint64_t i = c * 32 + uint64_t(lane);
    uint4 x[NX];
    make(i, i < count, r, x);
    const uint64_t cn = c + nw;
    if (cn * 32 < count) {
      const uint64_t in = cn * 32 + uint64_t(lane);
      fetch(in, in < count, r);
    }
    __syncwarp();  // the previous chunk's fragments are read
#pragma unroll
    for (int k = 0; k < NX; ++k) dot_put(s, k, lane, x[k]);
    __syncwarp();
    DotFrag f[NX];
#pragma unroll
    for (int k = 0; k < NX; ++k) f[k] = dot_frag(s, k);
    step(f);
    if (++since == kDotFlush) {
      since = 0;
      flush();
    }
  }
  flush();
}

__device__ __forceinline__ uint4 ld4(const Fe* p) { return *reinterpret_cast<const uint4*>(p); }
__device__ __forceinline__ uint4 zero4() { return make_uint4(0u, 0u, 0u, 0u); }
// r[k] = ok ? p[k](index) : 0 for each of the N pointers.
template <int N>
__device__ __forceinline__ void fetch_n(bool ok, uint4 (&r)[N], const Fe* const (&p)[N]) {
#pragma unroll
  for (int k = 0; k < N; ++k) r[k] = ok ? ld4(p[k]) : zero4();
}
template <int N>
__device__ __forceinline__ void copy_n(const uint4 (&r)[N], uint4 (&x)[N]) {
#pragma unroll
  for (int k = 0; k < N; ++k) x[k] = r[k];
}
__device__ __forceinline__ Fr fr(uint4 u) { return unpack_fe(u); }

// ---------------------------------------------------------------- kernels
// sum a_i b_i (k_dot).
__global__ void __launch_bounds__(kDotThreads, 2) k_dot_mma(const Fe* __restrict__ a, const Fe* __restrict__ b, uint64_t n,
                                                         Fe* __restrict__ partials) {
  __shared__ __align__(16) uint32_t stage_s[kDotThreads / 32][2 * kDotStride];
  uint32_t* s = stage_s[threadIdx.x >> 5];
  DotAcc acc;
  dot_clear(acc);
  Fr v[1] = {zero()};
  dot_loop<2, 2>(
      s, n, [&](uint64_t i, bool ok, uint4 (&r)[2]) { fetch_n<2>(ok, r, {a + i, b + i}); },
      [&](uint64_t, bool, const uint4 (&r)[2], uint4 (&x)[2]) { copy_n<2>(r, x); },
      [&](const DotFrag (&f)[2]) { dot_mma(acc, f[0], f[1]); }, [&] { dot_flush(acc, v[0]); });
  block_reduce<1>(v);
  finish_reduction<1>(v, partials);
}

// LiteBullet cross pair of (L, R) with half h: sum L[i] R[h+i], sum L[h+i] R[i] (k_lb_cross).
__global__ void __launch_bounds__(kDotThreads, 2) k_lb_cross_mma(const Fe* __restrict__ L, const Fe* __restrict__ R, uint64_t n,
                                                              Fe* __restrict__ partials) {
  __shared__ __align__(16) uint32_t stage_s[kDotThreads / 32][4 * kDotStride];
  uint32_t* s = stage_s[threadIdx.x >> 5];
  const uint64_t h = n / 2;
  DotAcc acc[2];
  dot_clear(acc[0]);
  dot_clear(acc[1]);
  Fr v[2] = {zero(), zero()};
  dot_loop<4, 4>(
      s, h, [&](uint64_t i, bool ok, uint4 (&r)[4]) { fetch_n<4>(ok, r, {L + i, L + h + i, R + i, R + h + i}); },
      [&](uint64_t, bool, const uint4 (&r)[4], uint4 (&x)[4]) { copy_n<4>(r, x); },
      [&](const DotFrag (&f)[4]) {
        dot_mma(acc[0], f[0], f[3]);
        dot_mma(acc[1], f[1], f[2]);
      },
      [&] {
        dot_flush(acc[0], v[0]);
        dot_flush(acc[1], v[1]);
      });
  block_reduce<2>(v);
  finish_reduction<2>(v, partials);
}

// L[i] += L[h+i] * wl, R[i] += R[h+i] * wr for i < h = n/2, in place, and the
// cross pair of the folded length-h vectors (k_lb_fold_cross).  Index i < n/4
// owns positions {i, i + n/4, i + n/2, i + 3n/4} (so the prefetch of a later
// chunk never reads a position this chunk writes); n >= 4.
__global__ void __launch_bounds__(kDotThreads, 2) k_lb_fold_cross_mma(Fe* __restrict__ L, Fe* __restrict__ R, uint64_t n, Fe wl,
                                                                   Fe wr, Fe* __restrict__ partials) {
  __shared__ __align__(16) uint32_t stage_s[kDotThreads / 32][4 * kDotStride];
  uint32_t* s = stage_s[threadIdx.x >> 5];
  const Fr fl = load(&wl), fw = load(&wr);
  const uint64_t h = n / 2, q = n / 4;
  DotAcc acc[2];
  dot_clear(acc[0]);
  dot_clear(acc[1]);
  Fr v[2] = {zero(), zero()};
  dot_loop<4, 8>(
      s, q,
      [&](uint64_t i, bool ok, uint4 (&r)[8]) {
        fetch_n<8>(ok, r, {L + i, L + i + h, L + i + q, L + i + q + h, R + i, R + i + h, R + i + q, R + i + q + h});
      },
      [&](uint64_t i, bool ok, const uint4 (&r)[8], uint4 (&x)[4]) {
        const Fr l0 = add(fr(r[0]), mul(fr(r[1]), fl)), l1 = add(fr(r[2]), mul(fr(r[3]), fl));
        const Fr r0 = add(fr(r[4]), mul(fr(r[5]), fw)), r1 = add(fr(r[6]), mul(fr(r[7]), fw));
        x[0] = pack_fe(l0);
        x[1] = pack_fe(l1);
        x[2] = pack_fe(r0);
        x[3] = pack_fe(r1);
        if (ok) {
          *reinterpret_cast<uint4*>(L + i) = x[0];
          *reinterpret_cast<uint4*>(L + i + q) = x[1];
          *reinterpret_cast<uint4*>(R + i) = x[2];
          *reinterpret_cast<uint4*>(R + i + q) = x[3];
        }
      },
      [&](const DotFrag (&f)[4]) {
        dot_mma(acc[0], f[0], f[3]);
        dot_mma(acc[1], f[1], f[2]);
      },
      [&] {
        dot_flush(acc[0], v[0]);
        dot_flush(acc[1], v[1]);
      });
  block_reduce<2>(v);
  finish_reduction<2>(v, partials);
}

// dot(w, q) and the first binary cross pair (k_eo_dot_cross): over pairs
// j < n/2, sum w[2j] q[2j] + w[2j+1] q[2j+1], sum w[2j] q[2j+1], sum w[2j+1] q[2j].
__global__ void __launch_bounds__(kDotThreads, 2) k_eo_dot_cross_mma(const Fe* __restrict__ w, const Fe* __restrict__ q, uint64_t n,
                                                                  Fe* __restrict__ partials) {
  __shared__ __align__(16) uint32_t stage_s[kDotThreads / 32][4 * kDotStride];
  uint32_t* s = stage_s[threadIdx.x >> 5];
  DotAcc acc[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) dot_clear(acc[k]);
  Fr v[3] = {zero(), zero(), zero()};
  dot_loop<4, 4>(
      s, n / 2, [&](uint64_t j, bool ok, uint4 (&r)[4]) { fetch_n<4>(ok, r, {w + 2 * j, w + 2 * j + 1, q + 2 * j, q + 2 * j + 1}); },
      [&](uint64_t, bool, const uint4 (&r)[4], uint4 (&x)[4]) { copy_n<4>(r, x); },
      [&](const DotFrag (&f)[4]) {
        dot_mma(acc[0], f[0], f[2]);
        dot_mma(acc[0], f[1], f[3]);
        dot_mma(acc[1], f[0], f[3]);
        dot_mma(acc[2], f[1], f[2]);
      },
      [&] {
#pragma unroll
        for (int k = 0; k < 3; ++k) dot_flush(acc[k], v[k]);
      });
  block_reduce<3>(v);
  finish_reduction<3>(v, partials);
}

// w'[i] = w[2i] + w[2i+1] inv, q'[i] = q[2i] + q[2i+1] ch and the next cross
// pair of (w', q') (k_eo_fold_cross); n >= 4.
__global__ void __launch_bounds__(kDotThreads, 2) k_eo_fold_cross_mma(const Fe* __restrict__ w, const Fe* __restrict__ q, uint64_t n,
                                                                   Fe inv, Fe ch, Fe* __restrict__ w_out, Fe* __restrict__ q_out,
                                                                   Fe* __restrict__ partials) {
  __shared__ __align__(16) uint32_t stage_s[kDotThreads / 32][4 * kDotStride];
  uint32_t* s = stage_s[threadIdx.x >> 5];
  const Fr fi = load(&inv), fc = load(&ch);
  DotAcc acc[2];
  dot_clear(acc[0]);
  dot_clear(acc[1]);
  Fr v[2] = {zero(), zero()};
  dot_loop<4, 8>(
      s, n / 4,
      [&](uint64_t j, bool ok, uint4 (&r)[8]) {
        fetch_n<8>(ok, r, {w + 4 * j, w + 4 * j + 1, w + 4 * j + 2, w + 4 * j + 3, q + 4 * j, q + 4 * j + 1, q + 4 * j + 2,
                           q + 4 * j + 3});
      },
      [&](uint64_t j, bool ok, const uint4 (&r)[8], uint4 (&x)[4]) {
        x[0] = pack_fe(add(fr(r[0]), mul(fr(r[1]), fi)));
        x[1] = pack_fe(add(fr(r[2]), mul(fr(r[3]), fi)));
        x[2] = pack_fe(add(fr(r[4]), mul(fr(r[5]), fc)));
        x[3] = pack_fe(add(fr(r[6]), mul(fr(r[7]), fc)));
        if (ok) {
          *reinterpret_cast<uint4*>(w_out + 2 * j) = x[0];
          *reinterpret_cast<uint4*>(w_out + 2 * j + 1) = x[1];
          *reinterpret_cast<uint4*>(q_out + 2 * j) = x[2];
          *reinterpret_cast<uint4*>(q_out + 2 * j + 1) = x[3];
        }
      },
      [&](const DotFrag (&f)[4]) {
        dot_mma(acc[0], f[0], f[3]);
        dot_mma(acc[1], f[1], f[2]);
      },
      [&] {
        dot_flush(acc[0], v[0]);
        dot_flush(acc[1], v[1]);
      });
  block_reduce<2>(v);
  finish_reduction<2>(v, partials);
}

// q'[i] = q[2i] + q[2i+1] ch next to the folded witness wf, and the cross
// pair of (wf, q') (k_eo_fold_query_cross); n >= 4.
__global__ void __launch_bounds__(kDotThreads, 2) k_eo_fold_query_cross_mma(const Fe* __restrict__ wf, const Fe* __restrict__ q,
                                                                         uint64_t n, Fe ch, Fe* __restrict__ q_out,
                                                                         Fe* __restrict__ partials) {
  __shared__ __align__(16) uint32_t stage_s[kDotThreads / 32][4 * kDotStride];
  uint32_t* s = stage_s[threadIdx.x >> 5];
  const Fr fc = load(&ch);
  DotAcc acc[2];
  dot_clear(acc[0]);
  dot_clear(acc[1]);
  Fr v[2] = {zero(), zero()};
  dot_loop<4, 6>(
      s, n / 4,
      [&](uint64_t j, bool ok, uint4 (&r)[6]) {
        fetch_n<6>(ok, r, {wf + 2 * j, wf + 2 * j + 1, q + 4 * j, q + 4 * j + 1, q + 4 * j + 2, q + 4 * j + 3});
      },
      [&](uint64_t j, bool ok, const uint4 (&r)[6], uint4 (&x)[4]) {
        x[0] = r[0];
        x[1] = r[1];
        x[2] = pack_fe(add(fr(r[2]), mul(fr(r[3]), fc)));
        x[3] = pack_fe(add(fr(r[4]), mul(fr(r[5]), fc)));
        if (ok) {
          *reinterpret_cast<uint4*>(q_out + 2 * j) = x[2];
          *reinterpret_cast<uint4*>(q_out + 2 * j + 1) = x[3];
        }
      },
      [&](const DotFrag (&f)[4]) {
        dot_mma(acc[0], f[0], f[3]);
        dot_mma(acc[1], f[1], f[2]);
      },
      [&] {
        dot_flush(acc[0], v[0]);
        dot_flush(acc[1], v[1]);
      });
  block_reduce<2>(v);
  finish_reduction<2>(v, partials);
}

// Degree-2 sumcheck message on (v, w) of length n: sum_{i<h} v_i w_i and
// sum (v_{i+h} - v_i)(w_{i+h} - w_i) (k_sum_message).
__global__ void __launch_bounds__(kDotThreads, 2) k_sum_message_mma(const Fe* __restrict__ v, const Fe* __restrict__ w, uint64_t n,
                                                                 Fe* __restrict__ partials) {
  __shared__ __align__(16) uint32_t stage_s[kDotThreads / 32][4 * kDotStride];
  uint32_t* s = stage_s[threadIdx.x >> 5];
  const uint64_t h = n / 2;
  DotAcc acc[2];
  dot_clear(acc[0]);
  dot_clear(acc[1]);
  Fr out[2] = {zero(), zero()};
  dot_loop<4, 4>(
      s, h, [&](uint64_t i, bool ok, uint4 (&r)[4]) { fetch_n<4>(ok, r, {v + i, w + i, v + i + h, w + i + h}); },
      [&](uint64_t, bool, const uint4 (&r)[4], uint4 (&x)[4]) {
        x[0] = r[0];
        x[1] = r[1];
        x[2] = pack_fe(sub(fr(r[2]), fr(r[0])));
        x[3] = pack_fe(sub(fr(r[3]), fr(r[1])));
      },
      [&](const DotFrag (&f)[4]) {
        dot_mma(acc[0], f[0], f[1]);
        dot_mma(acc[1], f[2], f[3]);
      },
      [&] {
        dot_flush(acc[0], out[0]);
        dot_flush(acc[1], out[1]);
      });
  block_reduce<2>(out);
  finish_reduction<2>(out, partials);
}

// Fold both vectors at ch (lo <- lo + ch (hi - lo)) and the next message of
// the folded vectors (k_sum_fold_message); index i < n/4 produces entries
// i and i + n/4 of the length-n/2 outputs; n >= 4.
__global__ void __launch_bounds__(kDotThreads, 2) k_sum_fold_message_mma(const Fe* __restrict__ v, const Fe* __restrict__ w,
                                                                      uint64_t n, Fe ch, Fe* __restrict__ v_out,
                                                                      Fe* __restrict__ w_out, Fe* __restrict__ partials) {
  __shared__ __align__(16) uint32_t stage_s[kDotThreads / 32][4 * kDotStride];
  uint32_t* s = stage_s[threadIdx.x >> 5];
  const Fr c = load(&ch);
  const uint64_t h = n / 2, q = n / 4;
  DotAcc acc[2];
  dot_clear(acc[0]);
  dot_clear(acc[1]);
  Fr out[2] = {zero(), zero()};
  dot_loop<4, 8>(
      s, q,
      [&](uint64_t i, bool ok, uint4 (&r)[8]) {
        fetch_n<8>(ok, r, {v + i, v + i + h, v + i + q, v + i + q + h, w + i, w + i + h, w + i + q, w + i + q + h});
      },
      [&](uint64_t i, bool ok, const uint4 (&r)[8], uint4 (&x)[4]) {
        const Fr a0 = fr(r[0]), b0 = fr(r[2]), x0 = fr(r[4]), y0 = fr(r[6]);
        const Fr nv0 = add(a0, mul(sub(fr(r[1]), a0), c)), nv1 = add(b0, mul(sub(fr(r[3]), b0), c));
        const Fr nw0 = add(x0, mul(sub(fr(r[5]), x0), c)), nw1 = add(y0, mul(sub(fr(r[7]), y0), c));
        if (ok) {
          store(v_out + i, nv0);
          store(v_out + i + q, nv1);
          store(w_out + i, nw0);
          store(w_out + i + q, nw1);
        }
        x[0] = pack_fe(nv0);
        x[1] = pack_fe(nw0);
        x[2] = pack_fe(sub(nv1, nv0));
        x[3] = pack_fe(sub(nw1, nw0));
      },
      [&](const DotFrag (&f)[4]) {
        dot_mma(acc[0], f[0], f[1]);
        dot_mma(acc[1], f[2], f[3]);
      },
      [&] {
        dot_flush(acc[0], out[0]);
        dot_flush(acc[1], out[1]);
      });
  block_reduce<2>(out);
  finish_reduction<2>(out, partials);
}

}  // namespace QFD_NS
