// Opening kernels: EO lane projections / witness / query fold / binary
// rounds, the batch opening's equality-table lane projection, weight images,
// block fold and degree-2 sumcheck, plus row/path gathers and the top-round
// row projection and Freivalds fold.
//
// Every sum is exact: small signed weights times canonical coefficients
// accumulate in 32-bit registers within a bounded tile and in 64-bit across
// threads, and are reduced mod p once (the reference's i64 / u64 raw-lane
// accumulators, tbv.rs:288-352, packed.rs:569-592).  Evaluation order does not
// change any canonical result.
#pragma once
#include <cstdint>

#include "../device/field_dev.cuh"

namespace QFD_NS {

// ---------------------------------------------------------------- reductions
// Exact signed sums to canonical form; every caller keeps |v| < 2^62.
__device__ __forceinline__ uint32_t mod_i64(int64_t v) { return red_signed(v); }
__device__ __forceinline__ Fr shfl_xor(const Fr& v, int m) {
  Fr r;
#pragma unroll
  for (int k = 0; k < kC; ++k) r.c[k] = __shfl_xor_sync(0xffffffffu, v.c[k], m);
  return r;
}
// Sums N field elements across the CTA; thread 0 receives the totals.
template <int N>
__device__ void block_reduce(Fr (&v)[N]) {
  __shared__ Fr red_s[32][N];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int n = 0; n < N; ++n) v[n] = add(v[n], shfl_xor(v[n], o));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
#pragma unroll
    for (int n = 0; n < N; ++n) red_s[warp][n] = v[n];
  __syncthreads();
  if (threadIdx.x == 0) {
    const int warps = (blockDim.x + 31) >> 5;
    for (int w = 1; w < warps; ++w)
#pragma unroll
      for (int n = 0; n < N; ++n) v[n] = add(v[n], red_s[w][n]);
  }
}
// One-launch reductions.  A reduction buffer holds a 4-element header and
// then one slot of N elements per CTA: header word 0 counts the CTAs that
// have finished (zero between launches), header elements 1..N receive the
// result.  Each CTA stores its totals in its slot; the last one to finish
// sums every slot, writes the result and re-arms the counter, so the host
// reads the result right after the producing kernel with no reduction launch.
constexpr int kRedHeader = 4;
template <int N>
__device__ void finish_reduction(Fr (&v)[N], Fe* __restrict__ buf) {
  __shared__ bool last_s;
  Fe* part = buf + kRedHeader;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int n = 0; n < N; ++n) store(part + size_t(blockIdx.x) * N + n, v[n]);
    __threadfence();
    last_s = atomicAdd(reinterpret_cast<unsigned*>(buf), 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last_s) return;
  __threadfence();
  Fr s[N];
#pragma unroll
  for (int n = 0; n < N; ++n) s[n] = zero();
  for (uint32_t i = threadIdx.x; i < gridDim.x; i += blockDim.x)
#pragma unroll
    for (int n = 0; n < N; ++n)  // other CTAs' stores: read through L2
      s[n] = add(s[n], unpack_fe(__ldcg(reinterpret_cast<const uint4*>(part + size_t(i) * N + n))));
  block_reduce<N>(s);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int n = 0; n < N; ++n) store(buf + 1 + n, s[n]);
    *reinterpret_cast<unsigned*>(buf) = 0u;
  }
}

// Two-level product table: t[i] = hi[i >> lb] * lo[i & (2^lb - 1)].
__device__ __forceinline__ Fr table_at(const Fe* hi, const Fe* lo, int lb, uint64_t i) {
  return mul(load(hi + (i >> lb)), load(lo + (i & ((uint64_t(1) << lb) - 1))));
}

// ---------------------------------------------------------------- TBV term tiles
// Tensor weights of LSB-first factor pairs (tbv.rs:45-76), built on the
// device: entry e of a table is scale * prod_k factors[k][bit k of e].
struct TableSpec {
  uint32_t out_off, count;  // entries [out_off, out_off + count) of the table array
  uint32_t fac_off, n_bits; // factor pairs [fac_off, fac_off + n_bits)
  Fe scale;
};
__global__ void k_factor_tables(const TableSpec* __restrict__ specs, int n_specs, const Fe* __restrict__ factors,
                                uint32_t total, Fe* __restrict__ out) {
  for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    int lo = 0, hi = n_specs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (specs[mid].out_off <= e) lo = mid; else hi = mid - 1;
    }
    const TableSpec& s = specs[lo];
    const uint32_t idx = e - s.out_off;
    Fr v = load(&s.scale);
    for (uint32_t k = 0; k < s.n_bits; ++k) v = mul(v, load(factors + 2 * (s.fac_off + k) + ((idx >> k) & 1)));
    store(out + e, v);
  }
}

// The tiles of one TBV term: tile i covers rows [i << lb, (i + 1) << lb) of the
// term (a row is `lanes` consecutive BVA entries from `offset` for the
// projection, one packed row from `offset` for the query fold).  Its weight
// is lo[r] * top[i >> mb] * mid[i & (2^mb - 1)], the term scale folded into top.
struct TermTiles {
  uint64_t offset, rows;
  uint32_t first_tile;
  uint32_t tile_skip;  // the term's tiles before the first one of this list entry (0 unless a term is split)
  uint32_t lo_off, mid_off, top_off;
  uint32_t lb, mb;
};
__device__ __forceinline__ int find_term(const TermTiles* __restrict__ t, int n, uint32_t tile) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (t[mid].first_tile <= tile) lo = mid; else hi = mid - 1;
  }
  return lo;
}
__device__ __forceinline__ Fr tile_high(const TermTiles& T, const Fe* __restrict__ tables, uint64_t i) {
  return mul(load(tables + T.top_off + (i >> T.mb)), load(tables + T.mid_off + (i & ((uint64_t(1) << T.mb) - 1))));
}

constexpr int kTermThreads = 256;
constexpr int kTilesPerCta = 4;  // consecutive tiles per CTA: one term search, then a forward scan

// Segmented sum of tile outputs: term k owns tiles [seg[k], seg[k+1]).
__global__ void k_sum_segments(const Fe* __restrict__ tile_out, const uint32_t* __restrict__ seg, int lanes,
                               Fe* __restrict__ term_out) {
  const uint32_t a = seg[blockIdx.x], b = seg[blockIdx.x + 1];
  for (int lane = 0; lane < lanes; ++lane) {
    Fr v[1] = {zero()};
    for (uint32_t t = a + threadIdx.x; t < b; t += blockDim.x) v[0] = add(v[0], load(tile_out + size_t(t) * lanes + lane));
    block_reduce<1>(v);
    if (threadIdx.x == 0) store(term_out + size_t(blockIdx.x) * lanes + lane, v[0]);
    __syncthreads();
  }
}

// Laurent cross sums of the large terms (Query::cross_terms, tbv.rs:353-392):
// block d - 1 (d = 1 .. stride - 1) sums pr[t][lane] * low[t][lane + d], block
// stride - 2 + d sums pr[t][lane + d] * low[t][lane], over terms t and lanes.
__global__ void k_laurent_cross(const Fe* __restrict__ pr, const Fe* __restrict__ low, int n_terms, int stride,
                                Fe* __restrict__ out) {
  const int d = int(blockIdx.x) % (stride - 1) + 1;
  const bool negative = int(blockIdx.x) >= stride - 1;
  const int per = stride - d;
  Fr acc[1] = {zero()};
  for (int e = threadIdx.x; e < n_terms * per; e += blockDim.x) {
    const int t = e / per, lane = e % per;
    const Fe* a = pr + size_t(t) * stride;
    const Fe* b = low + size_t(t) * stride;
    acc[0] = add(acc[0], negative ? mul(load(a + lane + d), load(b + lane)) : mul(load(a + lane), load(b + lane + d)));
  }
  block_reduce<1>(acc);
  if (threadIdx.x == 0) store(out + blockIdx.x, acc[0]);
}

// Copies the aligned stride-wide BVA window of each small term.
__global__ void k_gather_windows(const Wt* __restrict__ bva, uint64_t active, const uint64_t* __restrict__ starts,
                                 uint32_t count, int stride, Wt* __restrict__ out) {
  const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= uint64_t(count) * stride) return;
  const uint64_t g = starts[i / stride] + i % stride;
  out[i] = g < active ? bva[g] : Wt(0);
}

// ---------------------------------------------------------------- EO
// Query fold of large terms (tbv.rs:393-428): q[offset + row] += high(tile) *
// lo[r] for the rows of each tile.  Terms within one launch are disjoint.
__global__ void k_query_terms(const TermTiles* __restrict__ terms, int n_terms, uint32_t n_tiles,
                              const Fe* __restrict__ tables, Fe* __restrict__ q) {
  __shared__ int t_sel;
  const uint32_t tile0 = blockIdx.x * kTilesPerCta;
  if (threadIdx.x == 0) t_sel = find_term(terms, n_terms, tile0);
  __syncthreads();
  int ti = t_sel;
  for (uint32_t tile = tile0; tile < tile0 + kTilesPerCta && tile < n_tiles; ++tile) {
    while (ti + 1 < n_terms && terms[ti + 1].first_tile <= tile) ++ti;
    const TermTiles T = terms[ti];
    const uint64_t i = tile - T.first_tile + T.tile_skip;
    const uint64_t row0 = i << T.lb;
    const uint64_t span = uint64_t(1) << T.lb, left = T.rows - row0;
    const uint32_t nrows = uint32_t(left < span ? left : span);
    const Fr hi = tile_high(T, tables, i);
    Fe* dst = q + T.offset + row0;
    for (uint32_t r = threadIdx.x; r < nrows; r += blockDim.x)
      store(dst + r, add(load(dst + r), mul(load(tables + T.lo_off + r), hi)));
  }
}
__global__ void k_scatter_add(const uint64_t* __restrict__ idx, const Fe* __restrict__ vals, uint32_t n, Fe* __restrict__ q) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) store(q + idx[i], add(load(q + idx[i]), load(vals + i)));  // indices are unique
}

// dot(w, q) and the first binary cross pair.
__global__ void k_eo_dot_cross(const Fe* __restrict__ w, const Fe* __restrict__ q, uint64_t n, Fe* __restrict__ partials) {
  Acc acc[3] = {acc_zero(), acc_zero(), acc_zero()};
  for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n / 2; j += uint64_t(gridDim.x) * blockDim.x) {
    Fr w0 = load(w + 2 * j), w1 = load(w + 2 * j + 1), q0 = load(q + 2 * j), q1 = load(q + 2 * j + 1);
    mul_acc(acc[0], w0, q0);
    mul_acc(acc[0], w1, q1);
    mul_acc(acc[1], w0, q1);
    mul_acc(acc[2], w1, q0);
  }
  Fr v[3] = {acc_reduce(acc[0]), acc_reduce(acc[1]), acc_reduce(acc[2])};
  block_reduce<3>(v);
  finish_reduction<3>(v, partials);
}
// w'[i] = w[2i] + w[2i+1] * inv; q'[i] = q[2i] + q[2i+1] * ch, plus the next
// cross pair of (w', q') (eo.rs:141-160, fold_in_place 57-79).
__global__ void k_eo_fold_cross(const Fe* __restrict__ w, const Fe* __restrict__ q, uint64_t n, Fe inv, Fe ch,
                                Fe* __restrict__ w_out, Fe* __restrict__ q_out, Fe* __restrict__ partials) {
  const Fr fi = load(&inv), fc = load(&ch);
  Acc acc[2] = {acc_zero(), acc_zero()};
  if (n == 2) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      store(w_out, add(load(w), mul(load(w + 1), fi)));
      store(q_out, add(load(q), mul(load(q + 1), fc)));
    }
  } else {
    for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n / 4; j += uint64_t(gridDim.x) * blockDim.x) {
      Fr a0 = add(load(w + 4 * j), mul(load(w + 4 * j + 1), fi));
      Fr a1 = add(load(w + 4 * j + 2), mul(load(w + 4 * j + 3), fi));
      Fr b0 = add(load(q + 4 * j), mul(load(q + 4 * j + 1), fc));
      Fr b1 = add(load(q + 4 * j + 2), mul(load(q + 4 * j + 3), fc));
      store(w_out + 2 * j, a0);
      store(w_out + 2 * j + 1, a1);
      store(q_out + 2 * j, b0);
      store(q_out + 2 * j + 1, b1);
      mul_acc(acc[0], a0, b1);
      mul_acc(acc[1], a1, b0);
    }
  }
  Fr v[2] = {acc_reduce(acc[0]), acc_reduce(acc[1])};
  block_reduce<2>(v);
  finish_reduction<2>(v, partials);
}

// The same fold as k_eo_fold_cross, one vector at a time, so the full-length
// witness can be released before the query's half-length output exists:
// w'[i] = w[2i] + w[2i+1] * inv, then q'[i] = q[2i] + q[2i+1] * ch with the
// next cross pair of (w', q').
__global__ void k_eo_fold_vec(const Fe* __restrict__ w, uint64_t n, Fe f, Fe* __restrict__ out) {
  const Fr ff = load(&f);
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n / 2; i += uint64_t(gridDim.x) * blockDim.x)
    store(out + i, add(load(w + 2 * i), mul(load(w + 2 * i + 1), ff)));
}
__global__ void k_eo_fold_query_cross(const Fe* __restrict__ wf, const Fe* __restrict__ q, uint64_t n, Fe ch,
                                      Fe* __restrict__ q_out, Fe* __restrict__ partials) {
  const Fr fc = load(&ch);
  Acc acc[2] = {acc_zero(), acc_zero()};
  if (n == 2) {
    if (blockIdx.x == 0 && threadIdx.x == 0) store(q_out, add(load(q), mul(load(q + 1), fc)));
  } else {
    for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n / 4; j += uint64_t(gridDim.x) * blockDim.x) {
      const Fr a0 = load(wf + 2 * j), a1 = load(wf + 2 * j + 1);
      const Fr b0 = add(load(q + 4 * j), mul(load(q + 4 * j + 1), fc));
      const Fr b1 = add(load(q + 4 * j + 2), mul(load(q + 4 * j + 3), fc));
      store(q_out + 2 * j, b0);
      store(q_out + 2 * j + 1, b1);
      mul_acc(acc[0], a0, b1);
      mul_acc(acc[1], a1, b0);
    }
  }
  Fr v[2] = {acc_reduce(acc[0]), acc_reduce(acc[1])};
  block_reduce<2>(v);
  finish_reduction<2>(v, partials);
}

// ---------------------------------------------------------------- batch opening
// weights[i] = hi[i >> lb] * lo[i & mask]  (an equality or tensor table).
__global__ void k_table(const Fe* __restrict__ hi, const Fe* __restrict__ lo, int lb, uint64_t m, Fe* __restrict__ out) {
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x)
    store(out + i, table_at(hi, lo, lb, i));
}

constexpr int kEqThreads = 256, kEqChunk = 2048, kEqBlocks = 8;
constexpr int kEqRaw = kC * kC;  // raw lane sums per block: lane j, coefficient k at j * kC + k

// w <- sum_j w.c[j] * images[j]  (apply_weight_images, packed.rs:634-650).
// With kC canonical coefficients a sum of kC products stays below 2^64.
__global__ void k_apply_images(Fe* __restrict__ weights, uint64_t m, const Fe* __restrict__ images) {
  __shared__ uint32_t img[kC][kC];
  if (threadIdx.x < kC * kC) img[threadIdx.x / kC][threadIdx.x % kC] = images[threadIdx.x / kC].c[threadIdx.x % kC];
  __syncthreads();
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += uint64_t(gridDim.x) * blockDim.x) {
    Fr w = load(weights + i);
    Fr o;
#pragma unroll
    for (int k = 0; k < kC; ++k) {
      uint64_t s = 0;
#pragma unroll
      for (int j = 0; j < kC; ++j) s += uint64_t(w.c[j]) * img[j][k];
      o.c[k] = red_sum(s);
    }
    store(weights + i, o);
  }
}

// Degree-2 sumcheck message on (v, w) of length n: sum_{i<h} v_i w_i and
// sum (v_{i+h} - v_i)(w_{i+h} - w_i) (round_message, packed.rs:652-667).
__global__ void k_sum_message(const Fe* __restrict__ v, const Fe* __restrict__ w, uint64_t n, Fe* __restrict__ partials) {
  const uint64_t h = n / 2;
  Acc acc[2] = {acc_zero(), acc_zero()};
  for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < h; i += uint64_t(gridDim.x) * blockDim.x) {
    Fr a = load(v + i), b = load(w + i), c = load(v + i + h), d = load(w + i + h);
    mul_acc(acc[0], a, b);
    mul_acc(acc[1], sub(c, a), sub(d, b));
  }
  Fr s[2] = {acc_reduce(acc[0]), acc_reduce(acc[1])};
  block_reduce<2>(s);
  finish_reduction<2>(s, partials);
}
// Fold both vectors at ch (lo <- lo + ch (hi - lo), packed.rs:674-696) and
// emit the next message of the folded vectors.  Thread i < n/4 produces
// entries i and i + n/4 of the new length-n/2 vectors.
__global__ void k_sum_fold_message(const Fe* __restrict__ v, const Fe* __restrict__ w, uint64_t n, Fe ch,
                                   Fe* __restrict__ v_out, Fe* __restrict__ w_out, Fe* __restrict__ partials) {
  const Fr c = load(&ch);
  const uint64_t h = n / 2, q = n / 4;
  Acc acc[2] = {acc_zero(), acc_zero()};
  if (n == 2) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      Fr a = load(v), b = load(v + 1);
      store(v_out, add(a, mul(sub(b, a), c)));
      Fr x = load(w), y = load(w + 1);
      store(w_out, add(x, mul(sub(y, x), c)));
    }
  } else {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < q; i += uint64_t(gridDim.x) * blockDim.x) {
      Fr a0 = load(v + i), a1 = load(v + i + h), b0 = load(v + i + q), b1 = load(v + i + q + h);
      Fr nv0 = add(a0, mul(sub(a1, a0), c)), nv1 = add(b0, mul(sub(b1, b0), c));
      Fr x0 = load(w + i), x1 = load(w + i + h), y0 = load(w + i + q), y1 = load(w + i + q + h);
      Fr nw0 = add(x0, mul(sub(x1, x0), c)), nw1 = add(y0, mul(sub(y1, y0), c));
      store(v_out + i, nv0);
      store(v_out + i + q, nv1);
      store(w_out + i, nw0);
      store(w_out + i + q, nw1);
      mul_acc(acc[0], nv0, nw0);
      mul_acc(acc[1], sub(nv1, nv0), sub(nw1, nw0));
    }
  }
  Fr s[2] = {acc_reduce(acc[0]), acc_reduce(acc[1])};
  block_reduce<2>(s);
  finish_reduction<2>(s, partials);
}

// ---------------------------------------------------------------- codeword access
__global__ void k_gather_rows(const Fe* __restrict__ cw, uint64_t n_ext, int n_cols, const uint64_t* __restrict__ idx,
                              uint32_t count, Fe* __restrict__ out) {
  const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= uint64_t(count) * n_cols) return;
  const uint64_t q = t / n_cols, c = t % n_cols;
  out[t] = cw[c * n_ext + idx[q]];
}
// Sibling digests of each queried leaf, leaf level first.
__global__ void k_gather_paths(const uint4* __restrict__ tree, const uint64_t* __restrict__ level_off, int depth,
                               const uint64_t* __restrict__ idx, uint32_t count, uint4* __restrict__ out) {
  const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= uint64_t(count) * depth) return;
  const uint64_t q = t / depth;
  const int l = int(t % depth);
  const uint64_t node = (idx[q] >> l) ^ 1;
  const uint64_t off = level_off[l] + node;
  out[2 * t] = tree[2 * off];
  out[2 * t + 1] = tree[2 * off + 1];
}
// Wire records of sampled rows (the partial form of write_rows): per query,
// u64 n_cols, the row's n_cols elements (16 canonical bytes each, which is
// their device layout), u64 depth, then the depth sibling digests leaf level
// first (32 bytes each, the tree's little-endian words).  Record q occupies
// rec_words = 2 + 2 n_cols + 4 depth u64 words from out + q * rec_words; one
// thread writes one element, one sibling or one length.
__global__ void k_binding_records(const Fe* __restrict__ cw, uint64_t n_ext, int n_cols, const uint4* __restrict__ tree,
                                  const uint64_t* __restrict__ level_off, int depth, const uint64_t* __restrict__ idx,
                                  uint32_t count, uint64_t* __restrict__ out) {
  const uint64_t per = uint64_t(n_cols) + uint64_t(depth) + 2;
  const uint64_t rec_words = 2 + 2 * uint64_t(n_cols) + 4 * uint64_t(depth);
  const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= uint64_t(count) * per) return;
  const uint64_t q = t / per, k = t % per;
  uint64_t* rec = out + q * rec_words;
  if (k < uint64_t(n_cols)) {
    const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(cw + k * n_ext + idx[q]);
    rec[1 + 2 * k] = v.x;
    rec[2 + 2 * k] = v.y;
  } else if (k < uint64_t(n_cols) + depth) {
    const int l = int(k - n_cols);
    const uint64_t off = level_off[l] + ((idx[q] >> l) ^ 1);
    const ulonglong2 a = *reinterpret_cast<const ulonglong2*>(tree + 2 * off);
    const ulonglong2 b = *reinterpret_cast<const ulonglong2*>(tree + 2 * off + 1);
    uint64_t* d = rec + 2 + 2 * uint64_t(n_cols) + 4 * uint64_t(l);
    d[0] = a.x; d[1] = a.y; d[2] = b.x; d[3] = b.y;
  } else if (k == uint64_t(n_cols) + depth) {
    rec[0] = uint64_t(n_cols);
  } else {
    rec[1 + 2 * uint64_t(n_cols)] = uint64_t(depth);
  }
}
// out[c] partials: sum_{r in chunk} w[r] * cw[c * n_ext + r], r < n_rows.
__global__ void k_row_project(const Fe* __restrict__ cw, uint64_t n_ext, uint64_t n_rows, const Fe* __restrict__ hi,
                              const Fe* __restrict__ lo, int lb, Fe* __restrict__ partials) {
  const int c = blockIdx.y;
  Acc acc = acc_zero();
  for (uint64_t r = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < n_rows; r += uint64_t(gridDim.x) * blockDim.x)
    mul_acc(acc, table_at(hi, lo, lb, r), load(cw + uint64_t(c) * n_ext + r));
  Fr s[1] = {acc_reduce(acc)};
  block_reduce<1>(s);
  if (threadIdx.x == 0) store(partials + size_t(c) * gridDim.x + blockIdx.x, s[0]);
}
// out[r] = sum_c fw[c] * cw[c * n_ext + r], r < n_rows (base_systematic_fold).
__global__ void k_row_fold(const Fe* __restrict__ cw, uint64_t n_ext, uint64_t n_rows, int n_cols, const Fe* __restrict__ fw,
                           Fe* __restrict__ out) {
  __shared__ Fe f_s[64];
  if (threadIdx.x < n_cols) f_s[threadIdx.x] = fw[threadIdx.x];
  __syncthreads();
  for (uint64_t r = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; r < n_rows; r += uint64_t(gridDim.x) * blockDim.x) {
    Fr s = zero();
    for (int c = 0; c < n_cols; ++c) s = add(s, mul(load(f_s + c), load(cw + uint64_t(c) * n_ext + r)));
    store(out + r, s);
  }
}

}  // namespace QFD_NS

// Kernels that read the BVA entries themselves (their arithmetic depends on
// the entry width and the modulus).
#if defined(QF_FIELD_KB)
#include "weights_kb.cuh"
#else
#include "weights_f65521.cuh"
#endif
