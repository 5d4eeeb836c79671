/* C ABI of the B200 QAFold commit+open library (libparcomm_qafold.so).
 *
 * Each entry point replaces one public call of the reference Rust prover
 * (qafold/f65521/src/protocol.rs, tbv.rs, main.rs).  Every call returns 0 or
 * a negative QF_E_* code; qf_last_error() returns the message of the last
 * failure on the calling thread (the reference's `check` strings and
 * mikros_qafold::Error variants, vendor/qafold/src/lib.rs:20-35).
 *
 * Wire formats
 *   points : per matrix, in shape order: row point then column point, each
 *            coordinate a 16-byte canonical extension element; the row
 *            point has log2(next_pow2(rows)) coordinates, the column point
 *            log2(next_pow2(cols)) (tbv.rs:128-142).
 *   claims : per matrix: row point, column point, value (16 bytes each).
 *   proof  : the reference's bincode-fixint Proof (protocol.rs:88-107).
 */
#ifndef PARCOMM_QAFOLD_H
#define PARCOMM_QAFOLD_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QF_FIELD_F65521 1    /* F65521^8, signed 8-bit weights */
#define QF_FIELD_KOALABEAR 2 /* KoalaBear^4, signed 16-bit payloads */

#define QF_OK 0
#define QF_E_ENCODING -1
#define QF_E_HASHING -2
#define QF_E_INVALID_COMMITMENT -3
#define QF_E_INVALID_NUMBER_OF_VARIABLES -4
#define QF_E_INVALID_PARAMETERS -5
#define QF_E_TRANSCRIPT -6
#define QF_E_PROTOCOL -7
#define QF_E_CUDA -8
#define QF_E_ARGUMENT -9
#define QF_E_NO_DEVICE -10

typedef struct qf_params qf_params;       /* Parameters (protocol.rs:41-46) */
typedef struct qf_committed qf_committed; /* Committed, device-resident (protocol.rs:47-51) */

typedef struct {
  uint64_t rows, cols;
} qf_shape; /* layout::Shape (layout.rs:4-8) */

typedef struct {
  uint32_t chunk_log, packed_log, query_rf_bits;
} qf_config; /* protocol::Config (protocol.rs:18-32) */

typedef struct {
  double commit_ms, upload_ms, eo_ms, projection_ms, folding_ms, sumcheck_ms, binding_ms, native_opening_ms, decide_ms,
      open_ms;
  uint64_t kernel_launches;
} qf_profile; /* ProverProfile (protocol.rs:67-80), milliseconds */

/* Parameters::new(shapes, config) (protocol.rs:109-130).  The setup's large
 * levels are encoded and their rows hashed on the current device when the
 * process has one (the rest of the setup, and all of it in a process
 * without a device, runs on the host threads); either way the parameter
 * digest is the same.  A parameter set's setup is built once per process. */
int qf_params_new(int field, const qf_shape* shapes, size_t n_shapes, const qf_config* config, qf_params** out);
void qf_params_free(qf_params* params);
/* Layout facts and Commitment::parameter_digest (layout.rs:56-114, packed.rs:161). */
int qf_params_info(const qf_params* params, uint64_t* active, uint64_t* logical, uint64_t* blocks, uint64_t* buckets,
                   uint8_t parameter_digest[32]);

/* Parameters::commit / commit_recomputed (protocol.rs:131-185): validates the
 * BVA padding, keeps the weights and codewords in HBM and writes the block
 * roots (blocks * 32 bytes).  `bva` holds `n_values` signed entries (int8 for
 * F65521, int16 for KoalaBear) in host memory, or in device memory when
 * `bva_on_device` is nonzero.  The library reads device weights on its own
 * streams: the caller's writes to them must be complete (synchronise the
 * stream that produced them) before the call.  Both cache modes produce identical bytes. */
int qf_commit(const qf_params* params, const void* bva, uint64_t n_values, int bva_on_device, qf_committed** out,
              uint8_t* roots_out);
void qf_committed_free(qf_committed* committed);

/* Parameters::commit_recomputed (protocol.rs:131-185, the reference's
 * `--cache-mode recompute`): only the block roots stay in HBM, and binding
 * re-encodes every block.  `host_bva` holds n_values entries in host memory
 * (for weight sets larger than HBM; page-locked memory lets the copies
 * overlap the compute) or in device memory (weights resident, codewords
 * recomputed: a pool of many commitments; its producer must have finished
 * writing it, as for qf_commit).  It stays owned by the caller and must stay
 * valid and unchanged until the committed handle is freed.  Every pass that reads the
 * weights (commit, EO cross terms and witness, projection, block fold) stages
 * them into HBM one PCS block at a time, and binding re-encodes each block
 * and checks its root.  The first resident_bytes / (2^chunk_log * entry size)
 * blocks are kept in HBM after the first pass; QF_RESIDENT_AUTO sizes that
 * from the device's free memory less the proof's own peak.  Needs at least
 * two PCS blocks.  Writes the same roots, claims and proof bytes as
 * qf_commit. */
#define QF_RESIDENT_AUTO UINT64_MAX
int qf_commit_streamed(const qf_params* params, const void* host_bva, uint64_t n_values, uint64_t resident_bytes,
                       qf_committed** out, uint8_t* roots_out);
/* For a qf_commit_streamed handle: bytes of weights copied host->device so
 * far, and the PCS blocks kept in HBM out of the blocks holding weights (all
 * 0 for qf_commit handles).  Any output pointer may be NULL.  No reference
 * counterpart. */
int qf_committed_stream_info(const qf_committed* committed, uint64_t* h2d_bytes, uint64_t* resident_blocks,
                             uint64_t* live_blocks);

/* serde_json of the Commitment statement (protocol.rs:33-40), as absorbed. */
int qf_statement_json(const qf_params* params, const uint8_t* roots, char* buf, size_t cap, size_t* len);

/* The demo/benchmark points of main.rs:190-204 derived from the statement. */
int qf_benchmark_points(const qf_params* params, const uint8_t* roots, uint8_t* points, size_t cap, size_t* len);

/* tbv::evaluate_claims (tbv.rs:143-185) over the committed weights. */
int qf_eval_claims(const qf_params* params, const qf_committed* committed, const uint8_t* points, size_t points_len,
                   uint8_t* claims, size_t cap, size_t* len);

/* Parameters::prove + Proof::to_bytes (protocol.rs:201-263, 88-96).  The
 * proof buffer is allocated by the library; release it with qf_free_bytes.
 * The committed state is consumed (as in the reference) and must still be
 * released with qf_committed_free. */
int qf_prove(const qf_params* params, qf_committed* committed, const uint8_t* claims, size_t claims_len, uint8_t** proof,
             size_t* proof_len, qf_profile* profile);

/* Like qf_prove, but leaves the committed handle usable for further
 * openings (a serving pool answers many claims on one commitment).  Calls on
 * one handle must not overlap; handles are independent.  No reference
 * counterpart: the reference's prove consumes Committed. */
int qf_open(const qf_params* params, const qf_committed* committed, const uint8_t* claims, size_t claims_len,
            uint8_t** proof, size_t* proof_len, qf_profile* profile);

/* Proof::from_bytes + Parameters::verify (protocol.rs:97-107, 266-320). Host only. */
int qf_verify(const qf_params* params, const uint8_t* roots, const uint8_t* claims, size_t claims_len, const uint8_t* proof,
              size_t proof_len);

/* LogUp range audit of committed weights over the entry type's table: the
 * 256 values -128..127 for int8 weights, the 65536 values -32768..32767 for
 * int16 payloads.  It is a check beside the proof: nothing of it enters a
 * transcript or the proof bytes, and it has no reference counterpart (the
 * values enter the field through field::small, field.rs:24-29).
 *
 * alpha is an extension element outside the base field, drawn from `seed` by
 * BLAKE2s (domain "parcomm-b200/logup-range-audit/v1"; bind it to the
 * commitment by hashing the roots into the seed).  On the device, one pass
 * over the committed weights accumulates lhs = sum_i 1 / (alpha - v_i) value by
 * value and counts each table value's multiplicity m_t; then rhs =
 * sum_t m_t / (alpha - t).  Writes the multiplicities (n_bins must be 256 or
 * 65536 to match the field; bin k counts the value k - 128 or k - 32768),
 * alpha, lhs and rhs (16 canonical bytes each) and *holds = 1 when lhs == rhs
 * and the multiplicities add up to the active entries, else 0.  Any output
 * pointer may be NULL.  Works on qf_commit and qf_commit_streamed handles
 * (streamed weights are staged block by block as in the proof's passes). */
int qf_range_audit(const qf_params* params, const qf_committed* committed, const uint8_t seed[32], uint64_t* multiplicities,
                   size_t n_bins, uint8_t alpha[16], uint8_t lhs[16], uint8_t rhs[16], int* holds);

void qf_free_bytes(uint8_t* bytes);

/* One proof over PCS blocks spread across ranks (one process per device), no
 * reference counterpart: the batch opening of Parameters::prove
 * (protocol.rs:201-263) with rank `rank` of `world` holding the contiguous
 * run of blocks [B rank / world, B (rank + 1) / world).  Every rank passes the
 * same host BVA and claims (null: the benchmark points, each rank's part of
 * the claim values summed); only its blocks are copied to the current
 * device.  The ranks exchange through the caller's collectives:
 *   gather(ctx, in, n, out): out = every rank's n bytes of `in`, in rank order;
 *   reduce(ctx, data, n): data[i] = the sum over the ranks of data[i]
 *     (64-bit, below 2^63); may be null, the sums then use `gather`.
 * Both return 0 on success.  Every rank gets the roots (blocks x 32 bytes)
 * and the proof that one device holding all blocks writes (malloc'd; free
 * with qf_free_bytes).  Calls on the ranks must be made together: a rank that
 * fails leaves the others waiting in their collectives until those time
 * out.  Needs 1 <= world <= blocks. */
typedef int (*qf_gather_fn)(void* ctx, const void* in, size_t n, void* out);
typedef int (*qf_reduce_fn)(void* ctx, uint64_t* data, size_t n);
int qf_prove_sharded(const qf_params* params, const void* host_bva, uint64_t n_values, int rank, int world,
                     qf_gather_fn gather, qf_reduce_fn reduce, void* ctx, const uint8_t* claims, size_t claims_len,
                     uint8_t* roots_out, uint8_t** proof, size_t* proof_len);

/* Diagnostics (no reference counterpart): per-kernel device time measured with
 * CUDA events on each kernel's launching stream.  qf_kernel_timing(1) resets
 * and enables recording; qf_kernel_stats writes JSON
 * {"kernel": {"launches": n, "ms": t}, ...}.  qf_kernel_launches counts every
 * kernel launched by this library since load. */
int qf_kernel_timing(int enable);
int qf_kernel_stats(char* buf, size_t cap, size_t* len);
uint64_t qf_kernel_launches(void);
/* Diagnostics, no reference counterpart: the current device's integer issue
 * peaks in thread-level operations per second, measured by a microbenchmark
 * (independent chains of 32-bit XORs, of 32-bit multiply-adds, of both
 * interleaved, of 32 x 32 -> 64-bit multiply-adds, of dp4a and of funnel-shift
 * rotations): out[0] the ALU pipe, out[1] the FMA pipe, out[2] both, out[3]
 * widening multiply-adds, out[4] dp4a, out[5] rotations.  They are the
 * denominators of the integer roofline; qf_kernel_stats reports each kernel's
 * algorithmic integer operations as "ops". */
int qf_kernel_int_peaks(double out[6]);
/* Diagnostics, no reference counterpart: process-wide kernel choices that
 * write identical bytes, for comparisons.  "imma" (default 0): 1 makes the
 * F65521 weight passes (EO witness, block fold, equality-table lane sums)
 * contract on the tensor cores with exact integer limbs instead of the dp4a
 * / IMAD kernels (measured slower on B200; kept for the comparison).  "per_matrix"
 * (default 0): 1 issues the weight passes one launch per term, bucket or
 * block instead of one launch over all of them.  "core_dots" chooses where
 * the sums of extension products of the EO binary rounds, the sumcheck
 * messages and the LiteBullet rounds run: 0 (default) per kernel, as
 * measured fastest on B200; 1 all with CUDA-core multiply-adds; 2 all as
 * exact integer-limb tensor-core products.  Set it between calls, not while
 * another call runs. */
int qf_kernel_option(const char* name, int value);

/* Device buffers released by the library are cached for reuse (no cudaMalloc
 * on repeated proofs); at most `bytes` stay cached, the rest is freed at once
 * (default: unlimited).  A request that does not fit frees cached blocks,
 * largest first, until it fits, then waits up to half a second for
 * concurrent work to release memory.
 * A caller that budgets HBM itself (a serving loop) sets a limit.  No
 * reference counterpart. */
int qf_device_cache_limit(uint64_t bytes);
size_t qf_last_error(char* buf, size_t cap);

/* No counterpart in the reference: a commitment entry point that allocates
 * no device memory, for callers that cannot (a serving engine that reserves
 * nearly all of HBM for its own pool; a latency-bound loop that cannot take
 * the synchronisation cudaMalloc/cudaFree may imply).
 *
 * Writes the root of PCS block `block` (the bytes qf_commit writes at
 * roots_out + 32 * block) to the 32 device bytes `d_root`, asynchronously on
 * `stream` (a cudaStream_t; NULL is the legacy default stream).  `d_bva` is
 * a device pointer to the n_values active int8 entries.  Unlike qf_commit it
 * neither copies the weights nor checks the layout's zero padding.
 *
 * Limit: F65521 blocks of at most 2^QF_NOALLOC_MAX_CHUNK_LOG weights
 * (config chunk_log <= 20); larger blocks return QF_E_ARGUMENT.  All working
 * buffers live in one static device array of QF_NOALLOC_SCRATCH_BYTES, which
 * every GPU that loads the library holds until the process exits.  The call
 * runs on the current device and uses that device's copy of the array:
 * d_bva, d_root and the stream must belong to it (QF_E_ARGUMENT otherwise).
 * The first call on a device looks up that array's address there
 * (cudaGetSymbolAddress), and looks it up again if the device's context has
 * changed since (after cudaDeviceReset); make that first call before any
 * stream capture.  The array also holds the code's alpha table: a call whose
 * parameter set differs from the previous call's on that device copies the
 * table in from host memory and waits for that copy (the host blocks until
 * the stream reaches it); calls with the same parameter set copy nothing.
 * Every call shares the array, which keeps the last call's contents (nothing
 * in it has to start at zero: each word a call reads, the same call or the
 * table copy wrote first); calls that overlap on the GPU (other streams or
 * host threads on the same device) race, so serialise them. */
#define QF_NOALLOC_MAX_CHUNK_LOG 20
#define QF_NOALLOC_SCRATCH_BYTES (5u << 20)
int qf_commit_block_noalloc(const qf_params* params, const int8_t* d_bva, uint64_t n_values, uint64_t block,
                            uint8_t* d_root, void* stream);

#ifdef __cplusplus
}
#endif
#endif
