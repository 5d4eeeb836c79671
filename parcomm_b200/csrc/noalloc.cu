// qf_commit_block_noalloc: the commitment root of one PCS block, computed in a
// fixed device array instead of allocated memory.
//
// Some callers cannot allocate device memory from this library.  A serving
// engine that reserves nearly all of HBM up front for its own pool (KV cache,
// weights) has nothing left for cudaMalloc, and a latency-bound loop cannot
// afford the device-wide synchronisation that cudaMalloc/cudaFree may imply.
// For them this entry point takes every working buffer (codeword, Merkle
// tree, alpha table) from g_noalloc_scratch, a static __device__ array that
// each GPU loading the library holds until the process exits.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/parcomm_qafold.h"
#include "capi_internal.h"
#include "gpu_backend.cuh"

namespace {

using qf::check;
using qf::fail;
using qfd::Fe;

// Largest block: 2^20 weights = 2^17 packed elements, 32 columns of R = 2^12
// message rows.  Codeword 2 * 2^17 * 16 B = 4 MiB, tree 4 * 2R * 16 B =
// 512 KiB, alpha R * 16 B = 64 KiB.
constexpr uint32_t kMaxChunkLog = QF_NOALLOC_MAX_CHUNK_LOG;
constexpr size_t kMaxPacked = size_t(1) << (kMaxChunkLog - 3);
constexpr size_t kScratchBytes = QF_NOALLOC_SCRATCH_BYTES;

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

size_t align256(size_t v) { return (v + 255) / 256 * 256; }

struct ScratchLayout {
  size_t cw = 0, tree = 0, alpha = 0, end = 0;
  ScratchLayout(size_t packed, size_t cols) {
    const size_t R = packed / cols;
    cw = 0;
    tree = align256(cw + 2 * packed * sizeof(Fe));
    alpha = align256(tree + 4 * (2 * R) * sizeof(uint4));
    end = align256(alpha + R * sizeof(Fe));
  }
};
static_assert(2 * kMaxPacked * 16 + 4 * (2 * (kMaxPacked / 32)) * 16 + (kMaxPacked / 32) * 16 + 3 * 256 <= kScratchBytes,
              "scratch too small for the largest block");

// Device address of g_noalloc_scratch, resolved once per device with that
// device current (the first call on a device does it).
constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};

void* scratch_on_current_device() {
  int dev = 0;
  QF_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) fail(QF_E_ARGUMENT, "device index out of range");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      fail(QF_E_CUDA, std::string("CUDA: cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
    g_scratch_addr[dev] = p;
  }
  return g_scratch_addr[dev];
}

}  // namespace

extern "C" int qf_commit_block_noalloc(const qf_params* params, const int8_t* d_bva, uint64_t n_values, uint64_t block,
                                       uint8_t* d_root, void* stream) {
  return qfc::guarded([&] {
    if (!params || !d_root || (!d_bva && n_values)) fail(QF_E_ARGUMENT, "null argument");
    if (params->field != QF_FIELD_F65521) fail(QF_E_ARGUMENT, "qf_commit_block_noalloc supports F65521 only");
    const auto& P = *static_cast<const qf::Parameters<qf::Fp8>*>(params->P.get());
    if (P.chunk_log() > kMaxChunkLog)
      fail(QF_E_ARGUMENT, "qf_commit_block_noalloc: block of 2^" + std::to_string(P.chunk_log()) +
                              " weights exceeds the limit of 2^" + std::to_string(kMaxChunkLog) + " (" +
                              std::to_string(kScratchBytes >> 20) + " MiB static scratch); use qf_commit");
    check(n_values == P.layout.active, "active BVA length mismatch");
    if (block >= P.blocks()) fail(QF_E_ARGUMENT, "block index out of range");
    qfc::require_device();
    const size_t packed = P.pcs.packed_len(), cols = P.pcs.pp->extension_columns;
    const ScratchLayout L(packed, cols);
    check(L.end <= kScratchBytes, "scratch layout exceeds the static array");
    unsigned char* base = static_cast<unsigned char*>(scratch_on_current_device());
    qfg::commit_block_into(P, d_bva, n_values, size_t(block), reinterpret_cast<Fe*>(base + L.cw),
                           reinterpret_cast<uint4*>(base + L.tree), reinterpret_cast<Fe*>(base + L.alpha), d_root,
                           static_cast<cudaStream_t>(stream));
  });
}
