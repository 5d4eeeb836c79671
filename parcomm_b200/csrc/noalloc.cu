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
#include <cuda.h>
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

// Per-device set-up state.  The array's device address is looked up once per
// device, with that device current, and again only if the device's context
// changed since (cudaDeviceReset, or a primary context released and made
// again, loads the module anew at another address).  `alpha_digest` names the
// parameter set whose top-code alpha table the array holds.
constexpr int kMaxDevices = 64;
struct DeviceState {
  unsigned long long ctx_id = 0;
  void* addr = nullptr;
  bool has_alpha = false;
  qf::Digest alpha_digest{};
};
std::mutex g_mu;
DeviceState g_state[kMaxDevices];

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Unique id of the calling thread's current context (the driver's
// cuCtxGetId, reached through the runtime so that no libcuda link is needed).
unsigned long long current_context_id() {
  static CtxGetCurrentFn get_current = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q1, q2;
    void* f1 = nullptr;
    void* f2 = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
        q1 == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<CtxGetCurrentFn>(f1);
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
        q2 == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f2);
  });
  if (!get_current || !get_id) fail(QF_E_CUDA, "CUDA: cuCtxGetCurrent/cuCtxGetId entry points unavailable");
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
    fail(QF_E_CUDA, "CUDA: no current context on the calling thread");
  return id;
}

// A device pointer on device `dev` (device or managed memory).
bool on_device(const void* p, int dev) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // clear the error of a pointer the runtime does not know
    return false;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == dev;
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
    // Everything runs on the current device, with its copy of the array: the
    // weights, the root and the stream must belong to it.
    int dev = 0;
    QF_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) fail(QF_E_ARGUMENT, "device index out of range");
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    if ((n_values && !on_device(d_bva, dev)) || !on_device(d_root, dev))
      fail(QF_E_ARGUMENT, "qf_commit_block_noalloc: d_bva and d_root must be memory of the current device");
    int sdev = dev;
    if (cudaStreamGetDevice(s, &sdev) == cudaSuccess && sdev != dev)
      fail(QF_E_ARGUMENT, "qf_commit_block_noalloc: the stream belongs to another device");
    const size_t packed = P.pcs.packed_len(), cols = P.pcs.pp->extension_columns;
    const ScratchLayout L(packed, cols);
    check(L.end <= kScratchBytes, "scratch layout exceeds the static array");
    unsigned char* base = nullptr;
    {
      std::lock_guard<std::mutex> lock(g_mu);
      DeviceState& st = g_state[dev];
      const unsigned long long ctx = current_context_id();
      if (!st.addr || st.ctx_id != ctx) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
          fail(QF_E_CUDA, std::string("CUDA: cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(e));
        st = DeviceState{};
        st.addr = p;
        st.ctx_id = ctx;
      }
      base = static_cast<unsigned char*>(st.addr);
      // The alpha table is the same for every block of a parameter set: it is
      // copied in only when the parameter set differs from the one whose
      // table the array holds, and the copy is waited for, so that a later
      // call on any stream finds it complete.
      const qf::Digest& dg = P.pcs.parameter_digest();
      if (!st.has_alpha || st.alpha_digest != dg) {
        const auto& alphas = P.pcs.pp->seq.top().alphas[1];
        check(alphas.size() * sizeof(Fe) <= L.end - L.alpha, "alpha table exceeds its scratch region");
        st.has_alpha = false;
        QF_CK(cudaMemcpyAsync(base + L.alpha, alphas.data(), alphas.size() * sizeof(Fe), cudaMemcpyHostToDevice, s));
        QF_CK(cudaStreamSynchronize(s));
        st.has_alpha = true;
        st.alpha_digest = dg;
      }
    }
    qfg::commit_block_into(P, d_bva, n_values, size_t(block), reinterpret_cast<Fe*>(base + L.cw),
                           reinterpret_cast<uint4*>(base + L.tree), reinterpret_cast<const Fe*>(base + L.alpha), d_root, s);
  });
}
