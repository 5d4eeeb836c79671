// Shared pieces of the extern "C" boundary: the parameter and commitment
// handles (field-independent, with the field's own state behind them), the
// per-field function table, the per-thread last-error message and the
// exception guard that turns a QfError into its QF_E_* return code.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/parcomm_qafold.h"
#include "host/protocol.h"

// State of one commitment, owned by the field's implementation.
struct qf_committed_state {
  virtual ~qf_committed_state() {}
};

struct qf_params {
  int field = 0;
  std::shared_ptr<void> P;       // qf::Parameters<F> of the field
  std::shared_ptr<void> tables;  // the field's device code tables, shared by its commitments
};

struct qf_committed {
  const qf_params* params = nullptr;
  std::unique_ptr<qf_committed_state> state;
  bool consumed = false;
};

namespace qfc {

// One field's implementation of the C ABI calls (capi_field.cu, compiled once
// per field).  Arguments are already checked for null.
struct FieldApi {
  size_t weight_bytes;  // bytes of one BVA entry
  void (*make_params)(qf_params* out, const std::vector<qf::Shape>& shapes, const qf::Config& config);
  void (*info)(const qf_params* p, uint64_t* active, uint64_t* logical, uint64_t* blocks, uint64_t* buckets,
               uint8_t digest[32]);
  void (*commit)(const qf_params* p, const void* bva, uint64_t n_values, int on_device, qf_committed* c,
                 uint8_t* roots_out);
  void (*commit_streamed)(const qf_params* p, const void* host_bva, uint64_t n_values, uint64_t resident_bytes,
                          qf_committed* c, uint8_t* roots_out);
  std::string (*statement_json)(const qf_params* p, const uint8_t* roots);
  std::vector<uint8_t> (*benchmark_points)(const qf_params* p, const uint8_t* roots);
  std::vector<uint8_t> (*eval_claims)(const qf_params* p, const qf_committed* c, const uint8_t* points, size_t len);
  std::vector<uint8_t> (*prove)(const qf_params* p, qf_committed* c, const uint8_t* claims, size_t len, qf_profile* profile);
  void (*verify)(const qf_params* p, const uint8_t* roots, const uint8_t* claims, size_t claims_len, const uint8_t* proof,
                 size_t proof_len);
  // Streamed weights: host->device bytes copied so far, resident and live blocks.
  void (*stream_info)(const qf_committed* c, uint64_t* h2d_bytes, uint64_t* resident_blocks, uint64_t* live_blocks);
  // One rank of a block-sharded proof (host/sharded.h) on the current device.
  std::vector<uint8_t> (*prove_sharded)(const qf_params* p, const void* host_bva, uint64_t n_values, int rank, int world,
                                        qf_gather_fn gather, qf_reduce_fn reduce, void* ctx, const uint8_t* claims,
                                        size_t claims_len, uint8_t* roots_out);
  // LogUp range audit of the committed weights (not part of the proof).
  void (*range_audit)(const qf_params* p, const qf_committed* c, const uint8_t seed[32], uint64_t* mult, size_t n_bins,
                      uint8_t alpha[16], uint8_t lhs[16], uint8_t rhs[16], int* holds);
};

inline thread_local std::string g_last_error;

inline int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

template <class Fn>
int guarded(Fn&& fn) {
  try {
    fn();
    return QF_OK;
  } catch (const qf::QfError& e) {
    return set_error(e.code, e.what());
  } catch (const std::bad_alloc&) {
    return set_error(QF_E_ARGUMENT, "host allocation failed");
  } catch (const std::exception& e) {
    return set_error(QF_E_PROTOCOL, e.what());
  }
}

inline void require_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) qf::fail(QF_E_NO_DEVICE, "no CUDA device available");
}

}  // namespace qfc

namespace qfg {
extern const qfc::FieldApi kFieldApi;  // F65521^8, int8 weights
}
namespace qfgkb {
extern const qfc::FieldApi kFieldApi;  // KoalaBear^4, int16 payloads
}
