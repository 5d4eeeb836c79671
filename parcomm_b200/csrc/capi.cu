// extern "C" boundary of libparcomm_qafold.so (declared in include/parcomm_qafold.h).
// Argument checks and the field dispatch live here; each field's bodies are
// in capi_field.cu, compiled once per field.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>

#include "capi_internal.h"
#include "gpu_common.cuh"

using namespace qf;
using qfc::guarded;
using qfc::require_device;

namespace {

const qfc::FieldApi& api(int field) {
  if (field == QF_FIELD_F65521) return qfg::kFieldApi;
  if (field == QF_FIELD_KOALABEAR) return qfgkb::kFieldApi;
  fail(QF_E_INVALID_PARAMETERS, "unknown field");
}

void copy_out(const std::vector<uint8_t>& src, uint8_t* dst, size_t cap, size_t* len) {
  if (len) *len = src.size();
  if (dst) {
    if (cap < src.size()) fail(QF_E_ARGUMENT, "output buffer too small");
    std::memcpy(dst, src.data(), src.size());
  }
}

}  // namespace

extern "C" {

int qf_params_new(int field, const qf_shape* shapes, size_t n_shapes, const qf_config* config, qf_params** out) {
  return guarded([&] {
    if (!out || !config || (!shapes && n_shapes)) fail(QF_E_ARGUMENT, "null argument");
    const qfc::FieldApi& f = api(field);
    std::vector<Shape> sh;
    for (size_t i = 0; i < n_shapes; ++i) sh.push_back({size_t(shapes[i].rows), size_t(shapes[i].cols)});
    Config c;
    c.chunk_log = config->chunk_log;
    c.packed_log = config->packed_log;
    c.query_rf_bits = config->query_rf_bits;
    auto p = std::make_unique<qf_params>();
    p->field = field;
    f.make_params(p.get(), sh, c);
    *out = p.release();
  });
}

void qf_params_free(qf_params* params) { delete params; }

int qf_params_info(const qf_params* params, uint64_t* active, uint64_t* logical, uint64_t* blocks, uint64_t* buckets,
                   uint8_t parameter_digest[32]) {
  return guarded([&] {
    if (!params) fail(QF_E_ARGUMENT, "null params");
    api(params->field).info(params, active, logical, blocks, buckets, parameter_digest);
  });
}

int qf_commit(const qf_params* params, const void* bva, uint64_t n_values, int bva_on_device, qf_committed** out,
              uint8_t* roots_out) {
  return guarded([&] {
    if (!params || !out || (!bva && n_values)) fail(QF_E_ARGUMENT, "null argument");
    require_device();
    auto c = std::make_unique<qf_committed>();
    c->params = params;
    api(params->field).commit(params, bva, n_values, bva_on_device, c.get(), roots_out);
    *out = c.release();
  });
}

int qf_commit_streamed(const qf_params* params, const void* host_bva, uint64_t n_values, uint64_t resident_bytes,
                       qf_committed** out, uint8_t* roots_out) {
  return guarded([&] {
    if (!params || !out || (!host_bva && n_values)) fail(QF_E_ARGUMENT, "null argument");
    require_device();
    auto c = std::make_unique<qf_committed>();
    c->params = params;
    api(params->field).commit_streamed(params, host_bva, n_values, resident_bytes, c.get(), roots_out);
    *out = c.release();
  });
}

void qf_committed_free(qf_committed* committed) { delete committed; }

int qf_committed_stream_info(const qf_committed* committed, uint64_t* h2d_bytes, uint64_t* resident_blocks,
                             uint64_t* live_blocks) {
  return guarded([&] {
    if (!committed) fail(QF_E_ARGUMENT, "null argument");
    if (committed->state) {
      api(committed->params->field).stream_info(committed, h2d_bytes, resident_blocks, live_blocks);
    } else {
      for (uint64_t* p : {h2d_bytes, resident_blocks, live_blocks})
        if (p) *p = 0;
    }
  });
}

int qf_statement_json(const qf_params* params, const uint8_t* roots, char* buf, size_t cap, size_t* len) {
  return guarded([&] {
    if (!params || !roots) fail(QF_E_ARGUMENT, "null argument");
    std::string j = api(params->field).statement_json(params, roots);
    copy_out(std::vector<uint8_t>(j.begin(), j.end()), reinterpret_cast<uint8_t*>(buf), cap, len);
  });
}

int qf_benchmark_points(const qf_params* params, const uint8_t* roots, uint8_t* points, size_t cap, size_t* len) {
  return guarded([&] {
    if (!params || !roots) fail(QF_E_ARGUMENT, "null argument");
    copy_out(api(params->field).benchmark_points(params, roots), points, cap, len);
  });
}

int qf_eval_claims(const qf_params* params, const qf_committed* committed, const uint8_t* points, size_t points_len,
                   uint8_t* claims, size_t cap, size_t* len) {
  return guarded([&] {
    if (!params || !committed || !points) fail(QF_E_ARGUMENT, "null argument");
    if (committed->consumed) fail(QF_E_ARGUMENT, "committed state already consumed by prove");
    copy_out(api(params->field).eval_claims(params, committed, points, points_len), claims, cap, len);
  });
}

int qf_prove(const qf_params* params, qf_committed* committed, const uint8_t* claims, size_t claims_len, uint8_t** proof,
             size_t* proof_len, qf_profile* profile) {
  return guarded([&] {
    if (!params || !committed || !claims || !proof || !proof_len) fail(QF_E_ARGUMENT, "null argument");
    if (committed->consumed) fail(QF_E_ARGUMENT, "committed state already consumed by prove");
    committed->consumed = true;
    std::vector<uint8_t> bytes = api(params->field).prove(params, committed, claims, claims_len, profile);
    uint8_t* buf = static_cast<uint8_t*>(std::malloc(bytes.size()));
    if (!buf) fail(QF_E_ARGUMENT, "host allocation failed");
    std::memcpy(buf, bytes.data(), bytes.size());
    *proof = buf;
    *proof_len = bytes.size();
  });
}

int qf_verify(const qf_params* params, const uint8_t* roots, const uint8_t* claims, size_t claims_len, const uint8_t* proof,
              size_t proof_len) {
  return guarded([&] {
    if (!params || !roots || !claims || !proof) fail(QF_E_ARGUMENT, "null argument");
    api(params->field).verify(params, roots, claims, claims_len, proof, proof_len);
  });
}

int qf_open(const qf_params* params, const qf_committed* committed, const uint8_t* claims, size_t claims_len,
            uint8_t** proof, size_t* proof_len, qf_profile* profile) {
  return guarded([&] {
    if (!params || !committed || !claims || !proof || !proof_len) fail(QF_E_ARGUMENT, "null argument");
    if (committed->consumed) fail(QF_E_ARGUMENT, "committed state already consumed by prove");
    std::vector<uint8_t> bytes =
        api(params->field).prove(params, const_cast<qf_committed*>(committed), claims, claims_len, profile);
    uint8_t* buf = static_cast<uint8_t*>(std::malloc(bytes.size()));
    if (!buf) fail(QF_E_ARGUMENT, "host allocation failed");
    std::memcpy(buf, bytes.data(), bytes.size());
    *proof = buf;
    *proof_len = bytes.size();
  });
}

int qf_range_audit(const qf_params* params, const qf_committed* committed, const uint8_t seed[32], uint64_t* multiplicities,
                   size_t n_bins, uint8_t alpha[16], uint8_t lhs[16], uint8_t rhs[16], int* holds) {
  return guarded([&] {
    if (!params || !committed || !seed) fail(QF_E_ARGUMENT, "null argument");
    if (committed->consumed) fail(QF_E_ARGUMENT, "committed state already consumed by prove");
    require_device();
    api(params->field).range_audit(params, committed, seed, multiplicities, n_bins, alpha, lhs, rhs, holds);
  });
}

int qf_prove_sharded(const qf_params* params, const void* host_bva, uint64_t n_values, int rank, int world,
                     qf_gather_fn gather, qf_reduce_fn reduce, void* ctx, const uint8_t* claims, size_t claims_len,
                     uint8_t* roots_out, uint8_t** proof, size_t* proof_len) {
  return guarded([&] {
    if (!params || (!host_bva && n_values) || !gather || !proof || !proof_len) fail(QF_E_ARGUMENT, "null argument");
    if (world < 1 || rank < 0 || rank >= world) fail(QF_E_ARGUMENT, "rank and world: need 0 <= rank < world");
    require_device();
    std::vector<uint8_t> bytes = api(params->field).prove_sharded(params, host_bva, n_values, rank, world, gather, reduce,
                                                                  ctx, claims, claims_len, roots_out);
    uint8_t* buf = static_cast<uint8_t*>(std::malloc(bytes.size()));
    if (!buf) fail(QF_E_ARGUMENT, "host allocation failed");
    std::memcpy(buf, bytes.data(), bytes.size());
    *proof = buf;
    *proof_len = bytes.size();
  });
}

void qf_free_bytes(uint8_t* bytes) { std::free(bytes); }

int qf_kernel_timing(int enable) {
  return guarded([&] { qfg::KernelClock::reset(enable != 0); });
}

int qf_kernel_option(const char* name, int value) {
  return guarded([&] {
    const std::string n = name ? name : "";
    if (n == "imma") qfg::KernelOptions::imma = value != 0;
    else if (n == "per_matrix") qfg::KernelOptions::per_matrix = value != 0;
    else if (n == "core_dots") {
      if (value < 0 || value > 2) fail(QF_E_ARGUMENT, "core_dots takes 0, 1 or 2");
      qfg::KernelOptions::core_dots = value;
    }
    else fail(QF_E_ARGUMENT, "unknown kernel option: " + n);
  });
}

int qf_kernel_stats(char* buf, size_t cap, size_t* len) {
  return guarded([&] {
    std::string j = qfg::KernelClock::stats_json();
    copy_out(std::vector<uint8_t>(j.begin(), j.end()), reinterpret_cast<uint8_t*>(buf), cap, len);
  });
}

uint64_t qf_kernel_launches(void) { return qfg::KernelClock::launches.load(); }

int qf_device_cache_limit(uint64_t bytes) {
  return guarded([&] { qfg::DevicePool::set_limit(size_t(bytes)); });
}

size_t qf_last_error(char* buf, size_t cap) {
  if (buf && cap) {
    size_t n = std::min(cap - 1, qfc::g_last_error.size());
    std::memcpy(buf, qfc::g_last_error.data(), n);
    buf[n] = 0;
  }
  return qfc::g_last_error.size();
}

}  // extern "C"
