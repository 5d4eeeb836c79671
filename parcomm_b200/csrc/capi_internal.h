// Shared pieces of the extern "C" boundary: the parameter handle, the
// per-thread last-error message and the exception guard that turns a QfError
// into its QF_E_* return code.
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <new>
#include <stdexcept>
#include <string>

#include "host/protocol.h"

namespace qfg {
class DeviceTables;
}

struct qf_params {
  int field = 0;
  std::unique_ptr<qf::Parameters<qf::Fp8>> P;
  std::shared_ptr<qfg::DeviceTables> tables;  // device code tables shared by its commitments
};

namespace qfc {

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
