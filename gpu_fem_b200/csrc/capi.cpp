// Library-level C ABI: status strings, version, last-error text.
#include <atomic>
#include <cstdio>
#include <string>

#include "gf_internal.h"

namespace gf {
static thread_local std::string g_last_error;
void set_last_error(const char* where, cudaError_t e) {
  g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
}
void set_last_error_text(const std::string& text) { g_last_error = text; }
static std::atomic<long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
}  // namespace gf

extern "C" {

long long gf_launch_count(void) { return gf::g_launches.load(); }

const char* gf_status_string(gf_status s) {
  switch (s) {
    case GF_OK: return "ok";
    case GF_INVALID_ARG: return "invalid argument";
    case GF_OOM: return "out of device memory";
    case GF_ZERO_PIVOT: return "zero pivot in ILU factorization";
    case GF_NOT_CONVERGED: return "solver did not converge";
    case GF_NAN: return "NaN detected";
    case GF_TIMEOUT: return "device wait exceeded its spin limit";
    case GF_CUDA_ERROR: return "CUDA error";
    case GF_NO_DEVICE: return "no CUDA device";
    case GF_OVER_BUDGET: return "request exceeds the HBM budget";
  }
  return "unknown status";
}

const char* gf_version(void) { return "gpufem-b200 0.1 (sm_100a)"; }

const char* gf_last_error(void) { return gf::g_last_error.c_str(); }

}  // extern "C"
