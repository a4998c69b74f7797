// Error reporting, version and small helpers of the C ABI.
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "common.cuh"

namespace rst {

static thread_local char g_err[512] = "";
static std::atomic<long long> g_launches{0};
static std::mutex g_tune_mu;
static reset_tuning g_tune = {8, 64, 1, 0, {0, 0, 0, 0}};

reset_tuning tuning() {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  return g_tune;
}

void note_launch(int k) { g_launches.fetch_add(k, std::memory_order_relaxed); }

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

reset_status cuda_fail(cudaError_t e, const char* what, const char* file,
                       int line) {
  const char* base = strrchr(file, '/');
  set_error("%s failed: %s (%s:%d)", what, cudaGetErrorString(e),
            base ? base + 1 : file, line);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();  // allocation failures are not sticky: clear them
    return RESET_ERR_OOM;
  }
  return RESET_ERR_CUDA;
}

reset_status arg_fail(const char* what) {
  set_error("invalid argument: %s", what);
  return RESET_ERR_ARG;
}

int sm_count() {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 148;
}

}  // namespace rst

extern "C" {

const char* reset_last_error_string(void) { return rst::g_err; }

const char* reset_status_string(int32_t s) {
  switch (s) {
    case RESET_OK: return "RESET_OK";
    case RESET_ERR_CUDA: return "RESET_ERR_CUDA";
    case RESET_ERR_OOM: return "RESET_ERR_OOM";
    case RESET_ERR_ARG: return "RESET_ERR_ARG";
    case RESET_ERR_TABLE_FULL: return "RESET_ERR_TABLE_FULL";
    case RESET_ERR_PROBE_LIMIT: return "RESET_ERR_PROBE_LIMIT";
    case RESET_ERR_TIMEOUT: return "RESET_ERR_TIMEOUT";
    case RESET_ERR_UNSUPPORTED: return "RESET_ERR_UNSUPPORTED";
    case RESET_ERR_BUSY: return "RESET_ERR_BUSY";
    default: return "RESET_ERR_UNKNOWN";
  }
}

int32_t reset_abi_version(void) { return RESET_ABI_VERSION; }

int64_t reset_kernel_launches(void) {
  return rst::g_launches.load(std::memory_order_relaxed);
}

void reset_params_default(reset_params* p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->alpha = 0.2f;
  p->bucket = 5;
}

reset_status reset_get_tuning(reset_tuning* out) {
  if (!out) return rst::arg_fail("NULL tuning");
  *out = rst::tuning();
  return RESET_OK;
}

reset_status reset_set_tuning(const reset_tuning* in) {
  if (!in) return rst::arg_fail("NULL tuning");
  if (in->probe_rounds != 2 && in->probe_rounds != 4 && in->probe_rounds != 8)
    return rst::arg_fail("probe_rounds must be 2, 4 or 8");
  if (in->probe_rounds == 8 && in->probe_variant != 1)
    return rst::arg_fail("probe_rounds 8 needs probe_variant 1");
  if (in->warp_pair_min < 1 || in->warp_pair_min > (1 << 20))
    return rst::arg_fail("warp_pair_min must be in 1..2^20");
  if (in->probe_variant != 0 && in->probe_variant != 1)
    return rst::arg_fail("probe_variant must be 0 or 1");
  if (in->pair_method < 0 || in->pair_method > 2)
    return rst::arg_fail("pair_method must be 0, 1 or 2");
  std::lock_guard<std::mutex> lock(rst::g_tune_mu);
  rst::g_tune = *in;
  return RESET_OK;
}

reset_status reset_free(void* d_ptr) {
  if (d_ptr) RST_CUDA(cudaFree(d_ptr));
  return RESET_OK;
}

}  // extern "C"
