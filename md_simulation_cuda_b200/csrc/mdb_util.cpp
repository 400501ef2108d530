#include "mdb_util.h"

#include <string.h>

#include <atomic>

namespace mdb {

static thread_local std::string g_last_error;
static std::atomic<long long> g_launches{0};

int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_error(cudaError_t e, const char* what) {
  return set_error(MDB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorName(e) + " (" +
                                     cudaGetErrorString(e) + ")");
}

void count_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

}  // namespace mdb

extern "C" {

int mdb_last_error(char* buf, size_t cap) {
  if (!buf || cap == 0) return MDB_ERR_ARG;
  size_t k = mdb::g_last_error.size();
  if (k + 1 > cap) k = cap - 1;
  memcpy(buf, mdb::g_last_error.data(), k);
  buf[k] = '\0';
  return MDB_OK;
}

const char* mdb_version(void) { return "mdb200 0.1.0 (sm_100a)"; }

int64_t mdb_kernel_launches(void) { return (int64_t)mdb::g_launches.load(); }

}  // extern "C"
