// Error plumbing of the C ABI: every failure stores a message in a
// thread-local buffer (mdb_last_error) and returns a status code.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "mdb200.h"

namespace mdb {

int set_error(int code, const std::string& msg);
int cuda_error(cudaError_t e, const char* what);
void count_launches(long long n);

int config_from_json_text(const char* text, mdb_config_t* out);
std::string config_to_json_text(const mdb_config_t* cfg, int indent);
int config_apply_override(mdb_config_t* cfg, const char* key, const char* value);

}  // namespace mdb

#define MDB_CUDA(call)                                           \
  do {                                                           \
    cudaError_t mdb_e_ = (call);                                 \
    if (mdb_e_ != cudaSuccess) return ::mdb::cuda_error(mdb_e_, #call); \
  } while (0)
