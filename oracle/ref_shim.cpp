// extern "C" shim over the reference's own FileWriter/FileReader
// (src/md_common.cpp) and MDConfigManager (src/md_config.cpp), compiled
// together with those sources into oracle/_ref/libref_io.so.
// TEST INFRASTRUCTURE ONLY: used by tests/ to pin the PFRAME and config JSON
// formats against the reference implementation.
#include <cstring>
#include <string>
#include <vector>

#include "md_common.hpp"
#include "md_config.hpp"

namespace {
int put(const std::string& s, char* out, size_t cap) {
  if (s.size() + 1 > cap) return -1;
  std::memcpy(out, s.c_str(), s.size() + 1);
  return (int)s.size();
}
}  // namespace

extern "C" {

// deserialize(json) then serialize() (compact form).
int ref_config_roundtrip(const char* json_in, char* out, size_t cap) {
  try {
    MDConfigManager m;
    m.deserialize(json_in);
    return put(m.serialize(), out, cap);
  } catch (...) {
    return -2;
  }
}

// config_from_json(path) then config_to_json(path_out) (pretty, dump(4)).
int ref_config_file_roundtrip(const char* path_in, const char* path_out) {
  try {
    MDConfigManager m = MDConfigManager::config_from_json(path_in);
    m.config_to_json(path_out);
    return 0;
  } catch (...) {
    return -2;
  }
}

// deserialize(json), apply_override(key, value), serialize.
int ref_config_override(const char* json_in, const char* key, const char* value, char* out,
                        size_t cap) {
  try {
    MDConfigManager m;
    m.deserialize(json_in);
    if (!m.apply_override(key, value)) return -3;
    return put(m.serialize(), out, cap);
  } catch (...) {
    return -2;
  }
}

int ref_parse_override(const char* arg, char* key, size_t kcap, char* value, size_t vcap) {
  std::string k, v;
  if (!MDConfigManager::parse_override_argument(arg, k, v)) return 0;
  if (put(k, key, kcap) < 0 || put(v, value, vcap) < 0) return -1;
  return 1;
}

int ref_pframe_write(const char* path, int append, const void* frame, unsigned long long n,
                     unsigned long long index) {
  try {
    FileWriter w(path, append != 0);
    w.write_frame(static_cast<const Particle*>(frame), (std::size_t)n, index);
    return 0;
  } catch (...) {
    return -2;
  }
}

// Scans for frame `index`; returns its particle count (copies when it fits),
// -1 when absent, -2 on open errors, -4 when the file is corrupted.
long long ref_pframe_read(const char* path, unsigned long long index, void* out,
                          unsigned long long cap) {
  try {
    FileReader r(path);
    std::vector<Particle> buf;
    std::uint64_t idx = 0;
    while (r.next_frame(buf, idx)) {
      if (idx == index) {
        if (buf.size() <= cap) std::memcpy(out, buf.data(), buf.size() * sizeof(Particle));
        return (long long)buf.size();
      }
    }
    return r.corrupted() ? -4 : -1;
  } catch (...) {
    return -2;
  }
}

}  // extern "C"
