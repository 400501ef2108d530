// PFRAME v2 trajectory files (include/md_common.hpp:17-31,
// src/md_common.cpp:110-320): a 16-byte file header {"PFRAME\0\0", u32 version
// = 2, u32 reserved = 0}, then per frame a packed 36-byte header
// {u64 frame_index, u64 n_particles, u64 uncompressed_bytes,
// u64 compressed_bytes, u32 crc32 of the uncompressed bytes} and the zlib
// compress2(level 9) payload of Particle[n]. The layout has to match the
// reference byte for byte so both programs read each other's files.
#include <stdio.h>
#include <string.h>
#include <zlib.h>

#include <string>
#include <vector>

#include "mdb200.h"
#include "mdb_util.h"

namespace mdb {
namespace {

#pragma pack(push, 1)
struct FileHeader {
  char magic[8];
  uint32_t version;
  uint32_t reserved;
};
struct FrameHeader {
  uint64_t frame_index;
  uint64_t n_particles;
  uint64_t uncompressed_bytes;
  uint64_t compressed_bytes;
  uint32_t crc32;
};
#pragma pack(pop)
static_assert(sizeof(FileHeader) == 16, "FileHeader layout");
static_assert(sizeof(FrameHeader) == 36, "FrameHeader layout");
static_assert(sizeof(mdb_particle_t) == 64, "Particle layout");

bool read_exact(FILE* f, void* buf, size_t n) {
  if (n == 0) return true;
  return fread(buf, 1, n, f) == n;
}

int check_header(FILE* f, const char* path) {
  FileHeader h;
  if (!read_exact(f, &h, sizeof(h)))
    return set_error(MDB_ERR_IO, std::string("Failed to read file header: ") + path);
  if (memcmp(h.magic, "PFRAME", 6) != 0)
    return set_error(MDB_ERR_IO, std::string("Not a valid PFRAME file: ") + path);
  if (h.version == 1)
    return set_error(MDB_ERR_IO,
                     "File format v1 is incompatible with the v2 Particle layout (theta field)");
  if (h.version != 2)
    return set_error(MDB_ERR_IO, "Unknown file version: " + std::to_string(h.version));
  return MDB_OK;
}

// Reads the next frame. Returns 1 with a frame, 0 at a clean end, <0 on a
// corrupt or truncated frame.
int next_frame(FILE* f, FrameHeader& fh, std::vector<unsigned char>& raw) {
  size_t got = fread(&fh, 1, sizeof(fh), f);
  if (got == 0) return 0;
  if (got != sizeof(fh)) return -1;
  if (fh.uncompressed_bytes != fh.n_particles * sizeof(mdb_particle_t) ||
      fh.compressed_bytes == 0)
    return -2;
  std::vector<unsigned char> comp((size_t)fh.compressed_bytes);
  if (!read_exact(f, comp.data(), comp.size())) return -3;
  raw.resize((size_t)fh.uncompressed_bytes);
  uLongf dl = (uLongf)fh.uncompressed_bytes;
  int z = uncompress(raw.data(), &dl, comp.data(), (uLong)comp.size());
  if (z != Z_OK || dl != fh.uncompressed_bytes) return -4;
  uint32_t crc = (uint32_t)crc32(0L, Z_NULL, 0);
  crc = (uint32_t)crc32(crc, raw.data(), (uInt)raw.size());
  if (crc != fh.crc32) return -5;
  return 1;
}

}  // namespace
}  // namespace mdb

extern "C" {

int mdb_pframe_write(const char* path, int32_t append, const mdb_particle_t* frame, int64_t n,
                     uint64_t frame_index) {
  using namespace mdb;
  if (!path || n < 0 || (n > 0 && !frame)) return set_error(MDB_ERR_ARG, "bad arguments");
  FILE* f = nullptr;
  if (append) {
    f = fopen(path, "r+b");
    if (!f) return set_error(MDB_ERR_IO, std::string("Failed to open file for append: ") + path);
    FileHeader h;
    if (!read_exact(f, &h, sizeof(h))) {
      fclose(f);
      return set_error(MDB_ERR_IO, "Failed to read existing header for append");
    }
    if (memcmp(h.magic, "PFRAME", 6) != 0 || (h.version != 1 && h.version != 2)) {
      fclose(f);
      return set_error(MDB_ERR_IO, "Not a valid PFRAME v1/v2 file");
    }
    if (fseek(f, 0, SEEK_END) != 0) {
      fclose(f);
      return set_error(MDB_ERR_IO, "Failed to seek to end of file");
    }
  } else {
    f = fopen(path, "wb");
    if (!f) return set_error(MDB_ERR_IO, std::string("Failed to open file for writing: ") + path);
    FileHeader h;
    memset(&h, 0, sizeof(h));
    memcpy(h.magic, "PFRAME", 6);
    h.version = 2;
    h.reserved = 0;
    if (fwrite(&h, 1, sizeof(h), f) != sizeof(h)) {
      fclose(f);
      return set_error(MDB_ERR_IO, "Failed to write to file");
    }
  }
  const uint64_t raw_bytes = (uint64_t)n * sizeof(mdb_particle_t);
  const unsigned char* raw = reinterpret_cast<const unsigned char*>(frame);
  uint32_t crc = (uint32_t)crc32(0L, Z_NULL, 0);
  crc = (uint32_t)crc32(crc, raw, (uInt)raw_bytes);
  uLong bound = compressBound((uLong)raw_bytes);
  std::vector<unsigned char> comp(bound);
  uLongf dl = bound;
  if (compress2(comp.data(), &dl, raw, (uLong)raw_bytes, Z_BEST_COMPRESSION) != Z_OK) {
    fclose(f);
    return set_error(MDB_ERR_IO, "compress2 failed");
  }
  FrameHeader fh;
  fh.frame_index = frame_index;
  fh.n_particles = (uint64_t)n;
  fh.uncompressed_bytes = raw_bytes;
  fh.compressed_bytes = (uint64_t)dl;
  fh.crc32 = crc;
  bool ok = fwrite(&fh, 1, sizeof(fh), f) == sizeof(fh) && fwrite(comp.data(), 1, dl, f) == dl;
  ok = (fclose(f) == 0) && ok;
  if (!ok) return set_error(MDB_ERR_IO, "Failed to write to file");
  return MDB_OK;
}

int mdb_pframe_read(const char* path, uint64_t frame_index, mdb_particle_t* out, int64_t cap,
                    int64_t* n_out) {
  using namespace mdb;
  if (!path) return set_error(MDB_ERR_ARG, "null path");
  FILE* f = fopen(path, "rb");
  if (!f) return set_error(MDB_ERR_IO, std::string("Failed to open file for reading: ") + path);
  int rc = check_header(f, path);
  if (rc != MDB_OK) {
    fclose(f);
    return rc;
  }
  FrameHeader fh;
  std::vector<unsigned char> raw;
  for (;;) {
    int r = next_frame(f, fh, raw);
    if (r == 0) {
      fclose(f);
      return set_error(MDB_ERR_IO, "Frame index " + std::to_string(frame_index) +
                                       " not found in " + path);
    }
    if (r < 0) {
      fclose(f);
      return set_error(MDB_ERR_IO, std::string("File ") + path + " is corrupted");
    }
    if (fh.frame_index == frame_index) break;
  }
  fclose(f);
  const int64_t n = (int64_t)fh.n_particles;
  if (n_out) *n_out = n;
  if (n > cap || (n > 0 && !out))
    return set_error(MDB_ERR_CAPACITY, "output buffer smaller than the frame");
  if (n > 0) memcpy(out, raw.data(), raw.size());
  return MDB_OK;
}

int mdb_pframe_count(const char* path, int64_t* n_frames, uint64_t* last_index) {
  using namespace mdb;
  if (!path) return set_error(MDB_ERR_ARG, "null path");
  FILE* f = fopen(path, "rb");
  if (!f) return set_error(MDB_ERR_IO, std::string("Failed to open file for reading: ") + path);
  int rc = check_header(f, path);
  if (rc != MDB_OK) {
    fclose(f);
    return rc;
  }
  int64_t k = 0;
  uint64_t last = 0;
  FrameHeader fh;
  std::vector<unsigned char> raw;
  int r;
  while ((r = next_frame(f, fh, raw)) == 1) {
    ++k;
    last = fh.frame_index;
  }
  fclose(f);
  if (n_frames) *n_frames = k;
  if (last_index) *last_index = last;
  if (r < 0) return set_error(MDB_ERR_IO, std::string("File ") + path + " has a corrupted tail");
  return MDB_OK;
}

}  // extern "C"
