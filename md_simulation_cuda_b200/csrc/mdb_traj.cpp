// Asynchronous PFRAME trajectory writer.
//
// The reference's save_env (src/md_env.cu:4106-4124) gathers the frame to the
// host, compresses it (zlib level 9) and appends it to the file before the
// next step can start. Here a write call only queues, on the simulation's own
// stream, the export of the frame into a pinned host slot and an event after
// it, and returns: the steps issued afterwards run while a writer thread waits
// for the event, compresses and appends the frame with the same byte format
// (mdb_pframe_write). `depth` slots bound the frames in flight; a write call
// waits for a free slot when all are taken.
#include <cuda_runtime.h>
#include <string.h>

#include <condition_variable>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "mdb200.h"
#include "mdb_engine.h"
#include "mdb_util.h"

namespace {

struct Slot {
  mdb_particle_t* host = nullptr;  // pinned
  int64_t cap = 0;
  cudaEvent_t ev = nullptr;
  int device = -1;
  int64_t n = 0;
  uint64_t index = 0;
  bool busy = false;
};

}  // namespace

struct mdb_traj_writer {
  std::string path;
  bool append_next = false;  // later frames append to the file
  std::vector<Slot> slots;
  std::deque<int> queue;
  std::mutex mu;
  std::condition_variable cv;  // queue changes and freed slots
  int error = MDB_OK;
  std::string message;
  bool stop = false;
  std::thread worker;

  void run() {
    for (;;) {
      int k;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return stop || !queue.empty(); });
        if (queue.empty()) return;  // stop with nothing left
        k = queue.front();
      }
      Slot& s = slots[k];
      int rc = MDB_OK;
      std::string msg;
      cudaSetDevice(s.device);
      const cudaError_t e = cudaEventSynchronize(s.ev);
      if (e != cudaSuccess) {
        rc = MDB_ERR_CUDA;
        msg = std::string("cudaEventSynchronize: ") + cudaGetErrorString(e);
      } else {
        rc = mdb_pframe_write(path.c_str(), append_next ? 1 : 0, s.host, s.n, s.index);
        if (rc != MDB_OK) {
          char buf[512];
          mdb_last_error(buf, sizeof buf);
          msg = buf;
        } else {
          append_next = true;
        }
      }
      std::lock_guard<std::mutex> lk(mu);
      if (rc != MDB_OK && error == MDB_OK) {
        error = rc;
        message = msg;
      }
      queue.pop_front();
      s.busy = false;
      cv.notify_all();
    }
  }
};

extern "C" {

int mdb_traj_writer_open(const char* path, int32_t append, int32_t depth,
                         mdb_traj_writer_t** out) {
  if (!path || !out || depth <= 0 || depth > 64)
    return mdb::set_error(MDB_ERR_ARG, "bad arguments (depth must be 1..64)");
  *out = nullptr;
  mdb_traj_writer_t* w = new (std::nothrow) mdb_traj_writer();
  if (!w) return mdb::set_error(MDB_ERR_CAPACITY, "out of host memory");
  w->path = path;
  w->append_next = append != 0;
  w->slots.resize((size_t)depth);
  w->worker = std::thread([w] { w->run(); });
  *out = w;
  return MDB_OK;
}

int mdb_traj_writer_write(mdb_traj_writer_t* w, mdb_sim_t* sim, uint64_t frame_index) {
  if (!w || !sim) return mdb::set_error(MDB_ERR_ARG, "null argument");
  const int64_t n = mdb::sim_particles(sim);
  const int dev = mdb::sim_device(sim);
  int k = -1;
  {
    std::unique_lock<std::mutex> lk(w->mu);
    if (w->error != MDB_OK) return mdb::set_error(w->error, w->message);
    w->cv.wait(lk, [&] {
      for (size_t i = 0; i < w->slots.size(); ++i)
        if (!w->slots[i].busy) return true;
      return false;
    });
    for (size_t i = 0; i < w->slots.size(); ++i)
      if (!w->slots[i].busy) {
        k = (int)i;
        break;
      }
    w->slots[k].busy = true;
  }
  Slot& s = w->slots[k];
  int rc = MDB_OK;
  cudaError_t e = cudaSetDevice(dev);
  if (e == cudaSuccess && (s.cap < n || s.device != dev)) {
    if (s.host) cudaFreeHost(s.host);
    if (s.ev) cudaEventDestroy(s.ev);
    s.host = nullptr;
    s.ev = nullptr;
    s.cap = 0;
    e = cudaHostAlloc((void**)&s.host, sizeof(mdb_particle_t) * (size_t)(n > 0 ? n : 1),
                      cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming);
    if (e == cudaSuccess) {
      s.cap = n;
      s.device = dev;
    }
  }
  if (e != cudaSuccess) rc = mdb::cuda_error(e, "trajectory writer staging");
  if (rc == MDB_OK) rc = mdb::sim_export_async(sim, s.host, s.ev);
  std::lock_guard<std::mutex> lk(w->mu);
  if (rc != MDB_OK) {
    s.busy = false;
    w->cv.notify_all();
    return rc;
  }
  s.n = n;
  s.index = frame_index;
  w->queue.push_back(k);
  w->cv.notify_all();
  return MDB_OK;
}

int mdb_traj_writer_flush(mdb_traj_writer_t* w) {
  if (!w) return mdb::set_error(MDB_ERR_ARG, "null argument");
  std::unique_lock<std::mutex> lk(w->mu);
  w->cv.wait(lk, [&] { return w->queue.empty(); });
  if (w->error != MDB_OK) return mdb::set_error(w->error, w->message);
  return MDB_OK;
}

int mdb_traj_writer_close(mdb_traj_writer_t* w) {
  if (!w) return MDB_OK;
  {
    std::lock_guard<std::mutex> lk(w->mu);
    w->stop = true;
  }
  w->cv.notify_all();
  if (w->worker.joinable()) w->worker.join();
  const int rc = w->error;
  const std::string msg = w->message;
  for (Slot& s : w->slots) {
    if (s.device >= 0) cudaSetDevice(s.device);
    if (s.host) cudaFreeHost(s.host);
    if (s.ev) cudaEventDestroy(s.ev);
  }
  delete w;
  if (rc != MDB_OK) return mdb::set_error(rc, msg);
  return MDB_OK;
}

}  // extern "C"
