// Asynchronous per-step OBJ output (the headless replacement of the viewer's
// frames): Environment::SaveObj / Save, sim/Environment.h:295-327.
//
// A fixed ring of staging slots; enqueue copies a state into a free slot (an
// asynchronous device-to-host copy on the scene's stream, followed by an
// event, or a host memcpy) and hands the slot to one writer thread, which
// waits for the copy, formats every body's file and frees the slot.  The
// simulation only waits when all slots are in flight.
#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/dfem.h"

namespace dfem {
int report_error(int code, const std::string& msg);
cudaStream_t scene_stream(dfem_scene* sc);
int scene_device(dfem_scene* sc);
}  // namespace dfem

using dfem::report_error;

struct dfem_obj_writer {
  struct Slot {
    double* x = nullptr;
    bool pinned = false;
    cudaEvent_t ev = nullptr;
    bool on_device = false;
    int device = 0;
    std::string prefix;
  };
  int nb = 0;
  std::vector<int> voff, foff, faces;
  std::vector<std::string> suffix;
  size_t n3 = 0;
  std::vector<Slot> slots;
  std::deque<int> free_q, work_q;
  std::mutex mu;
  std::condition_variable cv;
  int busy = 0;      // slots queued or being written
  bool stop = false;
  int first_error = DFEM_OK;
  std::string error_msg;
  std::thread worker;

  void run() {
    std::vector<char> buf;
    for (;;) {
      int k;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return stop || !work_q.empty(); });
        if (work_q.empty()) return;
        k = work_q.front();
        work_q.pop_front();
      }
      Slot& s = slots[k];
      int rc = DFEM_OK;
      std::string msg;
      if (s.on_device) {
        cudaSetDevice(s.device);
        const cudaError_t e = cudaEventSynchronize(s.ev);
        if (e != cudaSuccess) { rc = DFEM_ERR_CUDA; msg = std::string("obj writer: ") + cudaGetErrorString(e); }
      }
      for (int b = 0; b < nb && rc == DFEM_OK; ++b) {
        const std::string name = s.prefix + suffix[b];
        FILE* f = std::fopen(name.c_str(), "w");
        if (!f) { rc = DFEM_ERR_INVALID; msg = "obj writer: cannot open " + name; break; }
        char line[128];
        buf.clear();
        for (int i = voff[b]; i < voff[b + 1]; ++i) {
          const int n = std::snprintf(line, sizeof(line), "v %06f %06f %06f\n", s.x[3 * (size_t)i],
                                      s.x[3 * (size_t)i + 1], s.x[3 * (size_t)i + 2]);
          buf.insert(buf.end(), line, line + n);
        }
        for (int q = foff[b]; q < foff[b + 1]; ++q) {
          const int n = std::snprintf(line, sizeof(line), "f %d %d %d\n", faces[3 * (size_t)q] + 1,
                                      faces[3 * (size_t)q + 1] + 1, faces[3 * (size_t)q + 2] + 1);
          buf.insert(buf.end(), line, line + n);
        }
        const bool ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
        if (std::fclose(f) != 0 || !ok) { rc = DFEM_ERR_INVALID; msg = "obj writer: write failed: " + name; }
      }
      std::lock_guard<std::mutex> lk(mu);
      if (rc != DFEM_OK && first_error == DFEM_OK) { first_error = rc; error_msg = msg; }
      free_q.push_back(k);
      --busy;
      cv.notify_all();
    }
  }
};

extern "C" {

int dfem_obj_writer_create(int32_t n_bodies, const int32_t* vertex_offsets, const int32_t* face_offsets,
                           const int32_t* faces, const char* const* suffixes, int32_t depth,
                           dfem_obj_writer** out) {
  if (!out || n_bodies < 1 || !vertex_offsets || !face_offsets || !suffixes || depth < 1 || depth > 1024)
    return report_error(DFEM_ERR_INVALID, "obj writer: bad arguments");
  *out = nullptr;
  if (vertex_offsets[0] != 0 || face_offsets[0] != 0) return report_error(DFEM_ERR_INVALID, "obj writer: offsets must start at 0");
  for (int b = 0; b < n_bodies; ++b) {
    if (vertex_offsets[b + 1] < vertex_offsets[b] || face_offsets[b + 1] < face_offsets[b] || !suffixes[b])
      return report_error(DFEM_ERR_INVALID, "obj writer: decreasing offsets or missing suffix");
    const int nv = vertex_offsets[b + 1] - vertex_offsets[b];
    for (int q = 3 * face_offsets[b]; q < 3 * face_offsets[b + 1]; ++q)
      if (!faces || faces[q] < 0 || faces[q] >= nv) return report_error(DFEM_ERR_INVALID, "obj writer: face vertex out of range");
  }
  std::unique_ptr<dfem_obj_writer> w(new dfem_obj_writer());
  w->nb = n_bodies;
  w->voff.assign(vertex_offsets, vertex_offsets + n_bodies + 1);
  w->foff.assign(face_offsets, face_offsets + n_bodies + 1);
  if (face_offsets[n_bodies] > 0) w->faces.assign(faces, faces + 3 * (size_t)face_offsets[n_bodies]);
  for (int b = 0; b < n_bodies; ++b) w->suffix.emplace_back(suffixes[b]);
  w->n3 = 3 * (size_t)vertex_offsets[n_bodies];
  w->slots.resize(depth);
  for (int k = 0; k < depth; ++k) {
    auto& s = w->slots[k];
    void* p = nullptr;
    // pinned staging when a device is present (asynchronous copies), else plain
    if (cudaHostAlloc(&p, std::max<size_t>(1, w->n3) * sizeof(double), cudaHostAllocDefault) == cudaSuccess) {
      s.pinned = true;
    } else {
      cudaGetLastError();
      p = std::malloc(std::max<size_t>(1, w->n3) * sizeof(double));
      if (!p) return report_error(DFEM_ERR_NOMEM, "obj writer: staging allocation failed");
    }
    s.x = static_cast<double*>(p);
    w->free_q.push_back(k);
  }
  dfem_obj_writer* raw = w.release();
  raw->worker = std::thread([raw] { raw->run(); });
  *out = raw;
  return DFEM_OK;
}

int dfem_obj_writer_enqueue(dfem_obj_writer* w, dfem_scene* scene, const char* prefix, const double* x, int mem) {
  if (!w || !prefix || !x) return report_error(DFEM_ERR_INVALID, "obj writer: null argument");
  if (mem != DFEM_MEM_HOST && mem != DFEM_MEM_DEVICE) return report_error(DFEM_ERR_INVALID, "obj writer: bad mem");
  if (mem == DFEM_MEM_DEVICE && !scene) return report_error(DFEM_ERR_INVALID, "obj writer: a device state needs its scene");
  int k;
  {
    std::unique_lock<std::mutex> lk(w->mu);
    w->cv.wait(lk, [&] { return !w->free_q.empty(); });
    k = w->free_q.front();
    w->free_q.pop_front();
  }
  auto& s = w->slots[k];
  s.prefix = prefix;
  s.on_device = mem == DFEM_MEM_DEVICE;
  int rc = DFEM_OK;
  if (s.on_device) {
    s.device = dfem::scene_device(scene);
    cudaError_t e = cudaSetDevice(s.device);
    if (e == cudaSuccess && !s.ev) e = cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming);
    const cudaStream_t st = dfem::scene_stream(scene);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s.x, x, w->n3 * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(s.ev, st);
    if (e != cudaSuccess) rc = report_error(DFEM_ERR_CUDA, std::string("obj writer: ") + cudaGetErrorString(e));
  } else {
    std::memcpy(s.x, x, w->n3 * sizeof(double));
  }
  std::lock_guard<std::mutex> lk(w->mu);
  if (rc != DFEM_OK) {
    w->free_q.push_back(k);
  } else {
    ++w->busy;
    w->work_q.push_back(k);
  }
  w->cv.notify_all();
  return rc;
}

int dfem_obj_writer_flush(dfem_obj_writer* w) {
  if (!w) return report_error(DFEM_ERR_INVALID, "obj writer: null argument");
  std::unique_lock<std::mutex> lk(w->mu);
  w->cv.wait(lk, [&] { return w->busy == 0; });
  const int rc = w->first_error;
  const std::string msg = w->error_msg;
  w->first_error = DFEM_OK;
  w->error_msg.clear();
  lk.unlock();
  return rc == DFEM_OK ? DFEM_OK : report_error(rc, msg);
}

int dfem_obj_writer_destroy(dfem_obj_writer* w) {
  if (!w) return DFEM_OK;
  {
    std::unique_lock<std::mutex> lk(w->mu);
    w->cv.wait(lk, [&] { return w->busy == 0; });
    w->stop = true;
  }
  w->cv.notify_all();
  if (w->worker.joinable()) w->worker.join();
  for (auto& s : w->slots) {
    if (s.ev) { cudaSetDevice(s.device); cudaEventDestroy(s.ev); }
    if (s.pinned) cudaFreeHost(s.x);
    else std::free(s.x);
  }
  delete w;
  return DFEM_OK;
}

}  // extern "C"
