// ae_mpm_server.cu -- continuous-batching MPM server (ae_mpm_server_* in include/ae_mpm.h).
//
// One device thread owns a "batch": a world holding every admitted scene.  Each tick it
//   1. drops cancelled requests and admits waiting ones while their estimated device state fits
//      the HBM budget (ae_engine/src/vram_manager.rs:4-146 keeps a VRAM budget per subsystem; this
//      is the device analogue for resident MPM scenes),
//   2. rebuilds the batch world when membership changed, moving continuing scenes' state
//      device-to-device (their particles never return to the host mid-run),
//   3. runs min(substeps_per_tick, smallest remaining substep count) batched substeps,
//   4. copies finished scenes into their callers' buffers and frees their memory.
// Requests submitted while a tick runs wait at most one tick before joining the batch, so the
// device work of old and new requests overlaps in the same launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/ae_mpm.h"
#include "mpm_world.cuh"


namespace {

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// Size-class caching allocator: batch rebuilds reuse freed blocks instead of cudaMalloc/cudaFree.
class CachingAlloc final : public aemp::DevAlloc {
 public:
  ~CachingAlloc() override { trim(); }
  cudaError_t alloc(void** p, size_t bytes) override {
    size_t cls = round(bytes);
    auto it = free_.find(cls);
    if (it != free_.end() && !it->second.empty()) {
      *p = it->second.back();
      it->second.pop_back();
      sizes_[*p] = cls;
      return cudaSuccess;
    }
    cudaError_t e = cudaMalloc(p, cls);
    if (e == cudaErrorMemoryAllocation) {  // give cached blocks back and retry once
      cudaGetLastError();
      trim();
      e = cudaMalloc(p, cls);
    }
    if (e == cudaSuccess) sizes_[*p] = cls;
    return e;
  }
  void release(void* p) override {
    auto it = sizes_.find(p);
    if (it == sizes_.end()) {
      cudaFree(p);
      return;
    }
    free_[it->second].push_back(p);
    sizes_.erase(it);
  }
  void trim() {
    for (auto& kv : free_)
      for (void* p : kv.second) cudaFree(p);
    free_.clear();
  }

 private:
  static size_t round(size_t b) {  // 1/8-octave size classes, >= 512 B
    if (b < 512) return 512;
    size_t top = 1;
    while ((top << 1) <= b) top <<= 1;
    size_t step = std::max<size_t>(top / 8, 256);
    return (b + step - 1) / step * step;
  }
  std::map<size_t, std::vector<void*>> free_;
  std::map<void*, size_t> sizes_;
};

struct Request {
  uint64_t id = 0;
  ae_mpm_scene_desc desc{};
  std::vector<ae_mpm_material> mats;
  // host copy of the input particles (reference layout), kept until the scene is on the device
  std::vector<float> pos, vel, F, J, C, mass;
  std::vector<uint16_t> mat;
  uint64_t n = 0;
  uint32_t substeps = 0, done = 0;
  ae_mpm_particles out{};
  double submit_s = 0, admit_s = 0, done_s = 0;
  uint64_t bytes = 0;
  int status = AE_MPM_OK;
  bool cancelled = false, on_device = false;
  int slot = -1;  // scene index in the current batch world
};

}  // namespace

struct ae_mpm_server {
  int device = 0;
  ae_mpm_server_opts opts{};
  std::thread thr;
  std::mutex mu;
  std::condition_variable cv;
  bool stop = false;
  uint64_t next_id = 1;
  std::deque<Request*> waiting;
  std::vector<Request*> running;
  std::vector<ae_mpm_request_result> finished;
  uint64_t resident_bytes = 0;
  uint64_t ticks = 0, particle_substeps = 0;
  uint64_t outstanding = 0;  // submitted and not yet finished
  std::string fatal;
  // device-thread state
  std::unique_ptr<CachingAlloc> alloc;
  aemp::WorldBase* world = nullptr;
  bool rebuild = false;

  void finish(Request* r, int status) {  // mu held
    r->status = status;
    r->done_s = now_s();
    finished.push_back(ae_mpm_request_result{r->id, status, r->submit_s, r->admit_s, r->done_s});
    if (outstanding) --outstanding;
    cv.notify_all();
  }

  int upload_new(aemp::WorldBase* w, Request* r) {
    ae_mpm_particles v{r->pos.data(), r->vel.data(), r->F.data(), r->J.data(), r->C.data(), r->mass.data(), r->mat.data()};
    int rc = w->upload(uint32_t(r->slot), &v, r->n, false);
    if (rc == AE_MPM_OK) {
      r->on_device = true;
      // the device copy is authoritative from here on
      std::vector<float>().swap(r->pos);
      std::vector<float>().swap(r->vel);
      std::vector<float>().swap(r->F);
      std::vector<float>().swap(r->J);
      std::vector<float>().swap(r->C);
      std::vector<float>().swap(r->mass);
      std::vector<uint16_t>().swap(r->mat);
    }
    return rc;
  }

  // builds a world for `batch`; continuing scenes are copied from the old world
  int rebuild_world(std::vector<Request*>& batch) {
    std::vector<ae_mpm_scene_desc> descs(batch.size());
    for (size_t i = 0; i < batch.size(); ++i) {
      descs[i] = batch[i]->desc;
      descs[i].materials = batch[i]->mats.data();
      descs[i].max_particles = batch[i]->n;
    }
    std::string why;
    int st = 0;
    aemp::WorldBase* nw = descs.empty() ? nullptr : aemp::make_world(descs.data(), uint32_t(descs.size()), opts.exec, why, &st, alloc.get());
    if (!descs.empty() && !nw) {
      fatal = why;
      return st ? st : AE_MPM_ECUDA;
    }
    if (world) cudaStreamSynchronize(world->stream());
    for (size_t i = 0; i < batch.size(); ++i) {
      Request* r = batch[i];
      int rc;
      if (r->on_device && world) {
        // accumulate the old world's error word before it goes away
        uint32_t word = 0;
        world->errors(uint32_t(r->slot), &word, nullptr);
        if (word & aemp::kErrNaN) r->status = AE_MPM_ENAN;
        else if ((word & aemp::kErrDomain) && r->status == AE_MPM_OK) r->status = AE_MPM_EDOMAIN;
        rc = nw->copy_scene_from(uint32_t(i), world, uint32_t(r->slot));
        r->slot = int(i);
      } else {
        r->slot = int(i);
        rc = upload_new(nw, r);
      }
      if (rc) {
        fatal = nw->err;
        delete nw;
        return rc;
      }
    }
    if (nw) cudaStreamSynchronize(nw->stream());
    delete world;
    world = nw;
    return AE_MPM_OK;
  }

  void loop() {
    cudaSetDevice(device);
    alloc.reset(new CachingAlloc());
    while (true) {
      std::vector<Request*> done_now;
      {
        std::unique_lock<std::mutex> lk(mu);
        // cancellations
        for (size_t i = 0; i < running.size();) {
          Request* r = running[i];
          if (r->cancelled) {
            resident_bytes -= r->bytes;
            finish(r, AE_MPM_EINVAL);
            delete r;
            running.erase(running.begin() + i);
            rebuild = true;
          } else {
            ++i;
          }
        }
        for (size_t i = 0; i < waiting.size();) {
          if (waiting[i]->cancelled) {
            finish(waiting[i], AE_MPM_EINVAL);
            delete waiting[i];
            waiting.erase(waiting.begin() + i);
          } else {
            ++i;
          }
        }
        // admission by HBM budget (FIFO: a request that does not fit blocks later ones)
        while (!waiting.empty() && running.size() < opts.max_scenes &&
               resident_bytes + waiting.front()->bytes <= opts.hbm_budget_bytes) {
          Request* r = waiting.front();
          waiting.pop_front();
          r->admit_s = now_s();
          resident_bytes += r->bytes;
          running.push_back(r);
          rebuild = true;
        }
        if (running.empty()) {
          if (stop) break;
          cv.wait_for(lk, std::chrono::milliseconds(1));
          continue;
        }
      }
      if (rebuild) {
        int rc = rebuild_world(running);
        rebuild = false;
        if (rc) {  // the batch cannot run: fail every running request
          std::lock_guard<std::mutex> lk(mu);
          for (Request* r : running) {
            resident_bytes -= r->bytes;
            finish(r, rc);
            delete r;
          }
          running.clear();
          delete world;
          world = nullptr;
          continue;
        }
      }
      uint32_t k = opts.substeps_per_tick;
      for (Request* r : running) k = std::min(k, r->substeps - r->done);
      int rc = world->step(k);
      if (rc == AE_MPM_OK) rc = world->sync();
      if (rc == AE_MPM_ENAN || rc == AE_MPM_EDOMAIN) rc = AE_MPM_OK;  // attributed per scene below
      uint64_t parts = 0;
      for (Request* r : running) {
        r->done += k;
        parts += r->n;
      }
      std::vector<Request*> keep;
      for (Request* r : running) {
        if (r->done < r->substeps && rc == AE_MPM_OK) {
          keep.push_back(r);
          continue;
        }
        int st = rc;
        if (st == AE_MPM_OK) {
          uint32_t word = 0;
          world->errors(uint32_t(r->slot), &word, nullptr);
          st = r->status;
          if (word & aemp::kErrNaN) st = AE_MPM_ENAN;
          else if ((word & aemp::kErrDomain) && st == AE_MPM_OK) st = AE_MPM_EDOMAIN;
          int d = world->download(uint32_t(r->slot), &r->out, false);
          if (d) st = d;
        }
        r->status = st;
        done_now.push_back(r);
      }
      {
        std::lock_guard<std::mutex> lk(mu);
        ticks += 1;
        particle_substeps += parts * k;
        for (Request* r : done_now) {
          resident_bytes -= r->bytes;
          finish(r, r->status);
          delete r;
        }
        if (!done_now.empty()) rebuild = true;
        running.swap(keep);
      }
    }
    delete world;
    world = nullptr;
    alloc.reset();
  }
};

extern "C" {

int ae_mpm_server_create(ae_mpm_ctx* ctx, const ae_mpm_server_opts* opts, ae_mpm_server** out) {
  if (!ctx || !out) return AE_MPM_EINVAL;
  *out = nullptr;
  auto* s = new ae_mpm_server();
  s->device = aemp::ctx_device(ctx);
  if (opts) {
    s->opts = *opts;
  } else {
    std::memset(&s->opts, 0, sizeof(s->opts));
    ae_mpm_exec_opts_default(&s->opts.exec);
  }
  if (s->opts.substeps_per_tick == 0) s->opts.substeps_per_tick = 10;
  if (s->opts.max_scenes == 0) s->opts.max_scenes = 4096;
  if (s->opts.exec.precision != 64) s->opts.exec.precision = 32;
  if (s->opts.exec.p2g_variant == AE_MPM_P2G_AUTO) {
    // options left to the library: batches are rebuilt whenever membership changes, so graphs
    // (captured per world) would be re-captured every few ticks; sort every 4th substep as the
    // autotuner usually picks for batched worlds
    s->opts.exec.p2g_variant = AE_MPM_P2G_LANES;
    s->opts.exec.use_graph = 0;
    if (s->opts.exec.sort_interval <= 1) s->opts.exec.sort_interval = 4;
  }
  if (s->opts.exec.block_threads == 0) s->opts.exec.block_threads = 256;
  if (s->opts.exec.sort_interval < 1) s->opts.exec.sort_interval = 1;
  if (s->opts.hbm_budget_bytes == 0) {
    size_t fr = 0, tot = 0;
    cudaSetDevice(s->device);
    cudaMemGetInfo(&fr, &tot);
    s->opts.hbm_budget_bytes = uint64_t(fr) / 2;
  }
  if (s->opts.exec.precision == 64) {  // the server moves f32 host buffers
    delete s;
    return AE_MPM_EINVAL;
  }
  s->thr = std::thread([s] { s->loop(); });
  *out = s;
  return AE_MPM_OK;
}

int ae_mpm_server_submit(ae_mpm_server* s, const ae_mpm_scene_desc* scene, const ae_mpm_particles* in, uint64_t n,
                         uint32_t substeps, ae_mpm_particles* out, uint64_t* request_id) {
  if (!s || !scene || !in || !out) return AE_MPM_EINVAL;
  if (scene->n_materials == 0 || !scene->materials || substeps == 0 || n == 0) return AE_MPM_EINVAL;
  if (!in->pos || !in->vel || !in->strain || !in->jacobian || !in->c || !in->mass || !in->material_idx) return AE_MPM_EINVAL;
  if (!out->pos || !out->vel || !out->strain || !out->jacobian || !out->c || !out->mass || !out->material_idx)
    return AE_MPM_EINVAL;
  auto* r = new Request();
  r->desc = *scene;
  r->desc.max_particles = n;
  r->mats.assign(scene->materials, scene->materials + scene->n_materials);
  r->n = n;
  r->substeps = substeps;
  r->out = *out;
  r->pos.assign(in->pos, in->pos + 3 * n);
  r->vel.assign(in->vel, in->vel + 3 * n);
  r->F.assign(in->strain, in->strain + 9 * n);
  r->J.assign(in->jacobian, in->jacobian + n);
  r->C.assign(in->c, in->c + 9 * n);
  r->mass.assign(in->mass, in->mass + n);
  r->mat.assign(in->material_idx, in->material_idx + n);
  r->bytes = aemp::scene_device_bytes(r->desc, 32);
  std::lock_guard<std::mutex> lk(s->mu);
  if (r->bytes > s->opts.hbm_budget_bytes) {
    delete r;
    return AE_MPM_EBUDGET;
  }
  r->id = s->next_id++;
  r->submit_s = now_s();
  if (request_id) *request_id = r->id;
  s->waiting.push_back(r);
  s->outstanding += 1;
  s->cv.notify_all();
  return AE_MPM_OK;
}

int ae_mpm_server_cancel(ae_mpm_server* s, uint64_t id) {
  if (!s) return AE_MPM_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  for (Request* r : s->waiting)
    if (r->id == id) {
      r->cancelled = true;
      return AE_MPM_OK;
    }
  for (Request* r : s->running)
    if (r->id == id) {
      r->cancelled = true;
      return AE_MPM_OK;
    }
  return AE_MPM_ENOTFOUND;
}

int ae_mpm_server_poll(ae_mpm_server* s, ae_mpm_request_result* results, uint32_t max, uint32_t* n_out) {
  if (!s || !n_out || (max > 0 && !results)) return AE_MPM_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  uint32_t k = uint32_t(std::min<size_t>(max, s->finished.size()));
  for (uint32_t i = 0; i < k; ++i) results[i] = s->finished[i];
  s->finished.erase(s->finished.begin(), s->finished.begin() + k);
  *n_out = k;
  return k > 0 ? AE_MPM_OK : AE_MPM_EAGAIN;
}

int ae_mpm_server_drain(ae_mpm_server* s, double timeout_s) {
  if (!s) return AE_MPM_EINVAL;
  std::unique_lock<std::mutex> lk(s->mu);
  bool ok = s->cv.wait_for(lk, std::chrono::duration<double>(timeout_s), [s] { return s->outstanding == 0; });
  return ok ? AE_MPM_OK : AE_MPM_ETIMEOUT;
}

int ae_mpm_server_stats(ae_mpm_server* s, uint64_t* resident_bytes, uint32_t* resident_scenes, uint64_t* ticks,
                        uint64_t* particle_substeps) {
  if (!s) return AE_MPM_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  if (resident_bytes) *resident_bytes = s->resident_bytes;
  if (resident_scenes) *resident_scenes = uint32_t(s->running.size());
  if (ticks) *ticks = s->ticks;
  if (particle_substeps) *particle_substeps = s->particle_substeps;
  return AE_MPM_OK;
}

int ae_mpm_server_destroy(ae_mpm_server* s) {
  if (!s) return AE_MPM_EINVAL;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    for (Request* r : s->waiting) r->cancelled = true;
    for (Request* r : s->running) r->cancelled = true;
    s->cv.notify_all();
  }
  if (s->thr.joinable()) s->thr.join();
  for (Request* r : s->waiting) delete r;
  for (Request* r : s->running) delete r;
  delete s;
  return AE_MPM_OK;
}

}  // extern "C"
