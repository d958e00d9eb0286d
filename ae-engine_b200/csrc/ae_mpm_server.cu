// ae_mpm_server.cu -- continuous-batching MPM server (ae_mpm_server_* in include/ae_mpm.h).
//
// One device thread owns a resident world whose scenes are *slots*: each slot was created with a
// grid, material and particle capacity, and holds one request's scene at a time.  Each tick it
//   1. drops cancelled requests and admits waiting ones (first come, first served) into free slots
//      that fit them; when none fits it grows the world by a batch of slots of the request's size
//      class, as long as the world stays within the HBM budget (ae_engine/src/vram_manager.rs:4-146
//      keeps a VRAM budget per subsystem; this is the device analogue for resident MPM scenes),
//   2. uploads the admitted scenes into their slots in place: no other scene moves,
//   3. runs min(substeps_per_tick, smallest remaining substep count) substeps of every occupied
//      slot in one batch,
//   4. copies finished scenes into their callers' buffers and vacates their slots.
// Requests submitted while a tick runs join at the next tick, so the device work of old and new
// requests overlaps in the same launches.  Growing is the only step that moves resident scenes
// (device to device, into a world with more slots); the slot count doubles per size class, so
// that happens a logarithmic number of times.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
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

// Page-locked host blocks, cached by power-of-two size class: request inputs are copied into one at
// submit and outputs come back through one, so every host<->device copy is one asynchronous DMA.
// Pinning memory is slow (the driver locks every page), so one pool serves every server of the
// process and keeps up to kPinnedCacheBytes of free blocks for the next requests.
class PinnedPool {
 public:
  static constexpr size_t kPinnedCacheBytes = size_t(8) << 30;
  static PinnedPool& process() {
    static PinnedPool* p = new PinnedPool();  // lives until exit: servers may outlive each other
    return *p;
  }
  void* get(size_t bytes, size_t* cls_out) {
    size_t cls = size_t(1) << 20;
    while (cls < bytes) cls <<= 1;
    *cls_out = cls;
    {
      std::lock_guard<std::mutex> lk(mu_);
      auto& v = free_[cls];
      if (!v.empty()) {
        void* p = v.back();
        v.pop_back();
        cached_ -= cls;
        return p;
      }
    }
    void* p = nullptr;
    if (cudaHostAlloc(&p, cls, cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    return p;
  }
  void put(void* p, size_t cls) {
    if (!p) return;
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (cached_ + cls <= kPinnedCacheBytes) {
        free_[cls].push_back(p);
        cached_ += cls;
        return;
      }
    }
    cudaFreeHost(p);
  }

 private:
  std::mutex mu_;
  std::map<size_t, std::vector<void*>> free_;
  size_t cached_ = 0;
};

// A particle block in the world's upload staging layout (pos 3n | vel 3n | F 9n | J n | C 9n |
// mass n floats, then n u16 material indices), so it crosses PCIe in one copy.
ae_mpm_particles staging_view(void* base, uint64_t n) {
  float* f = static_cast<float*>(base);
  return ae_mpm_particles{f, f + 3 * n, f + 6 * n, f + 15 * n, f + 16 * n, f + 25 * n,
                          reinterpret_cast<uint16_t*>(f + 26 * n)};
}
size_t staging_bytes(uint64_t n) { return (26 * sizeof(float) + sizeof(uint16_t)) * n; }

struct Request {
  uint64_t id = 0;
  ae_mpm_scene_desc desc{};
  std::vector<ae_mpm_material> mats;
  // pinned host block with the input particles (staging layout) until they are on the device,
  // then with the results on their way to the caller's buffers
  void* host = nullptr;
  size_t host_cls = 0;
  uint64_t n = 0;
  uint32_t substeps = 0, done = 0;
  ae_mpm_particles out{};
  double submit_s = 0, admit_s = 0, done_s = 0;
  int status = AE_MPM_OK;
  bool cancelled = false, on_device = false, uploaded = false;
  int slot = -1;        // its slot in the server's slot table
  int world_slot = -1;  // the scene index of that slot in the current world (once on the device)
};

// The size class a request's slot is made with: each grid axis rounded up to 16 nodes, the
// particle count to the next of 1024 * 2^(k/4) rounded to 256 (quarter-octave steps: at most 19 %
// of a slot's chunks stay empty), the material count to a power of two (at least 4).  A request
// fits any free slot at least that large whose particle capacity is at most 1.5 times its class.
struct SlotClass {
  uint32_t n[3];
  uint64_t particles;
  uint32_t materials;
};
uint64_t pow2_at_least(uint64_t v, uint64_t lo) {
  uint64_t p = lo;
  while (p < v) p <<= 1;
  return p;
}
uint64_t particle_class(uint64_t n) {
  static const double kStep[4] = {1.0, 1.189207115002721, 1.414213562373095, 1.681792830507429};  // 2^(k/4)
  for (uint64_t p2 = 1024;; p2 <<= 1)
    for (int k = 0; k < 4; ++k) {
      const uint64_t c = (uint64_t(double(p2) * kStep[k]) + 255) / 256 * 256;
      if (c >= n) return c;
    }
}
SlotClass class_of(const ae_mpm_scene_desc& d, uint64_t n) {
  SlotClass c;
  for (int a = 0; a < 3; ++a) c.n[a] = std::max<uint32_t>(16u, (d.n[a] + 15u) / 16u * 16u);
  c.particles = particle_class(n);
  c.materials = uint32_t(pow2_at_least(d.n_materials, 4));
  return c;
}
uint64_t grid_blocks(const uint32_t* n) { return uint64_t((n[0] + 3) / 4) * ((n[1] + 3) / 4) * ((n[2] + 3) / 4) + 1; }

constexpr uint64_t kCompactMin = uint64_t(1) << 22;  // particle capacity below which a world is not compacted

struct Slot {
  SlotClass cls{};
  uint64_t bytes = 0;     // estimated device bytes of the slot
  Request* r = nullptr;   // occupant
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
  uint64_t ticks = 0, particle_substeps = 0;
  uint64_t outstanding = 0;  // submitted and not yet finished
  std::string fatal;
  // slots (guarded by mu; the device thread alone changes them)
  std::vector<Slot> slots;
  uint64_t slot_bytes = 0;   // sum of the slots' estimated bytes: the world's footprint
  uint64_t layout = 0;       // bumped whenever the slot table grows or is compacted
  uint64_t world_layout = ~0ull;  // the layout the current world was built with
  ae_mpm_material filler{};  // material of the slots' creation descriptors
  // device-thread state
  aemp::WorldBase* world = nullptr;
  uint64_t worlds_built = 0;
  PinnedPool* pool = &PinnedPool::process();
  // host seconds of the device thread per phase, printed at destroy when AE_MPM_SERVER_PROFILE is
  // set: [admission, world rebuilds, uploads, queueing substeps, deliveries, waiting for the
  // device, finishing scenes (error words, downloads)]
  double phase_s[7] = {0, 0, 0, 0, 0, 0, 0};
  std::vector<Request*> outgoing;  // results in pinned blocks, copied to callers while the next tick runs

  ae_mpm_scene_desc slot_desc(const Slot& s, std::vector<ae_mpm_material>& mats) const {
    ae_mpm_scene_desc d{};
    d.mode = AE_MPM_MODE_PHYSICS;
    for (int a = 0; a < 3; ++a) d.n[a] = s.cls.n[a];
    d.dx = 1.0f / float(s.cls.n[0]);
    d.dt = 0.0f;
    d.wall_mode = AE_MPM_WALL_STICKY;
    d.wall_margin = 3;
    d.n_materials = s.cls.materials;
    mats.assign(s.cls.materials, filler);
    d.materials = mats.data();
    d.max_particles = s.cls.particles;
    return d;
  }

  void finish(Request* r, int status) {  // mu held
    r->status = status;
    r->done_s = now_s();
    finished.push_back(ae_mpm_request_result{r->id, status, r->submit_s, r->admit_s, r->done_s});
    if (outstanding) --outstanding;
    cv.notify_all();
  }

  // a free slot r fits, the smallest one (mu held); -1 if none
  int find_slot(const Request* r) const {
    const SlotClass want = class_of(r->desc, r->n);
    int best = -1;
    for (size_t i = 0; i < slots.size(); ++i) {
      const Slot& s = slots[i];
      if (s.r || s.cls.particles < r->n || 2 * s.cls.particles > 3 * want.particles ||
          s.cls.materials < r->desc.n_materials || grid_blocks(s.cls.n) < grid_blocks(r->desc.n))
        continue;
      if (best < 0 || s.bytes < slots[best].bytes) best = int(i);
    }
    return best;
  }

  // grows the slot table within the budget (mu held); false if not even one slot of r's class
  // fits.  Growing rebuilds the world, so one growth sizes every class for what is waiting: each
  // class present in the queue (r's included) gets slots for all its waiting requests plus half
  // as many again, at least 4 and at least as many as it has (so a class at least doubles), and
  // every other class without a free slot doubles too.
  bool grow_for(const Request* r) {
    std::vector<std::pair<Slot, uint64_t>> want;  // class representative, slots to add
    auto index_of = [&](const SlotClass& c) {
      for (size_t i = 0; i < want.size(); ++i)
        if (std::memcmp(&want[i].first.cls, &c, sizeof(SlotClass)) == 0) return int(i);
      return -1;
    };
    auto count_class = [&](const SlotClass& c, bool free_only) {
      uint64_t k = 0;
      for (const Slot& o : slots)
        if (std::memcmp(&o.cls, &c, sizeof(SlotClass)) == 0 && (!free_only || !o.r)) ++k;
      return k;
    };
    auto add_want = [&](const SlotClass& c) {
      int i = index_of(c);
      if (i < 0) {
        Slot s;
        s.cls = c;
        std::vector<ae_mpm_material> tmp;
        s.bytes = aemp::scene_device_bytes(slot_desc(s, tmp), 32);
        want.emplace_back(s, 0);
        i = int(want.size()) - 1;
      }
      return i;
    };
    add_want(class_of(r->desc, r->n));
    for (const Request* q : waiting) want[size_t(add_want(class_of(q->desc, q->n)))].second += 1;
    for (auto& w : want) {
      const uint64_t have = count_class(w.first.cls, false), free_now = count_class(w.first.cls, true);
      const uint64_t need = w.second > free_now ? w.second - free_now : 0;
      w.second = std::max<uint64_t>({4, have, need + need / 2});
    }
    for (const Slot& o : slots)
      if (index_of(o.cls) < 0 && count_class(o.cls, true) == 0) {
        const int i = add_want(o.cls);
        want[size_t(i)].second = std::max<uint64_t>(4, count_class(o.cls, false));
      }
    bool first = true, ok = false;
    for (auto& w : want) {  // r's class first: if even one of it does not fit, nothing grows
      uint64_t k = w.second;
      while (k > 0 && slot_bytes + k * w.first.bytes > opts.hbm_budget_bytes) --k;
      if (first && k == 0) return false;
      first = false;
      for (uint64_t i = 0; i < k; ++i) slots.push_back(w.first);
      slot_bytes += k * w.first.bytes;
      ok = ok || k > 0;
    }
    if (ok) ++layout;
    return ok;
  }

  // drops the vacant slots (mu held): the budget they hold goes back to admission; the occupied
  // ones are renumbered and move to the next world with it
  bool compact() {
    std::vector<Slot> kept;
    uint64_t bytes = 0;
    for (Slot& sl : slots)
      if (sl.r) {
        sl.r->slot = int(kept.size());
        kept.push_back(sl);
        bytes += sl.bytes;
      }
    if (kept.size() == slots.size()) return false;
    slots.swap(kept);
    slot_bytes = bytes;
    ++layout;
    return true;
  }

  ae_mpm_scene_desc request_desc(Request* r) const {
    ae_mpm_scene_desc d = r->desc;
    d.materials = r->mats.data();
    d.max_particles = r->n;
    return d;
  }

  // queues the request's particles (one DMA from its pinned block) into its slot; the block goes
  // back to the pool once the tick's work has finished
  int upload_new(Request* r) {
    ae_mpm_particles v = staging_view(r->host, r->n);
    int rc = world->assign_scene(uint32_t(r->slot), request_desc(r), &v, r->n);
    if (rc == AE_MPM_OK) {
      r->on_device = true;
      r->uploaded = true;
      r->world_slot = r->slot;
    }
    return rc;
  }

  // results of finished scenes: from their pinned blocks into the callers' buffers, then reported
  // (runs while the device works on the next tick)
  void deliver() {
    for (Request* r : outgoing) {
      if (r->host && r->status == AE_MPM_OK) {
        const ae_mpm_particles v = staging_view(r->host, r->n);
        const uint64_t n = r->n;
        std::memcpy(r->out.pos, v.pos, sizeof(float) * 3 * n);
        std::memcpy(r->out.vel, v.vel, sizeof(float) * 3 * n);
        std::memcpy(r->out.strain, v.strain, sizeof(float) * 9 * n);
        std::memcpy(r->out.jacobian, v.jacobian, sizeof(float) * n);
        std::memcpy(r->out.c, v.c, sizeof(float) * 9 * n);
        std::memcpy(r->out.mass, v.mass, sizeof(float) * n);
        std::memcpy(r->out.material_idx, v.material_idx, sizeof(uint16_t) * n);
      }
      pool->put(r->host, r->host_cls);
      r->host = nullptr;
    }
    std::lock_guard<std::mutex> lk(mu);
    for (Request* r : outgoing) {
      finish(r, r->status);
      delete r;
    }
    outgoing.clear();
  }

  // a world with every slot; resident scenes move over device to device (their particles never
  // return to the host mid-run)
  int rebuild_world(size_t n_slots, uint64_t lay, const std::vector<Request*>& resident) {
    std::vector<ae_mpm_scene_desc> descs(n_slots);
    std::vector<std::vector<ae_mpm_material>> mats(n_slots);
    for (size_t i = 0; i < n_slots; ++i) descs[i] = slot_desc(slots[i], mats[i]);
    std::string why;
    int st = 0;
    aemp::WorldBase* nw = aemp::make_world(descs.data(), uint32_t(n_slots), opts.exec, why, &st, nullptr);
    if (!nw) {
      fatal = why;
      return st ? st : AE_MPM_ECUDA;
    }
    if (world) cudaStreamSynchronize(world->stream());
    for (Request* r : resident) {
      if (!r->on_device || !world) continue;
      // particles and error word move device to device
      int rc = nw->assign_scene(uint32_t(r->slot), request_desc(r), nullptr, 0);
      if (rc == AE_MPM_OK) rc = nw->copy_scene_from(uint32_t(r->slot), world, uint32_t(r->world_slot));
      if (rc) {
        fatal = nw->err;
        delete nw;
        return rc;
      }
    }
    cudaStreamSynchronize(nw->stream());
    delete world;
    world = nw;
    world_layout = lay;
    for (Request* r : resident) r->world_slot = r->slot;
    ++worlds_built;
    return AE_MPM_OK;
  }

  void fail_all(int rc) {  // mu held; the world goes too (the next admission builds a new one)
    for (Request* r : running) {
      if (r->slot >= 0) slots[size_t(r->slot)].r = nullptr;
      pool->put(r->host, r->host_cls);
      finish(r, rc);
      delete r;
    }
    running.clear();
    delete world;
    world = nullptr;
    world_layout = ~0ull;
  }

  void loop() {
    cudaSetDevice(device);
    filler.young_modulus = 1.0e4f;
    filler.poisson_ratio = 0.2f;
    filler.density = 1.0f;
    filler.model = AE_MPM_PHYS_JELLY;
    while (true) {
      std::vector<Request*> admitted;
      std::vector<int> vacate;
      size_t n_slots = 0;
      uint64_t lay = 0;
      std::vector<Request*> resident;
      double t = now_s();
      auto lap = [&](int ph) {
        const double u = now_s();
        phase_s[ph] += u - t;
        t = u;
      };
      {
        std::unique_lock<std::mutex> lk(mu);
        // cancellations
        for (size_t i = 0; i < running.size();) {
          Request* r = running[i];
          if (r->cancelled) {
            if (r->on_device) vacate.push_back(r->world_slot);
            slots[size_t(r->slot)].r = nullptr;
            pool->put(r->host, r->host_cls);
            finish(r, AE_MPM_EINVAL);
            delete r;
            running.erase(running.begin() + i);
          } else {
            ++i;
          }
        }
        for (size_t i = 0; i < waiting.size();) {
          if (waiting[i]->cancelled) {
            pool->put(waiting[i]->host, waiting[i]->host_cls);
            finish(waiting[i], AE_MPM_EINVAL);
            delete waiting[i];
            waiting.erase(waiting.begin() + i);
          } else {
            ++i;
          }
        }
        // admission into free slots, growing the world within the HBM budget (first come, first
        // served: a request that does not fit blocks later ones)
        while (!waiting.empty() && running.size() < opts.max_scenes) {
          Request* r = waiting.front();
          int s = find_slot(r);
          if (s < 0 && grow_for(r)) s = find_slot(r);
          if (s < 0 && compact() && grow_for(r)) s = find_slot(r);
          if (s < 0) break;
          waiting.pop_front();
          r->slot = s;
          slots[size_t(s)].r = r;
          r->admit_s = now_s();
          running.push_back(r);
          admitted.push_back(r);
        }
        if (running.empty() && outgoing.empty()) {
          if (stop) break;
          cv.wait_for(lk, std::chrono::milliseconds(1));
          if (vacate.empty()) continue;
        }
        n_slots = slots.size();
        lay = layout;
        resident = running;
      }
      int rc = AE_MPM_OK;
      if (world)
        for (int s : vacate) world->vacate_scene(uint32_t(s));
      if (resident.empty()) {
        deliver();
        continue;
      }
      lap(0);
      if (!world || lay != world_layout) rc = rebuild_world(n_slots, lay, resident);
      lap(1);
      for (Request* r : admitted)
        if (rc == AE_MPM_OK) {
          rc = upload_new(r);
          if (rc) fatal = world->err;
        }
      lap(2);
      if (rc) {  // the batch cannot run: fail every running request
        deliver();
        std::lock_guard<std::mutex> lk(mu);
        fail_all(rc);
        continue;
      }
      uint32_t k = opts.substeps_per_tick;
      for (Request* r : resident) k = std::min(k, r->substeps - r->done);
      rc = world->step(k);  // queued: the host copies below overlap the device work
      lap(3);
      deliver();
      lap(4);
      if (rc == AE_MPM_OK) rc = world->sync();
      lap(5);
      if (rc == AE_MPM_ENAN || rc == AE_MPM_EDOMAIN) rc = AE_MPM_OK;  // attributed per scene below
      // the uploads of this tick are complete: their input blocks can be reused
      for (Request* r : admitted)
        if (r->uploaded && r->host) {
          pool->put(r->host, r->host_cls);
          r->host = nullptr;
        }
      uint64_t parts = 0;
      for (Request* r : resident) {
        r->done += k;
        parts += r->n;
      }
      std::vector<Request*> done_now;
      for (Request* r : resident) {
        if (r->done < r->substeps && rc == AE_MPM_OK) continue;
        int st = rc;
        if (st == AE_MPM_OK) {
          uint32_t word = 0;
          world->errors(uint32_t(r->world_slot), &word, nullptr);
          st = r->status;
          if (word & aemp::kErrNaN) st = AE_MPM_ENAN;
          else if ((word & aemp::kErrDomain) && st == AE_MPM_OK) st = AE_MPM_EDOMAIN;
          // results into a pinned block (one DMA); the caller's buffers get them next tick
          r->host = pool->get(staging_bytes(r->n), &r->host_cls);
          if (!r->host) {
            st = AE_MPM_ENOMEM;
          } else {
            ae_mpm_particles v = staging_view(r->host, r->n);
            int d = world->download(uint32_t(r->world_slot), &v, false);
            if (d) st = d;
          }
        }
        world->vacate_scene(uint32_t(r->world_slot));
        r->status = st;
        done_now.push_back(r);
      }
      lap(6);
      {
        std::lock_guard<std::mutex> lk(mu);
        ticks += 1;
        particle_substeps += parts * k;
        for (Request* r : done_now) {
          slots[size_t(r->slot)].r = nullptr;
          running.erase(std::find(running.begin(), running.end(), r));
          outgoing.push_back(r);
        }
        // A large world whose slots stand mostly empty still sorts its whole capacity and launches
        // a CTA per chunk of every slot each substep: with nothing waiting, a capacity above
        // kCompactMin particles and under a quarter of it in use, drop the vacant slots (the next
        // tick rebuilds the world from the occupied ones).  Small worlds are left alone: their
        // empty slots cost less than the rebuild, and arrivals would grow them again.
        if (!done_now.empty() && waiting.empty() && !running.empty()) {
          uint64_t live = 0, cap = 0;
          for (const Slot& sl : slots) cap += sl.cls.particles;
          for (const Request* r : running) live += r->n;
          if (cap > kCompactMin && 4 * live < cap) compact();
        }
      }
    }
    deliver();
    delete world;
    world = nullptr;
    if (std::getenv("AE_MPM_SERVER_PROFILE"))
      std::fprintf(stderr,
                   "ae_mpm_server: %llu ticks, %llu worlds built; seconds: admission %.3f rebuild %.3f upload %.3f "
                   "queue %.3f deliver %.3f device-wait %.3f finish %.3f\n",
                   (unsigned long long)ticks, (unsigned long long)worlds_built, phase_s[0], phase_s[1], phase_s[2],
                   phase_s[3], phase_s[4], phase_s[5], phase_s[6]);
  }
};

extern "C" {

int ae_mpm_server_slot_class(const ae_mpm_scene_desc* scene, uint64_t n_particles, uint32_t grid_out[3],
                             uint64_t* particles_out, uint32_t* materials_out) {
  if (!scene || !grid_out || !particles_out || !materials_out) return AE_MPM_EINVAL;
  const SlotClass c = class_of(*scene, n_particles);
  for (int a = 0; a < 3; ++a) grid_out[a] = c.n[a];
  *particles_out = c.particles;
  *materials_out = c.materials;
  return AE_MPM_OK;
}

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
    // options left to the library: slot particle counts change at every admission and completion,
    // which changes the chunk table a captured graph replays, so substeps are launched eagerly;
    // sort every 8th substep as the autotuner picks for the batched scene set
    s->opts.exec.p2g_variant = AE_MPM_P2G_LANES;
    s->opts.exec.use_graph = 0;
    if (s->opts.exec.sort_interval <= 1) s->opts.exec.sort_interval = 8;
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
  // the slots' world steps physics-mode scenes (the reference-mode drop-in is a per-call path)
  if (scene->mode != AE_MPM_MODE_PHYSICS || scene->wall_margin < 1 || !(scene->dx > 0.0f) || !(scene->dt >= 0.0f))
    return AE_MPM_EINVAL;
  for (int a = 0; a < 3; ++a)
    if (scene->n[a] < 4 || scene->n[a] > 1024) return AE_MPM_EINVAL;
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
  // the request's slot class must fit the budget on its own
  {
    const SlotClass c = class_of(r->desc, n);
    ae_mpm_scene_desc cd = r->desc;
    for (int a = 0; a < 3; ++a) cd.n[a] = c.n[a];
    cd.max_particles = c.particles;
    if (aemp::scene_device_bytes(cd, 32) > s->opts.hbm_budget_bytes) {
      delete r;
      return AE_MPM_EBUDGET;
    }
  }
  // the particles are copied now, into a pinned block in the upload staging layout
  {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    r->host = s->pool->get(staging_bytes(n), &r->host_cls);
    cudaSetDevice(prev);
  }
  if (!r->host) {
    delete r;
    return AE_MPM_ENOMEM;
  }
  {
    const ae_mpm_particles v = staging_view(r->host, n);
    std::memcpy(v.pos, in->pos, sizeof(float) * 3 * n);
    std::memcpy(v.vel, in->vel, sizeof(float) * 3 * n);
    std::memcpy(v.strain, in->strain, sizeof(float) * 9 * n);
    std::memcpy(v.jacobian, in->jacobian, sizeof(float) * n);
    std::memcpy(v.c, in->c, sizeof(float) * 9 * n);
    std::memcpy(v.mass, in->mass, sizeof(float) * n);
    std::memcpy(v.material_idx, in->material_idx, sizeof(uint16_t) * n);
  }
  std::lock_guard<std::mutex> lk(s->mu);
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
  if (resident_bytes) *resident_bytes = s->slot_bytes;
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
  for (Request* r : s->waiting) {
    s->pool->put(r->host, r->host_cls);
    delete r;
  }
  for (Request* r : s->running) {
    s->pool->put(r->host, r->host_cls);
    delete r;
  }
  delete s;
  return AE_MPM_OK;
}

}  // extern "C"
