// bb_server.cu -- serving loop with continuous batching: step requests for many device-resident
// worlds, packed as slots into batched worlds that advance together, admitted by an HBM budget.
//
// No reference counterpart: the reference steps one scene per frame from its render loop
// (src/renderer_manager.cpp:254-257 -> RigidBodyManager::simulate).  This is the serving
// pattern built on the batched step (bb_add_world): one bb_world object holds many independent
// worlds in slots, and one graph launch per step advances all of them.
//
//   * Requests are grouped by step class (solver parameters, dt, substeps: one batch steps with
//     one set).  A batch of a step class holds worlds of every size, each in a slot of its size
//     class (a power of two >= the world's bodies, 64 at least), up to 2^19 bodies (fewer when a
//     batch that size would take more than half of the HBM budget).  A step of a batch costs
//     nearly the same for a few small worlds as for many (the colour sweeps and AVBD's
//     per-colour passes are latency-bound), so one batch per step class advances the most
//     worlds per step.
//   * A request is admitted as soon as a slot and the budget allow: its world is put into a free
//     slot of its size class (bb_world_refill), a new slot where the batch has room
//     (bb_add_world), or, when it is already resident in a batch of its step class, resumed in
//     place (bb_world_pause(.., 0)).  From then on it advances with every step of its batch;
//     requests that arrive while others run join at the next step boundary.
//   * After its last step a world is paused in its slot: it keeps its device state (bodies,
//     warm-start contacts, sort order) exactly until its next request, whatever the other
//     slots do.  A world's results therefore do not depend on what else is in flight.
//   * A request whose step class differs from the batch its world sits in moves the world: its
//     body state goes to the host and into a slot of a batch of the new class, and its warm
//     starts restart there.  The same happens to a world evicted to make room: under budget
//     pressure, batches with no running request are destroyed least recently used first and
//     their worlds' body states kept on the host.
//   * Device error bits are per batch; a request reports those seen by the time its last step
//     ended (they may come from any slot of its batch).
//   * All batches step on one stream of the server.  A batch's persistent kernels size their grids
//     for the whole GPU and synchronise with grid barriers, so two batches' steps must not run at
//     the same time (their blocks could not all be resident); one stream orders them, and every
//     step has the whole GPU.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/beatbox.h"

bb_status bb_fail(bb_status code, const char* msg);
bb_status bb_world_read_range(void* world, uint32_t first, uint32_t count, float* position, float* rotation,
                              float* velocity, float* omega, uint32_t* flags);
const uint32_t* bb_world_error_word(void* world);
bb_status bb_world_move_in(void* dst_world, uint32_t widx, const bb_batch_world_desc* desc, void* src_world,
                           uint32_t src_widx, uint32_t count);
const uint32_t* bb_world_error_site_word(void* world);

namespace {

using Clock = std::chrono::steady_clock;
constexpr uint32_t kBatchBodies = 1u << 19;  // body capacity of one batch (at least its largest slot)
constexpr uint32_t kInFlight = 2;           // steps a batch may have queued on its stream

uint64_t fnv1a(const void* data, size_t bytes, uint64_t h = 1469598103934665603ull) {
  const uint8_t* b = static_cast<const uint8_t*>(data);
  for (size_t i = 0; i < bytes; ++i) h = (h ^ b[i]) * 1099511628211ull;
  return h;
}

uint32_t class_of(uint32_t n) {
  uint32_t c = 6;  // smallest slot: 64 bodies
  while ((1ull << c) < n) ++c;
  return c;
}

struct Batch;
struct Req;

struct WorldRec {
  uint64_t key = 0;
  std::vector<bb_shape_desc> shapes;
  std::vector<bb_body_desc> bodies;  // as given; pose, velocity and flags refreshed when it leaves a slot
  float wmin[3] = {0, 0, 0}, wext[3] = {1, 1, 1};
  Batch* batch = nullptr;  // resident: the batch and slot it sits in
  uint32_t slot = 0;
  bool busy = false;     // a request of this world is running
  bool reading = false;  // bb_server_read_state is copying its state out
  uint64_t last_use = 0;
};

struct Slot {
  WorldRec* world = nullptr;  // resident world (running or paused), nullptr = free
  Req* req = nullptr;         // running request
  uint32_t remaining = 0;     // its steps not yet enqueued
  uint32_t cls = 0, first = 0;  // size class (2^cls bodies) and first body id in the batch
};

struct Batch {
  void* w = nullptr;
  cudaStream_t stream = nullptr;
  uint64_t step_key = 0;
  float dt = 0;
  uint32_t substeps = 1;
  uint32_t cap = 0, used = 0;  // body capacity, bodies taken by its slots
  std::vector<Slot> slots;
  std::map<std::tuple<uint32_t, float, float, float>, uint32_t> shape_handle;
  uint32_t park_shape = 0;
  std::deque<cudaEvent_t> inflight;
  uint32_t* err_host = nullptr;  // pinned copies of the batch's error bits and error site after each step
  uint64_t bytes = 0, last_use = 0;
  uint32_t running = 0;
};

struct Req {
  uint64_t ticket = 0;
  bb_request r = {};
  uint64_t step_key = 0;
  std::vector<bb_shape_desc> shapes;  // copies for a new world
  std::vector<bb_body_desc> bodies;
  double submit_s = 0, start_s = 0, finish_s = 0;
  bb_status result = BB_OK;
  uint32_t error_flags = 0, error_site = 0;
  bool done = false;
  cudaEvent_t ev = nullptr;  // after the request's last step
  Batch* batch = nullptr;
  WorldRec* w = nullptr;
};

// step class of a request: its solver parameters without the Morton box (each world of a batch
// keeps its own), dt and substeps
uint64_t step_key_of(const bb_request& r) {
  bb_solver_params p = r.params;
  std::memset(p.world_min, 0, sizeof(p.world_min));
  std::memset(p.world_extent, 0, sizeof(p.world_extent));
  p.bounds_mode = BB_BOUNDS_FIXED;
  uint64_t h = fnv1a(&p, sizeof(p));
  h = fnv1a(&r.dt, sizeof(r.dt), h);
  return fnv1a(&r.substeps, sizeof(r.substeps), h);
}

}  // namespace

struct bb_server_impl {
  bb_server_desc desc = {};
  Clock::time_point t0;
  cudaStream_t stream = nullptr;  // every batch steps on it
  std::mutex mu;      // queue, requests, worlds, bookkeeping
  std::mutex gpu_mu;  // calls on the batch objects (the worker's, and bb_server_read_state's)
  std::condition_variable cv;
  std::deque<Req*> queue;  // submitted, not yet admitted (FIFO)
  std::vector<Req*> issued;  // every step enqueued, waiting for the last one to end
  std::unordered_map<uint64_t, std::unique_ptr<Req>> reqs;
  std::unordered_map<uint64_t, std::unique_ptr<WorldRec>> worlds;
  std::vector<std::unique_ptr<Batch>> batches;
  uint64_t held_bytes = 0;
  uint64_t next_ticket = 1, use_clock = 0;
  uint32_t running = 0;  // admitted requests not finished
  bb_server_stats st = {};
  bool stop = false;
  std::thread worker;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
  uint32_t ppb() const { return desc.pairs_per_body ? desc.pairs_per_body : 8; }

  // body state of a resident world's slot to its host copy (it restarts from there elsewhere)
  void save_world(WorldRec* wr) {
    Batch* b = wr->batch;
    const uint32_t n = uint32_t(wr->bodies.size());
    const uint32_t first = b->slots[wr->slot].first;
    std::vector<float> pos(3 * size_t(n)), rot(4 * size_t(n)), vel(3 * size_t(n)), om(3 * size_t(n));
    std::vector<uint32_t> fl(n);
    if (bb_world_read_range(b->w, first, n, pos.data(), rot.data(), vel.data(), om.data(), fl.data()) == BB_OK) {
      for (uint32_t i = 0; i < n; ++i) {
        bb_body_desc& d = wr->bodies[i];
        std::memcpy(d.position, &pos[3 * size_t(i)], 12);
        std::memcpy(d.rotation, &rot[4 * size_t(i)], 16);
        std::memcpy(d.velocity, &vel[3 * size_t(i)], 12);
        std::memcpy(d.omega, &om[3 * size_t(i)], 12);
        d.flags = fl[i];
      }
    }
    b->slots[wr->slot].world = nullptr;
    wr->batch = nullptr;
    ++st.evictions;
  }

  void destroy_batch(Batch* b) {
    for (auto& s : b->slots)
      if (s.world) save_world(s.world);
    for (cudaEvent_t e : b->inflight) cudaEventDestroy(e);
    b->inflight.clear();
    if (b->err_host) cudaFreeHost(b->err_host);
    held_bytes -= b->bytes;
    bb_world_destroy(b->w);
    for (size_t i = 0; i < batches.size(); ++i)
      if (batches[i].get() == b) {
        batches.erase(batches.begin() + long(i));
        break;
      }
  }

  // destroy batches with no running request (least recently used first) until `need` more
  // bytes fit the budget
  bool make_room(uint64_t need) {
    while (held_bytes + need > desc.hbm_budget_bytes) {
      Batch* lru = nullptr;
      for (auto& b : batches)
        if (b->running == 0 && b->inflight.empty() && (!lru || b->last_use < lru->last_use)) lru = b.get();
      if (!lru) return false;
      bool reading = false;
      for (auto& s : lru->slots) reading |= s.world && s.world->reading;
      if (reading) return false;
      destroy_batch(lru);
    }
    return true;
  }

  Batch* create_batch(const Req* q, uint32_t cls, bb_status* err) {
    // capacity kBatchBodies, at least the first slot's size; under a small budget smaller: one
    // batch should not take more than half of it
    uint32_t cap = std::max(kBatchBodies, 1u << cls);
    while (cap > (1u << cls) && bb_world_bytes_for(cap, ppb()) > desc.hbm_budget_bytes / 2) cap /= 2;
    const uint64_t need = bb_world_bytes_for(cap, ppb());
    if (need > desc.hbm_budget_bytes) {
      *err = BB_E_BUDGET;
      return nullptr;
    }
    if (!make_room(need)) {
      *err = BB_OK;  // wait for running requests to end
      return nullptr;
    }
    auto b = std::make_unique<Batch>();
    bb_world_desc wd = {};
    wd.max_bodies = cap;
    wd.pairs_per_body = ppb();
    wd.device = desc.device;
    wd.stream = stream;
    if (bb_world_create(&wd, &b->w) != BB_OK) {
      *err = BB_E_CUDA;
      return nullptr;
    }
    b->stream = static_cast<cudaStream_t>(bb_world_stream(b->w));
    b->step_key = q->step_key;
    b->dt = q->r.dt;
    b->substeps = q->r.substeps;
    b->cap = cap;
    bb_solver_params p = q->r.params;
    p.bounds_mode = BB_BOUNDS_FIXED;
    for (int k = 0; k < 3; ++k) {
      p.world_min[k] = 0.f;
      p.world_extent[k] = 1.f;
    }
    bb_status s = bb_set_solver_params(b->w, &p);
    if (s == BB_OK) s = bb_add_box_shape(b->w, 0.001f, 0.001f, 0.001f, &b->park_shape);
    if (s == BB_OK && cudaMallocHost(&b->err_host, 2 * sizeof(uint32_t)) != cudaSuccess) s = BB_E_CUDA;
    if (s != BB_OK) {
      bb_world_destroy(b->w);
      *err = s;
      return nullptr;
    }
    b->err_host[0] = b->err_host[1] = 0;
    b->bytes = bb_world_device_bytes(b->w);
    held_bytes += b->bytes;
    ++st.worlds_created;
    batches.push_back(std::move(b));
    return batches.back().get();
  }

  // the world's bodies with their shape handles in batch b (shapes added once per batch)
  bb_status batch_bodies(Batch* b, const WorldRec* wr, std::vector<bb_body_desc>& out) {
    std::vector<uint32_t> handle(wr->shapes.size());
    for (size_t k = 0; k < wr->shapes.size(); ++k) {
      const bb_shape_desc& sh = wr->shapes[k];
      auto key = std::make_tuple(sh.type, sh.half[0], sh.type == BB_SHAPE_SPHERE ? 0.f : sh.half[1],
                                 sh.type == BB_SHAPE_SPHERE ? 0.f : sh.half[2]);
      auto it = b->shape_handle.find(key);
      if (it == b->shape_handle.end()) {
        uint32_t h = 0;
        bb_status s = sh.type == BB_SHAPE_SPHERE ? bb_add_sphere_shape(b->w, sh.half[0], &h)
                                                 : bb_add_box_shape(b->w, sh.half[0], sh.half[1], sh.half[2], &h);
        if (s != BB_OK) return s;
        it = b->shape_handle.emplace(key, h).first;
      }
      handle[k] = it->second;
    }
    out = wr->bodies;
    for (auto& d : out) {
      d.shape = handle[d.shape];
      d.flags &= BB_BODY_DYNAMIC | BB_BODY_GRAVITY | BB_BODY_SLEEPING;
    }
    return BB_OK;
  }

  // world wr into slot k of batch b: a refill of a free slot of its size class, or a new slot
  // of 2^cls bodies (k == slots.size()) padded with parked bodies
  bb_status place(Batch* b, uint32_t k, uint32_t cls, WorldRec* wr) {
    const uint32_t slot_cap = 1u << cls;
    // A world still resident in a batch of another step class moves by device copies (same
    // stream, so after that batch's queued steps); its host copy is stale and not needed.
    Batch* from = wr->batch;
    std::vector<bb_body_desc> bodies;
    bb_status s = BB_OK;
    if (from) {
      bodies.resize(slot_cap);  // a new slot starts parked, then takes the moved bodies
    } else {
      s = batch_bodies(b, wr, bodies);
      if (s != BB_OK) return s;
    }
    bb_batch_world_desc wd = {};
    std::memcpy(wd.world_min, wr->wmin, sizeof(wd.world_min));
    std::memcpy(wd.world_extent, wr->wext, sizeof(wd.world_extent));
    const uint32_t n_real = uint32_t(wr->bodies.size());
    if (from && k < b->slots.size()) {
      s = bb_world_move_in(b->w, k, &wd, from->w, wr->slot, n_real);
    } else if (k < b->slots.size()) {
      s = bb_world_refill(b->w, k, &wd, bodies.data(), uint32_t(bodies.size()));
    } else {
      const uint32_t n = from ? 0u : uint32_t(bodies.size());
      bodies.resize(slot_cap);
      for (uint32_t i = n; i < slot_cap; ++i) {
        bb_body_desc& d = bodies[i];
        std::memset(&d, 0, sizeof(d));
        d.position[0] = wr->wmin[0] - 1000.0f - 0.01f * float(i - n);
        d.position[1] = wr->wmin[1] - 1000.0f;
        d.position[2] = wr->wmin[2] - 1000.0f;
        d.rotation[3] = 1.0f;
        d.shape = b->park_shape;
      }
      uint32_t widx = 0, first = 0;
      s = bb_add_world(b->w, &wd, bodies.data(), slot_cap, &widx, &first);
      if (s == BB_OK) {
        b->slots.emplace_back();
        b->slots.back().cls = cls;
        b->slots.back().first = first;
        b->used += slot_cap;
      }
      if (s == BB_OK && from) s = bb_world_move_in(b->w, k, &wd, from->w, wr->slot, n_real);
    }
    if (s != BB_OK) return s;
    if (from) from->slots[wr->slot].world = nullptr;
    b->slots[k].world = wr;
    wr->batch = b;
    wr->slot = k;
    return BB_OK;
  }

  // Admission of q: a slot for its world in a batch of its step class.  Returns false when q
  // must wait (no slot and no room yet); sets *fail when it can never run.
  bool admit(Req* q, bb_status* fail) {
    *fail = BB_OK;
    WorldRec* wr = q->w;
    Batch* b = wr->batch;
    if (b && b->step_key == q->step_key) {  // resident in a batch of its class: resume in place
      bb_status s = bb_world_pause(b->w, wr->slot, 0);
      if (s != BB_OK) *fail = s;
      return true;
    }
    // otherwise it moves to a batch of its new step class (its warm starts restart there); it
    // stays registered in its old slot until placed, so a batch destroyed to make room saves it
    // A free slot of its size class in a batch of its step class (the busiest such batch: more
    // worlds per step), else a new slot where a batch has room, else the slot of an idle world
    // of that size class (saved to the host), else a new batch.
    const uint32_t cls = class_of(uint32_t(wr->bodies.size()));
    Batch* best = nullptr;
    uint32_t best_k = 0;
    for (auto& c : batches) {
      if (c->step_key != q->step_key) continue;
      uint32_t k = 0;
      while (k < c->slots.size() && (c->slots[k].world || c->slots[k].cls != cls)) ++k;
      if (k == c->slots.size()) continue;
      if (!best || c->running > best->running) {
        best = c.get();
        best_k = k;
      }
    }
    if (!best) {
      for (auto& c : batches) {
        if (c->step_key != q->step_key || c->used + (1u << cls) > c->cap) continue;
        if (!best || c->running > best->running) {
          best = c.get();
          best_k = uint32_t(c->slots.size());
        }
      }
    }
    if (!best) {
      // a slot of this size class holding an idle paused world can be taken over
      for (auto& c : batches) {
        if (c->step_key != q->step_key) continue;
        for (uint32_t k = 0; k < c->slots.size(); ++k) {
          Slot& sl = c->slots[k];
          if (sl.cls == cls && sl.world && !sl.world->busy && !sl.world->reading && !sl.req) {
            save_world(sl.world);
            best = c.get();
            best_k = k;
            break;
          }
        }
        if (best) break;
      }
    }
    if (!best) {
      bb_status err = BB_OK;
      best = create_batch(q, cls, &err);
      if (!best) {
        *fail = err;
        return err != BB_OK;
      }
      best_k = 0;
    }
    const auto t = Clock::now();
    bb_status s = place(best, best_k, cls, wr);
    st.materialise_s += std::chrono::duration<double>(Clock::now() - t).count();
    if (s != BB_OK) *fail = s;
    return true;
  }

  void finish(Req* q, bb_status result) {
    q->result = result;
    q->finish_s = now();
    q->done = true;
    if (q->ev) {
      cudaEventDestroy(q->ev);
      q->ev = nullptr;
    }
    if (q->w) {
      q->w->busy = false;
      q->w->last_use = ++use_clock;
    }
    ++st.completed;
    if (result == BB_OK) st.body_steps += uint64_t(q->w->bodies.size()) * q->r.steps;
    else ++st.failed;
  }

  void loop() {
    if (desc.device >= 0) cudaSetDevice(desc.device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      // retire requests whose last step ended
      for (size_t i = 0; i < issued.size();) {
        Req* q = issued[i];
        if (cudaEventQuery(q->ev) == cudaSuccess) {
          const uint32_t e = q->batch->err_host[0];
          q->error_flags = e;
          q->error_site = q->batch->err_host[1];
          bb_status res = BB_OK;
          if (e & (BB_ERRF_PAIR_OVERFLOW | BB_ERRF_CONTACT_OVERFLOW)) res = BB_E_CAPACITY;
          else if (e) res = BB_E_DEVICE_LIMIT;
          --q->batch->running;
          --running;
          finish(q, res);
          issued[i] = issued.back();
          issued.pop_back();
        } else {
          ++i;
        }
      }
      // admit in arrival order; a world runs one request at a time (later ones wait in order)
      {
        std::lock_guard<std::mutex> g(gpu_mu);
        const uint32_t cap = desc.max_active ? desc.max_active : 64;
        for (auto it = queue.begin(); it != queue.end() && running < cap;) {
          Req* q = *it;
          if (q->w->busy || q->w->reading) {
            ++it;
            continue;
          }
          bb_status fail = BB_OK;
          if (!admit(q, &fail)) {
            ++it;
            continue;
          }
          it = queue.erase(it);
          q->start_s = now();
          q->w->busy = true;
          if (fail != BB_OK) {
            finish(q, fail);
            continue;
          }
          Batch* b = q->w->batch;
          q->batch = b;
          b->slots[q->w->slot].req = q;
          b->slots[q->w->slot].remaining = q->r.steps;
          ++b->running;
          ++running;
        }
        // step every batch with running requests, keeping a few steps queued per batch
        const auto t = Clock::now();
        for (auto& bp : batches) {
          Batch* b = bp.get();
          while (!b->inflight.empty() && cudaEventQuery(b->inflight.front()) == cudaSuccess) {
            cudaEventDestroy(b->inflight.front());
            b->inflight.pop_front();
          }
          while (b->running && b->inflight.size() < kInFlight) {
            bool any = false;
            for (auto& sl : b->slots) any |= sl.req && sl.remaining > 0;
            if (!any) break;
            bb_status s = bb_step(b->w, b->dt, b->substeps);
            ++st.batch_steps;
            cudaMemcpyAsync(b->err_host, bb_world_error_word(b->w), sizeof(uint32_t), cudaMemcpyDeviceToHost,
                            b->stream);
            cudaMemcpyAsync(b->err_host + 1, bb_world_error_site_word(b->w), sizeof(uint32_t),
                            cudaMemcpyDeviceToHost, b->stream);
            cudaEvent_t ev = nullptr;
            cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
            cudaEventRecord(ev, b->stream);
            b->inflight.push_back(ev);
            b->last_use = ++use_clock;
            for (uint32_t k = 0; k < b->slots.size(); ++k) {
              Slot& sl = b->slots[k];
              if (!sl.req || sl.remaining == 0) continue;
              ++st.slot_steps;
              if (s != BB_OK) sl.req->result = s;
              if (--sl.remaining == 0) {  // its last step: stop the world after it, then retire
                Req* q = sl.req;
                bb_world_pause(b->w, k, 1);
                cudaEventCreateWithFlags(&q->ev, cudaEventDisableTiming);
                cudaEventRecord(q->ev, b->stream);
                sl.req = nullptr;
                issued.push_back(q);
              }
            }
          }
        }
        st.issue_s += std::chrono::duration<double>(Clock::now() - t).count();
      }
      st.resident_bytes = held_bytes;
      st.active = running;
      st.queued = uint32_t(queue.size());
      if (stop && queue.empty() && running == 0) break;
      cv.notify_all();
      if (running == 0 && queue.empty()) cv.wait(lk);
      else cv.wait_for(lk, std::chrono::microseconds(50));
    }
  }
};

namespace {
bb_server_impl* S(void* s) { return static_cast<bb_server_impl*>(s); }
}  // namespace

bb_status bb_server_create(const bb_server_desc* desc, void** out_server) {
  if (!desc || !out_server || desc->hbm_budget_bytes == 0) return bb_fail(BB_E_INVALID, "bb_server_create: bad arguments");
  auto* s = new bb_server_impl();
  s->desc = *desc;
  s->t0 = Clock::now();
  if (desc->device >= 0 && cudaSetDevice(desc->device) != cudaSuccess) {
    delete s;
    return bb_fail(BB_E_CUDA, "bb_server_create: cudaSetDevice failed");
  }
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete s;
    return bb_fail(BB_E_CUDA, "bb_server_create: cudaStreamCreate failed");
  }
  s->worker = std::thread([s] { s->loop(); });
  *out_server = s;
  return BB_OK;
}

bb_status bb_server_destroy(void* server) {
  bb_server_impl* s = S(server);
  if (!s) return bb_fail(BB_E_INVALID, "bb_server_destroy: null server");
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv.notify_all();
  s->worker.join();
  cudaStreamSynchronize(s->stream);
  for (auto& b : s->batches) {
    for (cudaEvent_t e : b->inflight) cudaEventDestroy(e);
    if (b->err_host) cudaFreeHost(b->err_host);
    bb_world_destroy(b->w);
  }
  cudaStreamDestroy(s->stream);
  delete s;
  return BB_OK;
}

bb_status bb_server_submit(void* server, const bb_request* req, uint64_t* out_ticket) {
  bb_server_impl* s = S(server);
  if (!s || !req || !out_ticket || req->steps == 0 || !(req->dt > 0) || req->substeps == 0)
    return bb_fail(BB_E_INVALID, "bb_server_submit: bad arguments");
  const double t_submit = s->now();  // before waiting for the lock
  auto q = std::make_unique<Req>();
  q->r = *req;
  q->step_key = step_key_of(*req);
  if (req->n_bodies) {
    if (!req->bodies || (req->n_shapes && !req->shapes)) return bb_fail(BB_E_INVALID, "bb_server_submit: null arrays");
    for (uint32_t i = 0; i < req->n_bodies; ++i)
      if (req->bodies[i].shape >= req->n_shapes) return bb_fail(BB_E_INVALID, "bb_server_submit: shape index out of range");
    for (uint32_t i = 0; i < req->n_shapes; ++i)
      if (req->shapes[i].type != BB_SHAPE_BOX && req->shapes[i].type != BB_SHAPE_SPHERE)
        return bb_fail(BB_E_INVALID, "bb_server_submit: served worlds take box and sphere shapes");
    q->bodies.assign(req->bodies, req->bodies + req->n_bodies);
    q->shapes.assign(req->shapes, req->shapes + req->n_shapes);
  }
  q->r.bodies = nullptr;
  q->r.shapes = nullptr;
  std::lock_guard<std::mutex> lk(s->mu);
  auto wit = s->worlds.find(req->world);
  WorldRec* wr = nullptr;
  if (wit == s->worlds.end()) {
    if (q->bodies.empty()) return bb_fail(BB_E_INVALID, "bb_server_submit: unknown world and no bodies");
    auto w = std::make_unique<WorldRec>();
    w->key = req->world;
    w->bodies = std::move(q->bodies);
    w->shapes = std::move(q->shapes);
    std::memcpy(w->wmin, req->world_min, sizeof(w->wmin));
    std::memcpy(w->wext, req->world_extent, sizeof(w->wext));
    for (int k = 0; k < 3; ++k)
      if (!(w->wext[k] > 0)) return bb_fail(BB_E_INVALID, "bb_server_submit: world_extent must be positive");
    wr = w.get();
    s->worlds.emplace(req->world, std::move(w));
  } else {
    if (!q->bodies.empty()) return bb_fail(BB_E_INVALID, "bb_server_submit: world exists; bodies must be NULL");
    wr = wit->second.get();
  }
  q->w = wr;
  q->ticket = s->next_ticket++;
  q->submit_s = t_submit;
  *out_ticket = q->ticket;
  s->queue.push_back(q.get());
  s->reqs.emplace(q->ticket, std::move(q));
  ++s->st.submitted;
  s->cv.notify_all();
  return BB_OK;
}

static void fill_status(const Req& q, bb_request_status* out) {
  out->done = q.done ? 1u : 0u;
  out->result = q.result;
  out->submit_s = q.submit_s;
  out->start_s = q.start_s;
  out->finish_s = q.finish_s;
  out->error_flags = q.error_flags;
  out->error_site = q.error_site;
}

bb_status bb_server_poll(void* server, uint64_t ticket, bb_request_status* out) {
  bb_server_impl* s = S(server);
  if (!s || !out) return bb_fail(BB_E_INVALID, "bb_server_poll: bad arguments");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return bb_fail(BB_E_INVALID, "bb_server_poll: unknown ticket");
  fill_status(*it->second, out);
  return BB_OK;
}

bb_status bb_server_wait(void* server, uint64_t ticket, bb_request_status* out) {
  bb_server_impl* s = S(server);
  if (!s) return bb_fail(BB_E_INVALID, "bb_server_wait: bad arguments");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return bb_fail(BB_E_INVALID, "bb_server_wait: unknown ticket");
  Req* q = it->second.get();
  s->cv.wait(lk, [q] { return q->done; });
  if (out) fill_status(*q, out);
  return BB_OK;
}

bb_status bb_server_read_state(void* server, uint64_t world, float* position, float* rotation, float* velocity,
                               float* omega, uint32_t* n_bodies) {
  bb_server_impl* s = S(server);
  if (!s) return bb_fail(BB_E_INVALID, "bb_server_read_state: null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->worlds.find(world);
  if (it == s->worlds.end()) return bb_fail(BB_E_INVALID, "bb_server_read_state: unknown world");
  WorldRec* wr = it->second.get();
  s->cv.wait(lk, [wr] { return !wr->busy && !wr->reading; });
  const uint32_t n = uint32_t(wr->bodies.size());
  if (n_bodies) *n_bodies = n;
  if (wr->batch) {  // resident (paused in its slot): copy its range out of the batch
    wr->reading = true;
    Batch* b = wr->batch;
    const uint32_t first = b->slots[wr->slot].first;
    lk.unlock();
    bb_status st;
    {
      std::lock_guard<std::mutex> g(s->gpu_mu);
      st = bb_world_read_range(b->w, first, n, position, rotation, velocity, omega, nullptr);
    }
    lk.lock();
    wr->reading = false;
    s->cv.notify_all();
    return st;
  }
  for (uint32_t i = 0; i < n; ++i) {  // not resident: the saved state
    const bb_body_desc& b = wr->bodies[i];
    if (position) std::memcpy(position + 3 * size_t(i), b.position, 12);
    if (rotation) std::memcpy(rotation + 4 * size_t(i), b.rotation, 16);
    if (velocity) std::memcpy(velocity + 3 * size_t(i), b.velocity, 12);
    if (omega) std::memcpy(omega + 3 * size_t(i), b.omega, 12);
  }
  return BB_OK;
}

bb_status bb_server_get_stats(void* server, bb_server_stats* out) {
  bb_server_impl* s = S(server);
  if (!s || !out) return bb_fail(BB_E_INVALID, "bb_server_get_stats: bad arguments");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->st;
  out->resident_bytes = s->held_bytes;
  uint32_t res = 0;
  for (auto& kv : s->worlds)
    if (kv.second->batch) ++res;
  out->resident_worlds = res;
  out->known_worlds = uint32_t(s->worlds.size());
  return BB_OK;
}
