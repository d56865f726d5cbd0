// bb_server.cu -- serving loop: step requests for many device-resident worlds, admitted by an
// HBM budget, their work overlapping on the device.
//
// No reference counterpart: the reference steps one scene per frame from its render loop
// (src/renderer_manager.cpp:254-257 -> RigidBodyManager::simulate).  This is the serving
// pattern built on the same step: every world is a bb_world (own stream, own CUDA graphs); a
// worker thread admits queued requests while the concurrency slots and the HBM budget allow,
// enqueues all of a request's steps on its world's stream at once, and retires requests as
// their completion events fire, so requests that arrive while others run start at once.
//
// A world keeps its device state (bodies, warm-start contacts, sort order) between requests
// while it stays resident.  When memory is needed for a new world, idle worlds are evicted:
// their body state (pose, velocity, sleep flag) is saved on the host and the world is rebuilt
// from it when a later request continues it (an evicted world restarts its warm-start state).
// World objects are pooled by capacity class (powers of two) and reused through bb_world_clear.
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
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/beatbox.h"

bb_status bb_fail(bb_status code, const char* msg);

namespace {

using Clock = std::chrono::steady_clock;

struct WorldRec {
  uint64_t key = 0;
  void* world = nullptr;             // resident bb_world, or nullptr when evicted
  uint32_t cls = 0;                  // capacity class of `world` (bodies = 1 << cls)
  std::vector<bb_shape_desc> shapes;
  std::vector<bb_body_desc> bodies;  // as given; pose, velocity and flags refreshed on eviction
  float wmin[3] = {0, 0, 0}, wext[3] = {1, 1, 1};
  bool busy = false;
  uint64_t last_use = 0;
};

struct Req {
  uint64_t ticket = 0;
  bb_request r = {};
  std::vector<bb_shape_desc> shapes;  // copies for a new world
  std::vector<bb_body_desc> bodies;
  double submit_s = 0, start_s = 0, finish_s = 0;
  bb_status result = BB_OK;
  bool done = false;
  cudaEvent_t ev = nullptr;
  WorldRec* w = nullptr;
};

uint32_t class_of(uint32_t n) {
  uint32_t c = 6;  // smallest pooled world: 64 bodies
  while ((1ull << c) < n) ++c;
  return c;
}

}  // namespace

struct bb_server_impl {
  bb_server_desc desc = {};
  Clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Req*> queue;  // submitted, not yet admitted (FIFO)
  std::vector<Req*> active;
  std::unordered_map<uint64_t, std::unique_ptr<Req>> reqs;
  std::unordered_map<uint64_t, std::unique_ptr<WorldRec>> worlds;
  std::map<uint32_t, std::vector<void*>> pool;  // free bb_world objects by capacity class
  std::map<uint32_t, uint64_t> class_bytes;     // device bytes of one world of each class
  uint64_t held_bytes = 0;                      // device bytes of resident + pooled worlds
  uint64_t next_ticket = 1, use_clock = 0;
  bb_server_stats st = {};
  bool stop = false;
  std::thread worker;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

  uint64_t bytes_of_class(uint32_t c) {
    auto it = class_bytes.find(c);
    if (it != class_bytes.end()) return it->second;
    const uint64_t b = bb_world_bytes_for(1u << c, desc.pairs_per_body ? desc.pairs_per_body : 8);
    class_bytes[c] = b;
    return b;
  }

  // free pooled objects, then evict idle resident worlds (least recently used first), until
  // `need` more bytes fit the budget
  bool make_room(uint64_t need) {
    while (held_bytes + need > desc.hbm_budget_bytes) {
      bool freed = false;
      for (auto& kv : pool) {
        if (kv.second.empty()) continue;
        void* w = kv.second.back();
        kv.second.pop_back();
        held_bytes -= bb_world_device_bytes(w);
        bb_world_destroy(w);
        freed = true;
        break;
      }
      if (freed) continue;
      WorldRec* lru = nullptr;
      for (auto& kv : worlds) {
        WorldRec* wr = kv.second.get();
        if (!wr->busy && wr->world && (!lru || wr->last_use < lru->last_use)) lru = wr;
      }
      if (!lru) return false;
      evict(lru);
    }
    return true;
  }

  void evict(WorldRec* wr) {  // save the body state, return the object to the pool
    const uint32_t n = bb_body_count(wr->world);
    std::vector<float> pos(3 * size_t(n)), rot(4 * size_t(n)), vel(3 * size_t(n)), om(3 * size_t(n));
    std::vector<uint32_t> fl(n);
    bb_read_state(wr->world, pos.data(), rot.data(), vel.data(), om.data());
    bb_read_flags(wr->world, fl.data());
    for (uint32_t i = 0; i < n && i < wr->bodies.size(); ++i) {
      bb_body_desc& b = wr->bodies[i];
      std::memcpy(b.position, &pos[3 * size_t(i)], 12);
      std::memcpy(b.rotation, &rot[4 * size_t(i)], 16);
      std::memcpy(b.velocity, &vel[3 * size_t(i)], 12);
      std::memcpy(b.omega, &om[3 * size_t(i)], 12);
      b.flags = fl[i];
    }
    pool[wr->cls].push_back(wr->world);
    wr->world = nullptr;
    ++st.evictions;
  }

  // Admission reserves what request q needs while the lock is held: a pooled world object of
  // its class, or budget for a new one.  The slow part (creating the world, loading bodies,
  // enqueueing the steps) runs after the lock is released, so submitters never wait on it.
  struct Start {
    Req* q = nullptr;
    void* pooled = nullptr;  // reused world object (cleared before use)
    uint64_t reserved = 0;   // budget reserved for a new world object
    bb_status result = BB_OK;
    double materialise_s = 0, issue_s = 0;
  };

  // outside the lock: materialise the world if needed, set parameters, enqueue all steps
  void run_start(Start& sp) {
    Req* q = sp.q;
    WorldRec* wr = q->w;
    bb_status s = BB_OK;
    const auto t0 = Clock::now();
    if (!wr->world) {
      void* w = sp.pooled;
      if (w) {
        s = bb_world_clear(w);
      } else {
        bb_world_desc wd = {};
        wd.max_bodies = 1u << wr->cls;
        wd.pairs_per_body = desc.pairs_per_body ? desc.pairs_per_body : 8;
        wd.device = desc.device;
        s = bb_world_create(&wd, &w);
        if (s != BB_OK) w = nullptr;
      }
      for (size_t k = 0; k < wr->shapes.size() && s == BB_OK; ++k) {  // handles come out as 0, 1, 2, ...
        const bb_shape_desc& sh = wr->shapes[k];
        uint32_t h = 0;
        s = sh.type == BB_SHAPE_SPHERE ? bb_add_sphere_shape(w, sh.half[0], &h)
                                       : bb_add_box_shape(w, sh.half[0], sh.half[1], sh.half[2], &h);
      }
      uint32_t first = 0;
      if (s == BB_OK) s = bb_add_bodies(w, wr->bodies.data(), uint32_t(wr->bodies.size()), &first);
      sp.pooled = w;  // the object now held for this world (nullptr if creation failed)
      if (s != BB_OK) {
        sp.result = s;
        return;
      }
    }
    void* w = wr->world ? wr->world : sp.pooled;
    const auto t1 = Clock::now();
    sp.materialise_s = std::chrono::duration<double>(t1 - t0).count();
    bb_solver_params p = q->r.params;
    std::memcpy(p.world_min, wr->wmin, sizeof(p.world_min));
    std::memcpy(p.world_extent, wr->wext, sizeof(p.world_extent));
    p.bounds_mode = BB_BOUNDS_FIXED;
    s = bb_set_solver_params(w, &p);
    for (uint32_t k = 0; k < q->r.steps && s == BB_OK; ++k) s = bb_step(w, q->r.dt, q->r.substeps);
    if (s == BB_OK && cudaEventCreateWithFlags(&q->ev, cudaEventDisableTiming) != cudaSuccess) s = BB_E_CUDA;
    if (s == BB_OK && cudaEventRecord(q->ev, static_cast<cudaStream_t>(bb_world_stream(w))) != cudaSuccess) s = BB_E_CUDA;
    sp.issue_s = std::chrono::duration<double>(Clock::now() - t1).count();
    sp.result = s;
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
    std::vector<Start> todo;
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      // retire finished requests
      for (size_t i = 0; i < active.size();) {
        Req* q = active[i];
        if (cudaEventQuery(q->ev) == cudaSuccess) {
          bb_status s = bb_sync(q->w->world);  // device error flags of the world
          finish(q, s);
          active[i] = active.back();
          active.pop_back();
        } else {
          ++i;
        }
      }
      // admit in arrival order; a world runs one request at a time (later ones wait in order)
      todo.clear();
      const uint32_t slots = desc.max_active ? desc.max_active : 64;
      for (auto it = queue.begin(); it != queue.end() && active.size() + todo.size() < slots;) {
        Req* q = *it;
        WorldRec* wr = q->w;
        if (wr->busy) {
          ++it;
          continue;
        }
        Start sp;
        sp.q = q;
        if (!wr->world) {
          wr->cls = class_of(uint32_t(wr->bodies.size()));
          auto pit = pool.find(wr->cls);
          if (pit != pool.end() && !pit->second.empty()) {
            sp.pooled = pit->second.back();
            pit->second.pop_back();
          } else {
            const uint64_t need = bytes_of_class(wr->cls);
            if (need > desc.hbm_budget_bytes) {  // can never fit
              it = queue.erase(it);
              q->start_s = now();
              finish(q, BB_E_BUDGET);
              continue;
            }
            if (!make_room(need)) {  // wait for running requests to free memory
              ++it;
              continue;
            }
            held_bytes += need;
            sp.reserved = need;
          }
        }
        wr->busy = true;
        q->start_s = now();
        it = queue.erase(it);
        todo.push_back(sp);
      }
      if (!todo.empty()) {
        lk.unlock();
        // independent worlds: materialise and enqueue them from several host threads (graph
        // capture and world creation are host-heavy; each world is touched by one thread)
        const size_t nt = std::min<size_t>(todo.size(), 8);
        if (nt <= 1) {
          for (Start& sp : todo) run_start(sp);
        } else {
          std::vector<std::thread> th;
          for (size_t t = 0; t < nt; ++t)
            th.emplace_back([this, &todo, t, nt] {
              if (desc.device >= 0) cudaSetDevice(desc.device);
              for (size_t k = t; k < todo.size(); k += nt) run_start(todo[k]);
            });
          for (auto& x : th) x.join();
        }
        lk.lock();
        for (Start& sp : todo) {
          Req* q = sp.q;
          WorldRec* wr = q->w;
          st.materialise_s += sp.materialise_s;
          st.issue_s += sp.issue_s;
          if (sp.reserved) {  // a new world object: account its real size
            held_bytes -= sp.reserved;
            if (sp.pooled) {
              held_bytes += bb_world_device_bytes(sp.pooled);
              ++st.worlds_created;
            }
          }
          if (!wr->world && sp.pooled) {
            if (sp.result == BB_OK) wr->world = sp.pooled;
            else pool[wr->cls].push_back(sp.pooled);
          }
          if (sp.result != BB_OK) finish(q, sp.result);
          else active.push_back(q);
        }
      }
      st.resident_bytes = held_bytes;
      st.active = uint32_t(active.size());
      st.queued = uint32_t(queue.size());
      if (stop && queue.empty() && active.empty()) break;
      cv.notify_all();
      if (active.empty() && queue.empty()) cv.wait(lk);
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
  for (auto& kv : s->worlds)
    if (kv.second->world) bb_world_destroy(kv.second->world);
  for (auto& kv : s->pool)
    for (void* w : kv.second) bb_world_destroy(w);
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
  if (req->n_bodies) {
    if (!req->bodies || (req->n_shapes && !req->shapes)) return bb_fail(BB_E_INVALID, "bb_server_submit: null arrays");
    for (uint32_t i = 0; i < req->n_bodies; ++i)
      if (req->bodies[i].shape >= req->n_shapes) return bb_fail(BB_E_INVALID, "bb_server_submit: shape index out of range");
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
  s->cv.wait(lk, [wr] { return !wr->busy; });
  const uint32_t n = uint32_t(wr->bodies.size());
  if (n_bodies) *n_bodies = n;
  if (wr->world) return bb_read_state(wr->world, position, rotation, velocity, omega);
  for (uint32_t i = 0; i < n; ++i) {  // evicted: the saved state
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
    if (kv.second->world) ++res;
  out->resident_worlds = res;
  out->known_worlds = uint32_t(s->worlds.size());
  return BB_OK;
}
