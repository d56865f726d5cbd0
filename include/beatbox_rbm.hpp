// beatbox_rbm.hpp -- header-only C++ facade with the reference's RigidBodyManager surface
// (src/rigid_body_manager.hpp:12-70) over the C ABI of beatbox.h.
//
// Names, argument meaning and error behaviour follow the reference class: create() returns
// false when already created (RBM:123-126); simulate() returns false when not created (the
// reference returns !initialized, RBM:1608-1611, i.e. true on that error -- this facade reports
// the error instead); flag setters return the new flag word.  The world state lives on the
// GPU; bodies come from SceneManager-style RigidBody descriptions (add_rigid_body).
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "beatbox.h"

namespace beatbox {

enum SimSolverType : uint32_t { PGS = BB_SOLVER_PGS, PGS_SOFT = BB_SOLVER_PGS_SOFT, AVBD = BB_SOLVER_AVBD };

// The SimConfig counters the reference reads back each frame (include/shared.inl:571-665).
struct SimConfig {
  SimSolverType solver_type = AVBD;
  uint32_t rigid_body_count = 0, active_rigid_body_count = 0, island_count = 0;
  uint32_t broad_phase_collision_count = 0, collision_count = 0, contact_count = 0;
  uint32_t graph_color_count = 0, graph_color_violations = 0, graph_color_overflow = 0;
  uint32_t sleeping_count = 0, avbd_color_count = 0, avbd_violations = 0, avbd_stick_count = 0;
  uint32_t dbg_fresh = 0, dbg_pen_mm = 0, error_flags = 0;
  float dt = 0.01667f, gravity = -9.81f;
  uint32_t flags = BB_SIM_DEFAULT_FLAGS;
};

// One body as the reference's scenes describe it (RigidBody fields used by the step).
struct RigidBodyDesc {
  uint32_t flags = BB_BODY_DYNAMIC | BB_BODY_GRAVITY;
  float position[3] = {0, 0, 0};
  float rotation[4] = {0, 0, 0, 1};  // x y z w
  float minimum[3] = {-0.5f, -0.5f, -0.5f}, maximum[3] = {0.5f, 0.5f, 0.5f};
  float mass = 1.0f;
  float velocity[3] = {0, 0, 0}, omega[3] = {0, 0, 0};
  float restitution = 0.0f, friction = 0.5f;
  bool sphere = false;  // sphere of radius maximum[0] (no reference counterpart)
};

class RigidBodyManager {
 public:
  static constexpr float TIME_STEP = 0.01667f;  // include/defines.hpp:354

  explicit RigidBodyManager(uint32_t max_bodies = 1024, uint32_t substeps = 1)
      : max_bodies_(max_bodies), substeps_(substeps) {}
  ~RigidBodyManager() { destroy(); }
  RigidBodyManager(const RigidBodyManager&) = delete;
  RigidBodyManager& operator=(const RigidBodyManager&) = delete;

  // RBM::create (src/rigid_body_manager.cpp:121-283): false if already created.
  bool create(const char* /*name*/ = "", uint32_t iterations = 5) {
    if (world_) return false;
    bb_world_desc d{max_bodies_, 0, -1, nullptr};
    if (bb_world_create(&d, &world_) != BB_OK) return false;
    bb_default_solver_params(&params_);
    params_.iterations = params_.relax_iterations = iterations;
    return bb_set_solver_params(world_, &params_) == BB_OK;
  }
  void destroy() {
    if (world_) bb_world_destroy(world_);
    world_ = nullptr;
  }

  // SceneManager::load_scene body assignment (src/scene_manager.hpp:850-887): returns the id.
  // `reference_inertia` reproduces cuboid_get_inverse_intertia(inv_mass, ...) (:861).
  uint32_t add_rigid_body(const RigidBodyDesc& b, bool reference_inertia = true) {
    if (!world_) throw std::runtime_error("RigidBodyManager: create() first");
    uint32_t shape = 0;
    float hx = 0.5f * (b.maximum[0] - b.minimum[0]), hy = 0.5f * (b.maximum[1] - b.minimum[1]),
          hz = 0.5f * (b.maximum[2] - b.minimum[2]);
    bb_status s = b.sphere ? bb_add_sphere_shape(world_, b.maximum[0], &shape) : bb_add_box_shape(world_, hx, hy, hz, &shape);
    if (s != BB_OK) throw std::runtime_error(bb_last_error_string());
    bb_body_desc d{};
    for (int k = 0; k < 3; ++k) {
      d.position[k] = b.position[k];
      d.velocity[k] = b.velocity[k];
      d.omega[k] = b.omega[k];
    }
    for (int k = 0; k < 4; ++k) d.rotation[k] = b.rotation[k];
    d.shape = shape;
    d.flags = b.flags;
    d.mass = b.mass;
    d.friction = b.friction;
    d.restitution = b.restitution;
    d.inertia_mode = reference_inertia ? BB_INERTIA_REFERENCE : BB_INERTIA_PHYSICAL;
    uint32_t id = 0;
    if (bb_add_bodies(world_, &d, 1, &id) != BB_OK) throw std::runtime_error(bb_last_error_string());
    return id;
  }

  // RBM::simulate (RBM:1606-1622): one fixed step of TIME_STEP, run as `substeps` passes.
  bool simulate() {
    if (!world_) return false;
    return bb_step(world_, TIME_STEP, substeps_) == BB_OK;
  }
  // RBM::read_back_sim_config (RBM:1681-1693)
  bool read_back_sim_config() {
    if (!world_) return false;
    bb_step_stats st{};
    if (bb_read_stats(world_, &st) != BB_OK) return false;
    cfg_.solver_type = SimSolverType(params_.solver);
    cfg_.rigid_body_count = st.body_count;
    cfg_.active_rigid_body_count = st.active_body_count;
    cfg_.island_count = st.island_count;
    cfg_.broad_phase_collision_count = st.pair_count;
    cfg_.collision_count = st.manifold_count;
    cfg_.contact_count = st.contact_count;
    cfg_.graph_color_count = st.graph_color_count;
    cfg_.graph_color_violations = st.graph_color_violations;
    cfg_.graph_color_overflow = st.graph_color_overflow;
    cfg_.sleeping_count = st.sleeping_count;
    cfg_.avbd_color_count = st.avbd_color_count;
    cfg_.avbd_violations = st.avbd_violations;
    cfg_.avbd_stick_count = st.stick_count;
    cfg_.dbg_fresh = st.fresh_contacts;
    cfg_.dbg_pen_mm = uint32_t(st.max_penetration * 1000.0f);
    cfg_.error_flags = st.error_flags;
    cfg_.flags = params_.flags;
    cfg_.gravity = params_.gravity;
    cfg_.dt = TIME_STEP / float(substeps_);
    return true;
  }
  SimConfig& get_sim_config_reference() { return cfg_; }

  void skip_warm_starting_once() {
    if (world_) bb_skip_warm_starting_once(world_);
  }
  uint32_t get_sim_flags() const { return params_.flags; }
  uint32_t set_sim_flags(uint32_t flags) {
    params_.flags |= flags;
    apply();
    return params_.flags;
  }
  uint32_t clear_sim_flags(uint32_t flags) {
    params_.flags &= ~flags;
    apply();
    return params_.flags;
  }
  void set_sim_type(SimSolverType type) {
    params_.solver = type;
    apply();
  }
  SimSolverType get_sim_type() const { return SimSolverType(params_.solver); }
  bb_solver_params& params() { return params_; }
  bool apply() { return world_ && bb_set_solver_params(world_, &params_) == BB_OK; }

  // transforms for a renderer (the reference feeds them to the TLAS, AS_mngr.slang:5-36)
  bool read_transforms(std::vector<float>& position, std::vector<float>& rotation) {
    if (!world_) return false;
    uint32_t n = bb_body_count(world_);
    position.resize(3 * size_t(n));
    rotation.resize(4 * size_t(n));
    return bb_read_state(world_, position.data(), rotation.data(), nullptr, nullptr) == BB_OK;
  }
  void* world() { return world_; }

 private:
  uint32_t max_bodies_, substeps_;
  void* world_ = nullptr;
  bb_solver_params params_{};
  SimConfig cfg_;
};

}  // namespace beatbox
