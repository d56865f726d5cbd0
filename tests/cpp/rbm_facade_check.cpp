// Compiled by tests/test_rbm_facade.py against include/beatbox_rbm.hpp and libbeatbox.so: the
// C++ drop-in for the reference's RigidBodyManager (src/rigid_body_manager.hpp:14-70).
//
//   rbm_facade_check nogpu   create() must return false (no device to create a world on)
//   rbm_facade_check gpu     a box stack built through the facade and 10 simulate() calls must
//                            equal the same bodies stepped through the C ABI bit for bit, and
//                            read_back_sim_config() must equal bb_read_stats of that world
#include <cstdio>
#include <cstring>
#include <vector>

#include "beatbox_rbm.hpp"

namespace {
int fail(const char* what) {
  std::printf("FAIL %s: %s\n", what, bb_last_error_string());
  return 1;
}

// a 4 x 4 x 3 stack of unit boxes with small offsets, over a static ground box
std::vector<beatbox::RigidBodyDesc> scene() {
  std::vector<beatbox::RigidBodyDesc> v;
  beatbox::RigidBodyDesc g;
  g.flags = 0;
  g.position[1] = -50.0f;
  for (int k = 0; k < 3; ++k) {
    g.minimum[k] = -50.0f;
    g.maximum[k] = 50.0f;
  }
  g.mass = 0.0f;
  v.push_back(g);
  for (int l = 0; l < 3; ++l)
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c) {
        beatbox::RigidBodyDesc b;
        b.position[0] = -1.65f + 1.1f * c + 0.01f * l;
        b.position[1] = 0.6f + 1.1f * l;
        b.position[2] = -1.65f + 1.1f * r - 0.01f * l;
        b.mass = 1000.0f;
        b.velocity[0] = 0.05f * (c - 1.5f);
        v.push_back(b);
      }
  return v;
}
}  // namespace

int main(int argc, char** argv) {
  const bool gpu = argc > 1 && std::strcmp(argv[1], "gpu") == 0;
  beatbox::RigidBodyManager m(64, 4);
  if (!gpu) {
    if (m.create("no gpu")) {
      std::printf("FAIL create() succeeded without a GPU\n");
      return 1;
    }
    if (m.simulate()) {
      std::printf("FAIL simulate() succeeded without a world\n");
      return 1;
    }
    std::printf("ok nogpu\n");
    return 0;
  }
  if (!m.create("facade", 8)) return fail("create");
  if (m.create("again")) {
    std::printf("FAIL second create() returned true\n");
    return 1;
  }
  m.set_sim_type(beatbox::PGS_SOFT);
  m.params().quirks = BB_QUIRKS_PHYSICAL;
  if (!m.apply()) return fail("apply");
  const std::vector<beatbox::RigidBodyDesc> bodies = scene();
  for (const auto& b : bodies) m.add_rigid_body(b, false);

  // the same world through the C ABI
  bb_world_desc wd{64, 0, -1, nullptr};
  void* w = nullptr;
  if (bb_world_create(&wd, &w) != BB_OK) return fail("bb_world_create");
  for (const auto& b : bodies) {
    uint32_t shape = 0;
    if (bb_add_box_shape(w, 0.5f * (b.maximum[0] - b.minimum[0]), 0.5f * (b.maximum[1] - b.minimum[1]),
                         0.5f * (b.maximum[2] - b.minimum[2]), &shape) != BB_OK)
      return fail("bb_add_box_shape");
    bb_body_desc d{};
    std::memcpy(d.position, b.position, sizeof(d.position));
    std::memcpy(d.rotation, b.rotation, sizeof(d.rotation));
    std::memcpy(d.velocity, b.velocity, sizeof(d.velocity));
    std::memcpy(d.omega, b.omega, sizeof(d.omega));
    d.shape = shape;
    d.flags = b.flags;
    d.mass = b.mass;
    d.friction = b.friction;
    d.restitution = b.restitution;
    d.inertia_mode = BB_INERTIA_PHYSICAL;
    uint32_t id = 0;
    if (bb_add_bodies(w, &d, 1, &id) != BB_OK) return fail("bb_add_bodies");
  }
  bb_solver_params p = m.params();
  if (bb_set_solver_params(w, &p) != BB_OK) return fail("bb_set_solver_params");

  for (int s = 0; s < 10; ++s) {
    if (!m.simulate()) return fail("simulate");
    if (bb_step(w, beatbox::RigidBodyManager::TIME_STEP, 4) != BB_OK) return fail("bb_step");
  }
  if (bb_sync(m.world()) != BB_OK || bb_sync(w) != BB_OK) return fail("bb_sync");
  const uint32_t n = bb_body_count(w);
  if (n != bodies.size() || bb_body_count(m.world()) != n) {
    std::printf("FAIL body counts\n");
    return 1;
  }
  std::vector<float> pa(3 * n), qa(4 * n), va(3 * n), wa(3 * n), pb(3 * n), qb(4 * n), vb(3 * n), wb(3 * n);
  if (bb_read_state(m.world(), pa.data(), qa.data(), va.data(), wa.data()) != BB_OK) return fail("read facade");
  if (bb_read_state(w, pb.data(), qb.data(), vb.data(), wb.data()) != BB_OK) return fail("read abi");
  if (std::memcmp(pa.data(), pb.data(), pa.size() * 4) || std::memcmp(qa.data(), qb.data(), qa.size() * 4) ||
      std::memcmp(va.data(), vb.data(), va.size() * 4) || std::memcmp(wa.data(), wb.data(), wa.size() * 4)) {
    std::printf("FAIL facade and C ABI states differ\n");
    return 1;
  }
  // the stack must have moved: gravity acted on it
  if (pa[3 * 1 + 1] >= 0.6f) {
    std::printf("FAIL the bodies did not move\n");
    return 1;
  }
  std::vector<float> tp, tq;
  if (!m.read_transforms(tp, tq) || std::memcmp(tp.data(), pa.data(), pa.size() * 4)) {
    std::printf("FAIL read_transforms\n");
    return 1;
  }
  if (!m.read_back_sim_config()) return fail("read_back_sim_config");
  bb_step_stats st{};
  if (bb_read_stats(w, &st) != BB_OK) return fail("bb_read_stats");
  const beatbox::SimConfig& c = m.get_sim_config_reference();
  if (c.rigid_body_count != st.body_count || c.active_rigid_body_count != st.active_body_count ||
      c.broad_phase_collision_count != st.pair_count || c.collision_count != st.manifold_count ||
      c.contact_count != st.contact_count || c.island_count != st.island_count ||
      c.graph_color_count != st.graph_color_count || c.sleeping_count != st.sleeping_count ||
      c.error_flags != st.error_flags || c.solver_type != beatbox::PGS_SOFT || st.manifold_count == 0) {
    std::printf("FAIL SimConfig differs from bb_read_stats\n");
    return 1;
  }
  bb_world_destroy(w);
  std::printf("ok gpu %u bodies %u manifolds\n", n, st.manifold_count);
  return 0;
}
