// bb_voxel_build.hpp -- host build of a voxel shape from an occupancy grid.
//
// Follows SceneManager::build_voxel_shape (src/scene_manager.hpp:488-560): the body origin is
// the centre of mass of the solid cells (computed in double), the occupancy bits are x-major
// (bit = x + y*nx + z*nx*ny), and the surface list holds every solid cell with an empty face
// neighbour, in z, y, x order, tagged with the first empty direction in the order -x, +x, -y,
// +y, -z, +z.  Mass properties are per unit density: each cell contributes its point term and
// its own cube term (m vs^2 / 6) about the centre of mass.  The reference accumulates the
// inertia in float and inverts it with glm; this build accumulates and inverts in double and
// rounds once.
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>

struct VoxelBuild {
  uint32_t dims[3] = {0, 0, 0};
  float vs = 0;
  float origin[3] = {0, 0, 0};
  float hi[3] = {0, 0, 0};
  uint32_t solid = 0;
  std::vector<uint32_t> occ;   // ceil(nx*ny*nz / 32) words
  std::vector<uint32_t> surf;  // x | y<<8 | z<<16 | dir<<24
  float unit_mass = 0;
  float unit_inv[6] = {0, 0, 0, 0, 0, 0};  // xx yy zz xy xz yz
};

inline bool voxel_build(uint32_t nx, uint32_t ny, uint32_t nz, float vs, const uint8_t* solid, VoxelBuild& b) {
  if (nx == 0 || ny == 0 || nz == 0 || nx > 256 || ny > 256 || nz > 256 || !(vs > 0) || !solid) return false;
  b = VoxelBuild();
  b.dims[0] = nx;
  b.dims[1] = ny;
  b.dims[2] = nz;
  b.vs = vs;
  auto at = [&](int x, int y, int z) -> bool {
    if (x < 0 || y < 0 || z < 0 || x >= int(nx) || y >= int(ny) || z >= int(nz)) return false;
    return solid[size_t(x) + size_t(y) * nx + size_t(z) * nx * ny] != 0;
  };
  double com[3] = {0, 0, 0};
  for (uint32_t z = 0; z < nz; ++z)
    for (uint32_t y = 0; y < ny; ++y)
      for (uint32_t x = 0; x < nx; ++x)
        if (at(int(x), int(y), int(z))) {
          com[0] += x + 0.5;
          com[1] += y + 0.5;
          com[2] += z + 0.5;
          ++b.solid;
        }
  if (b.solid == 0) return false;
  for (int k = 0; k < 3; ++k) {
    com[k] = com[k] / double(b.solid) * double(vs);
    b.origin[k] = -float(com[k]);
    b.hi[k] = b.origin[k] + float(b.dims[k]) * vs;
  }
  const uint64_t bits = uint64_t(nx) * ny * nz;
  b.occ.assign(size_t((bits + 31) / 32), 0u);
  static const int nb[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
  const double v = double(vs), m = v * v * v;
  double I[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (uint32_t z = 0; z < nz; ++z)
    for (uint32_t y = 0; y < ny; ++y)
      for (uint32_t x = 0; x < nx; ++x) {
        if (!at(int(x), int(y), int(z))) continue;
        const uint64_t bit = uint64_t(x) + uint64_t(y) * nx + uint64_t(z) * nx * ny;
        b.occ[size_t(bit / 32)] |= 1u << (bit % 32);
        const double c[3] = {double(b.origin[0]) + (x + 0.5) * v, double(b.origin[1]) + (y + 0.5) * v,
                             double(b.origin[2]) + (z + 0.5) * v};
        const double r2 = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) I[i][j] += m * ((i == j ? r2 : 0.0) - c[i] * c[j]) + (i == j ? m * v * v / 6.0 : 0.0);
        for (uint32_t dd = 0; dd < 6; ++dd)
          if (!at(int(x) + nb[dd][0], int(y) + nb[dd][1], int(z) + nb[dd][2])) {
            b.surf.push_back(x | (y << 8) | (z << 16) | (dd << 24));
            break;
          }
      }
  b.unit_mass = float(m * b.solid);
  // inverse by cofactors; the result is symmetric up to rounding, averaged to make it exact
  const double c00 = I[1][1] * I[2][2] - I[1][2] * I[2][1], c01 = I[1][2] * I[2][0] - I[1][0] * I[2][2],
               c02 = I[1][0] * I[2][1] - I[1][1] * I[2][0];
  const double det = I[0][0] * c00 + I[0][1] * c01 + I[0][2] * c02;
  if (!(std::fabs(det) > 0)) return false;
  const double inv[3][3] = {
      {c00 / det, (I[0][2] * I[2][1] - I[0][1] * I[2][2]) / det, (I[0][1] * I[1][2] - I[0][2] * I[1][1]) / det},
      {c01 / det, (I[0][0] * I[2][2] - I[0][2] * I[2][0]) / det, (I[0][2] * I[1][0] - I[0][0] * I[1][2]) / det},
      {c02 / det, (I[0][1] * I[2][0] - I[0][0] * I[2][1]) / det, (I[0][0] * I[1][1] - I[0][1] * I[1][0]) / det}};
  b.unit_inv[0] = float(inv[0][0]);
  b.unit_inv[1] = float(inv[1][1]);
  b.unit_inv[2] = float(inv[2][2]);
  b.unit_inv[3] = float(0.5 * (inv[0][1] + inv[1][0]));
  b.unit_inv[4] = float(0.5 * (inv[0][2] + inv[2][0]));
  b.unit_inv[5] = float(0.5 * (inv[1][2] + inv[2][1]));
  return true;
}
