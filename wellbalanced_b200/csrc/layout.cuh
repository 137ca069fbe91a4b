// Device-side layout of the patch state pools and the work lists of the fused kernels.
//
// A state pool holds every patch of a hierarchy, each patch a block of fields with a
// halo of two cells. All fields of a patch share one padded node-shaped layout:
//   2D: (X + 1) x (Y + 1) with X = nx + 4, Y = ny + 4; element (i, j) at i * pitch0 + j;
//   3D: (X + 1) x (Y + 1) x (Z + 1); element (i, j, k) at i * pitch0 + j * pitch1 + k.
// Cell fields use the cell range, node / edge fields their node ranges. Field f of the
// patch starts at `off + f * fstride`.
//   2D fields: 0 rho, 1 m_x, 2 m_y, 3 m_z, 4 E, 5 B_z, 6 A_z (nodes)
//   3D fields: 0 rho, 1 m_x, 2 m_y, 3 m_z, 4 E, 5 A_x, 6 A_y, 7 A_z (edges)
#pragma once

#include <cstdint>

namespace wb {

constexpr int kHalo = 2;

// flags of PatchDesc
constexpr int kWallLo0 = 1 << 0;  // a conducting wall at the lower face along axis 0
constexpr int kWallHi0 = 1 << 1;
constexpr int kWallLo1 = 1 << 2;
constexpr int kWallHi1 = 1 << 3;
constexpr int kWallLo2 = 1 << 4;
constexpr int kWallHi2 = 1 << 5;
constexpr int kOwnLast0 = 1 << 8;  // the patch computes its last node plane along axis 0
constexpr int kOwnLast1 = 1 << 9;
constexpr int kOwnLast2 = 1 << 10;
// a dense block standing for a box of another rank's patch (mailboxes, proxies): the
// copy, interpolation, restriction and face-flux kernels address it like the patch
constexpr int kProxy = 1 << 30;

struct PatchDesc {
  int64_t off;       // element offset of field 0 in the pool
  int64_t fstride;   // elements between fields
  int64_t pitch0;    // elements per step along axis 0
  int64_t pitch1;    // elements per step along axis 1 (3D), 0 in 2D
  int32_t n[3];      // interior cells per axis (n[2] = 1 in 2D)
  int32_t instance;  // index of the time-step slot of this patch
  int32_t flags;
  int32_t level;
  double dx[3];
  int64_t bflux;     // offset of the patch's boundary-face fluxes, -1 if none
};

// One work item of a fused stage kernel: a tile of a patch (origin in interior cells).
struct Tile {
  int32_t patch;
  int32_t x0, y0, z0;
};

}  // namespace wb
