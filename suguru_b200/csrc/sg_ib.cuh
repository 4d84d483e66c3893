// sg_ib.cuh -- Lagrangian <-> Eulerian transfer on the staggered MAC grid.
//
// Replaces eulr2lagr (interp_spread.f90:12-475) and lagr2eulr
// (interp_spread.f90:510-922) on one GPU.  The reference's master/slave image
// copies and MPI halo exchange reduce, on a single domain, to periodic index
// wrap in x and y and clipping of the stencil to [1,kmax] in z
// (interp_spread.f90:340-351, 846-851); the force halo is the copy of
// bound.f90:141-190.
//
// Points are binned by output tile: a counting sort lists, for every tile,
// each point whose stencil reaches it.  Interpolation is a per-point gather.
// Spreading runs one CTA per tile over that list and sums in fixed point in
// shared memory (integer atomics, so the result does not depend on order).
#pragma once
#include "sg_common.cuh"

namespace sg {

// Spreading tile shapes (cells).  FP64 spreading takes shapes of at most 1024
// cells (three 32-bit limbs per cell and component in static shared memory).
// TX = 0 stands for whole x rows (TX = itot): FP32 row tiles, whose fixed-point
// sums take 3 (itot TY TZ + 32) words of dynamic shared memory, at most
// kRowTileSmemMax bytes.
struct TileShape {
  int TX, TY, TZ;
};
constexpr TileShape kTileShapes[] = {{32, 8, 4}, {16, 16, 8}, {32, 8, 8}, {8, 8, 4}, {0, 4, 4}, {0, 8, 4}, {32, 16, 4}};
constexpr int kNumTileShapes = 7;
constexpr unsigned kRowTileSmemMax = 200u * 1024u;

struct IBGrid {
  int itot, jtot, ktot;  // interior cells (imax, jmax, kmax)
  int ldi, ldj, ldk;     // itot+2, jtot+2, ktot+2 (halo of one cell)
  double dxi, dyi, dzi;  // inverse spacings
  double dvi;            // 1 / (dx dy dz)
  int shape;             // index into kTileShapes
  int TX, TY, TZ;        // tile shape
  int ntx, nty, ntz;     // tiles per dimension
  int ntiles;
};

// Per point after binning: base face index b = floor(c) per dimension (x, y
// wrapped into [0, n), z raw) and the fractional offsets c - b.
struct PointBins {
  int* bx;
  int* by;
  int* bz;
  int* tile;
};

}  // namespace sg
