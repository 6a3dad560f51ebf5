// Ghost images of interior cells, written by the kernel that produces the
// cell (internal to the library).  A ghost cell holds the periodic wrap or
// the mirror (with a per-field sign) of an interior cell
// (mhd_halo_exchange.hpp:51-265, boundary_condition.hpp:77-136); a producer
// writing every image of each cell it computes leaves the ghost layers,
// edges and corners filled without a separate pass.
#pragma once

#include "common.cuh"

namespace miso_b200 {

// ---------------------------------------------------------------------------
// Ghost images of an interior cell (faces, edges, corners): at most one
// image coordinate per axis (axis sizes >= 2 * margin), so at most 7.
// ---------------------------------------------------------------------------
struct Img {
  int off[7];             // element offset of image (mask-1) from the cell
  unsigned short neg[7];  // fields whose image is negated
  unsigned valid;         // bit (mask-1): image exists
};

__device__ __forceinline__ bool near_boundary(const Geom &g, int x0, int x1, int x2) {
  return x0 < g.m[0] || x0 >= g.n[0] - g.m[0] || x1 < g.m[1] || x1 >= g.n[1] - g.m[1] ||
         x2 < g.m[2] || x2 >= g.n[2] - g.m[2];
}

__device__ __forceinline__ void make_img(const Geom &g, int x0, int x1, int x2, Img &im) {
  const int xs[3] = {x0, x1, x2};
  int d[3];
  unsigned short nm[3];
  bool h[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int m = g.m[a], n = g.n[a], X = xs[a] + m;
    h[a] = false;
    d[a] = 0;
    nm[a] = 0;
    if (xs[a] < m && !g.ext[a][0]) {
      h[a] = true;
      d[a] = ((g.periodic[a] ? X + n : 2 * m - 1 - X) - X) * (int)g.st[a];
      nm[a] = g.negmask[a][0];
    } else if (xs[a] >= n - m && !g.ext[a][1]) {
      h[a] = true;
      d[a] = ((g.periodic[a] ? X - n : 2 * (m + n) - 1 - X) - X) * (int)g.st[a];
      nm[a] = g.negmask[a][1];
    }
  }
  im.valid = 0;
#pragma unroll
  for (int mask = 1; mask < 8; ++mask) {
    const bool ok = (!(mask & 1) || h[0]) && (!(mask & 2) || h[1]) && (!(mask & 4) || h[2]);
    im.off[mask - 1] = ((mask & 1) ? d[0] : 0) + ((mask & 2) ? d[1] : 0) + ((mask & 4) ? d[2] : 0);
    im.neg[mask - 1] = (unsigned short)(((mask & 1) ? nm[0] : 0) ^ ((mask & 2) ? nm[1] : 0) ^
                                        ((mask & 4) ? nm[2] : 0));
    if (ok) im.valid |= 1u << (mask - 1);
  }
}

// p[cell] = v and every ghost image; field f picks the mirror sign.
template <typename T>
__device__ __forceinline__ void store_img(T *p, long long cell, const Img &im, int f, T v) {
  p[cell] = v;
#pragma unroll
  for (int m = 0; m < 7; ++m)
    if ((im.valid >> m) & 1u) p[cell + im.off[m]] = ((im.neg[m] >> f) & 1u) ? -v : v;
}

template <typename T>
__device__ __forceinline__ void store_cell(T *p, long long cell, bool nb, const Img &im, int f,
                                           T v) {
  if (nb)
    store_img(p, cell, im, f, v);
  else
    p[cell] = v;
}

// Interior coordinate whose value the coordinate t of axis a holds, for t
// in [-m, n + m): t itself inside, else the periodic wrap or the mirror
// (the inverse of the image map above).  side = 0 / 1 on the low / high
// ghost layer (the mirror sign of the value is g.negmask[a][side]), -1
// inside and on a face shared with a neighbouring shard (whose ghost layer
// the halo exchange fills: t is returned as it is).  Lets a pass read a neighbour across a face without the ghost
// layer being filled.
__device__ __forceinline__ int ghost_src(const Geom &g, int a, int t, int &side) {
  const int n = g.n[a];
  if ((t < 0 && g.ext[a][0]) || (t >= n && g.ext[a][1])) {
    side = -1;  // a face shared with a neighbouring shard: its ghosts hold the neighbour's cells
    return t;
  }
  if (t < 0) {
    side = 0;
    return g.periodic[a] ? t + n : -1 - t;
  }
  if (t >= n) {
    side = 1;
    return g.periodic[a] ? t - n : 2 * n - 1 - t;
  }
  side = -1;
  return t;
}

__device__ __forceinline__ int cell_of(const Geom &g, int x0, int x1, int x2) {
  return (x0 + g.m[0]) * (int)g.st[0] + (x1 + g.m[1]) * (int)g.st[1] + (x2 + g.m[2]);
}

}  // namespace miso_b200
