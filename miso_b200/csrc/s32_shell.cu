// Ghost images of the interior shell of a 3-D grid, for several arrays at
// once (FP32; internal to the library).
//
// The streaming kernels of the split path write interior cells only; this
// kernel then gives every interior cell within `margin` of a face its ghost
// images -- the periodic wrap or the mirror with the per-field sign
// (mhd_halo_exchange.hpp:51-265, boundary_condition.hpp:77-136), faces,
// edges and corners -- exactly as the producing kernels would have written
// them (images.cuh).
//
// The shell is enumerated as one flat list, one cell per thread: (A) the
// i-shell planes, (B) the j-shell rows of the remaining planes, (C) the
// k-ends of the remaining rows, each in k-fastest order so neighbouring
// threads touch neighbouring cells.  A thread loads the cell's value in
// every array before it stores any image, so the loads overlap.  An image
// mask limits the work to the images the next pass reads (the faces of one
// axis for a sweep, the faces of all axes without edges and corners for the
// Runge-Kutta star stencil, everything for a step's final state).
#include "common.cuh"
#include "images.cuh"
#include "s32_tiled.h"

namespace miso_b200 {
namespace s32s {

constexpr int MAXA = 2 * NF + 1;

__device__ __forceinline__ void shell_coords(const Geom &g, long long idx, int &x0, int &x1,
                                             int &x2) {
  const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
  const int m0 = g.m[0], m1 = g.m[1], m2 = g.m[2];
  const long long a = 2LL * m0 * n1 * n2;
  if (idx < a) {  // (A) i-shell planes
    const long long plane = (long long)n1 * n2;
    const int p = (int)(idx / plane);
    const long long rem = idx - p * plane;
    x0 = p < m0 ? p : n0 - 2 * m0 + p;
    x1 = (int)(rem / n2);
    x2 = (int)(rem - (long long)x1 * n2);
    return;
  }
  idx -= a;
  const long long b = (long long)(n0 - 2 * m0) * 2 * m1 * n2;
  if (idx < b) {  // (B) j-shell rows of the inner planes
    const long long q = idx / n2;
    x2 = (int)(idx - q * n2);
    x0 = m0 + (int)(q / (2 * m1));
    const int j = (int)(q % (2 * m1));
    x1 = j < m1 ? j : n1 - 2 * m1 + j;
    return;
  }
  idx -= b;  // (C) k-ends of the inner rows
  const int e = (int)(idx % (2 * m2));
  const long long r = idx / (2 * m2);
  x2 = e < m2 ? e : n2 - 2 * m2 + e;
  x1 = m1 + (int)(r % (n1 - 2 * m1));
  x0 = m0 + (int)(r / (n1 - 2 * m1));
}

// cells of the two face slabs of axis `a` (k-fastest order)
__device__ __forceinline__ void slab_coords(const Geom &g, int a, long long idx, int &x0, int &x1,
                                            int &x2) {
  const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
  if (a == 0) {
    const long long plane = (long long)n1 * n2;
    const int p = (int)(idx / plane);
    const long long rem = idx - p * plane;
    x0 = p < g.m[0] ? p : n0 - 2 * g.m[0] + p;
    x1 = (int)(rem / n2);
    x2 = (int)(rem - (long long)x1 * n2);
  } else if (a == 1) {
    const int m = g.m[1];
    x2 = (int)(idx % n2);
    const long long q = idx / n2;
    const int e = (int)(q % (2 * m));
    x0 = (int)(q / (2 * m));
    x1 = e < m ? e : n1 - 2 * m + e;
  } else {
    const int m = g.m[2];
    const int e = (int)(idx % (2 * m));
    const long long r = idx / (2 * m);
    x2 = e < m ? e : n2 - 2 * m + e;
    x1 = (int)(r % n1);
    x0 = (int)(r / n1);
  }
}

__global__ void __launch_bounds__(256)
shell_kernel(const Geom g, const ShellArgs a, long long total) {
  unsigned any = 0;
#pragma unroll
  for (int n = 0; n < MAXA; ++n)
    if (n < a.n) any |= a.m[n];
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    int x0, x1, x2;
    if (a.slab >= 0)
      slab_coords(g, a.slab, idx, x0, x1, x2);
    else
      shell_coords(g, idx, x0, x1, x2);
    Img im;
    make_img(g, x0, x1, x2, im);
    if (!(im.valid & any)) continue;  // none of the images the next pass reads
    const int cell = cell_of(g, x0, x1, x2);
    float v[MAXA];
#pragma unroll
    for (int n = 0; n < MAXA; ++n)
      if (n < a.n && (im.valid & a.m[n])) v[n] = a.p[n][cell];
#pragma unroll
    for (int n = 0; n < MAXA; ++n) {
      if (n < a.n) {
        float *p = a.p[n];
        const int f = a.f[n];
        const unsigned valid = im.valid & a.m[n];
#pragma unroll
        for (int m = 0; m < 7; ++m)
          if ((valid >> m) & 1u) p[cell + im.off[m]] = ((im.neg[m] >> f) & 1u) ? -v[n] : v[n];
      }
    }
  }
}

}  // namespace s32s

long long s32_shell_cells(const Geom &g) {
  const long long n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
  const long long m0 = g.m[0], m1 = g.m[1], m2 = g.m[2];
  return 2 * m0 * n1 * n2 + (n0 - 2 * m0) * 2 * m1 * n2 + (n0 - 2 * m0) * (n1 - 2 * m1) * 2 * m2;
}

long long s32_shell_count(const Geom &g, int slab) {
  if (slab < 0) return s32_shell_cells(g);
  long long c = 2LL * g.m[slab];
  for (int a = 0; a < 3; ++a)
    if (a != slab) c *= g.n[a];
  return c;
}

void launch_s32_shell(const Geom &g, const ShellArgs &a, int grid, cudaStream_t st) {
  s32s::shell_kernel<<<grid, 256, 0, st>>>(g, a, s32_shell_count(g, a.slab));
}

}  // namespace miso_b200
