// C ABI of libmiso_b200.so (declared in include/miso_b200.h): handle
// lifetime, device buffers, step sequencing, CUDA-graph capture, monitors.
//
// Step sequence (Integrator::update, mhd_integrator_host.hpp:344-350):
//   divb parameters -> 4 RK stages (258-277), each followed by a ghost fill
//   -> characteristic speed -> AV sweeps x, y, z (280-300), each followed by a
//   ghost fill.
// The reference copies whole field sets between stages (Fields::copy_from,
// mhd_fields.hpp:161-172); here three field sets rotate instead, so a step
// makes no device-to-device copies.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/miso_b200.h"
#include "common.cuh"
#include "kernels.h"
#include "kernels_s32.h"
#include "s32_tiled.h"
#include "s32_flat.h"
#include "tma.cuh"
#include "view.h"

using namespace miso_b200;

namespace {

std::string g_create_error;
std::mutex g_create_mu;

constexpr size_t ALIGN = 256;

size_t round_up(size_t x) { return (x + ALIGN - 1) / ALIGN * ALIGN; }

// FP64 monitors: per-block partial sums of 8 quantities (interior cells).
// The conserved state and |div B| (4th-order central differences) of cell c,
// folded into the accumulators.  Neighbours across a face come from the
// ghost cells, which are current when the kernel runs (miso_b200_monitors
// brings the split form's lo images up to date first).
// DIVB_ONLY: |div B| alone (the sums come from the z sweep, monitor fusion).
template <bool SPLIT, bool DIVB_ONLY = false>
__device__ __forceinline__ void monitor_cell(const Geom &g, const FieldPtrs<const double> &q,
                                             const FieldPtrs<const float> &hi,
                                             const FieldPtrs<const float> &lo, long long c,
                                             double acc[8]) {
  double u[NF];
  if (DIVB_ONLY) {
  } else if (SPLIT) {
    for (int f = 0; f < NF; ++f) u[f] = (double)hi.f[f][c] + (double)lo.f[f][c];
  } else {
    const double ro = q.f[RO][c], vx = q.f[VX][c], vy = q.f[VY][c], vz = q.f[VZ][c];
    const double bx = q.f[BX][c], by = q.f[BY][c], bz = q.f[BZ][c];
    u[RO] = ro;
    u[MX] = ro * vx;
    u[MY] = ro * vy;
    u[MZ] = ro * vz;
    u[BX] = bx;
    u[BY] = by;
    u[BZ] = bz;
    u[ET] = ro * q.f[EI][c] + 0.5 * ro * (vx * vx + vy * vy + vz * vz) +
            PII8 * (bx * bx + by * by + bz * bz);
    u[PH] = q.f[PH][c];
  }
  double divb = 0.0;
  for (int d = 0; d < 3; ++d) {
    if (!g.s[d]) continue;
    const long long s = g.st[d];
    double p2, p1, m1, m2;
    if (SPLIT) {
      const float *h = hi.f[BX + d], *l = lo.f[BX + d];
      p2 = (double)h[c + 2 * s] + l[c + 2 * s];
      p1 = (double)h[c + s] + l[c + s];
      m1 = (double)h[c - s] + l[c - s];
      m2 = (double)h[c - 2 * s] + l[c - 2 * s];
    } else {
      const double *b = q.f[BX + d];
      p2 = b[c + 2 * s];
      p1 = b[c + s];
      m1 = b[c - s];
      m2 = b[c - 2 * s];
    }
    divb += (-p2 + 8.0 * p1 - 8.0 * m1 + m2) * INV12 * g.dsi[d];
  }
  acc[5] += fabs(divb);
  acc[6] = fmax(acc[6], fabs(divb));
  if (DIVB_ONLY) return;
  acc[0] += u[RO];
  acc[1] += u[MX];
  acc[2] += u[MY];
  acc[3] += u[MZ];
  acc[4] += u[ET];
  acc[7] += u[PH] * u[PH];
}

template <bool SPLIT, bool DIVB_ONLY = false>
__global__ void __launch_bounds__(256, 4)
monitor_kernel(Geom g, FieldPtrs<const double> q, FieldPtrs<const float> hi,
               FieldPtrs<const float> lo, double *__restrict__ partial) {
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const long long nint = (long long)g.n[0] * g.n[1] * g.n[2];
  const long long stride = (long long)gridDim.x * blockDim.x;
  long long lin = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (lin < nint) {
    // decode the interior index once, then step it by the grid stride with
    // carries (no 64-bit division per cell)
    const int n1 = g.n[1], n2 = g.n[2];
    int k = (int)(lin % n2);
    const long long r1 = lin / n2;
    int j = (int)(r1 % n1);
    int i = (int)(r1 / n1);
    const int dk = (int)(stride % n2);
    const long long s1 = stride / n2;
    const int dj = (int)(s1 % n1);
    const int di = (int)(s1 / n1);
    for (; lin < nint; lin += stride) {
      monitor_cell<SPLIT, DIVB_ONLY>(g, q, hi, lo,
                          (i + g.m[0]) * g.st[0] + (j + g.m[1]) * g.st[1] + k + g.m[2], acc);
      k += dk;
      int carry = k >= n2;
      if (carry) k -= n2;
      j += dj + carry;
      carry = j >= n1;
      if (carry) j -= n1;
      i += di + carry;
    }
  }
  __shared__ double red[8][256];
  for (int q8 = 0; q8 < 8; ++q8) red[q8][threadIdx.x] = acc[q8];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      for (int q8 = 0; q8 < 8; ++q8) {
        if (q8 == 6)
          red[q8][threadIdx.x] = fmax(red[q8][threadIdx.x], red[q8][threadIdx.x + w]);
        else
          red[q8][threadIdx.x] += red[q8][threadIdx.x + w];
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int q8 = 0; q8 < 8; ++q8) partial[blockIdx.x * 8 + q8] = red[q8][0];
}

// |div B| of the split state (the monitors with their sums folded into the
// z sweep), the monitor kernel's difference in FP64 from hi + lo, by a march
// along i.  A work item is a tile of DBM_TJ x DBM_TK (j, k) cells over a run
// of DBM_L planes; a thread owns DBM_NP pairs of neighbouring k cells, 64
// cells apart (one float2 of hi and one of lo per array and pair, tiled
// grids having k_total a multiple of 4).  bx of the planes i-2 .. i+2 stays
// in a register ring, so each bx word is read and widened to FP64 once per
// run (plus the four planes before it); by and bz of plane i go to shared
// memory as FP64, halo rows and columns included, and the y and z
// neighbours are read from there: about 7 widenings per cell instead of the
// 22 of a kernel that widens every neighbour it loads.  The next plane's
// words are loaded into registers before the plane's barrier, and the
// shared planes alternate between two buffers, so one barrier per plane
// suffices; two pairs per thread halve the barriers per cell.  The ghost
// layers of bx, by and bz (hi and lo) must be current.  Writes slots 5 and 6
// of the monitor kernel's per-block layout; the grid is at most 2 CTAs per
// SM, all resident, each taking every gridDim-th item.
constexpr int DBM_NP = 2, DBM_TJ = 8, DBM_TK = 64 * DBM_NP, DBM_L = 64;

struct Raw2 {
  float2 h, l;
};
__device__ __forceinline__ Raw2 ld_raw2(const float *h, const float *l, long long c) {
  return Raw2{__ldg(reinterpret_cast<const float2 *>(h + c)),
              __ldg(reinterpret_cast<const float2 *>(l + c))};
}
__device__ __forceinline__ double2 widen2(const Raw2 &r) {
  return make_double2((double)r.h.x + (double)r.l.x, (double)r.h.y + (double)r.l.y);
}

__global__ void __launch_bounds__(256, 2)
divb_march_kernel(Geom g, FieldPtrs<const float> hi, FieldPtrs<const float> lo,
                  double *__restrict__ partial) {
  __shared__ __align__(16) double sby[2][DBM_TJ + 4][DBM_TK];
  __shared__ __align__(16) double sbz[2][DBM_TJ][DBM_TK + 4];
  const int lane = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int n0 = g.n[0], n1 = g.n[1], n2 = g.n[2];
  const int njt = (n1 + DBM_TJ - 1) / DBM_TJ, nkt = (n2 + DBM_TK - 1) / DBM_TK;
  const int items = (n0 + DBM_L - 1) / DBM_L * njt * nkt;
  const float *bxh = hi.f[BX], *bxl = lo.f[BX], *byh = hi.f[BY], *byl = lo.f[BY];
  const float *bzh = hi.f[BZ], *bzl = lo.f[BZ];
  // halo duty: warps 0-3 load the by rows j0-2, j0-1, j0+8, j0+9; lanes
  // 0-15 of warp 4 the bz pairs at k0-2 and k0+DBM_TK of the tile's 8 rows
  const int hy_row = ty < 2 ? ty - 2 : ty + DBM_TJ - 2;  // tile-relative j of a by halo row
  const int hz_row = lane >> 1, hz_side = lane & 1;
  double sum = 0.0, mx = 0.0;
  int par = 0;  // shared buffer of the current plane; flips once per plane
  for (int it = blockIdx.x; it < items; it += gridDim.x) {
    int r = it;
    const int kt = r % nkt;
    r /= nkt;
    const int jt = r % njt;
    const int i0 = r / njt * DBM_L;
    const int i1 = min(i0 + DBM_L, n0);
    const int j0 = jt * DBM_TJ, k0 = kt * DBM_TK;
    const int j = j0 + ty;
    const int jh = j0 + hy_row, jz = j0 + hz_row, kh = hz_side ? k0 + DBM_TK : k0 - 2;
    const bool hz = ty == 4 && lane < 16 && jz < n1 && kh <= n2;
    const long long chz = (long long)(jz + g.m[1]) * g.st[1] + (kh + g.m[2]);
    bool own[DBM_NP], yv[DBM_NP], hy[DBM_NP];
    long long cj[DBM_NP], chy[DBM_NP];
#pragma unroll
    for (int h = 0; h < DBM_NP; ++h) {
      const int k = k0 + 64 * h + 2 * lane;  // interior k of this pair
      own[h] = j < n1 && k < n2;             // n2 is a multiple of 4: k + 1 < n2 too
      yv[h] = j <= n1 + 1 && k < n2;         // by pair that an owned cell reads
      hy[h] = ty < 4 && jh <= n1 + 1 && k < n2;
      cj[h] = (long long)(j + g.m[1]) * g.st[1] + (k + g.m[2]);
      chy[h] = (long long)(jh + g.m[1]) * g.st[1] + (k + g.m[2]);
    }
    // bz pair that an owned cell reads: k <= n2
    bool zv[DBM_NP];
#pragma unroll
    for (int h = 0; h < DBM_NP; ++h) zv[h] = j < n1 && k0 + 64 * h + 2 * lane <= n2;
    // bx of planes i-2, i-1, i (not in the stencil), i+1 per pair
    double2 x0[DBM_NP], x1[DBM_NP], x2[DBM_NP], x3[DBM_NP];
    Raw2 px[DBM_NP], py[DBM_NP], pz[DBM_NP], ph[DBM_NP], pq{};  // plane i's words
    {
      const long long ci = (long long)(i0 + g.m[0]) * g.st[0];
#pragma unroll
      for (int h = 0; h < DBM_NP; ++h) {
        x0[h] = x1[h] = x2[h] = x3[h] = make_double2(0.0, 0.0);
        px[h] = py[h] = pz[h] = ph[h] = Raw2{};
        if (own[h]) {
          const long long c = ci + cj[h];
          x0[h] = widen2(ld_raw2(bxh, bxl, c - 2 * g.st[0]));
          x1[h] = widen2(ld_raw2(bxh, bxl, c - g.st[0]));
          x2[h] = widen2(ld_raw2(bxh, bxl, c));
          x3[h] = widen2(ld_raw2(bxh, bxl, c + g.st[0]));
          px[h] = ld_raw2(bxh, bxl, c + 2 * g.st[0]);
        }
        if (yv[h]) py[h] = ld_raw2(byh, byl, ci + cj[h]);
        if (zv[h]) pz[h] = ld_raw2(bzh, bzl, ci + cj[h]);
        if (hy[h]) ph[h] = ld_raw2(byh, byl, ci + chy[h]);
      }
      if (hz) pq = ld_raw2(bzh, bzl, ci + chz);
    }
    for (int i = i0; i < i1; ++i, par ^= 1) {
      double2 x4[DBM_NP];
#pragma unroll
      for (int h = 0; h < DBM_NP; ++h) {
        const int c = 64 * h + 2 * lane;  // tile-relative k of the pair
        if (yv[h]) *reinterpret_cast<double2 *>(&sby[par][ty + 2][c]) = widen2(py[h]);
        if (zv[h]) *reinterpret_cast<double2 *>(&sbz[par][ty][c + 2]) = widen2(pz[h]);
        if (hy[h]) *reinterpret_cast<double2 *>(&sby[par][hy_row + 2][c]) = widen2(ph[h]);
        x4[h] = own[h] ? widen2(px[h]) : make_double2(0.0, 0.0);
      }
      if (hz)
        *reinterpret_cast<double2 *>(&sbz[par][hz_row][hz_side ? DBM_TK + 2 : 0]) = widen2(pq);
      if (i + 1 < i1) {  // the next plane's words, in flight across the barrier
        const long long ci = (long long)(i + 1 + g.m[0]) * g.st[0];
#pragma unroll
        for (int h = 0; h < DBM_NP; ++h) {
          if (own[h]) px[h] = ld_raw2(bxh, bxl, ci + 2 * g.st[0] + cj[h]);
          if (yv[h]) py[h] = ld_raw2(byh, byl, ci + cj[h]);
          if (zv[h]) pz[h] = ld_raw2(bzh, bzl, ci + cj[h]);
          if (hy[h]) ph[h] = ld_raw2(byh, byl, ci + chy[h]);
        }
        if (hz) pq = ld_raw2(bzh, bzl, ci + chz);
      }
      __syncthreads();
#pragma unroll
      for (int h = 0; h < DBM_NP; ++h) {
        if (own[h]) {
          const int c = 64 * h + 2 * lane;
          const double2 ym2 = *reinterpret_cast<const double2 *>(&sby[par][ty][c]);
          const double2 ym1 = *reinterpret_cast<const double2 *>(&sby[par][ty + 1][c]);
          const double2 yp1 = *reinterpret_cast<const double2 *>(&sby[par][ty + 3][c]);
          const double2 yp2 = *reinterpret_cast<const double2 *>(&sby[par][ty + 4][c]);
          // bz of k-2 .. k+3
          const double2 za = *reinterpret_cast<const double2 *>(&sbz[par][ty][c]);
          const double2 zb = *reinterpret_cast<const double2 *>(&sbz[par][ty][c + 2]);
          const double2 zc = *reinterpret_cast<const double2 *>(&sbz[par][ty][c + 4]);
          double divb = 0.0;
          divb += (-x4[h].x + 8.0 * x3[h].x - 8.0 * x1[h].x + x0[h].x) * INV12 * g.dsi[0];
          divb += (-yp2.x + 8.0 * yp1.x - 8.0 * ym1.x + ym2.x) * INV12 * g.dsi[1];
          divb += (-zc.x + 8.0 * zb.y - 8.0 * za.y + za.x) * INV12 * g.dsi[2];
          sum += fabs(divb);
          mx = fmax(mx, fabs(divb));
          divb = 0.0;
          divb += (-x4[h].y + 8.0 * x3[h].y - 8.0 * x1[h].y + x0[h].y) * INV12 * g.dsi[0];
          divb += (-yp2.y + 8.0 * yp1.y - 8.0 * ym1.y + ym2.y) * INV12 * g.dsi[1];
          divb += (-zc.y + 8.0 * zc.x - 8.0 * zb.x + za.y) * INV12 * g.dsi[2];
          sum += fabs(divb);
          mx = fmax(mx, fabs(divb));
        }
        x0[h] = x1[h];
        x1[h] = x2[h];
        x2[h] = x3[h];
        x3[h] = x4[h];
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sum += __shfl_xor_sync(0xffffffffu, sum, o);
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  __shared__ double red[8][2];
  if (lane == 0) {
    red[ty][0] = sum;
    red[ty][1] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0, m = 0.0;
    for (int w2 = 0; w2 < (int)(blockDim.x >> 5); ++w2) {
      s += red[w2][0];
      m = fmax(m, red[w2][1]);
    }
    partial[blockIdx.x * 8 + 5] = s;
    partial[blockIdx.x * 8 + 6] = m;
  }
}

// The time loop of ModelBase::run kept on the device
// (miso_b200_run_until): after every step, time += dt (Time::update,
// time.hpp), and the loop goes on while time < t_end and fewer than
// max_steps steps were taken (mhd_model_base.hpp:108-111).
struct RunState {
  double time, t_end;
  int steps, max_steps;
};

__global__ void advance_kernel(RunState *rs, const StepScalars *sc) {
  rs->time += sc->dt;
  rs->steps += 1;
}

// the same inside the loop's graph: the conditions of the WHILE node and
// (a body of two steps) of the IF node around the second step
__global__ void advance_cond_kernel(RunState *rs, const StepScalars *sc,
                                    cudaGraphConditionalHandle h_while,
                                    cudaGraphConditionalHandle h_if, int set_if) {
  rs->time += sc->dt;
  rs->steps += 1;
  const unsigned go = rs->time < rs->t_end && rs->steps < rs->max_steps ? 1u : 0u;
  cudaGraphSetConditional(h_while, go);
  if (set_if) cudaGraphSetConditional(h_if, go);
}

__global__ void set_scalars_kernel(StepScalars *sc, StepScalars v) {
  const unsigned int err = sc->err;
  *sc = v;
  sc->err = err;
}

}  // namespace

struct miso_b200_handle {
  Geom g{};
  miso_b200_params p{};
  int device = 0;
  int sms = 148;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;

  void *block = nullptr;  // one allocation holds every device buffer
  size_t bytes = 0;

  // FP64 form: three rotating field sets + characteristic speed
  double *q64[3][NF] = {};
  double *cc64 = nullptr;
  // FP32-split form: hi/lo state (two sets, swapped by the AV sweeps), two
  // stage buffers, characteristic speed, FP64 staging for upload/download
  float *hi[2][NF] = {}, *lo[2][NF] = {};
  float *stg[2][NF] = {};
  float *cc32 = nullptr;
  double *io64[NF] = {};
  int cur = 0;  // which hi/lo set holds the state

  float *partial = nullptr;
  int nparts = 0;         // CFL partial minima used by the FP64 / untiled passes
  int nparts_alloc = 0;   // capacity of `partial`

  // tiled FP32-split path (3-D grids); tiled_ok: the grid can take it (the
  // magnetosphere boundary, which reads every ghost between passes, runs
  // the per-cell kernels instead)
  bool tiled = false, tiled_ok = false;
  // built-in source term (miso_b200_set_source) and the cell centres it
  // reads, one array per axis (ghosts included)
  Source src{};
  Magneto mag{};               // the magnetosphere demo's boundary (FP64 form)
  double *blend_block = nullptr;  // its reference state (9 arrays), once set
  // a boundary callback (miso_b200_set_boundary_callback, FP64 form): called
  // after every pass in place of the mirror faces, which are then marked
  // shared (ext) so the fill leaves them to it; on_host: the set is staged
  // through pinned host memory around the call
  // a source functor of the caller's (FP64): before every RK stage it fills
  // src_dev (4 arrays) from the stage's argument state
  miso_b200_source_fn src_cb = nullptr;
  void *src_user = nullptr;
  bool src_host = false;
  double *src_dev = nullptr, *src_stage = nullptr;  // device terms; host staging (q then s)
  double *src_arg = nullptr;  // split form: the stage's argument state as FP64 primitives
  miso_b200_boundary_fn bc_cb = nullptr;
  void *bc_user = nullptr;
  bool bc_host = false;
  double *bc_stage = nullptr;
  double *axc[3] = {};
  // halo exchange with neighbouring shards (miso_b200_set_halo along i,
  // miso_b200_set_halo3 along any axis: callback with the axis); a j or k
  // face travels through face_buf, four regions of face_region bytes (send
  // lo, send hi, receive lo, receive hi)
  miso_b200_halo_ops halo_ops{};
  miso_b200_halo3_ops halo3{};
  bool halo_on = false, halo_axes = false;
  char *face_buf = nullptr;
  size_t face_region = 0;
  // overlap of the exchange with the next pass (miso_b200_set_halo_overlap):
  // the callback runs on `comm` after event ev_pass; the next pass finishes
  // the planes that need no ghost first and waits for ev_xchg before the
  // two boundary plane groups
  cudaStream_t comm = nullptr;
  cudaEvent_t ev_pass = nullptr, ev_xchg = nullptr;
  bool xchg_pending = false;
  alignas(64) unsigned char tm_hi[2][128];   // RK plane-tile maps of hi[set] (4-D: k, j, i, field)
  alignas(64) unsigned char tm_stg[2][128];  // RK plane-tile maps of stg[set]
  alignas(64) unsigned char tm_avh[2][128];  // AV line maps of hi[set]
  alignas(64) unsigned char tm_avl[2][128];  // AV line maps of lo[set]
  alignas(64) unsigned char tm_avc[128];     // AV line map of the characteristic speed
  alignas(64) unsigned char tm_avd[128];     // AV line map of stg[1] (deferred last-stage D)
  alignas(64) unsigned char tm_zwh[2][128];  // z line sweep: 8-wide wrap maps of hi[set]
  alignas(64) unsigned char tm_zwc[128];     // and of the characteristic speed
  alignas(64) unsigned char tm_zwl[2][128];  // fused y and z sweeps: wrap maps of lo[set]
  long long pitch = 0;                       // elements between consecutive field arrays
  int rk_L = 64, rk_tiles_j = 0, rk_tiles_k = 0, rk_items = 0, rk_grid = 0;
  int av_L = 128, av_grid = 0, z_grid = 0;
  int avp_grid = 0;  // warp-march x / y sweep: 2 resident CTAs of 8 warps per SM
  int zl_grid = 0;   // z line sweep: resident CTAs per SM x SMs
  int yz_grid = 0;   // fused y and z sweeps: resident CTAs per SM x SMs
  int shell_grid = 0;
  // The flat kernels run exactly one resident wave (grid = resident blocks)
  // and stride over tiles in order, so the CTAs in flight always cover one
  // contiguous band of planes and stencil neighbours are reused from L2.
  int flat_grid = 0;
  int z_parts = 0;  // CFL partial minima written by the last z sweep
  bool partials_valid = false;  // `partial` holds CFL minima of the current state
  bool lo_shell_stale = false;  // the lo ghost images lag the interior (filled on download)
  bool lo_b_fresh = false;      // while stale: those of bx, by and bz are current
  // kernel variant per class on the 3-D split path: 0 = tiled (TMA plane
  // tiles / streaming lines), 1 = flat (one thread per cell); 2: RK =
  // pipelined TMA planes with packed FP32x2 differences (default), x / y
  // sweeps = one warp per line segment marching along the sweep axis; 3:
  // RK = variant 2 with the last update deferred into the x sweep (default),
  // y sweep = the y and z sweeps fused into one pass (the z variant unused)
  int rk_var = 3;
  int av_var[3] = {0, 3, 0};  // the y and z sweeps fused by default
  // (a shared k face needs the y-swept state exchanged before the z sweep)
  bool fused_yz() const { return av_var[1] == 3 && !g.ext[2][0] && !g.ext[2][1]; }
  // hi / lo set swaps of one step: one per viscosity pass
  int sweep_passes() const {
    return tiled ? (fused_yz() ? 2 : 3) : g.s[0] + g.s[1] + g.s[2];
  }
  double *mon_partial = nullptr;
  int mon_blocks = 0;
  // monitors folded into the step (miso_b200_set_monitor_fusion, 3-D split
  // path): the z sweep leaves per-block sums of the new state in mon_z and
  // monitors() adds only the div B kernel
  bool mon_fuse = false;
  bool mon_valid = false;  // mon_z holds the sums of the current state
  double *mon_z = nullptr;

  StepScalars *sc = nullptr;

  double min_dxyz = 0.0, cfl_dx = 0.0;
  long long launches = 0;
  // bound (clock cycles) of the consumer waits for each plane's TMA copy in
  // the Runge-Kutta stage and x / y sweep kernels (miso_b200_set_wait_limit)
  long long wait_limit = s32t::WAIT_CYCLES;
  // armed by miso_b200_arm_timeout_test: the next pipelined Runge-Kutta
  // stage launched outside a graph capture stalls on a barrier phase that
  // nothing completes, with this bound (0: not armed)
  long long stall_cycles = 0;

  void drop_loop() {
    if (loop_exec) cudaGraphExecDestroy(loop_exec);
    if (loop_graph) cudaGraphDestroy(loop_graph);
    loop_exec = nullptr;
    loop_graph = nullptr;
    loop_cur = -1;
  }
  // the device-held time loop (miso_b200_run_until): one graph with a WHILE
  // node around one step (or two, the second under an IF node, where a step
  // swaps the hi / lo sets)
  RunState *rs = nullptr;
  cudaGraph_t loop_graph = nullptr;
  cudaGraphExec_t loop_exec = nullptr;
  int loop_cur = -1, loop_steps = 0;
  long long loop_kernels = 0;  // kernels per step

  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  int graph_steps = 0;          // steps captured in the graph (1 or 2)
  int graph_cur = 0;            // hi/lo set the captured graph starts from
  long long graph_kernels = 0;  // kernels per graph launch

  // Optional per-kernel CUDA-event timing (never active inside a graph
  // capture): each timed launch is bracketed by two events on the stream.
  struct Pending {
    const char *name;
    double bytes;
    cudaEvent_t a, b;
  };
  struct Acc {
    long long n = 0;
    double ms = 0.0, bytes = 0.0;
  };
  bool timing = false, capturing = false;
  std::vector<Pending> pend;
  std::vector<cudaEvent_t> pool;
  std::map<std::string, Acc> acc;

  cudaEvent_t ev() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
  int tb() {
    if (!timing || capturing) return -1;
    Pending pd{nullptr, 0.0, ev(), ev()};
    cudaEventRecord(pd.a, stream);
    pend.push_back(pd);
    return (int)pend.size() - 1;
  }
  void te(int slot, const char *name, double bytes) {
    ++launches;
    if (slot < 0) return;
    pend[slot].name = name;
    pend[slot].bytes = bytes;
    cudaEventRecord(pend[slot].b, stream);
  }
  void harvest() {
    for (auto &pd : pend) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, pd.a, pd.b);
      Acc &x = acc[pd.name ? pd.name : "?"];
      x.n++;
      x.ms += ms;
      x.bytes += pd.bytes;
      pool.push_back(pd.a);
      pool.push_back(pd.b);
    }
    pend.clear();
  }
  double interior() const { return (double)g.n[0] * g.n[1] * g.n[2]; }
  double ghost_cells() const { return (double)g.cells - interior(); }

  int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    err = buf;
    return code;
  }
  int cuda(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return MISO_B200_OK;
    cudaGetLastError();  // a non-sticky error must not surface at a later launch check
    return fail(MISO_B200_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  }
  int check_launch(const char *what) { return cuda(cudaGetLastError(), what); }

  bool split() const { return p.precision == MISO_B200_FP32_SPLIT; }

  FieldPtrs<double> f64(int set) {
    FieldPtrs<double> r;
    for (int f = 0; f < NF; ++f) r.f[f] = q64[set][f];
    return r;
  }
  FieldPtrs<const double> c64(int set) {
    FieldPtrs<const double> r;
    for (int f = 0; f < NF; ++f) r.f[f] = q64[set][f];
    return r;
  }
  template <typename T>
  static FieldPtrs<const T> cst(const FieldPtrs<T> &a) {
    FieldPtrs<const T> r;
    for (int f = 0; f < NF; ++f) r.f[f] = a.f[f];
    return r;
  }
  FieldPtrs<float> H(int s) {
    FieldPtrs<float> r;
    for (int f = 0; f < NF; ++f) r.f[f] = hi[s][f];
    return r;
  }
  FieldPtrs<float> L(int s) {
    FieldPtrs<float> r;
    for (int f = 0; f < NF; ++f) r.f[f] = lo[s][f];
    return r;
  }
  FieldPtrs<float> S(int s) {
    FieldPtrs<float> r;
    for (int f = 0; f < NF; ++f) r.f[f] = stg[s][f];
    return r;
  }
  FSet fs(float *const (&arr)[NF]) const {
    FSet r;
    for (int f = 0; f < NF; ++f) r.f[f] = arr[f];
    return r;
  }
  CFSet cfs(float *const (&arr)[NF]) const {
    CFSet r;
    for (int f = 0; f < NF; ++f) r.f[f] = arr[f];
    return r;
  }

  FieldPtrs<double> IO() {
    FieldPtrs<double> r;
    for (int f = 0; f < NF; ++f) r.f[f] = io64[f];
    return r;
  }

  // ghost fill of one field set (the split form fills hi and lo together)
  int fill64(int set) {
    const int t = tb();
    launch_fill_ghosts<double>(g, f64(set), NF, sms, stream);
    te(t, "fill_ghosts", ghost_cells() * NF * 16.0);
    launches += g.s[0] + g.s[1] + g.s[2] - 1;
    return check_launch("fill_ghosts");
  }
  // The tiled 3-D FP32-split path: tensor maps of the state, stage and
  // speed arrays (each set of 9 arrays at one pitch of `pb` bytes), work
  // items and grids.  Leaves `tiled` false where a map cannot be made.
  void setup_tiled(size_t pb) {
    const Geom &g_ = g;
    bool ok = s32_configure() == 0 && s32_rk_pipe_configure() == 0;
    for (int s = 0; s < 2 && ok; ++s) {
      ok = s32_make_tmap(g_, hi[s][0], pb, 0, tm_hi[s]) == 0 &&
           s32_make_tmap(g_, stg[s][0], pb, 0, tm_stg[s]) == 0 &&
           s32_make_tmap(g_, hi[s][0], pb, 1, tm_avh[s]) == 0 &&
           s32_make_tmap(g_, lo[s][0], pb, 1, tm_avl[s]) == 0;
    }
    if (ok) ok = s32_make_tmap_cc(g_, cc32, tm_avc) == 0;
    if (ok) ok = s32_make_tmap(g_, stg[1][0], pb, 1, tm_avd) == 0;
    for (int s = 0; s < 2 && ok; ++s)
      ok = s32_make_tmap(g_, hi[s][0], pb, 2, tm_zwh[s]) == 0 &&
           s32_make_tmap(g_, lo[s][0], pb, 2, tm_zwl[s]) == 0;
    if (ok) ok = s32_make_tmap_cc(g_, cc32, tm_zwc, 8) == 0;
    if (ok) {
      tiled = tiled_ok = true;
      s32_rk_items(g_, rk_L, rk_tiles_j, rk_tiles_k, rk_items);
      const int per_sm = 2;
      rk_grid = rk_items < per_sm * sms ? rk_items : per_sm * sms;
      av_grid = 2 * sms;  // line sweeps: two CTAs per SM
      avp_grid = 2 * sms;
      zl_grid = s32_zline_per_sm() * sms;
      yz_grid = s32_yz_per_sm() * sms;
      {
        const long long want = (s32_shell_cells(g_) + 255) / 256;
        shell_grid = (int)(want < 8LL * sms ? want : 8LL * sms);
      }
      flat_grid = 3 * sms;  // 256 threads x 80 registers: 3 resident CTAs per SM
      if (const char *v = getenv("MISO_B200_RK"))
        rk_var = strcmp(v, "flat") == 0    ? 1
                    : strcmp(v, "tiled") == 0 ? 0
                    : strcmp(v, "pipe") == 0  ? 2
                                              : 3;
      if (const char *v = getenv("MISO_B200_AV"))
        for (int d = 0; d < 3 && v[d]; ++d)
          av_var[d] = v[d] == 'f' ? 1 : v[d] == 'p' ? 2 : (v[d] == 'u' && d == 1) ? 3 : 0;
    }
  }

  // Integrator::apply_boundary_condition of the FP64 state: the mirror /
  // periodic fill, then the magnetosphere boundary where it is on (the
  // caller exchanges shared faces after both, as the reference's halo
  // exchange follows its boundary functor)
  int bc64(int set) {
    if (bc_cb) return bc_callback(set);
    int rc = fill64(set);
    if (rc || !mag.on) return rc;
    const int t = tb();
    launch_magneto_bc(g, f64(set), mag, p.gm, sms, stream);
    // every cell: 9 fields read and written, and the reference state read once set
    te(t, "magnetosphere_bc", (double)g.cells * (mag.blend[0] ? 216.0 : 144.0));
    launches += 1;
    return check_launch("magnetosphere boundary");
  }
  // the caller's source functor on the argument state of the stage at hand
  // (set `set`): its four terms into src_dev, which the stage kernel reads
  int src_callback(int set) { return src_callback_on(q64[set]); }
  // the split form: the stage's argument state (hi and, for U^n, lo words;
  // a stage buffer alone otherwise) as FP64 primitives in the io set first
  int src_callback_split(const FieldPtrs<const float> &arg, const FieldPtrs<const float> &lo) {
    FieldPtrs<double> q;
    double *qp[NF];
    for (int f = 0; f < NF; ++f) q.f[f] = qp[f] = src_arg + (size_t)f * g.cells;
    launch_s32_from_split(g.cells, arg, lo, q, sms, stream);
    launches++;
    if (int rc = check_launch("from_split")) return rc;
    return src_callback_on(qp);
  }
  int src_callback_on(double *const *qdev) {
    // a host callback reads host copies; a device callback enqueues its work
    // on the handle's stream behind the stage that wrote its argument
    int rc = MISO_B200_OK;
    const size_t bytes = (size_t)g.cells * sizeof(double);
    const double *qp[NF];
    double *sp[4];
    for (int f = 0; f < NF; ++f) {
      if (src_host) {
        double *dst = src_stage + (size_t)f * g.cells;
        if ((rc = cuda(cudaMemcpyAsync(dst, qdev[f], bytes, cudaMemcpyDeviceToHost, stream),
                       "stage the fields for the source callback")))
          return rc;
        qp[f] = dst;
      } else {
        qp[f] = qdev[f];
      }
    }
    for (int t = 0; t < 4; ++t)
      sp[t] = src_host ? src_stage + (size_t)(NF + t) * g.cells : src_dev + (size_t)t * g.cells;
    if (src_host && (rc = cuda(cudaStreamSynchronize(stream), "synchronize"))) return rc;
    const int r = src_cb(src_user, qp, sp, (void *)stream);
    if (r) return fail(MISO_B200_ERR_CALLBACK, "source callback returned %d", r);
    if (src_host)
      for (int t = 0; t < 4; ++t)
        if ((rc = cuda(cudaMemcpyAsync(src_dev + (size_t)t * g.cells, sp[t], bytes,
                                       cudaMemcpyHostToDevice, stream),
                       "return the source terms")))
          return rc;
    return MISO_B200_OK;
  }
  // the caller's boundary functor on the set just written, then the
  // periodic faces (the reference's bc.apply followed by its halo exchange,
  // mhd_integrator_cuda.cuh:396-401)
  int bc_callback(int set) {
    int rc = cuda(cudaStreamSynchronize(stream), "synchronize before the boundary callback");
    if (rc) return rc;
    const size_t bytes = (size_t)g.cells * sizeof(double);
    double *ptrs[NF];
    for (int f = 0; f < NF; ++f) {
      ptrs[f] = bc_host ? bc_stage + (size_t)f * g.cells : q64[set][f];
      if (bc_host &&
          (rc = cuda(cudaMemcpyAsync(ptrs[f], q64[set][f], bytes, cudaMemcpyDeviceToHost, stream),
                     "stage the fields for the boundary callback")))
        return rc;
    }
    if (bc_host && (rc = cuda(cudaStreamSynchronize(stream), "synchronize"))) return rc;
    const int r = bc_cb(bc_user, ptrs, (void *)stream);
    if (r) return fail(MISO_B200_ERR_CALLBACK, "boundary callback returned %d", r);
    if (bc_host)
      for (int f = 0; f < NF; ++f)
        if ((rc = cuda(cudaMemcpyAsync(q64[set][f], ptrs[f], bytes, cudaMemcpyHostToDevice,
                                       stream),
                       "return the fields from the boundary callback")))
          return rc;
    return fill64(set);
  }
  int fill_split(int s) {
    const int t = tb();
    launch_fill_ghosts<float>(g, H(s), NF, sms, stream);
    launch_fill_ghosts<float>(g, L(s), NF, sms, stream);
    te(t, "fill_ghosts", ghost_cells() * NF * 16.0);
    launches += 2 * (g.s[0] + g.s[1] + g.s[2]) - 1;
    return check_launch("fill_ghosts");
  }
  int fill_stage(int s) {
    const int t = tb();
    launch_fill_ghosts<float>(g, S(s), NF, sms, stream);
    te(t, "fill_ghosts", ghost_cells() * NF * 8.0);
    launches += g.s[0] + g.s[1] + g.s[2] - 1;
    return check_launch("fill_ghosts");
  }

  // the magnetosphere boundary on the split state (hi / lo of set s) or on
  // a stage buffer (stg[s]), after its mirror fill
  int magneto32(int s, bool stage) {
    if (!mag.on) return MISO_B200_OK;
    const int t = tb();
    if (stage)
      launch_s32_magneto(g, S(s), S(s), false, mag, p.gm, sms, stream);
    else
      launch_s32_magneto(g, H(s), L(s), true, mag, p.gm, sms, stream);
    te(t, "magnetosphere_bc", (double)g.cells * (stage ? 72.0 : 144.0) +
                                  (mag.blend[0] ? (double)g.cells * 72.0 : 0.0));
    launches += 1;
    return check_launch("magnetosphere boundary");
  }

  int fill_state() {
    int rc = join_xchg();
    if (rc) return rc;
    rc = split() ? fill_split(cur) : bc64(0);
    if (!rc && split()) rc = magneto32(cur, false);
    if (rc) return rc;
    return split() ? halo_f(hi[cur], lo[cur]) : halo_d(q64[0]);
  }

  // Exchange of the ghost layers of `n` arrays (element size `elem`) with
  // the neighbouring shards along the axes of `axes` (bit a: axis a) that
  // have a shared face, through the caller's callback; a no-op for a single
  // grid.
  int halo_exchange(void *const *arr, int n, size_t elem, unsigned axes = 7u) {
    if (!halo_on) return MISO_B200_OK;
    for (int a = 0; a < 3; ++a) {
      if (!((axes >> a) & 1u) || !(g.ext[a][0] || g.ext[a][1])) continue;
      const int rc = a == 0 ? halo_planes(arr, n, elem) : halo_face(a, arr, n, elem);
      if (rc) return rc;
    }
    return MISO_B200_OK;
  }
  int halo_call(int axis, int n, size_t bytes, void **slo, void **shi, void **rlo, void **rhi,
                cudaStream_t xs) {
    const int r = halo_axes ? halo3.exchange(halo3.user, axis, n, bytes, g.ext[axis][0],
                                             g.ext[axis][1], slo, shi, rlo, rhi, (void *)xs)
                            : halo_ops.exchange(halo_ops.user, n, bytes, g.ext[axis][0],
                                                g.ext[axis][1], slo, shi, rlo, rhi, (void *)xs);
    if (r) return fail(MISO_B200_ERR_HALO, "halo exchange callback returned %d", r);
    return MISO_B200_OK;
  }
  // a j or k face: its interior layers gathered into face_buf, the
  // callback, the received layers scattered into the ghost layers
  int halo_face(int a, void *const *arr, int n, size_t elem) {
    FaceArgs f;
    f.n = n;
    f.axis = a;
    f.ext[0] = g.ext[a][0];
    f.ext[1] = g.ext[a][1];
    for (int x = 0; x < 3; ++x) {
      f.d[x] = x == a ? g.m[a] : g.t[x];
      f.st[x] = g.st[x];
    }
    f.face = f.d[0] * f.d[1] * f.d[2];
    const size_t bytes = (size_t)f.face * elem;
    if ((size_t)n * bytes > face_region)
      return fail(MISO_B200_ERR_STATE, "face buffers too small for %d arrays", n);
    void *slo[2 * NF + 1], *shi[2 * NF + 1], *rlo[2 * NF + 1], *rhi[2 * NF + 1];
    for (int x = 0; x < n; ++x) {
      f.arr[x] = arr[x];
      slo[x] = face_buf + (size_t)x * bytes;
      shi[x] = face_buf + face_region + (size_t)x * bytes;
      rlo[x] = face_buf + 2 * face_region + (size_t)x * bytes;
      rhi[x] = face_buf + 3 * face_region + (size_t)x * bytes;
    }
    // interior layers m .. 2m-1 and n .. n+m-1 out; ghost layers 0 .. m-1
    // and n+m .. n+2m-1 in
    f.pack = 1;
    f.start[0] = g.m[a];
    f.start[1] = g.n[a];
    f.buf[0] = face_buf;
    f.buf[1] = face_buf + face_region;
    launch_face_copy(f, elem, sms, stream);
    launches++;
    int rc = check_launch("face_pack");
    if (!rc) rc = halo_call(a, n, bytes, slo, shi, rlo, rhi, stream);
    if (rc) return rc;
    f.pack = 0;
    f.start[0] = 0;
    f.start[1] = g.n[a] + g.m[a];
    f.buf[0] = face_buf + 2 * face_region;
    f.buf[1] = face_buf + 3 * face_region;
    launch_face_copy(f, elem, sms, stream);
    launches++;
    return check_launch("face_unpack");
  }
  // an i face: `margin` whole planes per array, exchanged in place
  int halo_planes(void *const *arr, int n, size_t elem) {
    const long long plane = (long long)g.t[1] * g.t[2];
    const int m = g.m[0], ni = g.n[0];
    void *slo[2 * NF + 1], *shi[2 * NF + 1], *rlo[2 * NF + 1], *rhi[2 * NF + 1];
    for (int a = 0; a < n; ++a) {
      char *b = (char *)arr[a];
      slo[a] = b + (size_t)m * plane * elem;           // interior planes 0 .. m-1
      shi[a] = b + (size_t)ni * plane * elem;          // interior planes n-m .. n-1
      rlo[a] = b;                                       // low ghost planes
      rhi[a] = b + (size_t)(ni + m) * plane * elem;    // high ghost planes
    }
    cudaStream_t xs = stream;
    if (comm) {
      // behind everything the pass wrote, on the exchange's own stream
      int rc = join_xchg();
      if (!rc) rc = cuda(cudaEventRecord(ev_pass, stream), "record pass event");
      if (!rc) rc = cuda(cudaStreamWaitEvent(comm, ev_pass, 0), "order the exchange");
      if (rc) return rc;
      xs = comm;
    }
    if (int rc = halo_call(0, n, (size_t)m * plane * elem, slo, shi, rlo, rhi, xs)) return rc;
    if (comm) {
      int rc = cuda(cudaEventRecord(ev_xchg, comm), "record exchange event");
      if (rc) return rc;
      xchg_pending = true;
    }
    return MISO_B200_OK;
  }
  // the ghost planes of the last exchange are in place before what follows
  // on the handle's stream
  int join_xchg() {
    if (!xchg_pending) return MISO_B200_OK;
    xchg_pending = false;
    return cuda(cudaStreamWaitEvent(stream, ev_xchg, 0), "wait for the exchange");
  }
  // the pass runs its planes that need no ghost before the exchange lands
  bool split_pass() const { return comm && xchg_pending && g.n[0] > 4; }
  int halo_d(double *const *set) {
    void *arr[NF];
    for (int f = 0; f < NF; ++f) arr[f] = set[f];
    return halo_exchange(arr, NF, sizeof(double));
  }
  int halo_f(float *const *a, float *const *b = nullptr, float *c = nullptr,
             unsigned axes = 7u) {
    void *arr[2 * NF + 1];
    int n = 0;
    for (int f = 0; f < NF; ++f) arr[n++] = a[f];
    if (b)
      for (int f = 0; f < NF; ++f) arr[n++] = b[f];
    if (c) arr[n++] = c;
    return halo_exchange(arr, n, sizeof(float), axes);
  }

  // the pipelined kernels of a 3-D split grid, unless the magnetosphere
  // boundary or a caller's source needs the per-cell kernels
  void retile() {
    const bool t = tiled_ok && !mag.on;
    if (t != tiled) partials_valid = false;
    tiled = t;
  }
  // the lo ghost images catch up with the interior before the state leaves
  // the device
  int fresh_lo_shell() {
    if (!lo_shell_stale) return MISO_B200_OK;
    lo_shell_stale = false;
    return shell(lo[cur], SHELL_ALL);
  }
  // the same for bx, by and bz alone (the div B stencil of the monitors);
  // the other lo images stay stale until a download
  int fresh_lo_b() {
    if (!lo_shell_stale || lo_b_fresh) return MISO_B200_OK;
    lo_b_fresh = true;
    ShellArgs sa;
    sa.n = 0;
    for (int f = BX; f <= BZ; ++f) {
      sa.p[sa.n] = lo[cur][f];
      sa.f[sa.n] = f;
      sa.m[sa.n++] = SHELL_ALL;
    }
    sa.slab = -1;
    const long long cells = s32_shell_count(g, sa.slab);
    long long grid = (cells + 255) / 256;
    if (grid > 8LL * sms) grid = 8LL * sms;
    const int t = tb();
    launch_s32_shell(g, sa, (int)grid, stream);
    te(t, "ghost_shell", (double)cells * 8.0 * sa.n);
    return check_launch("ghost_shell");
  }

  // ghost images of the interior shell: the 9 arrays of `set` with image
  // mask `mset`, and (when given) cc with mask `mcc`
  int shell(float *const *set, unsigned mset, float *ccp = nullptr, unsigned mcc = 0) {
    ShellArgs sa;
    sa.n = 0;
    if (set)
      for (int f = 0; f < NF; ++f) {
        sa.p[sa.n] = set[f];
        sa.f[sa.n] = f;
        sa.m[sa.n++] = mset;
      }
    if (ccp) {
      sa.p[sa.n] = ccp;
      sa.f[sa.n] = NF;
      sa.m[sa.n++] = mcc;
    }
    unsigned any = 0;
    for (int n = 0; n < sa.n; ++n) any |= sa.m[n];
    sa.slab = any == SHELL_FACES_I ? 0 : any == SHELL_FACES_J ? 1 : any == SHELL_FACES_K ? 2 : -1;
    const long long cells = s32_shell_count(g, sa.slab);
    long long grid = (cells + 255) / 256;
    if (grid > 8LL * sms) grid = 8LL * sms;
    const int t = tb();
    launch_s32_shell(g, sa, (int)grid, stream);
    te(t, "ghost_shell", (double)cells * 8.0 * sa.n);
    return check_launch("ghost_shell");
  }

  // host-side step scalars exactly as Integrator::divb_parameters_set and
  // runge_kutta_4step form them (host libm exp, as the reference's host path)
  StepScalars host_scalars(double dt) const {
    StepScalars v{};
    v.dt = dt;
    v.dts[0] = dt / 4.0;
    v.dts[1] = dt / 3.0;
    v.dts[2] = dt / 2.0;
    v.dts[3] = dt;
    volatile double ch = 0.8 * p.cfl_number * min_dxyz / dt;
    v.ch2 = ch * ch;
    v.tau = 2.0 * dt;
    for (int s = 0; s < 4; ++s) v.ph_decay[s] = std::exp(-v.dts[s] / v.tau);
    return v;
  }

  int enqueue_cfl() {
    const int t = tb();
    if (split() && tiled) {
      if (!partials_valid) {
        launch_s32_cfl_partial(g, cst(H(cur)), partial, z_grid, sc, p.gm, cfl_dx, stream, mag);
        te(t, "cfl", interior() * 32.0);
        const int t2 = tb();
        launch_cfl_finalize(partial, z_grid, sc, p.cfl_number, min_dxyz, stream);
        te(t2, "cfl_finalize", 0.0);
      } else {
        launch_cfl_finalize(partial, z_parts, sc, p.cfl_number, min_dxyz, stream);
        te(t, "cfl_finalize", 0.0);
      }
      return check_launch("cfl");
    }
    if (split()) {
      launch_s32_cfl_partial(g, cst(H(cur)), partial, nparts, sc, p.gm, cfl_dx, stream, mag,
                             cst(L(cur)));
      launch_cfl_finalize(partial, nparts, sc, p.cfl_number, min_dxyz, stream);
      te(t, "cfl", interior() * 32.0);
    } else {
      launch_fp64_cfl(g, c64(0), partial, sc, p.gm, p.cfl_number, cfl_dx, min_dxyz, mag, sms,
                      stream);
      te(t, "cfl", interior() * 64.0);
    }
    launches += 1;
    return check_launch("cfl");
  }

  int enqueue_update() {
    int rc;
    if (!split()) {
      // RK: qq(0) -> A(1) -> B(2) -> A -> B
      const int seq_a[4] = {0, 1, 2, 1};
      const int seq_r[4] = {1, 2, 1, 2};
      for (int s = 0; s < 4; ++s) {
        if (src_cb && (rc = src_callback(seq_a[s]))) return rc;
        const int t = tb();
        launch_fp64_rhs_stage(g, c64(0), c64(seq_a[s]), f64(seq_r[s]), sc, s, p.gm, src, sms,
                              stream);
        te(t, "rk_stage", interior() * (s == 0 ? 144.0 : 216.0));
        if ((rc = check_launch("rhs_stage"))) return rc;
        if ((rc = bc64(seq_r[s]))) return rc;
        if ((rc = halo_d(q64[seq_r[s]]))) return rc;
      }
      // AV on B(2): x: B -> qq, y: qq -> A, z: A -> qq
      int t = tb();
      launch_fp64_char_velocity(g, c64(2), cc64, p.gm, p.cs_fac, p.vv_fac, p.ca_fac, sms,
                                stream);
      te(t, "char_velocity", (double)g.cells * 72.0);
      const int src[3] = {2, 0, 1}, dst[3] = {0, 1, 0};
      for (int d = 0; d < 3; ++d) {
        t = tb();
        launch_fp64_av_sweep(g, c64(src[d]), f64(dst[d]), cc64, sc, d, p.ep, p.fh, sms, stream);
        te(t, "av_sweep", interior() * 152.0);
        if ((rc = check_launch("av_sweep"))) return rc;
        if ((rc = bc64(dst[d]))) return rc;
        if ((rc = halo_d(q64[dst[d]]))) return rc;
      }
      return MISO_B200_OK;
    }
    if (tiled) return enqueue_update_tiled();
    // FP32 split: stage 0 reads hi, stages write stg[0], stg[1], stg[0];
    // stage 3 accumulates into hi/lo of the current set.
    const int c = cur;
    for (int s = 0; s < 4; ++s) {
      FieldPtrs<const float> prev = s == 0 ? cst(H(c)) : cst(S((s - 1) & 1));
      FieldPtrs<float> out = s < 3 ? S(s & 1) : S(0);
      if (src_cb && (rc = src_callback_split(prev, s == 0 ? cst(L(c)) : FieldPtrs<const float>{})))
        return rc;
      const int t = tb();
      launch_s32_rk_stage(g, prev, H(c), L(c), out, sc, s, p.gm, src, sms, stream);
      te(t, "rk_stage", interior() * (s == 0 ? 72.0 : s < 3 ? 108.0 : 180.0));
      if ((rc = check_launch("rk_stage"))) return rc;
      if (s < 3) {
        if ((rc = fill_stage(s & 1))) return rc;
        if ((rc = magneto32(s & 1, true))) return rc;
        if ((rc = halo_f(stg[s & 1]))) return rc;
      } else {
        if ((rc = fill_split(c))) return rc;
        if ((rc = magneto32(c, false))) return rc;
        if ((rc = halo_f(hi[c], lo[c]))) return rc;
      }
    }
    int t = tb();
    launch_s32_char_velocity(g, cst(H(c)), cc32, p.gm, p.cs_fac, p.vv_fac, p.ca_fac, sms, stream);
    te(t, "char_velocity", (double)g.cells * 40.0);
    for (int d = 0; d < 3; ++d) {
      if (!g.s[d]) continue;  // a degenerate sweep leaves the conserved state unchanged
      t = tb();
      launch_s32_av_sweep(g, cst(H(cur)), cst(L(cur)), H(cur ^ 1), L(cur ^ 1), cc32, sc, d, p.ep,
                          p.fh, sms, stream);
      te(t, "av_sweep", interior() * 148.0);
      if ((rc = check_launch("av_sweep"))) return rc;
      cur ^= 1;
      if ((rc = fill_split(cur))) return rc;
      if ((rc = magneto32(cur, false))) return rc;
      if ((rc = halo_f(hi[cur], lo[cur]))) return rc;
    }
    return MISO_B200_OK;
  }

  // Tiled FP32-split step: 4 RK stage launches and 3 viscosity sweeps; ghost
  // images, the characteristic speed and the next step's CFL minima are
  // written by those kernels themselves.
  // RK variant 3: the pipelined stages with the last stage's update deferred
  // into the x line sweep (rk_pipe_kernel<4> writes its right-hand side D to
  // stg[1]; av_line_kernel<0, true> forms U^{n+1} from hi, lo and D as it
  // streams them).  Needs the line x sweep and no flat sweep, which would
  // read the images of U^{n+1} and its speed.
  // persistent grid of a line sweep: two CTAs per SM, or one per work item
  // on a small grid
  int line_grid(int d, int r0 = 0, int r1 = -1) const {
    const int items = s32_av_line_items(g, d, av_L, r0, r1 < 0 ? g.n[d] : r1);
    return items < av_grid ? items : av_grid;
  }
  bool defer_last() const {
    // (a caller's source heats the new total energy, which the deferred
    // update, formed in the x sweep, does not add)
    return rk_var == 3 && av_var[0] == 0 && av_var[1] != 1 && av_var[2] != 1 && src.kind != 2;
  }

  int enqueue_update_tiled() {
    int rc;
    const int c = cur;
    const bool defer = defer_last();
    for (int st = 0; st < 4; ++st) {
      if (src_cb) {
        // the caller's source on the stage's argument state (U^n with the
        // lo images current, or the last stage's output)
        if (st == 0 && (rc = fresh_lo_shell())) return rc;
        if ((rc = src_callback_split(st == 0 ? cst(H(c)) : cst(S((st - 1) & 1)),
                                     st == 0 ? cst(L(c)) : FieldPtrs<const float>{})))
          return rc;
      }
      RkArgs a;
      a.g = g;
      a.u0 = cfs(hi[c]);
      a.hi = fs(hi[c]);
      a.lo = fs(lo[c]);
      a.out = fs(defer && st == 3 ? stg[1] : stg[st & 1]);
      a.cc = cc32;
      a.sc = sc;
      a.err = &sc->err;
      a.gm = (float)p.gm;
      a.gm1 = (float)(p.gm - 1.0);
      a.cs_fac = (float)p.cs_fac;
      a.vv_fac = (float)p.vv_fac;
      a.ca_fac = (float)p.ca_fac;
      a.L = rk_L;
      a.tiles_j = rk_tiles_j;
      a.tiles_k = rk_tiles_k;
      a.items = rk_items;
      a.src = src;
      a.src_ro = st == 0 ? hi[c][RO] : stg[(st - 1) & 1][RO];
      a.wait_limit = wait_limit;
      a.stall_limit = 0;
      if (stall_cycles > 0 && rk_var >= 2 && !capturing) {
        a.stall_limit = stall_cycles;  // one launch only
        stall_cycles = 0;
      }
      a.i0 = 0;
      a.i1 = g.n[0];
      const void *tm = st == 0 ? (const void *)tm_hi[c] : (const void *)tm_stg[(st - 1) & 1];
      const int t = tb();
      if (rk_var >= 2 && split_pass()) {
        // a shard with the exchange in flight: the planes [2, n-2) first,
        // then, with the ghost planes in place, the two boundary groups
        const int n0 = g.n[0];
        const int ranges[3][2] = {{2, n0 - 2}, {0, 2}, {n0 - 2, n0}};
        for (int r = 0; r < 3; ++r) {
          if (r == 1 && (rc = join_xchg())) return rc;
          a.i0 = ranges[r][0];
          a.i1 = ranges[r][1];
          a.items = s32_rk_items_range(g, rk_L, a.i0, a.i1);
          const int grid = a.items < 2 * sms ? a.items : 2 * sms;
          launch_s32_rk_pipe(tm, a, defer && st == 3 ? 4 : st, grid, stream);
          a.stall_limit = 0;
        }
      } else {
        if ((rc = join_xchg())) return rc;
        if (rk_var == 1)
          launch_s32_rk_flat(st == 0 ? cfs(hi[c]) : cfs(stg[(st - 1) & 1]), a, st, flat_grid,
                             stream);
        else if (rk_var >= 2)
          launch_s32_rk_pipe(tm, a, defer && st == 3 ? 4 : st, rk_grid, stream);
        else
          launch_s32_rk_tiled(tm, a, st, rk_grid, stream);
      }
      te(t, "rk_stage",
         interior() * (st == 0 || (defer && st == 3) ? 72.0 : st < 3 ? 108.0 : 184.0));
      if ((rc = check_launch("rk_stage"))) return rc;
      if (rk_var >= 2) {  // interior-only writer: fill the images read next
        if (st < 3) {
          // the next stage's star stencil reads face ghosts only
          if ((rc = shell(stg[st & 1], SHELL_FACES))) return rc;
        } else if (av_var[0] == 1 || av_var[1] == 1 || av_var[2] == 1) {
          // a flat sweep reads hi across the i faces and cc across its own
          // faces (the line, march and z sweeps read the imaged interior)
          if ((rc = shell(hi[c], SHELL_FACES_I, cc32, SHELL_FACES))) return rc;
        }
      }
      // a shard's ghosts of the stage output come from the neighbours; after
      // the last stage only the i ghosts the x sweep reads: of hi and cc, or
      // of D when the update is deferred (the U^n ghosts are current since
      // the last step's exchange)
      if ((rc = st < 3 ? halo_f(stg[st & 1])
                : defer ? halo_f(stg[1], nullptr, nullptr, 1u)
                        : halo_f(hi[c], nullptr, cc32, 1u)))
        return rc;
    }
    for (int d = 0; d < 3; ++d) {
      AvArgs a;
      a.g = g;
      a.hi = cfs(hi[cur]);
      a.lo = cfs(lo[cur]);
      a.hi2 = fs(hi[cur ^ 1]);
      a.lo2 = fs(lo[cur ^ 1]);
      a.cc = cc32;
      a.sc = sc;
      a.err = &sc->err;
      a.partial = d == 2 ? partial : nullptr;
      a.ep = (float)p.ep;
      a.fh = (float)p.fh;
      a.gm = (float)p.gm;
      a.gm1 = (float)(p.gm - 1.0);
      a.cfl_dx = (float)cfl_dx;
      a.L = av_L;
      a.cc_out = cc32;
      a.cs_fac = (float)p.cs_fac;
      a.vv_fac = (float)p.vv_fac;
      a.ca_fac = (float)p.ca_fac;
      a.wait_limit = wait_limit;
      a.mon = d == 2 && mon_fuse && av_var[2] == 0 ? mon_z : nullptr;
      a.r0 = 0;
      a.r1 = d < 2 ? g.n[d] : 0;
      if (d == 1 && fused_yz()) {
        // the y and z sweeps in one pass: CFL minima and monitor sums as
        // the z sweep leaves them
        if ((rc = join_xchg())) return rc;
        a.partial = partial;
        a.mon = mon_fuse ? mon_z : nullptr;
        const int t = tb();
        launch_s32_av_yz(tm_avh[cur], tm_avl[cur], tm_avc, tm_zwh[cur], tm_zwl[cur], tm_zwc, a,
                         yz_grid, stream);
        te(t, "av_yz", interior() * 148.0);
        if ((rc = check_launch("av_yz"))) return rc;
        if ((rc = shell(hi[cur ^ 1], SHELL_ALL))) return rc;
        lo_shell_stale = true;
        lo_b_fresh = false;
        cur ^= 1;
        break;
      }
      const int t = tb();
      if (d == 0 && av_var[0] == 0 && split_pass()) {
        // a shard with the exchange in flight: the x sweep finishes the
        // planes [2, n-2) first, the boundary groups after the exchange
        const int n0 = g.n[0];
        const int ranges[3][2] = {{2, n0 - 2}, {0, 2}, {n0 - 2, n0}};
        for (int r = 0; r < 3; ++r) {
          if (r == 1 && (rc = join_xchg())) return rc;
          a.r0 = ranges[r][0];
          a.r1 = ranges[r][1];
          launch_s32_av_line(tm_avh[cur], tm_avl[cur], defer ? tm_avd : tm_avc, a, 0, defer,
                             line_grid(0, a.r0, a.r1), stream);
        }
      } else if (((rc = join_xchg()))) {
        return rc;
      } else if (av_var[d] == 1)
        launch_s32_av_flat(a, d, flat_grid, stream);
      else if (av_var[d] == 2 && d < 2)
        launch_s32_av_march(a, d, avp_grid, stream);
      else if (d == 0 && defer)
        launch_s32_av_line(tm_avh[cur], tm_avl[cur], tm_avd, a, 0, true, line_grid(0), stream);
      else if (d < 2)
        launch_s32_av_line(tm_avh[cur], tm_avl[cur], tm_avc, a, d, false, line_grid(d), stream);
      else if (av_var[2] == 2)
        launch_s32_av_zline(tm_avh[cur], tm_avl[cur], tm_avc, tm_zwh[cur], tm_zwc, a, zl_grid,
                            stream);
      else
        launch_s32_av_z(a, z_grid, stream);
      te(t, d == 0 ? "av_x" : d == 1 ? "av_y" : "av_z",
         interior() * (d == 0 && defer ? 184.0 : 148.0));
      if ((rc = check_launch("av_sweep"))) return rc;
      // interior-only writers (line, march and z sweeps): the step's final
      // state gets every hi image; within the step only a flat sweep reads
      // ghosts (the others read the imaged interior across a face); lo
      // images are read by a download only (see lo_shell_stale)
      if (av_var[d] != 1) {
        if (d == 2 || av_var[d + 1] == 1) {
          const unsigned m = d == 0 ? SHELL_FACES_J : d == 1 ? SHELL_FACES_K : SHELL_ALL;
          if ((rc = shell(hi[cur ^ 1], m))) return rc;
        }
        lo_shell_stale = true;
        lo_b_fresh = false;
      } else {
        lo_shell_stale = false;
      }
      cur ^= 1;
      // a shard's j ghosts of the x-swept state and the speed (read by the y
      // sweep), its k ghosts of the y-swept state and the speed (z sweep)
      if (d < 2 && (rc = halo_f(hi[cur], lo[cur], cc32, d == 0 ? 2u : 4u))) return rc;
    }
    // a shard: the step's final state (hi and lo, so that a download needs
    // no exchange) takes its i ghosts from the neighbouring shards
    if (halo_on) {
      if ((rc = fresh_lo_shell())) return rc;
      if ((rc = halo_f(hi[cur], lo[cur]))) return rc;
    }
    z_parts = fused_yz()        ? yz_grid
              : av_var[2] == 1 ? flat_grid
              : av_var[2] == 2 ? zl_grid
                               : z_grid;
    partials_valid = true;
    mon_valid = mon_fuse && (av_var[2] == 0 || fused_yz());
    return MISO_B200_OK;
  }

  int read_err() {
    unsigned int e = 0;
    int rc = join_xchg();
    if (rc) return rc;
    rc = cuda(cudaMemcpyAsync(&e, &sc->err, sizeof e, cudaMemcpyDeviceToHost, stream),
              "read error flags");
    if (rc) return rc;
    if ((rc = cuda(cudaStreamSynchronize(stream), "synchronize"))) return rc;
    if (e & (ERRBIT_NONFINITE | ERRBIT_TIMEOUT)) {
      unsigned int zero = 0;
      cudaMemcpy(&sc->err, &zero, sizeof zero, cudaMemcpyHostToDevice);
      if (e & ERRBIT_TIMEOUT)
        return fail(MISO_B200_ERR_TIMEOUT,
                    "a device-side wait for a TMA copy ran out; the step's result is invalid");
      return fail(MISO_B200_ERR_NONFINITE,
                  "non-positive or non-finite density / internal energy in the CFL pass");
    }
    return MISO_B200_OK;
  }
};

static bool valid_axis(int size, int margin) { return size >= 1 && (size == 1 || size >= margin); }

// Error text of handle-less calls (read back through miso_b200_last_error(NULL)).
void miso_b200_set_global_error(const std::string &msg) {
  std::lock_guard<std::mutex> lk(g_create_mu);
  g_create_error = msg;
}

extern "C" {

int miso_b200_pointer_kind(const void *p, int *kind) {
  if (!kind) return MISO_B200_ERR_ARG;
  *kind = 0;
  if (!p) return MISO_B200_OK;
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();  // not known to CUDA: host memory
    return MISO_B200_OK;
  }
  *kind = (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) ? 1 : 0;
  return MISO_B200_OK;
}

int miso_b200_alloc_shared(size_t bytes, void **ptr) {
  if (!ptr) return MISO_B200_ERR_ARG;
  *ptr = nullptr;
  if (!bytes) return MISO_B200_OK;
  if (cudaMallocManaged(ptr, bytes, cudaMemAttachGlobal) != cudaSuccess) {
    cudaGetLastError();
    *ptr = nullptr;
    return MISO_B200_ERR_NOMEM;
  }
  return MISO_B200_OK;
}

int miso_b200_free_shared(void *ptr) {
  if (!ptr) return MISO_B200_OK;
  if (cudaFree(ptr) != cudaSuccess) {
    cudaGetLastError();
    return MISO_B200_ERR_CUDA;
  }
  return MISO_B200_OK;
}

const char *miso_b200_version(void) { return "miso_b200 0.1 (sm_100a)"; }

const char *miso_b200_last_error(miso_b200_handle *h) {
  if (!h) {
    std::lock_guard<std::mutex> lk(g_create_mu);
    return g_create_error.c_str();
  }
  return h->err.c_str();
}

// Geometry, parameters and CFL spacing of a new handle from its descriptors
// (validated by the caller).
static void init_geom(miso_b200_handle *h, const miso_b200_grid_desc *gd,
                      const miso_b200_params *pp) {
  const int sz[3] = {gd->i_size, gd->j_size, gd->k_size};
  const double lo[3] = {gd->x_min, gd->y_min, gd->z_min};
  const double hi[3] = {gd->x_max, gd->y_max, gd->z_max};
  h->p = *pp;
  Geom &g = h->g;
  double ds[3];
  for (int a = 0; a < 3; ++a) {
    g.n[a] = sz[a];
    g.s[a] = sz[a] > 1 ? 1 : 0;
    g.m[a] = gd->margin * g.s[a];
    g.t[a] = sz[a] + 2 * g.m[a];
    g.periodic[a] = gd->periodic[a] ? 1 : 0;
    // grid.hpp:22-31 and 67-99: uniform spacing; degenerate axes 1e30 / 0
    const double sp = (hi[a] - lo[a]) / (double)sz[a];
    ds[a] = g.s[a] ? sp : 1.e30;
    g.dsi[a] = g.s[a] ? 1.0 / sp : 0.0;
    for (int side = 0; side < 2; ++side) {
      g.negmask[a][side] = 0;
      for (int f = 0; f < NF; ++f) {
        g.sign[a][side][f] = (float)(gd->sign[a][side][f] < 0 ? -1 : 1);
        if (!g.periodic[a] && gd->sign[a][side][f] < 0) g.negmask[a][side] |= (unsigned short)(1u << f);
      }
    }
  }
  g.st[2] = 1;
  g.st[1] = g.t[2];
  g.st[0] = (long long)g.t[1] * g.t[2];
  g.cells = (long long)g.t[0] * g.t[1] * g.t[2];
  // grid.hpp:241 and mhd_integrator_host.hpp:323-325, through float
  const float m3 = fminf(fminf((float)ds[0], (float)ds[1]), (float)ds[2]);
  h->min_dxyz = (double)m3;
  h->cfl_dx = pp->cfl_number * (double)m3;
}

int miso_b200_create(const miso_b200_grid_desc *gd, const miso_b200_params *pp, void *stream,
                     miso_b200_handle **out) {
  auto create_fail = [](int code, const std::string &msg) {
    std::lock_guard<std::mutex> lk(g_create_mu);
    g_create_error = msg;
    return code;
  };
  if (!gd || !pp || !out) return create_fail(MISO_B200_ERR_ARG, "null argument");
  *out = nullptr;
  if (gd->margin < 2)
    return create_fail(MISO_B200_ERR_ARG, "margin must be >= 2 for the 4th-order stencil");
  const int sz[3] = {gd->i_size, gd->j_size, gd->k_size};
  const double lo[3] = {gd->x_min, gd->y_min, gd->z_min};
  const double hi[3] = {gd->x_max, gd->y_max, gd->z_max};
  for (int a = 0; a < 3; ++a) {
    if (!valid_axis(sz[a], gd->margin))
      return create_fail(MISO_B200_ERR_ARG, "invalid grid size");
    if (!(lo[a] < hi[a])) return create_fail(MISO_B200_ERR_ARG, "invalid grid range");
  }
  if (!(pp->gm > 1.0) || !(pp->cfl_number > 0.0) || !(pp->ep >= 0.0) || !(pp->fh >= 0.0))
    return create_fail(MISO_B200_ERR_ARG, "invalid physics parameters");
  if (pp->precision != MISO_B200_FP64 && pp->precision != MISO_B200_FP32_SPLIT)
    return create_fail(MISO_B200_ERR_ARG, "unknown precision");

  auto *h = new miso_b200_handle();
  init_geom(h, gd, pp);
  Geom &g = h->g;

  cudaError_t e = cudaGetDevice(&h->device);
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->device);
  if (e != cudaSuccess) {
    delete h;
    return create_fail(MISO_B200_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
  }
  if (stream) {
    h->stream = (cudaStream_t)stream;
  } else {
    e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      delete h;
      return create_fail(MISO_B200_ERR_CUDA, "stream creation failed");
    }
    h->own_stream = true;
  }

  h->nparts = cfl_partial_blocks(h->sms);
  h->z_grid = 8 * h->sms;
  h->av_grid = 16 * h->sms;
  h->nparts_alloc = h->nparts > h->z_grid ? h->nparts : h->z_grid;
  h->mon_blocks = h->sms * 4;  // 4 x 148 CTAs of 256: 4.0 -> 2.5 ms at 512^3 against 2 per SM
  const size_t cells = (size_t)g.cells;
  size_t total = 0;
  std::vector<std::pair<void **, size_t>> plan;
  auto add = [&](void **p, size_t b) {
    plan.emplace_back(p, b);
    total += round_up(b);
  };
  if (!h->split()) {
    for (int s = 0; s < 3; ++s)
      for (int f = 0; f < NF; ++f) add((void **)&h->q64[s][f], cells * sizeof(double));
    add((void **)&h->cc64, cells * sizeof(double));
  } else {
    // each set of 9 arrays is contiguous with one pitch, so a 4-D tensor
    // map (k, j, i, field) can address it
    for (int s = 0; s < 2; ++s) {
      for (int f = 0; f < NF; ++f) add((void **)&h->hi[s][f], cells * sizeof(float));
      for (int f = 0; f < NF; ++f) add((void **)&h->lo[s][f], cells * sizeof(float));
    }
    for (int s = 0; s < 2; ++s)
      for (int f = 0; f < NF; ++f) add((void **)&h->stg[s][f], cells * sizeof(float));
    add((void **)&h->cc32, cells * sizeof(float));
  }
  add((void **)&h->partial, sizeof(float) * h->nparts_alloc);
  add((void **)&h->mon_partial, sizeof(double) * 8 * h->mon_blocks);
  if (h->split()) {
    add((void **)&h->mon_z, sizeof(double) * 6 * h->z_grid);
  }
  add((void **)&h->sc, sizeof(StepScalars));
  add((void **)&h->rs, sizeof(RunState));
  for (int a = 0; a < 3; ++a) add((void **)&h->axc[a], sizeof(double) * g.t[a]);
  e = cudaMalloc(&h->block, total);
  if (e != cudaSuccess) {
    if (h->own_stream) cudaStreamDestroy(h->stream);
    delete h;
    return create_fail(MISO_B200_ERR_NOMEM, "device allocation of " + std::to_string(total) +
                                                " bytes failed");
  }
  h->bytes = total;
  size_t off = 0;
  for (auto &pb : plan) {
    *pb.first = (char *)h->block + off;
    off += round_up(pb.second);
  }
  if (h->split()) {
    // The FP64 upload/download staging overlays the 18 consecutive FP32
    // stage arrays (18 * 4 bytes >= 9 * 8 bytes per cell), which hold no
    // state between steps.
    for (int f = 0; f < NF; ++f) h->io64[f] = (double *)h->stg[0][0] + (size_t)f * cells;
  }
  h->pitch = (long long)(round_up(cells * sizeof(float)) / sizeof(float));
  if (h->split() && s32_tiled_supported(g) && !getenv("MISO_B200_UNTILED"))
    h->setup_tiled(round_up(cells * sizeof(float)));
  e = cudaMemsetAsync(h->block, 0, total, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    cudaFree(h->block);
    if (h->own_stream) cudaStreamDestroy(h->stream);
    delete h;
    return create_fail(MISO_B200_ERR_CUDA, "device memset failed");
  }
  // cell centres per axis, placed as UniformAxisProvider::loc places them
  // (grid.hpp:22-31): x_min + (i_global + 0.5) * (x_max - x_min) / size
  for (int a = 0; a < 3; ++a) {
    std::vector<double> xs(g.t[a]);
    for (int i = 0; i < g.t[a]; ++i) {
      const int ig = i - g.m[a];
      const double sp = (hi[a] - lo[a]) / (double)sz[a];
      xs[i] = lo[a] + ((double)ig + 0.5) * sp;
    }
    // after the block's memset: the copy is ordered behind it on the stream
    e = cudaMemcpyAsync(h->axc[a], xs.data(), sizeof(double) * g.t[a], cudaMemcpyHostToDevice,
                        h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
      cudaFree(h->block);
      if (h->own_stream) cudaStreamDestroy(h->stream);
      delete h;
      return create_fail(MISO_B200_ERR_CUDA, "copy of the cell centres failed");
    }
  }
  h->src.kind = 0;
  h->src.g = 0.0;
  h->src.x = h->axc[0];
  h->src.y = h->axc[1];
  h->src.z = h->axc[2];
  *out = h;
  return MISO_B200_OK;
}

}  // extern "C"

// ---- views (view.h): the tiled step over arrays another owner holds
int miso_b200::b200_view_create(const miso_b200_grid_desc &gd, const miso_b200_params &pp,
                                cudaStream_t stream, float *const hi[2][NF],
                                float *const lo[2][NF], float *const stg[2][NF], float *cc,
                                size_t pitch_bytes, StepScalars *sc, miso_b200_handle **out) {
  *out = nullptr;
  if (pp.precision != MISO_B200_FP32_SPLIT) return MISO_B200_ERR_ARG;
  auto *h = new miso_b200_handle();
  init_geom(h, &gd, &pp);
  const Geom &g = h->g;
  if (!g.s[0] || !g.s[1] || !g.s[2] || !s32_tiled_supported(g)) {
    delete h;
    return MISO_B200_ERR_STATE;
  }
  cudaError_t e = cudaGetDevice(&h->device);
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->device);
  if (e != cudaSuccess) {
    delete h;
    return MISO_B200_ERR_CUDA;
  }
  h->stream = stream;
  h->own_stream = false;
  for (int s = 0; s < 2; ++s)
    for (int f = 0; f < NF; ++f) {
      h->hi[s][f] = hi[s][f];
      h->lo[s][f] = lo[s][f];
      h->stg[s][f] = stg[s][f];
    }
  h->cc32 = cc;
  h->sc = sc;
  h->pitch = (long long)(pitch_bytes / sizeof(float));
  // the view's own buffers: CFL and monitor partials, cell centres
  h->nparts = cfl_partial_blocks(h->sms);
  h->z_grid = 8 * h->sms;
  h->nparts_alloc = h->nparts > h->z_grid ? h->nparts : h->z_grid;
  h->mon_blocks = h->sms * 4;
  size_t total = 0;
  std::vector<std::pair<void **, size_t>> plan;
  auto add = [&](void **p, size_t b) {
    plan.emplace_back(p, b);
    total += round_up(b);
  };
  add((void **)&h->partial, sizeof(float) * h->nparts_alloc);
  add((void **)&h->mon_partial, sizeof(double) * 8 * h->mon_blocks);
  add((void **)&h->mon_z, sizeof(double) * 6 * h->z_grid);
  for (int a = 0; a < 3; ++a) add((void **)&h->axc[a], sizeof(double) * g.t[a]);
  e = cudaMalloc(&h->block, total);
  if (e == cudaSuccess) e = cudaMemsetAsync(h->block, 0, total, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) {
    if (h->block) cudaFree(h->block);
    delete h;
    return MISO_B200_ERR_NOMEM;
  }
  h->bytes = total;
  size_t off = 0;
  for (auto &pb : plan) {
    *pb.first = (char *)h->block + off;
    off += round_up(pb.second);
  }
  h->setup_tiled(pitch_bytes);
  if (!h->tiled) {
    cudaFree(h->block);
    delete h;
    return MISO_B200_ERR_STATE;
  }
  h->src.kind = 0;
  *out = h;
  return MISO_B200_OK;
}

int miso_b200::b200_view_step(miso_b200_handle *h, int cur, int *cur_out) {
  if (cur >= 0) h->cur = cur;
  int rc = h->enqueue_cfl();
  if (!rc) rc = h->enqueue_update();
  *cur_out = h->cur;
  return rc;
}

int miso_b200::b200_view_fill(miso_b200_handle *h, int cur) {
  h->cur = cur;
  h->partials_valid = false;
  h->mon_valid = false;
  h->lo_shell_stale = false;
  return h->fill_state();
}

int miso_b200::b200_view_fresh_lo(miso_b200_handle *h, int cur) {
  h->cur = cur;
  return h->fresh_lo_shell();
}

long long miso_b200::b200_view_launches(const miso_b200_handle *h) { return h->launches; }

int miso_b200::b200_view_cur(const miso_b200_handle *h) { return h->cur; }

void miso_b200::b200_view_set_cur(miso_b200_handle *h, int cur) { h->cur = cur; }

extern "C" {

int miso_b200_destroy(miso_b200_handle *h) {
  if (!h) return MISO_B200_ERR_ARG;
  h->join_xchg();
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->ev_pass) cudaEventDestroy(h->ev_pass);
  if (h->ev_xchg) cudaEventDestroy(h->ev_xchg);
  h->harvest();
  for (cudaEvent_t e : h->pool) cudaEventDestroy(e);
  if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  if (h->loop_exec) cudaGraphExecDestroy(h->loop_exec);
  if (h->loop_graph) cudaGraphDestroy(h->loop_graph);
  if (h->block) cudaFree(h->block);
  if (h->blend_block) cudaFree(h->blend_block);
  if (h->bc_stage) cudaFreeHost(h->bc_stage);
  if (h->src_stage) cudaFreeHost(h->src_stage);
  if (h->src_dev) cudaFree(h->src_dev);
  if (h->src_arg) cudaFree(h->src_arg);
  if (h->face_buf) cudaFree(h->face_buf);
  if (h->own_stream) cudaStreamDestroy(h->stream);
  delete h;
  return MISO_B200_OK;
}

int miso_b200_upload(miso_b200_handle *h, const double *const q[9]) {
  if (!h || !q) return MISO_B200_ERR_ARG;
  if (int rc0 = h->join_xchg()) return rc0;
  const size_t bytes = (size_t)h->g.cells * sizeof(double);
  int rc;
  for (int f = 0; f < NF; ++f) {
    if (!q[f]) return h->fail(MISO_B200_ERR_ARG, "null field pointer %d", f);
    double *dst = h->split() ? h->io64[f] : h->q64[0][f];
    if ((rc = h->cuda(cudaMemcpyAsync(dst, q[f], bytes, cudaMemcpyDefault, h->stream), "upload")))
      return rc;
  }
  if (h->split()) {
    FieldPtrs<const double> src;
    for (int f = 0; f < NF; ++f) src.f[f] = h->io64[f];
    h->cur = 0;
    h->partials_valid = false;
    h->mon_valid = false;
    h->lo_shell_stale = false;
    launch_s32_to_split(h->g.cells, src, h->H(0), h->L(0), h->sms, h->stream);
    h->launches++;
    if ((rc = h->check_launch("to_split"))) return rc;
  }
  return h->cuda(cudaStreamSynchronize(h->stream), "upload synchronize");
}

// Enqueue the conversion and the copies of miso_b200_download on the
// handle's stream without waiting; `event` (a cudaEvent_t, may be NULL) is
// recorded after the last copy.  Later work on the stream is ordered after
// the copies, so stepping on while a snapshot drains is safe.
int miso_b200_download_async(miso_b200_handle *h, double *const q[9], void *event) {
  if (!h || !q) return MISO_B200_ERR_ARG;
  const size_t bytes = (size_t)h->g.cells * sizeof(double);
  int rc = h->join_xchg();
  if (rc) return rc;
  for (int f = 0; f < NF; ++f)
    if (!q[f]) return h->fail(MISO_B200_ERR_ARG, "null field pointer %d", f);
  if ((rc = h->fresh_lo_shell())) return rc;
  if (h->split()) {
    launch_s32_from_split(h->g.cells, h->cst(h->H(h->cur)), h->cst(h->L(h->cur)), h->IO(), h->sms,
                          h->stream);
    h->launches++;
    if ((rc = h->check_launch("from_split"))) return rc;
  }
  for (int f = 0; f < NF; ++f) {
    const double *src = h->split() ? h->io64[f] : h->q64[0][f];
    if ((rc = h->cuda(cudaMemcpyAsync(q[f], src, bytes, cudaMemcpyDefault, h->stream),
                      "download")))
      return rc;
  }
  if (event) return h->cuda(cudaEventRecord((cudaEvent_t)event, h->stream), "record event");
  return MISO_B200_OK;
}

int miso_b200_download(miso_b200_handle *h, double *const q[9]) {
  if (!h || !q) return MISO_B200_ERR_ARG;
  const size_t bytes = (size_t)h->g.cells * sizeof(double);
  int rc = h->join_xchg();
  if (rc) return rc;
  if ((rc = h->fresh_lo_shell())) return rc;
  if (h->split()) {
    launch_s32_from_split(h->g.cells, h->cst(h->H(h->cur)), h->cst(h->L(h->cur)), h->IO(), h->sms,
                          h->stream);
    h->launches++;
    if ((rc = h->check_launch("from_split"))) return rc;
  }
  for (int f = 0; f < NF; ++f) {
    if (!q[f]) return h->fail(MISO_B200_ERR_ARG, "null field pointer %d", f);
    const double *src = h->split() ? h->io64[f] : h->q64[0][f];
    if ((rc = h->cuda(cudaMemcpyAsync(q[f], src, bytes, cudaMemcpyDefault, h->stream),
                      "download")))
      return rc;
  }
  return h->cuda(cudaStreamSynchronize(h->stream), "download synchronize");
}

int miso_b200_fill_ghosts(miso_b200_handle *h) {
  if (!h) return MISO_B200_ERR_ARG;
  return h->fill_state();
}

int miso_b200_cfl(miso_b200_handle *h, double *dt_out) {
  if (!h || !dt_out) return MISO_B200_ERR_ARG;
  int rc = h->enqueue_cfl();
  if (rc) return rc;
  StepScalars v;
  if ((rc = h->cuda(cudaMemcpyAsync(&v, h->sc, sizeof v, cudaMemcpyDeviceToHost, h->stream),
                    "read dt")))
    return rc;
  if ((rc = h->cuda(cudaStreamSynchronize(h->stream), "cfl synchronize"))) return rc;
  if (v.err & (ERRBIT_NONFINITE | ERRBIT_TIMEOUT)) return h->read_err();
  double dt = v.dt;
  // a shard: the minimum over all shards, as the reference's MPI_Allreduce
  int (*min_all)(void *, double *) = h->halo_axes ? h->halo3.min_all : h->halo_ops.min_all;
  if (h->halo_on && min_all) {
    const int r = min_all(h->halo_axes ? h->halo3.user : h->halo_ops.user, &dt);
    if (r) return h->fail(MISO_B200_ERR_HALO, "min_all callback returned %d", r);
  }
  *dt_out = dt;
  return MISO_B200_OK;
}

int miso_b200_set_source(miso_b200_handle *h, int kind, const double *params, int nparams) {
  if (!h) return MISO_B200_ERR_ARG;
  if (h->src_cb) return h->fail(MISO_B200_ERR_STATE, "a source callback is set");
  if (kind == MISO_B200_SOURCE_NONE) {
    h->src.kind = 0;
    h->src.g = 0.0;
  } else if (kind == MISO_B200_SOURCE_POINT_GRAVITY) {
    if (!params || nparams < 1 || !std::isfinite(params[0]))
      return h->fail(MISO_B200_ERR_ARG, "point gravity needs its constant g in params[0]");
    h->src.kind = 1;
    h->src.g = params[0];
    // the pipelined RK stage carries the source on 3-D grids
    if (h->tiled && h->rk_var < 2) h->rk_var = 2;
  } else {
    return h->fail(MISO_B200_ERR_ARG, "unknown source kind %d", kind);
  }
  if (h->graph_exec) {
    cudaGraphExecDestroy(h->graph_exec);
    cudaGraphDestroy(h->graph);
    h->graph_exec = nullptr;
    h->graph = nullptr;
    h->drop_loop();
  }
  return MISO_B200_OK;
}

int miso_b200_set_boundary(miso_b200_handle *h, int kind, const double *params, int nparams) {
  if (!h) return MISO_B200_ERR_ARG;
  if (kind == MISO_B200_BOUNDARY_FACES) {
    h->mag.on = 0;
    h->mag.mask_cfl = 0;
    h->retile();
  } else if (kind == MISO_B200_BOUNDARY_MAGNETOSPHERE) {
    if (h->split() && h->halo_on)
      return h->fail(MISO_B200_ERR_STATE,
                     "the split form's magnetosphere boundary runs on a single grid");
    if (h->bc_cb)
      return h->fail(MISO_B200_ERR_STATE, "a boundary callback is set");
    if (!params || nparams < 9)
      return h->fail(MISO_B200_ERR_ARG, "the magnetosphere boundary takes 9 parameters");
    for (int n = 0; n < 8; ++n)
      if (!std::isfinite(params[n]))
        return h->fail(MISO_B200_ERR_ARG, "non-finite boundary parameter %d", n);
    if (!(params[4] > 0.0) || !(params[0] > 0.0))
      return h->fail(MISO_B200_ERR_ARG, "radius and solar-wind density must be > 0");
    for (int a = 0; a < 3; ++a)
      if (h->g.s[a] && h->g.periodic[a])
        return h->fail(MISO_B200_ERR_ARG, "the magnetosphere boundary needs non-periodic axes");
    Magneto &m = h->mag;
    m.ro_sw = params[0];
    m.pr_sw = params[1];
    m.vx_sw = params[2];
    m.bz_sw = params[3];
    m.r_inner = params[4];
    m.a0 = params[5];
    m.ro_floor = params[6];
    m.pr_floor = params[7];
    m.mask_cfl = params[8] != 0.0;
    m.x = h->axc[0];
    m.y = h->axc[1];
    m.z = h->axc[2];
    m.on = 1;
    // the split form runs the per-cell kernels, which read every ghost
    // cell the boundary writes between passes
    if (int rc = h->fresh_lo_shell()) return rc;
    h->retile();
  } else {
    return h->fail(MISO_B200_ERR_ARG, "unknown boundary kind %d", kind);
  }
  h->partials_valid = false;
  if (h->graph_exec) {
    cudaGraphExecDestroy(h->graph_exec);
    cudaGraphDestroy(h->graph);
    h->graph_exec = nullptr;
    h->graph = nullptr;
    h->drop_loop();
  }
  return MISO_B200_OK;
}

int miso_b200_set_blend_state(miso_b200_handle *h, const double *const q[9]) {
  if (!h || !q) return MISO_B200_ERR_ARG;
  const size_t bytes = (size_t)h->g.cells * sizeof(double);
  int rc;
  if (!h->blend_block &&
      (rc = h->cuda(cudaMalloc((void **)&h->blend_block, bytes * NF), "allocate blend state")))
    return rc;
  for (int f = 0; f < NF; ++f) {
    if (!q[f]) return h->fail(MISO_B200_ERR_ARG, "null field pointer %d", f);
    double *dst = h->blend_block + (size_t)f * h->g.cells;
    if ((rc = h->cuda(cudaMemcpyAsync(dst, q[f], bytes, cudaMemcpyDefault, h->stream),
                      "upload blend state")))
      return rc;
    h->mag.blend[f] = dst;
  }
  return h->cuda(cudaStreamSynchronize(h->stream), "upload blend state");
}

int miso_b200_set_mirror_signs(miso_b200_handle *h, const double *sign) {
  if (!h || !sign) return MISO_B200_ERR_ARG;
  Geom &g = h->g;
  for (int a = 0; a < 3; ++a)
    for (int side = 0; side < 2; ++side) {
      g.negmask[a][side] = 0;
      for (int f = 0; f < NF; ++f) {
        const double v = sign[(a * 2 + side) * NF + f];
        if (v != 1.0 && v != -1.0) return h->fail(MISO_B200_ERR_ARG, "signs must be +1 or -1");
        g.sign[a][side][f] = (float)v;
        if (!g.periodic[a] && !g.ext[a][side] && v < 0)
          g.negmask[a][side] |= (unsigned short)(1u << f);
      }
    }
  if (h->graph_exec) {
    cudaGraphExecDestroy(h->graph_exec);
    cudaGraphDestroy(h->graph);
    h->graph_exec = nullptr;
    h->graph = nullptr;
    h->drop_loop();
  }
  return MISO_B200_OK;
}

int miso_b200_set_source_callback(miso_b200_handle *h, miso_b200_source_fn fn, void *user,
                                  int on_host) {
  if (!h) return MISO_B200_ERR_ARG;
  const size_t bytes = (size_t)h->g.cells * sizeof(double);
  if (fn) {
    if (h->halo_on)
      return h->fail(MISO_B200_ERR_STATE, "a source callback runs on a single grid");
    if (!h->src_dev && h->cuda(cudaMalloc((void **)&h->src_dev, 4 * bytes),
                               "allocate the source terms"))
      return MISO_B200_ERR_NOMEM;
    // the split form's stage buffers hold no FP64 primitives: a set of its own
    if (h->split() && !h->src_arg &&
        h->cuda(cudaMalloc((void **)&h->src_arg, NF * bytes), "allocate the source arguments"))
      return MISO_B200_ERR_NOMEM;
    if (on_host && !h->src_stage &&
        h->cuda(cudaMallocHost((void **)&h->src_stage, (NF + 4) * bytes),
                "allocate the source callback's host staging"))
      return MISO_B200_ERR_NOMEM;
    if (h->cuda(cudaMemsetAsync(h->src_dev, 0, 4 * bytes, h->stream), "clear the source terms"))
      return MISO_B200_ERR_CUDA;
    h->src.kind = 2;
    for (int t = 0; t < 4; ++t) h->src.arr[t] = h->src_dev + (size_t)t * h->g.cells;
  } else {
    if (h->src_stage) cudaFreeHost(h->src_stage);
    if (h->src_dev) {
      cudaStreamSynchronize(h->stream);
      cudaFree(h->src_dev);
    }
    if (h->src_arg) cudaFree(h->src_arg);
    h->src_stage = nullptr;
    h->src_dev = nullptr;
    h->src_arg = nullptr;
    if (h->src.kind == 2) h->src.kind = 0;
  }
  h->src_cb = fn;
  h->src_user = user;
  h->src_host = fn && on_host;

  if (h->graph_exec) {
    cudaGraphExecDestroy(h->graph_exec);
    cudaGraphDestroy(h->graph);
    h->graph_exec = nullptr;
    h->graph = nullptr;
    h->drop_loop();
  }
  return MISO_B200_OK;
}

int miso_b200_set_boundary_callback(miso_b200_handle *h, miso_b200_boundary_fn fn, void *user,
                                    int on_host) {
  if (!h) return MISO_B200_ERR_ARG;
  Geom &g = h->g;
  if (fn) {
    if (h->split())
      return h->fail(MISO_B200_ERR_STATE, "a boundary callback runs on the FP64 form");
    if (h->halo_on || h->mag.on)
      return h->fail(MISO_B200_ERR_STATE,
                     "a boundary callback excludes the halo exchange and the magnetosphere boundary");
    if (on_host && !h->bc_stage &&
        h->cuda(cudaMallocHost((void **)&h->bc_stage, (size_t)g.cells * NF * sizeof(double)),
                "allocate the boundary callback's host staging"))
      return MISO_B200_ERR_NOMEM;
  } else if (h->bc_stage) {
    cudaFreeHost(h->bc_stage);
    h->bc_stage = nullptr;
  }
  h->bc_cb = fn;
  h->bc_user = user;
  h->bc_host = fn && on_host;
  // the callback owns every non-periodic face: the fill leaves them alone
  for (int a = 0; a < 3; ++a)
    for (int side = 0; side < 2; ++side) {
      g.ext[a][side] = (fn && g.s[a] && !g.periodic[a]) ? 1 : 0;
      g.negmask[a][side] = 0;
      if (!g.ext[a][side] && !g.periodic[a])
        for (int f = 0; f < NF; ++f)
          if (g.sign[a][side][f] < 0) g.negmask[a][side] |= (unsigned short)(1u << f);
    }
  if (h->graph_exec) {
    cudaGraphExecDestroy(h->graph_exec);
    cudaGraphDestroy(h->graph);
    h->graph_exec = nullptr;
    h->graph = nullptr;
    h->drop_loop();
  }
  return MISO_B200_OK;
}

int miso_b200_set_halo_overlap(miso_b200_handle *h, void *comm_stream) {
  if (!h) return MISO_B200_ERR_ARG;
  if (int rc = h->join_xchg()) return rc;
  if (!comm_stream) {
    h->comm = nullptr;
    return MISO_B200_OK;
  }
  if (!h->halo_on) return h->fail(MISO_B200_ERR_STATE, "no halo exchange is set");
  if (h->g.ext[1][0] || h->g.ext[1][1] || h->g.ext[2][0] || h->g.ext[2][1])
    return h->fail(MISO_B200_ERR_STATE, "the overlapped exchange covers shared i faces only");
  if (!h->tiled || h->rk_var < 2 || h->av_var[0] != 0)
    return h->fail(MISO_B200_ERR_STATE,
                   "the overlapped exchange runs on the pipelined split path "
                   "(3-D FP32-split grid, Runge-Kutta variant 2 or 3, line x sweep)");
  int rc = MISO_B200_OK;
  if (!h->ev_pass)
    rc = h->cuda(cudaEventCreateWithFlags(&h->ev_pass, cudaEventDisableTiming), "event");
  if (!rc && !h->ev_xchg)
    rc = h->cuda(cudaEventCreateWithFlags(&h->ev_xchg, cudaEventDisableTiming), "event");
  if (rc) return rc;
  h->comm = (cudaStream_t)comm_stream;
  return MISO_B200_OK;
}

// miso_b200_set_halo (ops, along i) and miso_b200_set_halo3 (ops3, any
// axis); ext[2 * axis + side]
static int set_halo_impl(miso_b200_handle *h, const int *ext, const miso_b200_halo_ops *ops,
                         const miso_b200_halo3_ops *ops3) {
  if (int rc = h->join_xchg()) return rc;
  const bool on = ops != nullptr || ops3 != nullptr;
  if (!on) h->comm = nullptr;
  if (h->bc_cb || h->src_cb)
    return h->fail(MISO_B200_ERR_STATE, "a callback excludes the halo exchange");
  if (h->split() && h->mag.on && on)
    return h->fail(MISO_B200_ERR_STATE,
                   "the split form's magnetosphere boundary runs on a single grid");
  Geom &g = h->g;
  if ((ops && !ops->exchange) || (ops3 && !ops3->exchange))
    return h->fail(MISO_B200_ERR_ARG, "halo ops without exchange");
  bool any = false, jk = false;
  for (int a = 0; a < 3; ++a) {
    const bool shared = on && (ext[2 * a] || ext[2 * a + 1]);
    if (shared && !g.s[a])
      return h->fail(MISO_B200_ERR_ARG, "a shared face needs an axis of size > 1 (axis %d)", a);
    any = any || shared;
    jk = jk || (shared && a > 0);
  }
  if (jk && h->comm)
    return h->fail(MISO_B200_ERR_STATE, "the overlapped exchange covers shared i faces only");
  // face buffers: the largest j or k face of the widest exchange (2 * 9 + 1
  // float arrays, or 9 double arrays), four regions
  size_t region = 0;
  if (jk) {
    const long long fj = (long long)g.t[0] * g.m[1] * g.t[2];
    const long long fk = (long long)g.t[0] * g.t[1] * g.m[2];
    const long long face = fj > fk ? fj : fk;
    region = (size_t)face * (h->split() ? (2 * NF + 1) * sizeof(float) : NF * sizeof(double));
    region = (region + 255) / 256 * 256;
  }
  if (region != h->face_region) {
    if (h->face_buf) {
      if (h->stream) cudaStreamSynchronize(h->stream);
      cudaFree(h->face_buf);
    }
    h->face_buf = nullptr;
    h->face_region = 0;
    if (region) {
      if (h->cuda(cudaMalloc((void **)&h->face_buf, 4 * region), "allocate the face buffers"))
        return MISO_B200_ERR_NOMEM;
      h->face_region = region;
    }
  }
  h->halo_on = any;
  h->halo_axes = ops3 != nullptr;
  h->halo_ops = ops ? *ops : miso_b200_halo_ops{};
  h->halo3 = ops3 ? *ops3 : miso_b200_halo3_ops{};
  for (int a = 0; a < 3; ++a)
    for (int side = 0; side < 2; ++side) {
      const bool shared = any && ext[2 * a + side];
      g.ext[a][side] = shared ? 1 : 0;
      // no image across a shared face; elsewhere the descriptor's mirror signs
      g.negmask[a][side] = 0;
      if (!shared && !g.periodic[a])
        for (int f = 0; f < NF; ++f)
          if (g.sign[a][side][f] < 0) g.negmask[a][side] |= (unsigned short)(1u << f);
    }
  if (h->graph_exec) {
    cudaGraphExecDestroy(h->graph_exec);
    cudaGraphDestroy(h->graph);
    h->graph_exec = nullptr;
    h->graph = nullptr;
    h->drop_loop();
  }
  h->partials_valid = false;
  return MISO_B200_OK;
}

int miso_b200_set_halo(miso_b200_handle *h, int ext_lo, int ext_hi,
                       const miso_b200_halo_ops *ops) {
  if (!h) return MISO_B200_ERR_ARG;
  const int ext[6] = {ext_lo, ext_hi, 0, 0, 0, 0};
  return set_halo_impl(h, ext, ops, nullptr);
}

int miso_b200_set_halo3(miso_b200_handle *h, const int ext[6], const miso_b200_halo3_ops *ops) {
  if (!h) return MISO_B200_ERR_ARG;
  if (ops && !ext) return h->fail(MISO_B200_ERR_ARG, "no face flags");
  const int none[6] = {0, 0, 0, 0, 0, 0};
  return set_halo_impl(h, ops ? ext : none, nullptr, ops);
}

int miso_b200_update(miso_b200_handle *h, double dt) {
  if (!h) return MISO_B200_ERR_ARG;
  if (!(dt > 0.0) || !std::isfinite(dt)) return h->fail(MISO_B200_ERR_ARG, "dt must be > 0");
  set_scalars_kernel<<<1, 1, 0, h->stream>>>(h->sc, h->host_scalars(dt));
  h->launches++;
  int rc = h->check_launch("set_scalars");
  if (rc) return rc;
  return h->enqueue_update();
}

int miso_b200_update_device(miso_b200_handle *h) {
  if (!h) return MISO_B200_ERR_ARG;
  if (h->halo_on)
    return h->fail(MISO_B200_ERR_STATE, "a shard steps with cfl() and update(dt)");
  return h->enqueue_update();
}

int miso_b200_run(miso_b200_handle *h, int nsteps, int use_graph) {
  if (!h || nsteps < 0) return MISO_B200_ERR_ARG;
  if ((h->bc_cb || h->src_cb) && use_graph)
    return h->fail(MISO_B200_ERR_STATE, "a callback runs on the host between passes: no graph");
  if (h->halo_on)
    return h->fail(MISO_B200_ERR_STATE, "a shard steps with cfl() and update(dt)");
  int rc;
  if (!use_graph) {
    for (int n = 0; n < nsteps; ++n) {
      if ((rc = h->enqueue_cfl())) return rc;
      if ((rc = h->enqueue_update())) return rc;
    }
    return MISO_B200_OK;
  }
  // The tiled split path computes the next step's CFL minima inside the last
  // viscosity sweep; a captured step assumes they are present, so a state
  // that has not been stepped yet takes one eager step first.
  if (h->tiled && !h->partials_valid && nsteps > 0) {
    if ((rc = h->enqueue_cfl())) return rc;
    if ((rc = h->enqueue_update())) return rc;
    --nsteps;
  }
  if (nsteps == 0) return MISO_B200_OK;
  // The split form swaps its hi/lo sets once per AV sweep; when a step
  // swaps an odd number of times the captured graph covers two steps so
  // that it starts and ends on the same set.
  if (h->graph_exec && h->graph_cur != h->cur) {
    // captured for the other hi/lo set: capture again
    cudaGraphExecDestroy(h->graph_exec);
    cudaGraphDestroy(h->graph);
    h->graph_exec = nullptr;
    h->graph = nullptr;
    h->drop_loop();
  }
  if (!h->graph_exec) {
    const int before = h->cur;
    const bool valid_before = h->partials_valid;
    const long long l0 = h->launches;
    if ((rc = h->cuda(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal),
                      "begin capture")))
      return rc;
    h->capturing = true;
    int steps = 1;
    rc = h->enqueue_cfl();
    if (!rc) rc = h->enqueue_update();
    if (!rc && h->cur != before) {
      steps = 2;
      rc = h->enqueue_cfl();
      if (!rc) rc = h->enqueue_update();
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
    h->capturing = false;
    h->cur = before;
    h->partials_valid = valid_before;
    const long long kernels = h->launches - l0;
    h->launches = l0;
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if ((rc = h->cuda(e, "end capture"))) return rc;
    h->graph = graph;
    if ((rc = h->cuda(cudaGraphInstantiate(&h->graph_exec, graph, 0), "graph instantiate")))
      return rc;
    h->graph_steps = steps;
    h->graph_kernels = kernels;
    h->graph_cur = before;
  }
  const int reps = nsteps / h->graph_steps, rem = nsteps % h->graph_steps;
  for (int n = 0; n < reps; ++n) {
    if ((rc = h->cuda(cudaGraphLaunch(h->graph_exec, h->stream), "graph launch"))) return rc;
    h->launches += h->graph_kernels;
  }
  if (reps > 0 && h->tiled) h->partials_valid = true;
  for (int n = 0; n < rem; ++n) {
    if ((rc = h->enqueue_cfl())) return rc;
    if ((rc = h->enqueue_update())) return rc;
  }
  return MISO_B200_OK;
}

// The loop graph: WHILE { step; advance } with the condition set by the
// advance kernel; where a step swaps the hi / lo sets the body holds two
// steps, the second under an IF node with the same condition, so the loop
// still stops after the step that reaches t_end.
static int build_loop_graph(miso_b200_handle *h) {
  if (h->loop_exec) cudaGraphExecDestroy(h->loop_exec);
  if (h->loop_graph) cudaGraphDestroy(h->loop_graph);
  h->loop_exec = nullptr;
  h->loop_graph = nullptr;
  cudaGraph_t g = nullptr;
  int rc = h->cuda(cudaGraphCreate(&g, 0), "graph create");
  if (rc) return rc;
  cudaGraphConditionalHandle h_while;
  rc = h->cuda(cudaGraphConditionalHandleCreate(&h_while, g, 1, cudaGraphCondAssignDefault),
               "conditional handle");
  cudaGraphNodeParams wp = {};
  wp.type = cudaGraphNodeTypeConditional;
  wp.conditional.handle = h_while;
  wp.conditional.type = cudaGraphCondTypeWhile;
  wp.conditional.size = 1;
  cudaGraphNode_t wnode;
  if (!rc) rc = h->cuda(cudaGraphAddNode(&wnode, g, nullptr, 0, &wp), "while node");
  if (rc) {
    cudaGraphDestroy(g);
    return rc;
  }
  const int before = h->cur;
  const bool valid_before = h->partials_valid;
  const long long l0 = h->launches;
  cudaGraph_t tmp = nullptr;
  // where a step swaps the hi / lo sets (the split form's odd number of
  // viscosity sweeps) the body holds two steps, the second under an IF node
  const bool two = h->split() && (h->sweep_passes() & 1);
  cudaGraphConditionalHandle h_if = 0;
  if (two) {
    rc = h->cuda(cudaGraphConditionalHandleCreate(&h_if, wp.conditional.phGraph_out[0], 0,
                                                  cudaGraphCondAssignDefault),
                 "conditional handle");
    if (rc) {
      cudaGraphDestroy(g);
      return rc;
    }
  }
  h->capturing = true;
  rc = h->cuda(cudaStreamBeginCaptureToGraph(h->stream, wp.conditional.phGraph_out[0], nullptr,
                                             nullptr, 0, cudaStreamCaptureModeThreadLocal),
               "begin capture");
  if (!rc) rc = h->enqueue_cfl();
  if (!rc) rc = h->enqueue_update();
  const long long per_step = h->launches - l0 + 1;
  if (!rc && (h->cur != before) != two)
    rc = h->fail(MISO_B200_ERR_STATE, "a step swapped the state sets unexpectedly");
  if (!rc) {
    advance_cond_kernel<<<1, 1, 0, h->stream>>>(h->rs, h->sc, h_while, h_if, two ? 1 : 0);
    rc = h->check_launch("advance");
  }
  cudaGraphNodeParams ip = {};
  if (!rc && two) {
    // the second step under an IF node with the loop's condition
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    rc = h->cuda(cudaStreamGetCaptureInfo(h->stream, &cs, nullptr, &cg, &deps, &nd),
                 "capture info");
    ip.type = cudaGraphNodeTypeConditional;
    ip.conditional.handle = h_if;
    ip.conditional.type = cudaGraphCondTypeIf;
    ip.conditional.size = 1;
    cudaGraphNode_t inode;
    if (!rc) rc = h->cuda(cudaGraphAddNode(&inode, cg, deps, nd, &ip), "if node");
    if (!rc)
      rc = h->cuda(cudaStreamUpdateCaptureDependencies(h->stream, &inode, 1,
                                                        cudaStreamSetCaptureDependencies),
                   "capture dependencies");
  }
  cudaError_t e = cudaStreamEndCapture(h->stream, &tmp);
  if (!rc) rc = h->cuda(e, "end capture");
  if (!rc && two) {
    rc = h->cuda(cudaStreamBeginCaptureToGraph(h->stream, ip.conditional.phGraph_out[0], nullptr,
                                               nullptr, 0, cudaStreamCaptureModeThreadLocal),
                 "begin capture");
    if (!rc) rc = h->enqueue_cfl();
    if (!rc) rc = h->enqueue_update();
    if (!rc) {
      advance_cond_kernel<<<1, 1, 0, h->stream>>>(h->rs, h->sc, h_while, h_if, 0);
      rc = h->check_launch("advance");
    }
    e = cudaStreamEndCapture(h->stream, &tmp);
    if (!rc) rc = h->cuda(e, "end capture");
  }
  h->capturing = false;
  h->cur = before;
  h->partials_valid = valid_before;
  h->launches = l0;
  if (!rc) rc = h->cuda(cudaGraphInstantiate(&h->loop_exec, g, 0), "graph instantiate");
  if (rc) {
    cudaGraphDestroy(g);
    h->loop_exec = nullptr;
    return rc;
  }
  h->loop_graph = g;
  h->loop_cur = before;
  h->loop_steps = two ? 2 : 1;
  h->loop_kernels = per_step;
  return MISO_B200_OK;
}

int miso_b200_run_until(miso_b200_handle *h, double *time, double t_end, int max_steps,
                        int use_graph, int *steps_out) {
  if (!h || !time || !steps_out || max_steps < 0) return MISO_B200_ERR_ARG;
  *steps_out = 0;
  if (h->halo_on)
    return h->fail(MISO_B200_ERR_STATE, "a shard steps with cfl() and update(dt)");
  if (h->bc_cb || h->src_cb) use_graph = 0;  // a host callback between passes cannot be captured
  if (!(*time < t_end) || max_steps == 0) return MISO_B200_OK;
  RunState st{*time, t_end, 0, max_steps};
  int rc = h->cuda(cudaMemcpyAsync(h->rs, &st, sizeof st, cudaMemcpyHostToDevice, h->stream),
                   "set the run state");
  if (!rc) rc = h->cuda(cudaStreamSynchronize(h->stream), "synchronize");
  if (rc) return rc;
  // eager steps: without a graph, and until the tiled split path holds the
  // CFL minima its captured step relies on
  while (!use_graph || (h->tiled && !h->partials_valid)) {
    if ((rc = h->enqueue_cfl()) || (rc = h->enqueue_update())) return rc;
    advance_kernel<<<1, 1, 0, h->stream>>>(h->rs, h->sc);
    h->launches++;
    if ((rc = h->check_launch("advance"))) return rc;
    rc = h->cuda(cudaMemcpyAsync(&st, h->rs, sizeof st, cudaMemcpyDeviceToHost, h->stream),
                 "read the run state");
    if (!rc) rc = h->read_err();
    if (rc) return rc;
    *time = st.time;
    *steps_out = st.steps;
    if (!(st.time < t_end) || st.steps >= max_steps) return MISO_B200_OK;
  }
  if (!h->loop_exec || h->loop_cur != h->cur)
    if ((rc = build_loop_graph(h))) return rc;
  if ((rc = h->cuda(cudaGraphLaunch(h->loop_exec, h->stream), "graph launch"))) return rc;
  rc = h->cuda(cudaMemcpyAsync(&st, h->rs, sizeof st, cudaMemcpyDeviceToHost, h->stream),
               "read the run state");
  if (!rc) rc = h->read_err();
  if (rc) return rc;
  const int taken = st.steps - *steps_out;
  h->launches += h->loop_kernels * taken;
  // each step swaps the sets where the body holds two steps
  if (h->loop_steps == 2 && (taken & 1)) h->cur ^= 1;
  if (h->tiled) h->partials_valid = true;
  *time = st.time;
  *steps_out = st.steps;
  return MISO_B200_OK;
}

int miso_b200_sync(miso_b200_handle *h) {
  if (!h) return MISO_B200_ERR_ARG;
  return h->read_err();
}

int miso_b200_last_dt(miso_b200_handle *h, double *dt_out) {
  if (!h || !dt_out) return MISO_B200_ERR_ARG;
  StepScalars v;
  int rc = h->cuda(cudaMemcpyAsync(&v, h->sc, sizeof v, cudaMemcpyDeviceToHost, h->stream),
                   "read dt");
  if (rc) return rc;
  if ((rc = h->cuda(cudaStreamSynchronize(h->stream), "synchronize"))) return rc;
  *dt_out = v.dt;
  return MISO_B200_OK;
}

int miso_b200_monitors(miso_b200_handle *h, double out[8]) {
  if (!h || !out) return MISO_B200_ERR_ARG;
  if (int rc0 = h->join_xchg()) return rc0;
  FieldPtrs<const double> q{};
  FieldPtrs<const float> hs{}, ls{};
  int rc;
  double dv = 1.0;
  for (int a = 0; a < 3; ++a)
    if (h->g.s[a]) dv *= 1.0 / h->g.dsi[a];
  if (h->split() && h->mon_valid) {
    // the last z sweep summed the state; only |div B| is left to reduce (its
    // stencil reads the lo ghost words of bx, by and bz, which lag the
    // interior until refreshed)
    if ((rc = h->fresh_lo_b())) return rc;
    const Geom &g = h->g;
    const long long items = (long long)((g.n[0] + DBM_L - 1) / DBM_L) *
                            ((g.n[1] + DBM_TJ - 1) / DBM_TJ) * ((g.n[2] + DBM_TK - 1) / DBM_TK);
    const int nb = items < 2LL * h->sms ? (int)items : 2 * h->sms;  // <= mon_blocks
    divb_march_kernel<<<nb, 256, 0, h->stream>>>(g, h->cst(h->H(h->cur)), h->cst(h->L(h->cur)),
                                                 h->mon_partial);
    h->launches++;
    if ((rc = h->check_launch("divb"))) return rc;
    // per-block sums of the sweep that left them (z_parts blocks)
    std::vector<double> zs((size_t)h->z_parts * 6), db((size_t)nb * 8);
    if ((rc = h->cuda(cudaMemcpyAsync(zs.data(), h->mon_z, zs.size() * sizeof(double),
                                      cudaMemcpyDeviceToHost, h->stream),
                      "read monitors")) ||
        (rc = h->cuda(cudaMemcpyAsync(db.data(), h->mon_partial, db.size() * sizeof(double),
                                      cudaMemcpyDeviceToHost, h->stream),
                      "read monitors")) ||
        (rc = h->cuda(cudaStreamSynchronize(h->stream), "monitors synchronize")))
      return rc;
    for (int q8 = 0; q8 < 8; ++q8) out[q8] = 0.0;
    const int map[6] = {0, 1, 2, 3, 4, 7};  // ro, mx, my, mz, et, ph^2
    for (int b = 0; b < h->z_parts; ++b)
      for (int q = 0; q < 6; ++q) out[map[q]] += zs[(size_t)b * 6 + q];
    for (int b = 0; b < nb; ++b) {
      out[5] += db[(size_t)b * 8 + 5];
      out[6] = std::fmax(out[6], db[(size_t)b * 8 + 6]);
    }
    for (int q8 = 0; q8 < 8; ++q8)
      if (q8 != 6) out[q8] *= dv;
    return MISO_B200_OK;
  }
  if (h->split()) {
    // the stencil of div B reads lo ghost words, which lag the interior
    // between a step and a download
    if ((rc = h->fresh_lo_shell())) return rc;
    hs = h->cst(h->H(h->cur));
    ls = h->cst(h->L(h->cur));
    monitor_kernel<true><<<h->mon_blocks, 256, 0, h->stream>>>(h->g, q, hs, ls, h->mon_partial);
  } else {
    q = h->c64(0);
    monitor_kernel<false><<<h->mon_blocks, 256, 0, h->stream>>>(h->g, q, hs, ls, h->mon_partial);
  }
  h->launches++;
  rc = h->check_launch("monitors");
  if (rc) return rc;
  std::vector<double> part((size_t)h->mon_blocks * 8);
  if ((rc = h->cuda(cudaMemcpyAsync(part.data(), h->mon_partial, part.size() * sizeof(double),
                                    cudaMemcpyDeviceToHost, h->stream),
                    "read monitors")))
    return rc;
  if ((rc = h->cuda(cudaStreamSynchronize(h->stream), "monitors synchronize"))) return rc;
  for (int q8 = 0; q8 < 8; ++q8) out[q8] = 0.0;
  for (int b = 0; b < h->mon_blocks; ++b)
    for (int q8 = 0; q8 < 8; ++q8) {
      const double v = part[(size_t)b * 8 + q8];
      if (q8 == 6)
        out[6] = std::fmax(out[6], v);
      else
        out[q8] += v;
    }
  for (int q8 = 0; q8 < 8; ++q8)
    if (q8 != 6) out[q8] *= dv;
  return MISO_B200_OK;
}

int miso_b200_fields_view(miso_b200_handle *h, double *ptrs[9]) {
  if (!h || !ptrs) return MISO_B200_ERR_ARG;
  if (h->split())
    return h->fail(MISO_B200_ERR_STATE, "fields_view needs the FP64 form");
  for (int f = 0; f < NF; ++f) ptrs[f] = h->q64[0][f];
  return MISO_B200_OK;
}

int miso_b200_set_variant(miso_b200_handle *h, int kernel_class, int variant) {
  if (h && h->comm && ((kernel_class == 0 && variant < 2) || (kernel_class == 1 && variant != 0))) {
    h->join_xchg();
    h->comm = nullptr;  // the overlapped exchange needs the pipelined stage and the line x sweep
  }
  if (!h || kernel_class < 0 || kernel_class > 3 || variant < 0 ||
      variant > (kernel_class == 0 || kernel_class == 2 ? 3 : 2))
    return MISO_B200_ERR_ARG;
  if (!h->tiled) return h->fail(MISO_B200_ERR_STATE, "kernel variants apply to 3-D split grids");
  if (kernel_class == 0 && variant < 2 && h->src.kind != 0)
    return h->fail(MISO_B200_ERR_STATE, "with a source term the RK stage runs variant 2 or 3");
  if (kernel_class == 0)
    h->rk_var = variant;
  else
    h->av_var[kernel_class - 1] = variant;
  if (h->graph_exec) {
    cudaGraphExecDestroy(h->graph_exec);
    cudaGraphDestroy(h->graph);
    h->graph_exec = nullptr;
    h->graph = nullptr;
    h->drop_loop();
  }
  return MISO_B200_OK;
}

int miso_b200_set_chunks(miso_b200_handle *h, int rk_chunk, int av_chunk) {
  if (!h || rk_chunk < 1 || av_chunk < 1) return MISO_B200_ERR_ARG;
  if (!h->tiled) return h->fail(MISO_B200_ERR_STATE, "chunk lengths apply to 3-D split grids");
  h->rk_L = rk_chunk;
  h->av_L = av_chunk;
  s32_rk_items(h->g, h->rk_L, h->rk_tiles_j, h->rk_tiles_k, h->rk_items);
  h->rk_grid = h->rk_items < 2 * h->sms ? h->rk_items : 2 * h->sms;
  if (h->graph_exec) {
    cudaGraphExecDestroy(h->graph_exec);
    cudaGraphDestroy(h->graph);
    h->graph_exec = nullptr;
    h->graph = nullptr;
    h->drop_loop();
  }
  return MISO_B200_OK;
}

int miso_b200_set_monitor_fusion(miso_b200_handle *h, int on) {
  if (!h) return MISO_B200_ERR_ARG;
  if (!h->tiled) return h->fail(MISO_B200_ERR_STATE, "monitor fusion applies to 3-D split grids");
  h->mon_fuse = on != 0;
  h->mon_valid = false;
  if (h->graph_exec) {  // a captured graph holds the other z sweep
    cudaGraphExecDestroy(h->graph_exec);
    cudaGraphDestroy(h->graph);
    h->graph_exec = nullptr;
    h->graph = nullptr;
    h->drop_loop();
  }
  return MISO_B200_OK;
}

int miso_b200_set_wait_limit(miso_b200_handle *h, long long cycles) {
  if (!h) return MISO_B200_ERR_ARG;
  if (!h->tiled) return h->fail(MISO_B200_ERR_STATE, "the wait limit applies to 3-D split grids");
  h->wait_limit = cycles > 0 ? cycles : s32t::WAIT_CYCLES;
  if (h->graph_exec) {  // a captured graph holds the old bound
    cudaGraphExecDestroy(h->graph_exec);
    cudaGraphDestroy(h->graph);
    h->graph_exec = nullptr;
    h->graph = nullptr;
    h->drop_loop();
  }
  return MISO_B200_OK;
}

int miso_b200_arm_timeout_test(miso_b200_handle *h, long long cycles) {
  if (!h || cycles <= 0) return MISO_B200_ERR_ARG;
  if (!h->tiled || h->rk_var < 2)
    return h->fail(MISO_B200_ERR_STATE,
                   "the timeout test runs on the pipelined Runge-Kutta stage of 3-D split grids");
  h->stall_cycles = cycles;
  return MISO_B200_OK;
}

int miso_b200_get_variant(miso_b200_handle *h, int kernel_class, int *variant) {
  if (!h || !variant || kernel_class < 0 || kernel_class > 3) return MISO_B200_ERR_ARG;
  if (!h->tiled) {
    *variant = -1;
    return MISO_B200_OK;
  }
  *variant = kernel_class == 0 ? h->rk_var : h->av_var[kernel_class - 1];
  return MISO_B200_OK;
}

int miso_b200_set_timing(miso_b200_handle *h, int enable) {
  if (!h) return MISO_B200_ERR_ARG;
  int rc = h->cuda(cudaStreamSynchronize(h->stream), "synchronize");
  if (rc) return rc;
  h->harvest();
  h->acc.clear();
  h->timing = enable != 0;
  return MISO_B200_OK;
}

int miso_b200_timing_report(miso_b200_handle *h, char *buf, size_t len) {
  if (!h || !buf || len == 0) return MISO_B200_ERR_ARG;
  int rc = h->cuda(cudaStreamSynchronize(h->stream), "synchronize");
  if (rc) return rc;
  h->harvest();
  std::string out = "{";
  bool first = true;
  for (auto &kv : h->acc) {
    char item[256];
    snprintf(item, sizeof item, "%s\"%s\": {\"launches\": %lld, \"ms\": %.6f, \"bytes\": %.1f}",
             first ? "" : ", ", kv.first.c_str(), kv.second.n, kv.second.ms, kv.second.bytes);
    out += item;
    first = false;
  }
  out += "}";
  if (out.size() + 1 > len) return h->fail(MISO_B200_ERR_ARG, "buffer too small");
  memcpy(buf, out.c_str(), out.size() + 1);
  return MISO_B200_OK;
}

int miso_b200_device_bytes(miso_b200_handle *h, size_t *bytes) {
  if (!h || !bytes) return MISO_B200_ERR_ARG;
  *bytes = h->bytes;
  return MISO_B200_OK;
}

int miso_b200_launch_count(miso_b200_handle *h, long long *count) {
  if (!h || !count) return MISO_B200_ERR_ARG;
  *count = h->launches;
  return MISO_B200_OK;
}

}  // extern "C"
