// Tiled FP32 split-precision kernels for 3-D grids (every axis of size > 1).
//
// Runge-Kutta stage (rk_tiled_kernel):
//   A CTA owns a TJ x TK tile of (j, k) columns and marches along i over a
//   chunk of planes.  Each plane of the previous stage state -- 9 conserved
//   fields on the tile plus a 2-cell halo in j and k -- arrives in shared
//   memory by one TMA bulk-tensor copy (4-D tensor map: k, j, i, field),
//   NBUF planes in flight.  Every point's flux vectors along y and z are
//   formed once per plane and kept in shared memory for the 4th-order
//   differences; the flux along the march axis goes into a 5-plane register
//   queue, and each difference is formed as (F[-2] - F[+2]) + 8 (F[+1] -
//   F[-1]), exactly zero for a locally constant flux.  Results are written
//   with their ghost images (periodic wrap / mirror), so no ghost-fill pass
//   runs; the last stage also writes the characteristic speed.
//
// Artificial viscosity:
//   x and y sweeps (av_line_kernel) stream along their axis: four consumer
//   warps own 128 consecutive k cells of one line; per plane one TMA copy
//   each brings hi, lo and the characteristic speed (k box of 132 cells)
//   into a ring of slots that a fifth warp fills.  Full / empty mbarriers
//   order the ring, so no CTA barrier runs in the loop (a CTA barrier per
//   plane, with the first thread waiting for the copy, measured 1.1x
//   slower).  A register queue carries the limiter slopes and face fluxes,
//   so each face flux and each slope is evaluated once, on packed field
//   pairs.  The z sweep (contiguous axis, av_z_kernel) exchanges
//   neighbours with warp shuffles and folds the CFL candidate of the new
//   state into per-block minima.  The sweeps write the interior only; the ghost images follow
//   from the shell kernel (s32_shell.cu).
//
// Physics as in fp32s_kernels.cu (flux form of mhd_integrator_host.hpp:
// 57-247; limiter.hpp:11-37; mhd_artificial_viscosity_host.hpp:51-348).
#include <cuda.h>

#include "common.cuh"
#include "s32_tiled.h"
#include "s32_common.cuh"
#include "tma.cuh"

namespace miso_b200 {
namespace s32t {

// ---------------------------------------------------------------------------
// RK stage kernel
// ---------------------------------------------------------------------------
constexpr int TJ = 8, TK = 32, HJ = TJ + 4, HK = TK + 4;
constexpr int NTHR = TJ * TK;  // 256
constexpr int NBUF = 3;
constexpr int PLANE_BYTES = NF * HJ * HK * 4;                  // TMA bytes per plane
constexpr int PLANE_STRIDE = (PLANE_BYTES + 127) / 128 * 128;  // 128-byte aligned buffers

struct __align__(128) RkSmem {
  unsigned char plane[NBUF][PLANE_STRIDE];
  float fy[NF][HJ][TK];
  float fz[NF][TJ][HK];
  unsigned long long bar[NBUF];
  int abort;
};

struct March {
  float F1[NF], F2[NF], F3[NF], F4[NF];  // x flux at planes q-1 .. q-4
  float Dyz1[NF], Dyz2[NF];              // y+z differences of cells q-1, q-2
};

template <int STAGE>
__device__ __forceinline__ void rk_plane(const RkArgs &a, RkSmem &sm, const float *pl, March &ms,
                                         int q, int i_start, int i_end, int jj, int kk,
                                         int tid, float ch2, float dt, float decay) {
  const int ty = tid / TK, tx = tid % TK;
  const Geom &g = a.g;
  const float wx = (float)(g.dsi[0] * INV12);
  const float wy = (float)(g.dsi[1] * INV12);
  const float wz = (float)(g.dsi[2] * INV12);
  float Fn[NF];
  const bool need_yz = q >= i_start && q < i_end;
  {
    float u[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) u[f] = pl[(f * HJ + ty + 2) * HK + tx + 2];
    PrimF p;
    prim(u, a.gm1, p);
    if (need_yz) {
      float F[NF];
      flux_dir<1>(u, p, ch2, F);
#pragma unroll
      for (int f = 0; f < NF; ++f) sm.fy[f][ty + 2][tx] = F[f];
      flux_dir<2>(u, p, ch2, F);
#pragma unroll
      for (int f = 0; f < NF; ++f) sm.fz[f][ty][tx + 2] = F[f];
    }
    flux_dir<0>(u, p, ch2, Fn);
  }
  // halo fluxes (y rows above/below, z columns left/right)
  if (need_yz && tid < 4 * TK + 4 * TJ) {
    float uh[NF], Fh[NF];
    PrimF ph;
    if (tid < 4 * TK) {
      const int r = tid / TK, col = tid % TK;
      const int row = r < 2 ? r : TJ + r;  // 0, 1, TJ+2, TJ+3
#pragma unroll
      for (int f = 0; f < NF; ++f) uh[f] = pl[(f * HJ + row) * HK + col + 2];
      prim(uh, a.gm1, ph);
      flux_dir<1>(uh, ph, ch2, Fh);
#pragma unroll
      for (int f = 0; f < NF; ++f) sm.fy[f][row][col] = Fh[f];
    } else {
      const int e = tid - 4 * TK;
      const int row = e / 4, c = e % 4;
      const int col = c < 2 ? c : TK + c;  // 0, 1, TK+2, TK+3
#pragma unroll
      for (int f = 0; f < NF; ++f) uh[f] = pl[(f * HJ + row + 2) * HK + col];
      prim(uh, a.gm1, ph);
      flux_dir<2>(uh, ph, ch2, Fh);
#pragma unroll
      for (int f = 0; f < NF; ++f) sm.fz[f][row][col] = Fh[f];
    }
  }
  __syncthreads();  // (A) fluxes visible; the plane buffer is free
  float Dyz[NF];
  if (need_yz) {
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      const float dy = (sm.fy[f][ty][tx] - sm.fy[f][ty + 4][tx]) +
                       8.0f * (sm.fy[f][ty + 3][tx] - sm.fy[f][ty + 1][tx]);
      const float dz = (sm.fz[f][ty][tx] - sm.fz[f][ty][tx + 4]) +
                       8.0f * (sm.fz[f][ty][tx + 3] - sm.fz[f][ty][tx + 1]);
      Dyz[f] = wy * dy + wz * dz;
    }
  }
  // output of the centre cell c = q-2
  const int c = q - 2;
  const int jg = jj + ty, kg = kk + tx;
  if (c >= i_start && c < i_end && jg < g.n[1] && kg < g.n[2]) {
    float D[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f)
      D[f] = wx * ((ms.F4[f] - Fn[f]) + 8.0f * (ms.F1[f] - ms.F3[f])) + ms.Dyz2[f];
    const int cell = cell_of(g, c, jg, kg);
    const bool nb = near_boundary(g, c, jg, kg);
    Img im;
    if (nb) make_img(g, c, jg, kg, im);
    if (STAGE < 3) {
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        const float u0 = __ldg(a.u0.f[f] + cell);
        float v = u0 - dt * D[f];
        if (f == PH) v *= decay;
        store_cell(a.out.f[f], cell, nb, im, f, v);
      }
    } else {
      float sv[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        float *hp = a.hi.f[f];
        float *lp = a.lo.f[f];
        const float h = hp[cell], l = lp[cell];
        float e;
        if (f == PH) {
          float t;
          two_sum(h, l - dt * D[f], sv[f], t);
          const float pr = sv[f] * decay;
          const float pe = fmaf(sv[f], decay, -pr);
          two_sum(pr, pe + t * decay, sv[f], e);
        } else {
          two_sum(h, l - dt * D[f], sv[f], e);
        }
        store_cell(hp, cell, nb, im, f, sv[f]);
        store_cell(lp, cell, nb, im, f, e);
      }
      float cs, vv, ca, ein;
      speeds(sv, a.gm, a.gm1, cs, vv, ca, ein);
      store_cell(a.cc, cell, nb, im, NF, cs * a.cs_fac + vv * a.vv_fac + ca * a.ca_fac);
    }
  }
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    ms.F4[f] = ms.F3[f];
    ms.F3[f] = ms.F2[f];
    ms.F2[f] = ms.F1[f];
    ms.F1[f] = Fn[f];
    ms.Dyz2[f] = ms.Dyz1[f];
    ms.Dyz1[f] = need_yz ? Dyz[f] : 0.0f;
  }
}

struct Item {
  int tj, tk, i_start, i_end;
};

__device__ __forceinline__ Item item_of(const RkArgs &a, int it) {
  Item r;
  const int per_chunk = a.tiles_j * a.tiles_k;
  const int ch = it / per_chunk, rem = it % per_chunk;
  r.tj = rem / a.tiles_k;
  r.tk = rem % a.tiles_k;
  r.i_start = a.i0 + ch * a.L;
  r.i_end = min(a.i1, r.i_start + a.L);
  return r;
}

// Producer cursor over the (item, plane) sequence of this CTA.
struct RkCursor {
  int it, q;
  Item cur;
  __device__ void begin(const RkArgs &a) {
    it = blockIdx.x;
    if (it < a.items) {
      cur = item_of(a, it);
      q = cur.i_start - 2;
    }
  }
  __device__ bool valid(const RkArgs &a) const { return it < a.items; }
  __device__ void next(const RkArgs &a) {
    if (++q > cur.i_end + 1) {
      it += gridDim.x;
      if (it < a.items) {
        cur = item_of(a, it);
        q = cur.i_start - 2;
      }
    }
  }
};

template <int STAGE>
__global__ void __launch_bounds__(NTHR, 2)
rk_tiled_kernel(const __grid_constant__ CUtensorMap tm, const RkArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  RkSmem &sm = *reinterpret_cast<RkSmem *>(smem_raw);
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int b = 0; b < NBUF; ++b) mbar_init(&sm.bar[b], 1);
    sm.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if ((int)blockIdx.x >= a.items) return;
  const float ch2 = (float)a.sc->ch2;
  const float dt = (float)a.sc->dts[STAGE];
  const float decay = (float)a.sc->ph_decay[STAGE];

  RkCursor prod;
  int issued = 0;
  if (tid == 0) {
    prod.begin(a);
    for (int b = 0; b < NBUF && prod.valid(a); ++b) {
      mbar_expect_tx(&sm.bar[b], PLANE_BYTES);
      tma4(&tm, sm.plane[b], &sm.bar[b], prod.cur.tk * TK, prod.cur.tj * TJ, prod.q + a.g.m[0], 0);
      prod.next(a);
      ++issued;
    }
  }
  int seq = 0;
  March ms;
  for (int it = blockIdx.x; it < a.items; it += gridDim.x) {
    const Item itm = item_of(a, it);
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      ms.F1[f] = ms.F2[f] = ms.F3[f] = ms.F4[f] = 0.0f;
      ms.Dyz1[f] = ms.Dyz2[f] = 0.0f;
    }
    for (int q = itm.i_start - 2; q <= itm.i_end + 1; ++q, ++seq) {
      const int b = (int)(seq % NBUF);
      if (tid == 0 && !mbar_wait(&sm.bar[b], (unsigned)((seq / NBUF) & 1), a.wait_limit))
        sm.abort = 1;
      __syncthreads();
      if (sm.abort) {
        if (tid == 0) {
          atomicOr(a.err, ERRBIT_TIMEOUT);
          // drain the copies still in flight (bounded; the one whose wait
          // ran out included) before the CTA exits
          for (int s2 = seq; s2 < issued; ++s2)
            mbar_wait(&sm.bar[s2 % NBUF], (unsigned)((s2 / NBUF) & 1));
        }
        return;
      }
      const float *pl = reinterpret_cast<const float *>(sm.plane[b]);
      rk_plane<STAGE>(a, sm, pl, ms, q, itm.i_start, itm.i_end, itm.tj * TJ, itm.tk * TK, tid,
                      ch2, dt, decay);
      // every thread is past barrier (A) inside rk_plane: the plane buffer
      // is free; refill it with the plane NBUF ahead
      if (tid == 0 && prod.valid(a)) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&sm.bar[b], PLANE_BYTES);
        tma4(&tm, sm.plane[b], &sm.bar[b], prod.cur.tk * TK, prod.cur.tj * TJ,
             prod.q + a.g.m[0], 0);
        prod.next(a);
        ++issued;
      }
      __syncthreads();  // (B) fy/fz reads done before the next plane's writes
    }
  }
}

// ---------------------------------------------------------------------------
// Artificial viscosity
// ---------------------------------------------------------------------------
// ---- x / y line sweep ----
constexpr int LK = 128;       // k cells per CTA
constexpr int LBOX = LK + 4;  // k box of the TMA copies
constexpr int LNB = 5;        // slots (3 planes in use, 2 in flight; 6 measured slower)
constexpr int L_HI = 0;
constexpr int L_LO = (NF * LBOX * 4 + 127) / 128 * 128;
constexpr int L_CC = L_LO + L_LO;
constexpr int L_SLOT = L_CC + (LBOX * 4 + 127) / 128 * 128;
constexpr unsigned L_TX = 2 * NF * LBOX * 4 + LBOX * 4;  // bytes per slot fill
// x sweep with the last Runge-Kutta update deferred into it: the third
// block of a slot holds the stage's right-hand side D (9 fields) in place
// of the characteristic speed
constexpr int L_D = L_CC;
constexpr int L_SLOT_D = L_D + L_LO;
constexpr unsigned L_TX_D = 3 * NF * LBOX * 4;

constexpr int LCW = LK / 32;  // consumer warps; one more warp issues the copies

template <bool DEFER>
struct __align__(128) LineSmemT {
  unsigned char slot[LNB][DEFER ? L_SLOT_D : L_SLOT];
  unsigned long long full[LNB];   // copy of the slot landed (1 arrival + bytes)
  unsigned long long empty[LNB];  // slot read by every consumer warp (LCW arrivals)
};
using LineSmem = LineSmemT<false>;

// One field of U^{n+1} = (h, l) - dt D as a compensated pair (s, e), with
// the GLM damping of ph: the last Runge-Kutta stage's update, operation for
// operation as rk_pipe_kernel<3> forms it (s32_rk.cu).
template <int F>
__device__ __forceinline__ void last_stage_field(float h, float l, float d, float dt,
                                                 float decay, float &sv, float &e) {
  if (F == PH) {
    float t;
    two_sum(h, fmaf(-dt, d, l), sv, t);
    ph_damp(sv, t, decay, sv, e);
  } else {
    two_sum(h, fmaf(-dt, d, l), sv, e);
  }
}

// Characteristic speed of a state's hi words, with the sums of squares
// gathered in rk_pipe_kernel<3>'s order.
__device__ __forceinline__ float last_stage_cc(const float u[NF], const AvArgs &a) {
  float mm = u[MX] * u[MX];
  mm = fmaf(u[MY], u[MY], mm);
  mm = fmaf(u[MZ], u[MZ], mm);
  float bb2 = u[BX] * u[BX];
  bb2 = fmaf(u[BY], u[BY], bb2);
  bb2 = fmaf(u[BZ], u[BZ], bb2);
  return char_speed(u[RO], mm, bb2, u[ET], a.gm, a.gm1, a.cs_fac, a.vv_fac, a.ca_fac);
}

struct LineItem {
  int kb, u, t0, t1;
};

template <int DIR>
__device__ __forceinline__ LineItem line_item(const AvArgs &a, int it, int kblocks, int nu) {
  LineItem r;
  r.kb = it % kblocks;
  const int r1 = it / kblocks;
  r.u = r1 % nu;
  const int ch = r1 / nu;
  r.t0 = a.r0 + ch * a.L;
  r.t1 = min(a.r1, r.t0 + a.L);
  return r;
}

template <int DIR>
struct LineCursor {
  int it, p;
  LineItem cur;
  __device__ void begin(const AvArgs &a, int kblocks, int nu, int items) {
    it = blockIdx.x;
    if (it < items) {
      cur = line_item<DIR>(a, it, kblocks, nu);
      p = cur.t0 - 2;
    }
  }
  __device__ bool valid(int items) const { return it < items; }
  __device__ void next(const AvArgs &a, int kblocks, int nu, int items) {
    if (++p > cur.t1 + 1) {
      it += gridDim.x;
      if (it < items) {
        cur = line_item<DIR>(a, it, kblocks, nu);
        p = cur.t0 - 2;
      }
    }
  }
};

template <int DIR, bool DEFER>
__device__ __forceinline__ void line_issue(const CUtensorMap *thi, const CUtensorMap *tlo,
                                           const CUtensorMap *t3, LineSmemT<DEFER> &sm, int s,
                                           const Geom &g, const LineItem &it, int p) {
  unsigned char *sl = sm.slot[s];
  const int k0 = it.kb * LK;
  // a plane across a face comes from the interior plane it images
  int side;
  const int ps = ghost_src(g, DIR, p, side);
  const int cj = DIR == 0 ? it.u + g.m[1] : ps + g.m[1];
  const int ci = DIR == 0 ? ps + g.m[0] : it.u + g.m[0];
  mbar_expect_tx(&sm.full[s], DEFER ? L_TX_D : L_TX);
  tma4(thi, sl + L_HI, &sm.full[s], k0, cj, ci, 0);
  tma4(tlo, sl + L_LO, &sm.full[s], k0, cj, ci, 0);
  if (DEFER)
    tma4(t3, sl + L_D, &sm.full[s], k0, cj, ci, 0);
  else
    tma3(t3, sl + L_CC, &sm.full[s], k0, cj, ci);
}

// Plane p of a line sweep's march: wait for its slot (seq), then the
// limited quantities of the thread's cell -- with DEFER formed from U^n and
// the deferred stage's D, with the mirror signs of the sweep axis's face for
// a plane copied from the interior plane it images -- and its speed.  false
// (error bit set) when the wait ran out.
template <int DIR, bool DEFER>
__device__ __forceinline__ bool line_row(LineSmemT<DEFER> &sm, int seq, int p, const AvArgs &a,
                                         int tid, float dt4, float decay4, W9 &wp, float &ccp) {
  constexpr int NB = LNB;
  const int s = seq % NB;
  if (!mbar_wait(&sm.full[s], (unsigned)((seq / NB) & 1), a.wait_limit)) {
    atomicOr(a.err, ERRBIT_TIMEOUT);
    return false;
  }
  const float *shi = reinterpret_cast<const float *>(sm.slot[s] + L_HI);
  float u[NF];
  if (DEFER) {
    const float *slo = reinterpret_cast<const float *>(sm.slot[s] + L_LO);
    const float *sd = reinterpret_cast<const float *>(sm.slot[s] + L_D);
    const int o = tid + 2;
    float e;
    last_stage_field<RO>(shi[RO * LBOX + o], slo[RO * LBOX + o], sd[RO * LBOX + o], dt4, decay4, u[RO], e);
    last_stage_field<MX>(shi[MX * LBOX + o], slo[MX * LBOX + o], sd[MX * LBOX + o], dt4, decay4, u[MX], e);
    last_stage_field<MY>(shi[MY * LBOX + o], slo[MY * LBOX + o], sd[MY * LBOX + o], dt4, decay4, u[MY], e);
    last_stage_field<MZ>(shi[MZ * LBOX + o], slo[MZ * LBOX + o], sd[MZ * LBOX + o], dt4, decay4, u[MZ], e);
    last_stage_field<BX>(shi[BX * LBOX + o], slo[BX * LBOX + o], sd[BX * LBOX + o], dt4, decay4, u[BX], e);
    last_stage_field<BY>(shi[BY * LBOX + o], slo[BY * LBOX + o], sd[BY * LBOX + o], dt4, decay4, u[BY], e);
    last_stage_field<BZ>(shi[BZ * LBOX + o], slo[BZ * LBOX + o], sd[BZ * LBOX + o], dt4, decay4, u[BZ], e);
    last_stage_field<ET>(shi[ET * LBOX + o], slo[ET * LBOX + o], sd[ET * LBOX + o], dt4, decay4, u[ET], e);
    last_stage_field<PH>(shi[PH * LBOX + o], slo[PH * LBOX + o], sd[PH * LBOX + o], dt4, decay4, u[PH], e);
    ccp = last_stage_cc(u, a);
  } else {
#pragma unroll
    for (int f = 0; f < NF; ++f) u[f] = shi[f * LBOX + tid + 2];
    ccp = reinterpret_cast<const float *>(sm.slot[s] + L_CC)[tid + 2];
  }
  if (p < 0 || p >= a.g.n[DIR]) {
    // the plane was copied from the interior plane it images: apply the
    // mirror signs of that face (none on a periodic axis)
    const unsigned neg = a.g.negmask[DIR][p < 0 ? 0 : 1];
#pragma unroll
    for (int f = 0; f < NF; ++f)
      if ((neg >> f) & 1u) u[f] = -u[f];
  }
  limited_w9(u, wp);
  return true;
}

// Release the slots a consumer warp is done with after plane `seq` of an
// item: the plane two back (read for the cell just finished, or a leading
// halo plane), and after the item's last plane the two trailing halo planes.
template <bool DEFER>
__device__ __forceinline__ void line_release(LineSmemT<DEFER> &sm, int seq, int lane, bool last) {
  constexpr int NB = LNB;
  __syncwarp();
  if (lane == 0) {
    mbar_arrive(&sm.empty[(seq - 2) % NB]);
    if (last) {
      mbar_arrive(&sm.empty[(seq - 1) % NB]);
      mbar_arrive(&sm.empty[seq % NB]);
    }
  }
}

// DEFER (x sweep only): the state is U^{n+1} = (hi, lo) - dt_4 D of the
// deferred last Runge-Kutta stage (rk_pipe_kernel<4>); t3 maps D in place of
// the characteristic speed.  Each plane's state and speed are formed as the
// plane arrives, and the sweep writes the speed of the cells it finishes
// for the y and z sweeps.
// Registers are held to three CTAs' worth (<= 128), and the march's first
// four planes run apart from its steady loop so that the queue's leading
// entries are dead there; the grid keeps two CTAs per SM (three resident
// measured 1.2x slower: their copies in flight crowd each other).
template <int DIR, bool DEFER>
__global__ void __launch_bounds__(LK + 32, 3)
av_line_kernel(const __grid_constant__ CUtensorMap thi, const __grid_constant__ CUtensorMap tlo,
               const __grid_constant__ CUtensorMap t3, const AvArgs a) {
  static_assert(!DEFER || DIR == 0, "the deferred update rides on the x sweep");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  LineSmemT<DEFER> &sm = *reinterpret_cast<LineSmemT<DEFER> *>(smem_raw);
  const Geom &g = a.g;
  constexpr int OTH = DIR == 0 ? 1 : 0;
  constexpr int NB = LNB;
  const int tid = threadIdx.x, lane = tid & 31;
  const int nk = g.n[2], nu = g.n[OTH];
  const int kblocks = (nk + LK - 1) / LK;
  const int chunks = (a.r1 - a.r0 + a.L - 1) / a.L;
  const int items = kblocks * nu * chunks;
  if (tid == 0) {
    for (int b = 0; b < NB; ++b) {
      mbar_init(&sm.full[b], 1);
      mbar_init(&sm.empty[b], LCW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();  // the only CTA barrier
  if ((int)blockIdx.x >= items) return;

  if (tid >= LK) {
    // producer warp: one lane fills the slots in plane order, each once the
    // consumer warps have released its previous plane
    if (tid == LK) {
      LineCursor<DIR> prod;
      prod.begin(a, kblocks, nu, items);
      int s = 0;
      for (; prod.valid(items); ++s) {
        const int b = s % NB;
        if (s >= NB && !mbar_wait(&sm.empty[b], (unsigned)(((s / NB) - 1) & 1))) {
          atomicOr(a.err, ERRBIT_TIMEOUT);
          break;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        line_issue<DIR, DEFER>(&thi, &tlo, &t3, sm, b, g, prod.cur, prod.p);
        prod.next(a, kblocks, nu, items);
      }
      // the last copies land before the CTA exits (bounded)
      for (int s2 = s > NB ? s - NB : 0; s2 < s; ++s2)
        mbar_wait(&sm.full[s2 % NB], (unsigned)((s2 / NB) & 1));
    }
    return;
  }

  const float fac = (float)(g.dsi[DIR] * a.sc->dt);
  const float dt4 = DEFER ? (float)a.sc->dts[3] : 0.f;
  const float decay4 = DEFER ? (float)a.sc->ph_decay[3] : 0.f;
  int seq = 0;
  // limiter state on field pairs: W9 holds (ro, mx) (my, mz) (bx, by) (bz, ph)
  // as packed pairs and ro*e alone
  const float2 ep2 = vs<float2>(a.ep), fh2 = vs<float2>(a.fh), mfac2 = vs<float2>(-fac);
  for (int it = blockIdx.x; it < items; it += gridDim.x) {
    const LineItem li = line_item<DIR>(a, it, kblocks, nu);
    const int k = li.kb * LK + tid;
    const bool active = k < nk;
    // the first four planes of the item (t0-2 .. t0+1) give the limited
    // quantities of planes t0, t0+1, the slope of plane t0 and the flux of
    // face t0 - 1/2; they run apart from the steady loop, so the queue's
    // leading entries are dead there
    W9 w0, w1, dq0, F0;
    float cc0, cc1;
    {
      W9 wm2, wm1;
      float ccm1, cx;
      if (!line_row<DIR, DEFER>(sm, seq, li.t0 - 2, a, tid, dt4, decay4, wm2, cx)) return;
      ++seq;
      if (!line_row<DIR, DEFER>(sm, seq, li.t0 - 1, a, tid, dt4, decay4, wm1, ccm1)) return;
      ++seq;
      if (!line_row<DIR, DEFER>(sm, seq, li.t0, a, tid, dt4, decay4, w0, cc0)) return;
      line_release<DEFER>(sm, seq, lane, false);
      ++seq;
      if (!line_row<DIR, DEFER>(sm, seq, li.t0 + 1, a, tid, dt4, decay4, w1, cc1)) return;
      // -1/2 of the face speed 0.5 (cc[t-1] + cc[t])
      const float hcc = -0.25f * (ccm1 + cc0);
      const float2 hcc2 = vs<float2>(hcc);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float2 dqm = dqq_t(wm2.p[i], wm1.p[i], w0.p[i], ep2);
        dq0.p[i] = dqq_t(wm1.p[i], w0.p[i], w1.p[i], ep2);
        F0.p[i] = flux_t(wm1.p[i], w0.p[i], dqm, dq0.p[i], hcc2, fh2);
      }
      const float dqm = dqq_t(wm2.s, wm1.s, w0.s, a.ep);
      dq0.s = dqq_t(wm1.s, w0.s, w1.s, a.ep);
      F0.s = flux_t(wm1.s, w0.s, dqm, dq0.s, hcc, a.fh);
      line_release<DEFER>(sm, seq, lane, false);
      ++seq;
    }
    for (int p = li.t0 + 2; p <= li.t1 + 1; ++p, ++seq) {
      W9 wp;
      float ccp;
      if (!line_row<DIR, DEFER>(sm, seq, p, a, tid, dt4, decay4, wp, ccp)) return;
      // centre cell t = p - 2; its plane sits two slots back
      const int t = p - 2;
      const int sc_ = (int)((seq - 2) % LNB);
      const float *chi = reinterpret_cast<const float *>(sm.slot[sc_] + L_HI);
      const float *clo = reinterpret_cast<const float *>(sm.slot[sc_] + L_LO);
      const float *cd = reinterpret_cast<const float *>(sm.slot[sc_] + (DEFER ? L_D : L_LO));
      const float cct = cc0;  // speed of the centre cell
      const float hcc = -0.25f * (cc0 + cc1);
      const float2 hcc2 = vs<float2>(hcc);
      W9 dF;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float2 dq1 = dqq_t(w0.p[i], w1.p[i], wp.p[i], ep2);
        const float2 F1 = flux_t(w0.p[i], w1.p[i], dq0.p[i], dq1, hcc2, fh2);
        dF.p[i] = vsub(F1, F0.p[i]);
        F0.p[i] = F1;
        dq0.p[i] = dq1;
      }
      {
        const float dq1 = dqq_t(w0.s, w1.s, wp.s, a.ep);
        const float F1 = flux_t(w0.s, w1.s, dq0.s, dq1, hcc, a.fh);
        dF.s = vsub(F1, F0.s);
        F0.s = F1;
        dq0.s = dq1;
      }
      w0 = w1;
      w1 = wp;
      cc0 = cc1;
      cc1 = ccp;
      if (active) {
        const int x0 = DIR == 0 ? t : li.u;
        const int x1 = DIR == 0 ? li.u : t;
        const int cell = cell_of(g, x0, x1, k);
        const int o = tid + 2;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int f0 = field_of(2 * i), f1 = field_of(2 * i + 1);
          float2 h = make_float2(chi[f0 * LBOX + o], chi[f1 * LBOX + o]);
          float2 l = make_float2(clo[f0 * LBOX + o], clo[f1 * LBOX + o]);
          if (DEFER) {
            // the centre's U^{n+1} pair, formed again from its slot
            if (i == 0) {
              last_stage_field<RO>(h.x, l.x, cd[RO * LBOX + o], dt4, decay4, h.x, l.x);
              last_stage_field<MX>(h.y, l.y, cd[MX * LBOX + o], dt4, decay4, h.y, l.y);
            } else if (i == 1) {
              last_stage_field<MY>(h.x, l.x, cd[MY * LBOX + o], dt4, decay4, h.x, l.x);
              last_stage_field<MZ>(h.y, l.y, cd[MZ * LBOX + o], dt4, decay4, h.y, l.y);
            } else if (i == 2) {
              last_stage_field<BX>(h.x, l.x, cd[BX * LBOX + o], dt4, decay4, h.x, l.x);
              last_stage_field<BY>(h.y, l.y, cd[BY * LBOX + o], dt4, decay4, h.y, l.y);
            } else {
              last_stage_field<BZ>(h.x, l.x, cd[BZ * LBOX + o], dt4, decay4, h.x, l.x);
              last_stage_field<PH>(h.y, l.y, cd[PH * LBOX + o], dt4, decay4, h.y, l.y);
            }
          }
          float2 sv, e;
          two_sum(h, vfma(dF.p[i], mfac2, l), sv, e);
          // interior only: the shell kernel fills the images
          a.hi2.f[f0][cell] = sv.x;
          a.hi2.f[f1][cell] = sv.y;
          a.lo2.f[f0][cell] = e.x;
          a.lo2.f[f1][cell] = e.y;
        }
        {
          float h = chi[ET * LBOX + o], l = clo[ET * LBOX + o];
          if (DEFER) last_stage_field<ET>(h, l, cd[ET * LBOX + o], dt4, decay4, h, l);
          float sv, e;
          two_sum(h, vfma(dF.s, -fac, l), sv, e);
          a.hi2.f[ET][cell] = sv;
          a.lo2.f[ET][cell] = e;
        }
        if (DEFER) a.cc_out[cell] = cct;  // read by the y and z sweeps
      }
      line_release<DEFER>(sm, seq, lane, p == li.t1 + 1);
    }
  }
}

// ---- z sweep (contiguous axis) ----
// Each warp loads 32 consecutive cells of a row (hi words and the
// characteristic speed; lanes across a face read the interior cell they
// image) and updates the inner 28, loading their lo words for the update;
// neighbours come from warp shuffles, the limiter runs on packed field
// pairs.  The kernel is latency-bound and lives on warps in flight: 56
// registers give nine 128-thread CTAs per SM, and every variant that held
// more registers measured slower (the next segment's loads issued early:
// 1.2x; lo loaded with hi: 1.3x; a register cap with spills: 2.3x).
// Staging the segments in shared memory by TMA, a slot ring per warp,
// measured 2x slower: copies of 128-byte boxes keep the TMA unit busy for
// little data.  The CFL candidate of the new state is folded into a
// per-block minimum.
struct ZSeg {
  float u[NF], l[NF], cc;
};

__device__ __forceinline__ void z_load(const AvArgs &a, int wi, int segs, int lane, ZSeg &z,
                                       int &c, int &k) {
  const Geom &g = a.g;
  const int sg = wi % segs;
  const int row = wi / segs;
  const int j = row % g.n[1];
  const int i = row / g.n[1];
  k = sg * 28 + lane - 2;  // interior k of this lane
  // a lane across a face reads the interior cell it images (lanes past the
  // ghost layer, whose values no output uses, stay on its last cell)
  int side;
  const int ks = ghost_src(g, 2, min(k, g.n[2] + 1), side);
  c = cell_of(g, i, j, ks);
#pragma unroll
  for (int f = 0; f < NF; ++f) z.u[f] = __ldg(a.hi.f[f] + c);
  if (side >= 0) {
    const unsigned neg = g.negmask[2][side];
#pragma unroll
    for (int f = 0; f < NF; ++f)
      if ((neg >> f) & 1u) z.u[f] = -z.u[f];
  }
  z.cc = __ldg(a.cc + c);
}

template <bool MON>
__global__ void __launch_bounds__(128)
av_z_kernel(const AvArgs a) {
  const Geom &g = a.g;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nk = g.n[2];
  const int segs = (nk + 27) / 28;
  const int rows = g.n[0] * g.n[1];
  const int work = rows * segs;
  const float fac = (float)(g.dsi[2] * a.sc->dt);
  const int warps = gridDim.x * (blockDim.x >> 5);
  float best = 1.e10f;
  bool bad = false;
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // MON: ro, mx, my, mz, et, ph^2
  for (int wi = blockIdx.x * (blockDim.x >> 5) + wid; wi < work; wi += warps) {
    ZSeg cur;
    int c, k;
    z_load(a, wi, segs, lane, cur, c, k);
    W9 dF;
    z_flux_diff(cur.u, cur.cc, a.ep, a.fh, dF);
    if (lane >= 2 && lane < 30 && k < nk) {
      float s[NF], e[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) cur.l[f] = __ldg(a.lo.f[f] + c);
      av_update(cur.u, cur.l, dF, fac, s, e);
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        a.hi2.f[f][c] = s[f];  // interior only: the shell kernel fills the images
        a.lo2.f[f][c] = e[f];
      }
      if (MON) {
        // the monitors' sums of the new state, in FP64 from hi + lo
        acc[0] += (double)s[RO] + (double)e[RO];
        acc[1] += (double)s[MX] + (double)e[MX];
        acc[2] += (double)s[MY] + (double)e[MY];
        acc[3] += (double)s[MZ] + (double)e[MZ];
        acc[4] += (double)s[ET] + (double)e[ET];
        const double ph = (double)s[PH] + (double)e[PH];
        acc[5] += ph * ph;
      }
      if (a.partial) {
        // CFL candidate of the new state (mhd_integrator_host.hpp:303-334)
        float cs, vv, ca, ein;
        speeds(s, a.gm, a.gm1, cs, vv, ca, ein);
        const float tv = cs + vv + ca;
        best = fminf(best, a.cfl_dx / tv);
        bad |= !(s[RO] > 0.0f) || !(ein >= 0.0f) || !isfinite(tv);
      }
    }
  }
  if (a.partial) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = fminf(best, __shfl_xor_sync(0xffffffffu, best, o));
    __shared__ float red[4];
    if (lane == 0) red[wid] = best;
    if (bad) atomicOr(a.err, ERRBIT_NONFINITE);
    __syncthreads();
    if (threadIdx.x == 0) {
      float b = red[0];
      for (int w2 = 1; w2 < (int)(blockDim.x >> 5); ++w2) b = fminf(b, red[w2]);
      a.partial[blockIdx.x] = b;
    }
  }
  if (MON) {
    __shared__ double mred[4][6];
#pragma unroll
    for (int q = 0; q < 6; ++q) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
      if (lane == 0) mred[wid][q] = acc[q];
    }
    __syncthreads();
    if (threadIdx.x < 6) {
      double v = 0.0;
      for (int w2 = 0; w2 < (int)(blockDim.x >> 5); ++w2) v += mred[w2][threadIdx.x];
      a.mon[blockIdx.x * 6 + threadIdx.x] = v;
    }
  }
}

// ---- z sweep as a streaming line (sweep variant 2) ----
// The x / y line structure applied to the contiguous axis: a CTA owns ZK
// consecutive k cells of one i plane and walks a chunk of j rows; per row a
// producer warp copies hi, lo and the characteristic speed of the segment
// (k box of 132 from 2 cells before it) into a ring slot by TMA, and four
// consumer warps, each on 32 consecutive cells of which it updates the
// inner 28, take their neighbours by shuffles (z_flux_diff, as
// av_z_kernel).  A lane across a k face reads the interior cell it images:
// in the segment's own box for a mirror face, or, for a periodic face, in
// an 8-word box copied from the far end of the row.  Rows are independent,
// so the ring only keeps copies in flight; the CFL candidate of the new
// state is folded into a per-CTA minimum.
constexpr int ZK = 112;  // k cells a CTA updates per row (4 warps x 28)
constexpr int ZWB = 8;   // k box of the wrap copies
constexpr int ZNB = 6;   // ring slots
constexpr int ZL_HI = 0;
constexpr int ZL_LO = L_LO;
constexpr int ZL_CC = 2 * L_LO;
constexpr int ZL_WL = ZL_CC + (LBOX * 4 + 127) / 128 * 128;
constexpr int ZL_WLC = ZL_WL + (NF * ZWB * 4 + 127) / 128 * 128;
constexpr int ZL_WR = ZL_WLC + 128;
constexpr int ZL_WRC = ZL_WR + (NF * ZWB * 4 + 127) / 128 * 128;
constexpr int ZL_SLOT = ZL_WRC + 128;
constexpr unsigned ZL_TX = 2 * NF * LBOX * 4 + LBOX * 4;
constexpr unsigned ZL_TXW = (NF + 1) * ZWB * 4;

struct __align__(128) ZLineSmem {
  unsigned char slot[ZNB][ZL_SLOT];
  unsigned long long full[ZNB];
  unsigned long long empty[ZNB];
};

struct ZItem {
  int kb, i, t0, t1;
};

__device__ __forceinline__ ZItem z_item(const AvArgs &a, int it, int kblocks) {
  ZItem r;
  r.kb = it % kblocks;
  const int r1 = it / kblocks;
  r.i = r1 % a.g.n[0];
  const int ch = r1 / a.g.n[0];
  r.t0 = ch * a.L;
  r.t1 = min(a.g.n[1], r.t0 + a.L);
  return r;
}

__global__ void __launch_bounds__(LK + 32, 2)
av_zline_kernel(const __grid_constant__ CUtensorMap thi, const __grid_constant__ CUtensorMap tlo,
                const __grid_constant__ CUtensorMap tcc, const __grid_constant__ CUtensorMap twh,
                const __grid_constant__ CUtensorMap twc, const AvArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  ZLineSmem &sm = *reinterpret_cast<ZLineSmem *>(smem_raw);
  const Geom &g = a.g;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int nk = g.n[2];
  const int kblocks = (nk + ZK - 1) / ZK;
  const int chunks = (g.n[1] + a.L - 1) / a.L;
  const int items = kblocks * g.n[0] * chunks;
  const int xl = nk - nk % 4;  // first array column of the left wrap copy
  if (tid == 0) {
    for (int b = 0; b < ZNB; ++b) {
      mbar_init(&sm.full[b], 1);
      mbar_init(&sm.empty[b], LCW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();  // the only CTA-wide barrier
  if (tid >= LK) {
    // producer warp: one lane fills the slots row by row
    if (tid == LK) {
      int s = 0;
      bool stop = false;
      for (int it = blockIdx.x; it < items && !stop; it += gridDim.x) {
        const ZItem z = z_item(a, it, kblocks);
        // wrap copies for the blocks with lanes across a k face (the last
        // lane of block kb sits at k = kb * ZK + 113)
        const bool wl = g.periodic[2] && !g.ext[2][0] && z.kb == 0;
        const bool wr = g.periodic[2] && !g.ext[2][1] && z.kb * ZK + 4 * 28 + 1 >= nk;
        const unsigned tx = ZL_TX + (wl ? ZL_TXW : 0u) + (wr ? ZL_TXW : 0u);
        for (int j = z.t0; j < z.t1; ++j, ++s) {
          const int b = s % ZNB;
          if (s >= ZNB && !mbar_wait(&sm.empty[b], (unsigned)(((s / ZNB) - 1) & 1))) {
            atomicOr(a.err, ERRBIT_TIMEOUT);
            stop = true;
            break;
          }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          unsigned char *sl = sm.slot[b];
          const int x = z.kb * ZK, y = j + g.m[1], zc = z.i + g.m[0];
          mbar_expect_tx(&sm.full[b], tx);
          tma4(&thi, sl + ZL_HI, &sm.full[b], x, y, zc, 0);
          tma4(&tlo, sl + ZL_LO, &sm.full[b], x, y, zc, 0);
          tma3(&tcc, sl + ZL_CC, &sm.full[b], x, y, zc);
          if (wl) {
            tma4(&twh, sl + ZL_WL, &sm.full[b], xl, y, zc, 0);
            tma3(&twc, sl + ZL_WLC, &sm.full[b], xl, y, zc);
          }
          if (wr) {
            tma4(&twh, sl + ZL_WR, &sm.full[b], 0, y, zc, 0);
            tma3(&twc, sl + ZL_WRC, &sm.full[b], 0, y, zc);
          }
        }
      }
      // the last copies land before the CTA exits (bounded)
      for (int s2 = s > ZNB ? s - ZNB : 0; s2 < s; ++s2)
        mbar_wait(&sm.full[s2 % ZNB], (unsigned)((s2 / ZNB) & 1));
    }
    return;
  }

  const float fac = (float)(g.dsi[2] * a.sc->dt);
  float best = 1.e10f;
  bool bad = false, stop = false;
  int seq = 0;
  for (int it = blockIdx.x; it < items && !stop; it += gridDim.x) {
    const ZItem z = z_item(a, it, kblocks);
    const int k = z.kb * ZK + 28 * w + lane - 2;
    const int kk = min(k, nk + 1);
    // where this lane's words sit in a slot, and the mirror signs they take
    int region = 0, off = 28 * w + lane;
    unsigned neg = 0;
    if (kk < 0 || kk >= nk) {
      int side;
      const int img = ghost_src(g, 2, kk, side);
      if (side < 0) {
        off = kk - (z.kb * ZK - 2);  // a face shared with a neighbour: its ghost cell
      } else if (g.periodic[2]) {
        region = kk < 0 ? 1 : 2;
        off = img + 2 - (kk < 0 ? xl : 0);
      } else {
        off = img - (z.kb * ZK - 2);
        neg = g.negmask[2][side];
      }
    }
    const bool out = lane >= 2 && lane < 30 && k < nk;
    for (int j = z.t0; j < z.t1; ++j, ++seq) {
      const int s = seq % ZNB;
      if (!mbar_wait(&sm.full[s], (unsigned)((seq / ZNB) & 1))) {
        // leave the loops (every consumer warp still meets the barrier below)
        atomicOr(a.err, ERRBIT_TIMEOUT);
        stop = true;
        break;
      }
      const unsigned char *sl = sm.slot[s];
      const float *h = reinterpret_cast<const float *>(
          sl + (region == 0 ? ZL_HI : region == 1 ? ZL_WL : ZL_WR));
      const float *cp = reinterpret_cast<const float *>(
          sl + (region == 0 ? ZL_CC : region == 1 ? ZL_WLC : ZL_WRC));
      const int stride = region == 0 ? LBOX : ZWB;
      float u[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        u[f] = h[f * stride + off];
        if ((neg >> f) & 1u) u[f] = -u[f];
      }
      W9 dF;
      z_flux_diff(u, cp[off], a.ep, a.fh, dF);
      if (out) {
        const float *lo = reinterpret_cast<const float *>(sl + ZL_LO);
        float l[NF], sv[NF], e[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) l[f] = lo[f * LBOX + 28 * w + lane];
        av_update(u, l, dF, fac, sv, e);
        const int c = cell_of(g, z.i, j, k);
#pragma unroll
        for (int f = 0; f < NF; ++f) {
          a.hi2.f[f][c] = sv[f];  // interior only: the shell kernel fills the images
          a.lo2.f[f][c] = e[f];
        }
        if (a.partial) {
          float cs, vv, ca, ein;
          speeds(sv, a.gm, a.gm1, cs, vv, ca, ein);
          const float tv = cs + vv + ca;
          best = fminf(best, a.cfl_dx / tv);
          bad |= !(sv[RO] > 0.0f) || !(ein >= 0.0f) || !isfinite(tv);
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&sm.empty[s]);
    }
  }
  if (a.partial) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = fminf(best, __shfl_xor_sync(0xffffffffu, best, o));
    __shared__ float red[LCW];
    if (lane == 0) red[w] = best;
    if (bad) atomicOr(a.err, ERRBIT_NONFINITE);
    asm volatile("bar.sync 1, %0;" ::"r"(LK) : "memory");  // the consumer warps only
    if (tid == 0) {
      float b = red[0];
      for (int w2 = 1; w2 < LCW; ++w2) b = fminf(b, red[w2]);
      a.partial[blockIdx.x] = b;
    }
  }
}

// ---- y and z sweeps in one pass (y sweep variant 3) ----
// The two sweeps of one i plane fused: a CTA owns ZK consecutive k cells of
// a plane and marches along j over a chunk of rows, as the z line sweep
// does.  Per row a producer warp copies hi, lo and the characteristic speed
// of the x-swept state (k box of 132 from 2 cells before the block; for a
// periodic k face also the 8-wide wrap boxes of hi, lo and the speed) into
// a ring slot by TMA; rows across a j face come from the interior row they
// image.  Each lane of the four consumer warps runs the y sweep down its
// column with the line sweep's register queue, which yields the y-swept
// state of the row two back; the warp then runs the z sweep on that row by
// shuffles (z_flux_diff) and updates its inner 28 lanes.  A lane across a
// k face runs the y sweep of the interior column it images and takes the
// face's mirror signs afterwards -- the values the separate z sweep reads
// there -- so the pass gives the bits of the y line sweep followed by the z
// sweep, without writing the y-swept state and reading it back (144 B per
// cell).  The CFL candidate of the new state, and with MON the monitors'
// FP64 sums, are folded into per-CTA partials as the z sweep folds them.
// The first four rows of an item run apart from the steady loop, so the
// queue's leading entries are dead there: 128 registers, three CTAs (15
// warps) per SM beside 219 KB of slots.
constexpr int YZ_NB = 6;                                     // ring slots
constexpr int YZ_LO = L_LO;                                  // hi at 0, then lo
constexpr int YZ_CC = 2 * L_LO;                              // the speed
constexpr int YZ_WB = (NF * ZWB * 4 + 127) / 128 * 128;      // one 8-wide wrap box of 9 fields
constexpr int YZ_WL = YZ_CC + (LBOX * 4 + 127) / 128 * 128;  // left wrap: hi, lo, speed
constexpr int YZ_WR = YZ_WL + 2 * YZ_WB + 128;               // right wrap
constexpr int YZ_SLOT = YZ_WR + 2 * YZ_WB + 128;
constexpr unsigned YZ_TXW = (2 * NF + 1) * ZWB * 4;  // bytes of one side's wrap copies

struct __align__(128) YzSmem {
  unsigned char slot[YZ_NB][YZ_SLOT];
  unsigned long long full[YZ_NB];   // the row's copies landed
  unsigned long long empty[YZ_NB];  // the row read by every consumer warp (LCW arrivals)
};

// A consumer lane's place in a slot: offsets of its hi, lo and speed words
// (the main box or a wrap box) and the stride between fields.
struct YzLane {
  int o_hi, o_lo, o_cc, stride, off;
};

// Row p of the fused sweeps' march: wait for its slot (seq), then the
// limited quantities of the lane's column -- with the mirror signs of the
// j face for a row copied from the interior row it images -- and its speed.
// false (error bit set) when the wait ran out.
__device__ __forceinline__ bool yz_row(YzSmem &sm, int seq, long long limit, const YzLane &ln,
                                       int p, const Geom &g, W9 &wp, float &ccp,
                                       unsigned *err) {
  const int s = seq % YZ_NB;
  if (!mbar_wait(&sm.full[s], (unsigned)((seq / YZ_NB) & 1), limit)) {
    atomicOr(err, ERRBIT_TIMEOUT);
    return false;
  }
  const float *sh = reinterpret_cast<const float *>(sm.slot[s] + ln.o_hi);
  float u[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) u[f] = sh[f * ln.stride + ln.off];
  if (p < 0 || p >= g.n[1]) {
    const unsigned neg = g.negmask[1][p < 0 ? 0 : 1];
#pragma unroll
    for (int f = 0; f < NF; ++f)
      if ((neg >> f) & 1u) u[f] = -u[f];
  }
  limited_w9(u, wp);
  ccp = reinterpret_cast<const float *>(sm.slot[s] + ln.o_cc)[ln.off];
  return true;
}

// Release the slots a warp is done with after row `seq` of an item: the row
// two back (the centre just finished, or a leading halo row), and after the
// item's last row the two trailing halo rows.
__device__ __forceinline__ void yz_release(YzSmem &sm, int seq, int lane, bool last) {
  __syncwarp();
  if (lane == 0) {
    mbar_arrive(&sm.empty[(seq - 2) % YZ_NB]);
    if (last) {
      mbar_arrive(&sm.empty[(seq - 1) % YZ_NB]);
      mbar_arrive(&sm.empty[seq % YZ_NB]);
    }
  }
}

template <bool MON>
__global__ void __launch_bounds__(LK + 32, 3)
av_yz_kernel(const __grid_constant__ CUtensorMap thi, const __grid_constant__ CUtensorMap tlo,
             const __grid_constant__ CUtensorMap tcc, const __grid_constant__ CUtensorMap twh,
             const __grid_constant__ CUtensorMap twl, const __grid_constant__ CUtensorMap twc,
             const AvArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  YzSmem &sm = *reinterpret_cast<YzSmem *>(smem_raw);
  const Geom &g = a.g;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int nk = g.n[2];
  const int kblocks = (nk + ZK - 1) / ZK;
  const int chunks = (g.n[1] + a.L - 1) / a.L;
  const int items = kblocks * g.n[0] * chunks;
  const int xl = nk - nk % 4;  // first array column of the left wrap copy
  if (tid == 0) {
    for (int b = 0; b < YZ_NB; ++b) {
      mbar_init(&sm.full[b], 1);
      mbar_init(&sm.empty[b], LCW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();  // the only CTA-wide barrier
  if (tid >= LK) {
    // producer warp: one lane fills the slots row by row, rows t0-2 .. t1+1
    // of each item
    if (tid == LK) {
      int s = 0;
      bool stop = false;
      for (int it = blockIdx.x; it < items && !stop; it += gridDim.x) {
        const ZItem z = z_item(a, it, kblocks);
        // wrap copies for the blocks with lanes across a periodic k face
        // (the last lane of block kb sits at k = kb * ZK + 113)
        const bool wl = g.periodic[2] && !g.ext[2][0] && z.kb == 0;
        const bool wr = g.periodic[2] && !g.ext[2][1] && z.kb * ZK + 4 * 28 + 1 >= nk;
        const unsigned tx = ZL_TX + (wl ? YZ_TXW : 0u) + (wr ? YZ_TXW : 0u);
        for (int p = z.t0 - 2; p <= z.t1 + 1; ++p, ++s) {
          const int b = s % YZ_NB;
          if (s >= YZ_NB && !mbar_wait(&sm.empty[b], (unsigned)(((s / YZ_NB) - 1) & 1))) {
            atomicOr(a.err, ERRBIT_TIMEOUT);
            stop = true;
            break;
          }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          unsigned char *sl = sm.slot[b];
          int side;
          const int ps = ghost_src(g, 1, p, side);  // a row across a j face: its image
          const int x = z.kb * ZK, y = ps + g.m[1], zc = z.i + g.m[0];
          mbar_expect_tx(&sm.full[b], tx);
          tma4(&thi, sl, &sm.full[b], x, y, zc, 0);
          tma4(&tlo, sl + YZ_LO, &sm.full[b], x, y, zc, 0);
          tma3(&tcc, sl + YZ_CC, &sm.full[b], x, y, zc);
          if (wl) {
            tma4(&twh, sl + YZ_WL, &sm.full[b], xl, y, zc, 0);
            tma4(&twl, sl + YZ_WL + YZ_WB, &sm.full[b], xl, y, zc, 0);
            tma3(&twc, sl + YZ_WL + 2 * YZ_WB, &sm.full[b], xl, y, zc);
          }
          if (wr) {
            tma4(&twh, sl + YZ_WR, &sm.full[b], 0, y, zc, 0);
            tma4(&twl, sl + YZ_WR + YZ_WB, &sm.full[b], 0, y, zc, 0);
            tma3(&twc, sl + YZ_WR + 2 * YZ_WB, &sm.full[b], 0, y, zc);
          }
        }
      }
      // the last copies land before the CTA exits (bounded)
      for (int s2 = s > YZ_NB ? s - YZ_NB : 0; s2 < s; ++s2)
        mbar_wait(&sm.full[s2 % YZ_NB], (unsigned)((s2 / YZ_NB) & 1));
    }
    return;
  }

  const float facy = (float)(g.dsi[1] * a.sc->dt);
  const float facz = (float)(g.dsi[2] * a.sc->dt);
  const float2 ep2 = vs<float2>(a.ep), fh2 = vs<float2>(a.fh), mfac2 = vs<float2>(-facy);
  float best = 1.e10f;
  bool bad = false, stop = false;
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // MON: ro, mx, my, mz, et, ph^2
  int seq = 0;
  for (int it = blockIdx.x; it < items && !stop; it += gridDim.x) {
    const ZItem z = z_item(a, it, kblocks);
    const int k = z.kb * ZK + 28 * w + lane - 2;
    const int kk = min(k, nk + 1);
    // where this lane's words sit in a slot, and the k face's mirror signs
    // its y-swept values take
    int region = 0, off = 28 * w + lane;
    unsigned negz = 0;
    if (kk < 0 || kk >= nk) {
      int side;
      const int img = ghost_src(g, 2, kk, side);
      if (side < 0) {
        off = kk - (z.kb * ZK - 2);  // a face shared with a neighbour: its ghost cell
      } else if (g.periodic[2]) {
        region = kk < 0 ? 1 : 2;
        off = img + 2 - (kk < 0 ? xl : 0);
      } else {
        off = img - (z.kb * ZK - 2);
        negz = g.negmask[2][side];
      }
    }
    YzLane ln;
    ln.o_hi = region == 0 ? 0 : region == 1 ? YZ_WL : YZ_WR;
    ln.o_lo = region == 0 ? YZ_LO : ln.o_hi + YZ_WB;
    ln.o_cc = region == 0 ? YZ_CC : ln.o_hi + 2 * YZ_WB;
    ln.stride = region == 0 ? LBOX : ZWB;
    ln.off = off;
    const bool out = lane >= 2 && lane < 30 && k < nk;
    // the y sweep's queue on field pairs, as av_line_kernel: the first four
    // rows of the item (t0-2 .. t0+1) give the limited quantities of rows
    // t0, t0+1, the slope of row t0 and the flux of face t0 - 1/2
    W9 w0, w1, dq0, F0;
    float cc0, cc1;
    {
      W9 wm2, wm1;
      float ccm1, cx;
      // (a wait that ran out leaves the loops; every consumer warp still
      // meets the barrier below)
      if (!yz_row(sm, seq, a.wait_limit, ln, z.t0 - 2, g, wm2, cx, a.err)) break;
      ++seq;
      if (!yz_row(sm, seq, a.wait_limit, ln, z.t0 - 1, g, wm1, ccm1, a.err)) break;
      ++seq;
      if (!yz_row(sm, seq, a.wait_limit, ln, z.t0, g, w0, cc0, a.err)) break;
      yz_release(sm, seq, lane, false);
      ++seq;
      if (!yz_row(sm, seq, a.wait_limit, ln, z.t0 + 1, g, w1, cc1, a.err)) break;
      // -1/2 of the face speed 0.5 (cc[t-1] + cc[t])
      const float hcc = -0.25f * (ccm1 + cc0);
      const float2 hcc2 = vs<float2>(hcc);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float2 dqm = dqq_t(wm2.p[i], wm1.p[i], w0.p[i], ep2);
        dq0.p[i] = dqq_t(wm1.p[i], w0.p[i], w1.p[i], ep2);
        F0.p[i] = flux_t(wm1.p[i], w0.p[i], dqm, dq0.p[i], hcc2, fh2);
      }
      const float dqm = dqq_t(wm2.s, wm1.s, w0.s, a.ep);
      dq0.s = dqq_t(wm1.s, w0.s, w1.s, a.ep);
      F0.s = flux_t(wm1.s, w0.s, dqm, dq0.s, hcc, a.fh);
      yz_release(sm, seq, lane, false);
      ++seq;
    }
    for (int p = z.t0 + 2; p <= z.t1 + 1; ++p, ++seq) {
      W9 wp;
      float ccp;
      if (!yz_row(sm, seq, a.wait_limit, ln, p, g, wp, ccp, a.err)) {
        stop = true;
        break;
      }
      // centre row t = p - 2; its copies sit two slots back
      const int t = p - 2;
      const int sc_ = (int)((seq - 2) % YZ_NB);
      const float *chi = reinterpret_cast<const float *>(sm.slot[sc_] + ln.o_hi);
      const float *clo = reinterpret_cast<const float *>(sm.slot[sc_] + ln.o_lo);
      const float cct = cc0;  // speed of the centre cell
      const float hcc = -0.25f * (cc0 + cc1);
      const float2 hcc2 = vs<float2>(hcc);
      W9 dF;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float2 dq1 = dqq_t(w0.p[i], w1.p[i], wp.p[i], ep2);
        const float2 F1 = flux_t(w0.p[i], w1.p[i], dq0.p[i], dq1, hcc2, fh2);
        dF.p[i] = vsub(F1, F0.p[i]);
        F0.p[i] = F1;
        dq0.p[i] = dq1;
      }
      {
        const float dq1 = dqq_t(w0.s, w1.s, wp.s, a.ep);
        const float F1 = flux_t(w0.s, w1.s, dq0.s, dq1, hcc, a.fh);
        dF.s = vsub(F1, F0.s);
        F0.s = F1;
        dq0.s = dq1;
      }
      w0 = w1;
      w1 = wp;
      cc0 = cc1;
      cc1 = ccp;
      // the y-swept state of the centre cell (the y line sweep's update)
      float sy[NF], ey[NF];
      const int st = ln.stride, o = ln.off;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int f0 = field_of(2 * i), f1 = field_of(2 * i + 1);
        const float2 h = make_float2(chi[f0 * st + o], chi[f1 * st + o]);
        const float2 l = make_float2(clo[f0 * st + o], clo[f1 * st + o]);
        float2 sv, e;
        two_sum(h, vfma(dF.p[i], mfac2, l), sv, e);
        sy[f0] = sv.x;
        sy[f1] = sv.y;
        ey[f0] = e.x;
        ey[f1] = e.y;
      }
      two_sum(chi[ET * st + o], vfma(dF.s, -facy, clo[ET * st + o]), sy[ET], ey[ET]);
      if (negz) {
#pragma unroll
        for (int f = 0; f < NF; ++f)
          if ((negz >> f) & 1u) {
            sy[f] = -sy[f];
            ey[f] = -ey[f];
          }
      }
      // the z sweep of row t
      W9 dFz;
      z_flux_diff(sy, cct, a.ep, a.fh, dFz);
      if (out) {
        float sv[NF], e[NF];
        av_update(sy, ey, dFz, facz, sv, e);
        const int c = cell_of(g, z.i, t, k);
#pragma unroll
        for (int f = 0; f < NF; ++f) {
          a.hi2.f[f][c] = sv[f];  // interior only: the shell kernel fills the images
          a.lo2.f[f][c] = e[f];
        }
        if (MON) {
          acc[0] += (double)sv[RO] + (double)e[RO];
          acc[1] += (double)sv[MX] + (double)e[MX];
          acc[2] += (double)sv[MY] + (double)e[MY];
          acc[3] += (double)sv[MZ] + (double)e[MZ];
          acc[4] += (double)sv[ET] + (double)e[ET];
          const double ph = (double)sv[PH] + (double)e[PH];
          acc[5] += ph * ph;
        }
        if (a.partial) {
          // CFL candidate of the new state (mhd_integrator_host.hpp:303-334)
          float cs, vv, ca, ein;
          speeds(sv, a.gm, a.gm1, cs, vv, ca, ein);
          const float tv = cs + vv + ca;
          best = fminf(best, a.cfl_dx / tv);
          bad |= !(sv[RO] > 0.0f) || !(ein >= 0.0f) || !isfinite(tv);
        }
      }
      yz_release(sm, seq, lane, p == z.t1 + 1);
    }
  }
  __shared__ float red[LCW];
  __shared__ double mred[LCW][6];
  if (a.partial) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = fminf(best, __shfl_xor_sync(0xffffffffu, best, o));
    if (lane == 0) red[w] = best;
    if (bad) atomicOr(a.err, ERRBIT_NONFINITE);
  }
  if (MON) {
#pragma unroll
    for (int q = 0; q < 6; ++q) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
      if (lane == 0) mred[w][q] = acc[q];
    }
  }
  asm volatile("bar.sync 1, %0;" ::"r"(LK) : "memory");  // the consumer warps only
  if (a.partial && tid == 0) {
    float b = red[0];
    for (int w2 = 1; w2 < LCW; ++w2) b = fminf(b, red[w2]);
    a.partial[blockIdx.x] = b;
  }
  if (MON && tid < 6) {
    double v = 0.0;
    for (int w2 = 0; w2 < LCW; ++w2) v += mred[w2][tid];
    a.mon[blockIdx.x * 6 + tid] = v;
  }
}

}  // namespace s32t

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

bool s32_tiled_supported(const Geom &g) {
  if (!g.s[0] || !g.s[1] || !g.s[2]) return false;
  if (g.m[0] != 2 || g.m[1] != 2 || g.m[2] != 2) return false;
  if ((g.t[2] * 4) % 16) return false;  // TMA row pitch: multiple of 16 bytes
  for (int a = 0; a < 3; ++a)
    if (g.n[a] < 2 * g.m[a]) return false;  // one ghost image per axis side
  if (g.cells >= (1LL << 31) / 9) return false;  // 32-bit cell offsets
  return encode_fn() != nullptr;
}

int s32_make_tmap(const Geom &g, const float *field0, size_t pitch_bytes, int kind,
                  void *tm_out) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return -1;
  cuuint64_t dims[4] = {(cuuint64_t)g.t[2], (cuuint64_t)g.t[1], (cuuint64_t)g.t[0], NF};
  cuuint64_t strides[3] = {(cuuint64_t)g.t[2] * 4, (cuuint64_t)g.t[2] * g.t[1] * 4,
                           (cuuint64_t)pitch_bytes};
  cuuint32_t box_rk[4] = {s32t::HK, s32t::HJ, 1, NF};
  cuuint32_t box_av[4] = {kind == 2 ? (cuuint32_t)s32t::ZWB : (cuuint32_t)s32t::LBOX, 1, 1, NF};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = fn((CUtensorMap *)tm_out, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void *)field0,
                  dims, strides, kind == 0 ? box_rk : box_av, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -2;
}

int s32_make_tmap_cc(const Geom &g, const float *cc, void *tm_out, int kbox) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return -1;
  cuuint64_t dims[3] = {(cuuint64_t)g.t[2], (cuuint64_t)g.t[1], (cuuint64_t)g.t[0]};
  cuuint64_t strides[2] = {(cuuint64_t)g.t[2] * 4, (cuuint64_t)g.t[2] * g.t[1] * 4};
  cuuint32_t box[3] = {(cuuint32_t)kbox, 1, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn((CUtensorMap *)tm_out, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)cc, dims,
                  strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -2;
}

int s32_configure() {
  const int rk = (int)sizeof(s32t::RkSmem);
  const int ln = (int)sizeof(s32t::LineSmem);
  const int lnd = (int)sizeof(s32t::LineSmemT<true>);
  const int zl = (int)sizeof(s32t::ZLineSmem);
  const int yz = (int)sizeof(s32t::YzSmem);
  cudaError_t e = cudaSuccess;
#define MISO_SET(k, b) \
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, b)
  MISO_SET(s32t::rk_tiled_kernel<0>, rk);
  MISO_SET(s32t::rk_tiled_kernel<1>, rk);
  MISO_SET(s32t::rk_tiled_kernel<2>, rk);
  MISO_SET(s32t::rk_tiled_kernel<3>, rk);
  MISO_SET((s32t::av_line_kernel<0, false>), ln);
  MISO_SET((s32t::av_line_kernel<1, false>), ln);
  MISO_SET((s32t::av_line_kernel<0, true>), lnd);
  MISO_SET(s32t::av_zline_kernel, zl);
  MISO_SET(s32t::av_yz_kernel<false>, yz);
  MISO_SET(s32t::av_yz_kernel<true>, yz);
#undef MISO_SET
  return e == cudaSuccess ? 0 : -1;
}

int s32_rk_items_range(const Geom &g, int L, int i0, int i1) {
  const int tj = (g.n[1] + s32t::TJ - 1) / s32t::TJ;
  const int tk = (g.n[2] + s32t::TK - 1) / s32t::TK;
  return tj * tk * ((i1 - i0 + L - 1) / L);
}

void s32_rk_items(const Geom &g, int L, int &tiles_j, int &tiles_k, int &items) {
  tiles_j = (g.n[1] + s32t::TJ - 1) / s32t::TJ;
  tiles_k = (g.n[2] + s32t::TK - 1) / s32t::TK;
  const int chunks = (g.n[0] + L - 1) / L;
  items = tiles_j * tiles_k * chunks;
}

void launch_s32_rk_tiled(const void *tm, const RkArgs &a, int stage, int grid, cudaStream_t st) {
  const CUtensorMap &m = *(const CUtensorMap *)tm;
  const size_t smem = sizeof(s32t::RkSmem);
  switch (stage) {
    case 0: s32t::rk_tiled_kernel<0><<<grid, s32t::NTHR, smem, st>>>(m, a); break;
    case 1: s32t::rk_tiled_kernel<1><<<grid, s32t::NTHR, smem, st>>>(m, a); break;
    case 2: s32t::rk_tiled_kernel<2><<<grid, s32t::NTHR, smem, st>>>(m, a); break;
    default: s32t::rk_tiled_kernel<3><<<grid, s32t::NTHR, smem, st>>>(m, a); break;
  }
}

void launch_s32_av_line(const void *tm_hi, const void *tm_lo, const void *tm3, const AvArgs &a,
                        int dir, bool defer, int grid, cudaStream_t st) {
  const CUtensorMap &h = *(const CUtensorMap *)tm_hi;
  const CUtensorMap &l = *(const CUtensorMap *)tm_lo;
  const CUtensorMap &c = *(const CUtensorMap *)tm3;
  const size_t smem = sizeof(s32t::LineSmem);
  if (dir == 0 && defer)
    s32t::av_line_kernel<0, true>
        <<<grid, s32t::LK + 32, sizeof(s32t::LineSmemT<true>), st>>>(h, l, c, a);
  else if (dir == 0)
    s32t::av_line_kernel<0, false><<<grid, s32t::LK + 32, smem, st>>>(h, l, c, a);
  else
    s32t::av_line_kernel<1, false><<<grid, s32t::LK + 32, smem, st>>>(h, l, c, a);
}

int s32_av_line_items(const Geom &g, int dir, int L, int r0, int r1) {
  const int oth = dir == 0 ? 1 : 0;
  return ((g.n[2] + s32t::LK - 1) / s32t::LK) * g.n[oth] * ((r1 - r0 + L - 1) / L);
}

void launch_s32_av_z(const AvArgs &a, int grid, cudaStream_t st) {
  if (a.mon)
    s32t::av_z_kernel<true><<<grid, 128, 0, st>>>(a);
  else
    s32t::av_z_kernel<false><<<grid, 128, 0, st>>>(a);
}


int s32_zline_per_sm() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, s32t::av_zline_kernel, s32t::LK + 32,
                                                    sizeof(s32t::ZLineSmem)) != cudaSuccess ||
      n < 1)
    n = 1;
  return n;
}

void launch_s32_av_zline(const void *tm_hi, const void *tm_lo, const void *tm_cc,
                         const void *tm_wh, const void *tm_wc, const AvArgs &a, int grid,
                         cudaStream_t st) {
  s32t::av_zline_kernel<<<grid, s32t::LK + 32, sizeof(s32t::ZLineSmem), st>>>(
      *(const CUtensorMap *)tm_hi, *(const CUtensorMap *)tm_lo, *(const CUtensorMap *)tm_cc,
      *(const CUtensorMap *)tm_wh, *(const CUtensorMap *)tm_wc, a);
}

int s32_yz_per_sm() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, s32t::av_yz_kernel<true>, s32t::LK + 32,
                                                    sizeof(s32t::YzSmem)) != cudaSuccess ||
      n < 1)
    n = 1;
  return n;
}

void launch_s32_av_yz(const void *tm_hi, const void *tm_lo, const void *tm_cc, const void *tm_wh,
                      const void *tm_wl, const void *tm_wc, const AvArgs &a, int grid,
                      cudaStream_t st) {
  const CUtensorMap &h = *(const CUtensorMap *)tm_hi, &l = *(const CUtensorMap *)tm_lo;
  const CUtensorMap &c = *(const CUtensorMap *)tm_cc, &wh = *(const CUtensorMap *)tm_wh;
  const CUtensorMap &wl = *(const CUtensorMap *)tm_wl, &wc = *(const CUtensorMap *)tm_wc;
  const size_t smem = sizeof(s32t::YzSmem);
  if (a.mon)
    s32t::av_yz_kernel<true><<<grid, s32t::LK + 32, smem, st>>>(h, l, c, wh, wl, wc, a);
  else
    s32t::av_yz_kernel<false><<<grid, s32t::LK + 32, smem, st>>>(h, l, c, wh, wl, wc, a);
}

}  // namespace miso_b200
