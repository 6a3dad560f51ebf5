// FP32 split-precision viscosity sweep along x or y for 3-D grids, streamed
// along the sweep axis with no CTA-wide barrier in the march.
//
// A CTA of LK threads owns LK consecutive k cells of one line and marches
// along the sweep axis over a chunk of planes.  Per plane one TMA copy each
// brings hi, lo and the characteristic speed (132-cell k boxes, so every
// copy starts on a 16-byte boundary) into a slot of a ring in shared memory.
// Two mbarriers per slot run the ring: "full" completes when the copies have
// landed (every thread waits on it), "empty" when all LK threads have
// finished with the slot (thread 0 waits on it before refilling).  A thread
// reads only its own k column, so no other synchronisation is needed.
//
// Per plane p a thread forms the limited variables of cell p, the slope of
// cell p-1 and the limited face flux between p-2 and p-1, and finishes cell
// p-2 with the flux difference.  The limited variables of cells p-1, p-2
// are re-read from the ring (the conserved fields are the hi words; the
// internal-energy density is kept in a thread-private column of the slot),
// and the slope and face flux carried to the next plane ride a two-deep
// register ring rotated by unrolling the plane loop twice.
//
// Physics: mhd_artificial_viscosity_host.hpp:70-348 with limiter.hpp:11-37,
// in the compensated split form (two-sum update of the hi/lo pair).
#include <cuda.h>

#include "common.cuh"
#include "s32_common.cuh"
#include "s32_tiled.h"
#include "tma.cuh"

namespace miso_b200 {
namespace s32v {

using namespace s32t;

constexpr int LK = 128;       // k cells (threads) per CTA
constexpr int LBOX = LK + 4;  // k box of the TMA copies (starts 2 cells early: 16-byte aligned)
constexpr int NSLOT = 5;
constexpr int SZ_F = (NF * LBOX * 4 + 127) / 128 * 128;
constexpr int OFF_HI = 0, OFF_LO = SZ_F, OFF_CC = 2 * SZ_F;
constexpr int OFF_W8 = OFF_CC + (LBOX * 4 + 127) / 128 * 128;
constexpr int SLOT = OFF_W8 + LK * 4;
constexpr unsigned TX = 2 * NF * LBOX * 4 + LBOX * 4;  // bytes landed per slot fill

struct Geo {
  int kblocks, nu, items;
};

struct Item {
  int kb, u, t0, t1;
};

struct Producer {
  int it, p, issued;
  Item cur;
};

struct __align__(128) AvSmem {
  unsigned char slot[NSLOT][SLOT];
  unsigned long long full[NSLOT];
  unsigned long long empty[NSLOT];
  Producer prod;
};

template <int DIR>
__device__ __forceinline__ Item item_of(const AvArgs &a, const Geo &q, int it) {
  Item r;
  r.kb = it % q.kblocks;
  const int r1 = it / q.kblocks;
  r.u = r1 % q.nu;
  const int ch = r1 / q.nu;
  r.t0 = ch * a.L;
  r.t1 = min(a.g.n[DIR], r.t0 + a.L);
  return r;
}

__device__ __forceinline__ void mbar_arrive(unsigned long long *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// thread 0: issue the next plane of this CTA's sequence into slot s
template <int DIR>
__device__ __forceinline__ void produce(const CUtensorMap *thi, const CUtensorMap *tlo,
                                        const CUtensorMap *tcc, AvSmem &sm, int s,
                                        const AvArgs &a, const Geo &q) {
  Producer &pr = sm.prod;
  unsigned char *sl = sm.slot[s];
  const Geom &g = a.g;
  const int k0 = pr.cur.kb * LK;
  const int cj = DIR == 0 ? pr.cur.u + g.m[1] : pr.p + g.m[1];
  const int ci = DIR == 0 ? pr.p + g.m[0] : pr.cur.u + g.m[0];
  mbar_expect_tx(&sm.full[s], TX);
  tma4(thi, sl + OFF_HI, &sm.full[s], k0, cj, ci, 0);
  tma4(tlo, sl + OFF_LO, &sm.full[s], k0, cj, ci, 0);
  tma3(tcc, sl + OFF_CC, &sm.full[s], k0, cj, ci);
  ++pr.issued;
  if (++pr.p > pr.cur.t1 + 1) {
    pr.it += gridDim.x;
    if (pr.it < q.items) {
      pr.cur = item_of<DIR>(a, q, pr.it);
      pr.p = pr.cur.t0 - 2;
    }
  }
}

struct Ring {
  int seq;  // planes consumed
  int s;    // seq % NSLOT
};

// Thread 0, once the slot of plane seq-2 is released by every thread:
// refill it with the plane NSLOT ahead.  False on a timed-out wait.
template <int DIR>
__device__ __forceinline__ bool refill(const CUtensorMap *thi, const CUtensorMap *tlo,
                                       const CUtensorMap *tcc, AvSmem &sm, int seq_done,
                                       const AvArgs &a, const Geo &q) {
  if (sm.prod.it >= q.items) return true;  // nothing left to issue
  const int s = seq_done % NSLOT;
  if (!mbar_wait(&sm.empty[s], (unsigned)((seq_done / NSLOT) & 1))) return false;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  produce<DIR>(thi, tlo, tcc, sm, s, a, q);
  return true;
}

// One plane p of item `it`; dq_in / F_in are the slope of cell p-2 and the
// face flux between p-3 and p-2, dq_out / F_out receive those of p-1 and
// (p-2, p-1).  Returns false when a wait ran out.
template <int DIR>
__device__ __forceinline__ bool av_plane(const CUtensorMap *thi, const CUtensorMap *tlo,
                                         const CUtensorMap *tcc, AvSmem &sm, const AvArgs &a,
                                         const Geo &q, const Item &itm, int p, float fac,
                                         const float (&dq_in)[NW], const float (&F_in)[NW],
                                         float (&dq_out)[NW], float (&F_out)[NW], Ring &rg) {
  const Geom &g = a.g;
  const int tid = threadIdx.x;
  const int r = p - itm.t0;  // -2 .. t1-t0+1
  if (!mbar_wait(&sm.full[rg.s], (unsigned)((rg.seq / NSLOT) & 1))) return false;
  const int s1 = rg.s == 0 ? NSLOT - 1 : rg.s - 1;
  const int s2 = s1 == 0 ? NSLOT - 1 : s1 - 1;
  const float *h0 = reinterpret_cast<const float *>(sm.slot[rg.s] + OFF_HI) + tid + 2;
  float *w8_0 = reinterpret_cast<float *>(sm.slot[rg.s] + OFF_W8) + tid;
  float wp[NW];
  {
    float u[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) u[f] = h0[f * LBOX];
    limited_vars(u, wp);
    *w8_0 = wp[8];
  }
  if (r >= 0) {
    const float *h1 = reinterpret_cast<const float *>(sm.slot[s1] + OFF_HI) + tid + 2;
    const float *h2 = reinterpret_cast<const float *>(sm.slot[s2] + OFF_HI) + tid + 2;
    const float w8_1 = reinterpret_cast<const float *>(sm.slot[s1] + OFF_W8)[tid];
    const float w8_2 = reinterpret_cast<const float *>(sm.slot[s2] + OFF_W8)[tid];
    const float cc1 = reinterpret_cast<const float *>(sm.slot[s1] + OFF_CC)[tid + 2];
    const float cc2 = reinterpret_cast<const float *>(sm.slot[s2] + OFF_CC)[tid + 2];
    const float cface = 0.5f * (cc2 + cc1);
#pragma unroll
    for (int n = 0; n < NW; ++n) {
      const int f = field_of(n);
      const float w1 = n == 8 ? w8_1 : h1[f * LBOX];
      const float w2 = n == 8 ? w8_2 : h2[f * LBOX];
      dq_out[n] = dqq_eval(w2, w1, wp[n], a.ep);
      if (r >= 1) F_out[n] = flux_core(w2, w1, dq_in[n], dq_out[n], cface, a.fh);
    }
    const int c = p - 2;
    const int k = itm.kb * LK + tid;
    if (r >= 2 && k < g.n[2]) {
      const int x0 = DIR == 0 ? c : itm.u;
      const int x1 = DIR == 0 ? itm.u : c;
      const int cell = cell_of(g, x0, x1, k);
      const bool nb = near_boundary(g, x0, x1, k);
      Img im;
      if (nb) make_img(g, x0, x1, k, im);
      const float *l2 = reinterpret_cast<const float *>(sm.slot[s2] + OFF_LO) + tid + 2;
#pragma unroll
      for (int n = 0; n < NW; ++n) {
        const int f = field_of(n);
        float sv, e;
        two_sum(h2[f * LBOX], l2[f * LBOX] - (F_out[n] - F_in[n]) * fac, sv, e);
        store_cell(a.hi2.f[f], cell, nb, im, f, sv);
        store_cell(a.lo2.f[f], cell, nb, im, f, e);
      }
    }
  }
  // this thread is done with the slot of plane seq-2
  if (rg.seq >= 2) mbar_arrive(&sm.empty[s2]);
  if (tid == 0 && rg.seq >= 2 && !refill<DIR>(thi, tlo, tcc, sm, rg.seq - 2, a, q)) return false;
  ++rg.seq;
  rg.s = rg.s == NSLOT - 1 ? 0 : rg.s + 1;
  return true;
}

template <int DIR>
__global__ void __launch_bounds__(LK, 4)
av_pipe_kernel(const __grid_constant__ CUtensorMap thi, const __grid_constant__ CUtensorMap tlo,
               const __grid_constant__ CUtensorMap tcc, const AvArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  AvSmem &sm = *reinterpret_cast<AvSmem *>(smem_raw);
  const Geom &g = a.g;
  constexpr int OTH = DIR == 0 ? 1 : 0;
  Geo q;
  q.kblocks = (g.n[2] + LK - 1) / LK;
  q.nu = g.n[OTH];
  q.items = q.kblocks * q.nu * ((g.n[DIR] + a.L - 1) / a.L);
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < NSLOT; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], LK);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    Producer &pr = sm.prod;
    pr.issued = 0;
    pr.it = blockIdx.x;
    if (pr.it < q.items) {
      pr.cur = item_of<DIR>(a, q, pr.it);
      pr.p = pr.cur.t0 - 2;
      for (int s = 0; s < NSLOT && pr.it < q.items; ++s) produce<DIR>(&thi, &tlo, &tcc, sm, s, a, q);
    }
  }
  __syncthreads();
  if ((int)blockIdx.x >= q.items) return;
  const float fac = (float)(g.dsi[DIR] * a.sc->dt);
  Ring rg{0, 0};
  float dqA[NW], dqB[NW], FA[NW], FB[NW];
#pragma unroll
  for (int n = 0; n < NW; ++n) dqA[n] = dqB[n] = FA[n] = FB[n] = 0.0f;
  bool ok = true;
  for (int it = blockIdx.x; it < q.items && ok; it += gridDim.x) {
    const Item itm = item_of<DIR>(a, q, it);
    const int pe = itm.t1 + 1;
    for (int p = itm.t0 - 2; p <= pe; p += 2) {
      if (!(ok = av_plane<DIR>(&thi, &tlo, &tcc, sm, a, q, itm, p, fac, dqA, FA, dqB, FB, rg)))
        break;
      if (p + 1 > pe) break;
      if (!(ok = av_plane<DIR>(&thi, &tlo, &tcc, sm, a, q, itm, p + 1, fac, dqB, FB, dqA, FA, rg)))
        break;
    }
  }
  if (!ok) {
    atomicOr(a.err, ERRBIT_TIMEOUT);
    if (tid == 0) {
      // drain the copies still in flight (bounded) before the CTA exits
      for (int s2 = rg.seq; s2 < sm.prod.issued; ++s2)
        mbar_wait(&sm.full[s2 % NSLOT], (unsigned)((s2 / NSLOT) & 1));
    }
  }
}

}  // namespace s32v

int s32_av_pipe_configure() {
  const int bytes = (int)sizeof(s32v::AvSmem);
  cudaError_t e = cudaFuncSetAttribute(s32v::av_pipe_kernel<0>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(s32v::av_pipe_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             bytes);
  return e == cudaSuccess ? 0 : -1;
}

void launch_s32_av_pipe(const void *tm_hi, const void *tm_lo, const void *tm_cc, const AvArgs &a,
                        int dir, int grid, cudaStream_t st) {
  const CUtensorMap &h = *(const CUtensorMap *)tm_hi;
  const CUtensorMap &l = *(const CUtensorMap *)tm_lo;
  const CUtensorMap &c = *(const CUtensorMap *)tm_cc;
  const size_t smem = sizeof(s32v::AvSmem);
  if (dir == 0)
    s32v::av_pipe_kernel<0><<<grid, s32v::LK, smem, st>>>(h, l, c, a);
  else
    s32v::av_pipe_kernel<1><<<grid, s32v::LK, smem, st>>>(h, l, c, a);
}

}  // namespace miso_b200
