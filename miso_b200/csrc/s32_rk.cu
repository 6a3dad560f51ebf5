// FP32 split-precision Runge-Kutta stage for 3-D grids: TMA plane pipeline,
// packed FP32x2 differences, one CTA barrier per plane.
//
// A CTA owns a TJ x TK (8 x 32) tile of (j, k) columns and marches along i
// over a chunk of planes.  Each plane of the stage input -- 9 conserved
// fields on the tile plus a 2-cell halo in j and k -- arrives in shared
// memory by one TMA copy (4-D tensor map: k, j, i, field), three planes in
// flight; every thread waits on the plane's mbarrier itself.  Per plane a
// thread forms the primitive variables and the flux vectors of its point
// once (halo rows and columns: the one flux they feed), puts the y and z
// fluxes in a double-buffered shared array and keeps the x flux in a
// three-deep register ring.  After the single barrier of the plane it forms
// the y and z differences of its point and finishes the cell two planes
// back, whose centre values it loaded into registers before the wait.  Only
// the interior is written; the ghost images of the outputs are filled by the
// shell kernel (s32_shell.cu) that follows the stage.  (Splitting the plane
// barrier into an mbarrier arrival before the finish and a wait after it,
// so the finish overlaps the exchange, measured 1.1x slower than the
// hardware barrier: the polling waits take issue slots.)
// The ring is rotated by unrolling the plane loop three times, so no
// register moves are spent on it.
//
// Differences run on field pairs (ro,mx) (my,mz) (bx,by) (bz,et) with the
// packed FP32x2 operations of sm_100 (component-wise, round to nearest, so
// every field gets what the scalar operation gives); ph runs alone.  The
// 4th-order x difference of cell c is split into
//     P(c) = F(c-2) - 8 F(c-1)          formed at plane c,
//     N(c) = F(c+2) - 8 F(c+1) = -Q(c)  formed at plane c+2,
// and finished as D = (wx*P + Dyz) - wx*N with each product rounded on its
// own: for a locally constant flux P and N are the same number, so the x
// part cancels exactly, as it does in (F[-2] - F[+2]) + 8 (F[+1] - F[-1]).
//
// Physics: flux form of mhd_integrator_host.hpp:57-247 (Integrator::
// update_sc4) with the stage factors of runge_kutta_4step
// (mhd_integrator_host.hpp:258-277) and the GLM damping of ph.
//
// STAGE 0-3 are the four stages.  STAGE 4 is the last stage with its update
// deferred: it writes the stage's right-hand side D (source included) to
// `out` and reads no centre values; the x viscosity sweep then forms
// U^{n+1} = (hi, lo) - dt_4 D plane by plane as it streams the state in
// (av_line_kernel<0, true>), which saves the step one write and one read of
// the full split state.
#include <cuda.h>

#include "common.cuh"
#include "s32_common.cuh"
#include "s32_tiled.h"
#include "tma.cuh"

namespace miso_b200 {
namespace s32p {

using namespace s32t;

constexpr int TJ = 8, TK = 32, HJ = TJ + 4, HK = TK + 4;
constexpr int NTHR = TJ * TK;  // 256
constexpr int NBUF = 3;
constexpr int NPAIR = 4;  // packed field pairs; field 8 (ph) alone
constexpr int PLANE_BYTES = NF * HJ * HK * 4;
constexpr int PLANE_STRIDE = (PLANE_BYTES + 127) / 128 * 128;


// 9 values as 4 packed pairs and a single (ph)
struct V9 {
  float2 p[NPAIR];
  float s;
};

__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b, exactly rounded once: (-1) * b is exact
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(f2(-1.f, -1.f), b, a); }

// (A - E) + 8 (D - B) for A..E = F[-2], F[-1], F[+1], F[+2]
__device__ __forceinline__ float2 d4(float2 A, float2 B, float2 D, float2 E) {
  return fma2(f2(8.f, 8.f), sub2(D, B), sub2(A, E));
}
__device__ __forceinline__ float d4(float A, float B, float D, float E) {
  return fmaf(8.f, D - B, A - E);
}

struct Consts {
  float2 wx2, wy2, wz2, mdt2;
  float wx, wy, wz, dt, decay, ch2;
};

struct Item {
  int jj, kk, i_start, i_end;
};

__device__ __forceinline__ Item item_of(const RkArgs &a, int it) {
  const int per = a.tiles_j * a.tiles_k;
  const int ch = it / per, rem = it - ch * per;
  Item r;
  const int tj = rem / a.tiles_k;
  r.jj = tj * TJ;
  r.kk = (rem - tj * a.tiles_k) * TK;
  r.i_start = a.i0 + ch * a.L;
  r.i_end = min(a.i1, r.i_start + a.L);
  return r;
}

struct PipeSmem;
__device__ __forceinline__ void issue_plane(const CUtensorMap *tm, PipeSmem &sm, int b, int kk,
                                            int jj, int i);

// Producer cursor over this CTA's (item, plane) sequence; used by thread 0.
struct Producer {
  int it, q, issued;
  Item cur;
  __device__ void begin(const RkArgs &a) {
    issued = 0;
    it = blockIdx.x;
    if (it < a.items) {
      cur = item_of(a, it);
      q = cur.i_start - 2;
    }
  }
  __device__ bool valid(const RkArgs &a) const { return it < a.items; }
  __device__ void issue(const CUtensorMap *tm, PipeSmem &sm, int b, const RkArgs &a) {
    issue_plane(tm, sm, b, cur.kk, cur.jj, q + a.g.m[0]);
    ++issued;
    if (++q > cur.i_end + 1) {
      it += gridDim.x;
      if (it < a.items) {
        cur = item_of(a, it);
        q = cur.i_start - 2;
      }
    }
  }
};

struct __align__(128) PipeSmem {
  unsigned char plane[NBUF][PLANE_STRIDE];  // TMA destination: [field][HJ][HK]
  float2 fy2[2][NPAIR][HJ][TK];             // y fluxes (double-buffered by plane)
  float fy1[2][HJ][TK];
  float2 fz2[2][NPAIR][TJ][HK];             // z fluxes
  float fz1[2][TJ][HK];
  unsigned long long bar[NBUF];
  unsigned long long stall_bar;  // never arrived at (RkArgs::stall_limit)
  Consts k;       // stage constants (written once by thread 0)
  Producer prod;  // TMA issue cursor (thread 0 only)
};

__device__ __forceinline__ void issue_plane(const CUtensorMap *tm, PipeSmem &sm, int b, int kk,
                                            int jj, int i) {
  mbar_expect_tx(&sm.bar[b], PLANE_BYTES);
  tma4(tm, sm.plane[b], &sm.bar[b], kk, jj, i, 0);
}

// Consumer position in the plane ring.
struct Pipe {
  int seq;       // planes consumed by this CTA
  int b;         // seq % NBUF
  unsigned par;  // (seq / NBUF) & 1
};

template <int STAGE, bool SRC>
__device__ __forceinline__ bool plane_step(const RkArgs &a, PipeSmem &sm, const CUtensorMap *tm,
                                           const Item &itm, int q, V9 &Fn, const V9 &F1,
                                           const V9 &F2, V9 &Rn, const V9 &R2, Pipe &pp) {
  const Geom &g = a.g;
  const Consts &k = sm.k;
  Producer &prod = sm.prod;
  const int tid = threadIdx.x, ty = tid >> 5, tx = tid & 31;
  const int c = q - 2;  // the cell finished at this plane
  const int jg = itm.jj + ty, kg = itm.kk + tx;
  const bool out_ok = c >= itm.i_start && c < itm.i_end && jg < g.n[1] && kg < g.n[2];
  const bool need_yz = q >= itm.i_start && q < itm.i_end;
  const int cell = out_ok ? cell_of(g, c, jg, kg) : 0;

  // centre values of the finished cell, loaded before the wait so their
  // latency hides behind the flux work (an L1 prefetch instead measured
  // 1.3x slower: the lines do not survive in L1 next to 190 KB of shared
  // memory per SM)
  float A0[NF], A1[NF];
  if (STAGE < 4 && out_ok) {
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      if (STAGE < 3) {
        A0[f] = __ldg(a.u0.f[f] + cell);
      } else {
        A0[f] = a.hi.f[f][cell];
        A1[f] = a.lo.f[f][cell];
      }
    }
  }

  const bool ok = mbar_wait(&sm.bar[pp.b], pp.par, a.wait_limit);
  const float *pl = reinterpret_cast<const float *>(sm.plane[pp.b]);
  const int fb = pp.seq & 1;
  {
    float u[NF], F[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) u[f] = pl[(f * HJ + ty + 2) * HK + tx + 2];
    PrimF p;
    prim(u, a.gm1, p);
    flux_dir<0>(u, p, k.ch2, F);
#pragma unroll
    for (int i = 0; i < NPAIR; ++i) Fn.p[i] = f2(F[2 * i], F[2 * i + 1]);
    Fn.s = F[8];
    if (need_yz) {
      flux_dir<1>(u, p, k.ch2, F);
#pragma unroll
      for (int i = 0; i < NPAIR; ++i) sm.fy2[fb][i][ty + 2][tx] = f2(F[2 * i], F[2 * i + 1]);
      sm.fy1[fb][ty + 2][tx] = F[8];
      flux_dir<2>(u, p, k.ch2, F);
#pragma unroll
      for (int i = 0; i < NPAIR; ++i) sm.fz2[fb][i][ty][tx + 2] = f2(F[2 * i], F[2 * i + 1]);
      sm.fz1[fb][ty][tx + 2] = F[8];
    }
  }
  // halo fluxes: warps 0-3 the y rows above / below, warp 4 the z columns
  if (need_yz && tid < 4 * TK + 4 * TJ) {
    float uh[NF], Fh[NF];
    PrimF ph;
    if (tid < 4 * TK) {
      const int r = tid >> 5, col = tid & 31;
      const int row = r < 2 ? r : TJ + r;  // 0, 1, TJ+2, TJ+3
#pragma unroll
      for (int f = 0; f < NF; ++f) uh[f] = pl[(f * HJ + row) * HK + col + 2];
      prim(uh, a.gm1, ph);
      flux_dir<1>(uh, ph, k.ch2, Fh);
#pragma unroll
      for (int i = 0; i < NPAIR; ++i) sm.fy2[fb][i][row][col] = f2(Fh[2 * i], Fh[2 * i + 1]);
      sm.fy1[fb][row][col] = Fh[8];
    } else {
      const int e = tid - 4 * TK;
      const int row = e >> 2, cz = e & 3;
      const int col = cz < 2 ? cz : TK + cz;  // 0, 1, TK+2, TK+3
#pragma unroll
      for (int f = 0; f < NF; ++f) uh[f] = pl[(f * HJ + row + 2) * HK + col];
      prim(uh, a.gm1, ph);
      flux_dir<2>(uh, ph, k.ch2, Fh);
#pragma unroll
      for (int i = 0; i < NPAIR; ++i) sm.fz2[fb][i][row][col] = f2(Fh[2 * i], Fh[2 * i + 1]);
      sm.fz1[fb][row][col] = Fh[8];
    }
  }

  // The plane's one barrier: fluxes visible, the plane buffer free, and a
  // CTA-wide view of a timed-out wait.
  if (__syncthreads_or(!ok)) {
    if (tid == 0) {
      atomicOr(a.err, ERRBIT_TIMEOUT);
      // drain the copies still in flight (bounded) before the CTA exits
      for (int s2 = pp.seq; s2 < prod.issued; ++s2)
        mbar_wait(&sm.bar[s2 % NBUF], (unsigned)((s2 / NBUF) & 1));
    }
    return false;
  }
  if (tid == 0 && prod.valid(a)) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    prod.issue(tm, sm, pp.b, a);
  }

  if (need_yz) {
    // R(q) = wx * P(q) + Dyz(q),  P(q) = F(q-2) - 8 F(q-1)
#pragma unroll
    for (int i = 0; i < NPAIR; ++i) {
      const float2 *y = &sm.fy2[fb][i][ty][tx];
      const float2 *z = &sm.fz2[fb][i][ty][tx];
      const float2 dy = d4(y[0], y[TK], y[3 * TK], y[4 * TK]);
      const float2 dz = d4(z[0], z[1], z[3], z[4]);
      const float2 dyz = fma2(k.wz2, dz, mul2(k.wy2, dy));
      const float2 P = fma2(f2(-8.f, -8.f), F1.p[i], F2.p[i]);
      Rn.p[i] = add2(mul2(k.wx2, P), dyz);
    }
    const float *y = &sm.fy1[fb][ty][tx];
    const float *z = &sm.fz1[fb][ty][tx];
    const float dy = d4(y[0], y[TK], y[3 * TK], y[4 * TK]);
    const float dz = d4(z[0], z[1], z[3], z[4]);
    const float dyz = fmaf(k.wz, dz, k.wy * dy);
    const float P = fmaf(-8.f, F1.s, F2.s);
    Rn.s = __fadd_rn(__fmul_rn(k.wx, P), dyz);
  }

  if (out_ok) {
    // D(c) = R(c) - wx * N(c),  N(c) = F(c+2) - 8 F(c+1)
    V9 D;
#pragma unroll
    for (int i = 0; i < NPAIR; ++i) {
      const float2 N = fma2(f2(-8.f, -8.f), F1.p[i], Fn.p[i]);
      D.p[i] = sub2(R2.p[i], mul2(k.wx2, N));
    }
    D.s = __fsub_rn(R2.s, __fmul_rn(k.wx, fmaf(-8.f, F1.s, Fn.s)));
    // a caller's source functor: its heating enters the new total energy
    // outside the dt factor (mhd_integrator_host.hpp:241)
    float heat = 0.0f;
    if (SRC) {
      // the source's force enters the momentum RHS: D -= force
      float fx, fy, fz;
      if (a.src.kind == 2) {  // the functor's terms, filled before the stage
        fx = (float)__ldg(a.src.arr[0] + cell);
        fy = (float)__ldg(a.src.arr[1] + cell);
        fz = (float)__ldg(a.src.arr[2] + cell);
        heat = (float)__ldg(a.src.arr[3] + cell);
      } else {
        const float ro = STAGE == 0 ? A0[RO] : __ldg(a.src_ro + cell);
        gravity_force(a.src, ro, c + g.m[0], jg + g.m[1], kg + g.m[2], fx, fy, fz);
      }
      D.p[0].y -= fx;  // (ro, mx)
      D.p[1].x -= fy;  // (my, mz)
      D.p[1].y -= fz;
    }
    if (STAGE == 4) {
      // deferred update: the right-hand side itself
#pragma unroll
      for (int i = 0; i < NPAIR; ++i) {
        a.out.f[2 * i][cell] = D.p[i].x;
        a.out.f[2 * i + 1][cell] = D.p[i].y;
      }
      a.out.f[PH][cell] = D.s;
    } else if (STAGE < 3) {
#pragma unroll
      for (int i = 0; i < NPAIR; ++i) {
        const float2 u0 = f2(A0[2 * i], A0[2 * i + 1]);
        float2 v = fma2(k.mdt2, D.p[i], u0);
        if (SRC && i == 3) v.y = __fadd_rn(v.y, heat);  // (bz, et)
        a.out.f[2 * i][cell] = v.x;
        a.out.f[2 * i + 1][cell] = v.y;
      }
      const float u0 = A0[PH];
      a.out.f[PH][cell] = fmaf(-k.dt, D.s, u0) * k.decay;
    } else {
      // U^{n+1} = (hi, lo) - dt * D as a compensated (two-sum) pair, one
      // field pair at a time; the pieces of the characteristic speed are
      // gathered on the way
      float s_ro = 0.f, s_et = 0.f, mm = 0.f, bb2 = 0.f;
#pragma unroll
      for (int i = 0; i < NPAIR; ++i) {
        float *h0 = a.hi.f[2 * i], *h1 = a.hi.f[2 * i + 1];
        float *l0 = a.lo.f[2 * i], *l1 = a.lo.f[2 * i + 1];
        const float2 h = f2(A0[2 * i], A0[2 * i + 1]);
        float2 b = fma2(k.mdt2, D.p[i], f2(A1[2 * i], A1[2 * i + 1]));
        if (SRC && i == 3) b.y = __fadd_rn(b.y, heat);  // (bz, et)
        const float2 sm2 = add2(h, b);
        const float2 bb = sub2(sm2, h);
        const float2 e = add2(sub2(h, sub2(sm2, bb)), sub2(b, bb));
        h0[cell] = sm2.x;
        h1[cell] = sm2.y;
        l0[cell] = e.x;
        l1[cell] = e.y;
        // pairs: (ro, mx) (my, mz) (bx, by) (bz, et)
        if (i == 0) {
          s_ro = sm2.x;
          mm = sm2.y * sm2.y;
        } else if (i == 1) {
          mm = fmaf(sm2.x, sm2.x, mm);
          mm = fmaf(sm2.y, sm2.y, mm);
        } else if (i == 2) {
          bb2 = sm2.x * sm2.x;
          bb2 = fmaf(sm2.y, sm2.y, bb2);
        } else {
          bb2 = fmaf(sm2.x, sm2.x, bb2);
          s_et = sm2.y;
        }
      }
      {
        float *hp = a.hi.f[PH], *lp = a.lo.f[PH];
        float sv, t, e;
        two_sum(A0[PH], fmaf(-k.dt, D.s, A1[PH]), sv, t);
        ph_damp(sv, t, k.decay, sv, e);
        hp[cell] = sv;
        lp[cell] = e;
      }
      // characteristic speed of the new state
      a.cc[cell] = char_speed(s_ro, mm, bb2, s_et, a.gm, a.gm1, a.cs_fac, a.vv_fac, a.ca_fac);
    }
  }

  ++pp.seq;
  if (++pp.b == NBUF) {
    pp.b = 0;
    pp.par ^= 1u;
  }
  return true;
}

template <int STAGE, bool SRC>
__global__ void __launch_bounds__(NTHR, 2)
rk_pipe_kernel(const __grid_constant__ CUtensorMap tm, const RkArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  PipeSmem &sm = *reinterpret_cast<PipeSmem *>(smem_raw);
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int b = 0; b < NBUF; ++b) mbar_init(&sm.bar[b], 1);
    mbar_init(&sm.stall_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    Consts &k = sm.k;
    const Geom &g = a.g;
    k.wx = (float)(g.dsi[0] * INV12);
    k.wy = (float)(g.dsi[1] * INV12);
    k.wz = (float)(g.dsi[2] * INV12);
    k.dt = (float)a.sc->dts[STAGE < 4 ? STAGE : 3];
    k.decay = (float)a.sc->ph_decay[STAGE < 4 ? STAGE : 3];
    k.ch2 = (float)a.sc->ch2;
    k.wx2 = f2(k.wx, k.wx);
    k.wy2 = f2(k.wy, k.wy);
    k.wz2 = f2(k.wz, k.wz);
    k.mdt2 = f2(-k.dt, -k.dt);
    if ((int)blockIdx.x < a.items) {
      sm.prod.begin(a);
      for (int b = 0; b < NBUF && sm.prod.valid(a); ++b) sm.prod.issue(&tm, sm, b, a);
    }
  }
  __syncthreads();
  if ((int)blockIdx.x >= a.items) return;
  if (a.stall_limit > 0) {
    // test of the timeout path: a wait on a phase that nothing completes
    const bool ran_out = !mbar_wait(&sm.stall_bar, 0u, a.stall_limit);
    if (__syncthreads_or(ran_out)) {
      if (tid == 0) {
        atomicOr(a.err, ERRBIT_TIMEOUT);
        // the copies already issued land before the CTA exits (bounded)
        for (int s2 = 0; s2 < sm.prod.issued; ++s2)
          mbar_wait(&sm.bar[s2 % NBUF], (unsigned)((s2 / NBUF) & 1));
      }
      return;
    }
  }

  Pipe pp{0, 0, 0u};
  V9 FA, FB, FC, RA, RB, RC;
#pragma unroll
  for (int i = 0; i < NPAIR; ++i)
    FA.p[i] = FB.p[i] = FC.p[i] = RA.p[i] = RB.p[i] = RC.p[i] = f2(0.f, 0.f);
  FA.s = FB.s = FC.s = RA.s = RB.s = RC.s = 0.f;

  for (int it = blockIdx.x; it < a.items; it += gridDim.x) {
    const Item itm = item_of(a, it);
    const int qe = itm.i_end + 1;
    // ring slots: F(q) -> Fn, F(q-1) -> F1, F(q-2) -> F2 (R likewise)
    for (int q = itm.i_start - 2; q <= qe; q += 3) {
      if (!plane_step<STAGE, SRC>(a, sm, &tm, itm, q, FA, FC, FB, RA, RB, pp)) return;
      if (q + 1 > qe) break;
      if (!plane_step<STAGE, SRC>(a, sm, &tm, itm, q + 1, FB, FA, FC, RB, RC, pp)) return;
      if (q + 2 > qe) break;
      if (!plane_step<STAGE, SRC>(a, sm, &tm, itm, q + 2, FC, FB, FA, RC, RA, pp)) return;
    }
  }
}

}  // namespace s32p

int s32_rk_pipe_configure() {
  const int bytes = (int)sizeof(s32p::PipeSmem);
  cudaError_t e = cudaSuccess;
#define MISO_SET(kern) \
  if (e == cudaSuccess) e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)
  MISO_SET((s32p::rk_pipe_kernel<0, false>));
  MISO_SET((s32p::rk_pipe_kernel<1, false>));
  MISO_SET((s32p::rk_pipe_kernel<2, false>));
  MISO_SET((s32p::rk_pipe_kernel<3, false>));
  MISO_SET((s32p::rk_pipe_kernel<4, false>));
  MISO_SET((s32p::rk_pipe_kernel<0, true>));
  MISO_SET((s32p::rk_pipe_kernel<1, true>));
  MISO_SET((s32p::rk_pipe_kernel<2, true>));
  MISO_SET((s32p::rk_pipe_kernel<3, true>));
  MISO_SET((s32p::rk_pipe_kernel<4, true>));
#undef MISO_SET
  return e == cudaSuccess ? 0 : -1;
}

template <bool SRC>
static void launch_pipe(const CUtensorMap &m, const RkArgs &a, int stage, int grid,
                        cudaStream_t st) {
  const size_t smem = sizeof(s32p::PipeSmem);
  switch (stage) {
    case 0: s32p::rk_pipe_kernel<0, SRC><<<grid, s32p::NTHR, smem, st>>>(m, a); break;
    case 1: s32p::rk_pipe_kernel<1, SRC><<<grid, s32p::NTHR, smem, st>>>(m, a); break;
    case 2: s32p::rk_pipe_kernel<2, SRC><<<grid, s32p::NTHR, smem, st>>>(m, a); break;
    case 3: s32p::rk_pipe_kernel<3, SRC><<<grid, s32p::NTHR, smem, st>>>(m, a); break;
    default: s32p::rk_pipe_kernel<4, SRC><<<grid, s32p::NTHR, smem, st>>>(m, a); break;
  }
}

void launch_s32_rk_pipe(const void *tm, const RkArgs &a, int stage, int grid, cudaStream_t st) {
  const CUtensorMap &m = *(const CUtensorMap *)tm;
  if (a.src.kind != 0)
    launch_pipe<true>(m, a, stage, grid, st);
  else
    launch_pipe<false>(m, a, stage, grid, st);
}

}  // namespace miso_b200
