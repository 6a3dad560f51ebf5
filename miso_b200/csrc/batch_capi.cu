// C ABI of the batched solver (include/miso_b200.h, miso_b200_batch_*):
// many independent grids -- uneven sizes, their own parameters and time
// steps -- advanced together, one persistent launch per pass, a step
// captured once in a CUDA graph and replayed.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/miso_b200.h"
#include "batch.h"
#include "common.cuh"
#include "kernels_s32.h"
#include "s32_tiled.h"
#include "view.h"

using namespace miso_b200;

void miso_b200_set_global_error(const std::string &msg);  // capi.cu

namespace {
constexpr size_t ALIGN = 256;
size_t round_up(size_t x) { return (x + ALIGN - 1) / ALIGN * ALIGN; }
}  // namespace

struct miso_b200_batch {
  int count = 0;
  bool split = false;
  int sms = 148, grid = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;

  std::vector<BatchInst> insts;
  long long total = 0;       // elements per field array (all instances)
  long long max_cells = 0;   // largest instance (cells incl. ghosts)
  int ntiles = 0;
  int nbtiles = 0;
  int bgrid = 0;  // persistent grid of the FP32 block-tile kernels
  // FP32 warp-per-row items of the 1-D / 2-D instances: per axis pair for
  // the Runge-Kutta stage (28 cells along R), all of them for the sweep
  // along R, and 32-cell items for the sweep along C
  RowItem *d_rows = nullptr, *d_rows_c = nullptr;
  int row_off[ROW_COMBOS + 1] = {};
  int nrows = 0, nrows_c = 0;
  int rgrid = 0;
  bool sweep[3] = {false, false, false};  // some instance is non-degenerate along d
  bool defer_rows = true;  // RK variant 3: the rows' last update deferred into the first sweep
  bool sweep_c[3] = {false, false, false};  // d is the C axis of some 2-D instance

  void *block = nullptr;
  size_t bytes = 0;
  BatchInst *d_insts = nullptr;
  BatchTile *d_tiles = nullptr;
  TileGeo *d_btiles = nullptr;
  int4 *d_scells = nullptr;  // near-boundary interior cells (instance, x0, x1, x2)
  int nscells = 0;
  StepScalars *d_sc = nullptr;
  unsigned int *d_dtmin = nullptr;
  unsigned int *d_dtinit = nullptr;  // 1e10 per instance: the running minima's start
  unsigned int *d_err = nullptr;
  // FP64
  double *q64[3][NF] = {};
  double *cc64 = nullptr;
  // FP32 split
  float *hi[2][NF] = {}, *lo[2][NF] = {}, *stg[2][NF] = {};
  float *cc32 = nullptr;
  double *io64[NF] = {};
  int cur = 0;
  // FP32: the per-instance CFL minima of the current state were folded in
  // by the last sweep of the previous step (no separate CFL pass needed)
  bool cfl_valid = false;

  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  int graph_steps = 0, graph_cur = 0;
  long long launches = 0, graph_kernels = 0;

  // 3-D FP32-split instances stepped through views on their own streams
  // (at most VIEW_STREAMS; views on one stream run in turn), forked from
  // and joined back into the batch's stream every step
  static constexpr int VIEW_STREAMS = 64;
  struct View {
    int index;
    miso_b200_handle *h;
    int lane;  // which of the view streams; -1: the batch's own stream (a grid that fills the GPU)
  };
  std::vector<View> views;
  std::vector<int> view_at;  // per instance: its index in `views`, or -1
  std::vector<cudaStream_t> vstreams;
  std::vector<cudaEvent_t> vdone;
  cudaEvent_t vfork = nullptr;

  int enqueue_views() {
    if (views.empty()) return MISO_B200_OK;
    int rc = MISO_B200_OK;
    if (!vstreams.empty()) rc = cuda(cudaEventRecord(vfork, stream), "fork views");
    for (size_t s = 0; s < vstreams.size() && !rc; ++s)
      rc = cuda(cudaStreamWaitEvent(vstreams[s], vfork, 0), "fork views");
    if (rc) return rc;
    for (auto &v : views) {
      const long long l0 = b200_view_launches(v.h);
      int out_cur = 0;
      // each view steps from the set its own last step left it in
      if ((rc = b200_view_step(v.h, -1, &out_cur))) {
        err = std::string("instance ") + std::to_string(v.index) + ": " +
              miso_b200_last_error(v.h);
        return rc;
      }
      launches += b200_view_launches(v.h) - l0;
    }
    return MISO_B200_OK;
  }
  int join_views() {
    int rc = MISO_B200_OK;
    for (size_t s = 0; s < vstreams.size() && !rc; ++s) {
      rc = cuda(cudaEventRecord(vdone[s], vstreams[s]), "join views");
      if (!rc) rc = cuda(cudaStreamWaitEvent(stream, vdone[s], 0), "join views");
    }
    return rc;
  }
  // every view's ghost layers from its current state (after an upload or a
  // fill of the whole batch), ordered on the batch's stream
  int fill_views() {
    if (views.empty()) return MISO_B200_OK;
    int rc = vstreams.empty() ? MISO_B200_OK : cuda(cudaEventRecord(vfork, stream), "fork views");
    for (size_t s = 0; s < vstreams.size() && !rc; ++s)
      rc = cuda(cudaStreamWaitEvent(vstreams[s], vfork, 0), "fork views");
    for (auto &v : views)
      if (!rc && (rc = b200_view_fill(v.h, b200_view_cur(v.h))))
        err = std::string("instance ") + std::to_string(v.index) + ": " + miso_b200_last_error(v.h);
    int rj = join_views();
    return rc ? rc : rj;
  }

  int fail(int code, const std::string &m) {
    err = m;
    return code;
  }
  int cuda(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return MISO_B200_OK;
    return fail(MISO_B200_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  }
  BatchArgs args() const {
    BatchArgs a;
    a.insts = d_insts;
    a.tiles = d_tiles;
    a.ntiles = ntiles;
    a.btiles = d_btiles;
    a.nbtiles = nbtiles;
    a.count = count;
    a.sc = d_sc;
    a.dtmin = d_dtmin;
    a.err = d_err;
    return a;
  }
  template <typename T>
  static FieldPtrs<const T> cst(T *const (&arr)[NF]) {
    FieldPtrs<const T> r;
    for (int f = 0; f < NF; ++f) r.f[f] = arr[f];
    return r;
  }
  template <typename T>
  static FieldPtrs<T> mut(T *const (&arr)[NF]) {
    FieldPtrs<T> r;
    for (int f = 0; f < NF; ++f) r.f[f] = arr[f];
    return r;
  }

  int enqueue_step() {
    const BatchArgs a = args();
    // the 3-D split instances run their own pipelined steps concurrently
    if (int rc = enqueue_views()) return rc;
    if (!split) {
      b64_cfl(a, cst(q64[0]), grid, stream);
      b_finalize(a, stream);
      const int seq_a[4] = {0, 1, 2, 1}, seq_r[4] = {1, 2, 1, 2};
      for (int s = 0; s < 4; ++s)
        b64_rhs(a, cst(q64[0]), cst(q64[seq_a[s]]), mut(q64[seq_r[s]]), s, grid, stream);
      b64_cc(a, cst(q64[2]), cc64, grid, stream);
      // every sweep runs, degenerate ones included: in FP64 the reference's
      // degenerate sweep is a round-off step of its own
      const int src[3] = {2, 0, 1}, dst[3] = {0, 1, 0};
      for (int d = 0; d < 3; ++d) {
        // 3-D instances and degenerate axes on the tile list; the own axes
        // of the 1-D / 2-D instances by rows
        b64_av(a, cst(q64[src[d]]), mut(q64[dst[d]]), cc64, d, grid, stream);
        const int nc = sweep_c[d] ? nrows_c : 0;
        b64_av_rows(a, d_rows, nrows, d_rows_c, nc, cst(q64[src[d]]), mut(q64[dst[d]]), cc64, d,
                    grid, stream);
        launches += 1 + (nrows > 0) + (nc > 0);
      }
      launches += 2 + 4 + 1;
    } else {
      if (!cfl_valid) {
        // a replaced state: the minima the last sweep folded in are stale
        if (int rc = cuda(cudaMemcpyAsync(d_dtmin, d_dtinit, sizeof(unsigned int) * count,
                                          cudaMemcpyDeviceToDevice, stream),
                          "reset the CFL minima"))
          return rc;
        b32_cfl(a, cst(hi[cur]), grid, stream);
        ++launches;
      }
      b_finalize(a, stream);
      const int c = cur;
      // the 1-D / 2-D instances' last Runge-Kutta update deferred into the
      // step's first sweep (their fourth stage writes its right-hand side D
      // to stg[1]; the first sweep forms U^{n+1} from hi, lo and D)
      const bool defer = defer_rows && nrows > 0;
      int first = -1, last = -1;
      for (int d = 0; d < 3; ++d)
        if (sweep[d]) {
          if (first < 0) first = d;
          last = d;
        }
      for (int s = 0; s < 4; ++s) {
        FieldPtrs<const float> prev = s == 0 ? cst(hi[c]) : cst(stg[(s - 1) & 1]);
        if (nbtiles) {
          b32_rk(a, prev, cst(hi[c]), mut(hi[c]), mut(lo[c]), mut(stg[s & 1]), cc32, s, bgrid,
                 stream);
          ++launches;
        }
        for (int cb = 0; cb < ROW_COMBOS; ++cb) {
          const int n = row_off[cb + 1] - row_off[cb];
          if (!n) continue;
          b32_rk_rows(a, d_rows + row_off[cb], n, cb, prev, cst(hi[c]), mut(hi[c]), mut(lo[c]),
                      mut(stg[s & 1]), cc32, s, defer && s == 3 ? 1 : 0, rgrid, stream);
          ++launches;
        }
        // the block kernels write the interior; images of what the next pass reads
        if (s < 3 || defer) {  // the stage output, or with the deferred update D
          b32_shell_fill(a, d_scells, nscells, mut(stg[s & 1]), NF, -1, stream);
          ++launches;
        }
        if (s == 3 && (!defer || nbtiles)) {  // the block instances' new state and speed
          b32_shell_fill(a, d_scells, nscells, mut(hi[c]), NF, -1, stream);
          FieldPtrs<float> ccf{};
          ccf.f[0] = cc32;
          b32_shell_fill(a, d_scells, nscells, ccf, 1, NF, stream);
          launches += 2;
        }
      }
      launches += 1;
      FieldPtrs<const float> none{};
      for (int d = 0; d < 3; ++d) {
        if (!sweep[d]) continue;  // degenerate for every instance: the state is unchanged
        const int fuse = d == last ? 1 : 0;
        const bool dd = defer && d == first;  // the rows take the deferred update here
        const FieldPtrs<const float> d4 = dd ? cst(stg[1]) : none;
        float *cc_out = dd ? cc32 : nullptr;
        if (nbtiles) {
          b32_av(a, cst(hi[cur]), cst(lo[cur]), mut(hi[cur ^ 1]), mut(lo[cur ^ 1]), cc32, d, fuse,
                 bgrid, stream);
          ++launches;
        }
        if (nrows) {  // sweeps along R and degenerate ones of the 1-D / 2-D instances
          b32_av_rows_r(a, d_rows, nrows, cst(hi[cur]), cst(lo[cur]), mut(hi[cur ^ 1]),
                        mut(lo[cur ^ 1]), cc32, d, fuse, d4, cc_out, rgrid, stream);
          ++launches;
        }
        if (nrows_c && sweep_c[d]) {  // sweeps along C of the 2-D instances
          b32_av_rows_c(a, d_rows_c, nrows_c, cst(hi[cur]), cst(lo[cur]), mut(hi[cur ^ 1]),
                        mut(lo[cur ^ 1]), cc32, d, fuse, d4, cc_out, rgrid, stream);
          ++launches;
        }
        b32_shell_fill(a, d_scells, nscells, mut(hi[cur ^ 1]), NF, -1, stream);
        b32_shell_fill(a, d_scells, nscells, mut(lo[cur ^ 1]), NF, -1, stream);
        if (dd && d != last) {  // the speed the first sweep wrote, read across faces later
          FieldPtrs<float> ccf{};
          ccf.f[0] = cc32;
          b32_shell_fill(a, d_scells, nscells, ccf, 1, NF, stream);
          ++launches;
        }
        cur ^= 1;
        launches += 2;
      }
      cfl_valid = last >= 0;
    }
    if (int rc = join_views()) return rc;
    return cuda(cudaGetLastError(), "batch step");
  }

  int read_err() {
    unsigned int e = 0;
    int rc = cuda(cudaMemcpyAsync(&e, d_err, sizeof e, cudaMemcpyDeviceToHost, stream), "read");
    if (rc) return rc;
    if ((rc = cuda(cudaStreamSynchronize(stream), "synchronize"))) return rc;
    if (e) {
      cudaMemsetAsync(d_err, 0, sizeof e, stream);
      cudaStreamSynchronize(stream);
      if (e & ERRBIT_NONFINITE)
        return fail(MISO_B200_ERR_NONFINITE,
                    "non-positive or non-finite density / internal energy in a CFL pass");
    }
    if (!views.empty()) {
      // the views' kernels flag their instance's own step scalars
      std::vector<StepScalars> sc(count);
      if ((rc = cuda(cudaMemcpyAsync(sc.data(), d_sc, sizeof(StepScalars) * count,
                                     cudaMemcpyDeviceToHost, stream),
                     "read")) ||
          (rc = cuda(cudaStreamSynchronize(stream), "synchronize")))
        return rc;
      unsigned int ev = 0;
      for (auto &v : views) {
        if (!sc[v.index].err) continue;
        ev |= sc[v.index].err;
        cudaMemsetAsync(&d_sc[v.index].err, 0, sizeof(unsigned int), stream);
      }
      if (ev) {
        cudaStreamSynchronize(stream);
        if (ev & ERRBIT_TIMEOUT)
          return fail(MISO_B200_ERR_TIMEOUT, "a bounded device-side wait ran out");
        return fail(MISO_B200_ERR_NONFINITE,
                    "non-positive or non-finite density / internal energy in a CFL pass");
      }
    }
    return MISO_B200_OK;
  }
};

extern "C" {

int miso_b200_batch_create(int count, const miso_b200_grid_desc *grids,
                           const miso_b200_params *params, void *stream,
                           miso_b200_batch **out) {
  auto bad = [](int code, const std::string &m) {
    miso_b200_set_global_error("miso_b200_batch_create: " + m);
    return code;
  };
  if (count < 1 || !grids || !params || !out) return bad(MISO_B200_ERR_ARG, "null argument");
  *out = nullptr;
  auto *b = new miso_b200_batch();
  b->count = count;
  b->split = params[0].precision == MISO_B200_FP32_SPLIT;
  long long off = 0;
  std::vector<BatchTile> tiles;
  std::vector<TileGeo> btiles;
  std::vector<RowItem> rows[ROW_COMBOS], rows_c;
  std::vector<int4> scells;
  for (int n = 0; n < count; ++n) {
    const miso_b200_grid_desc &gd = grids[n];
    const miso_b200_params &pp = params[n];
    if (pp.precision != params[0].precision) {
      delete b;
      return bad(MISO_B200_ERR_ARG, "all instances of a batch share one precision");
    }
    if (gd.margin != 2 || !(pp.gm > 1.0) || !(pp.cfl_number > 0.0) || !(pp.ep >= 0.0) ||
        !(pp.fh >= 0.0)) {
      delete b;
      return bad(MISO_B200_ERR_ARG, "invalid margin or parameters of instance " +
                                        std::to_string(n));
    }
    BatchInst in{};
    Geom &g = in.g;
    const int sz[3] = {gd.i_size, gd.j_size, gd.k_size};
    const double lo[3] = {gd.x_min, gd.y_min, gd.z_min};
    const double hi[3] = {gd.x_max, gd.y_max, gd.z_max};
    double ds[3];
    for (int a = 0; a < 3; ++a) {
      if (sz[a] < 1 || (sz[a] > 1 && sz[a] < 2 * gd.margin) || !(lo[a] < hi[a])) {
        delete b;
        return bad(MISO_B200_ERR_ARG, "invalid size or range of instance " + std::to_string(n));
      }
      g.n[a] = sz[a];
      g.s[a] = sz[a] > 1 ? 1 : 0;
      g.m[a] = gd.margin * g.s[a];
      g.t[a] = sz[a] + 2 * g.m[a];
      g.periodic[a] = gd.periodic[a] ? 1 : 0;
      const double sp = (hi[a] - lo[a]) / (double)sz[a];
      ds[a] = g.s[a] ? sp : 1.e30;
      g.dsi[a] = g.s[a] ? 1.0 / sp : 0.0;
      for (int side = 0; side < 2; ++side) {
        g.negmask[a][side] = 0;
        for (int f = 0; f < NF; ++f) {
          g.sign[a][side][f] = (float)(gd.sign[a][side][f] < 0 ? -1 : 1);
          if (!g.periodic[a] && gd.sign[a][side][f] < 0)
            g.negmask[a][side] |= (unsigned short)(1u << f);
        }
      }
      if (g.s[a]) b->sweep[a] = true;
    }
    g.st[2] = 1;
    g.st[1] = g.t[2];
    g.st[0] = (long long)g.t[1] * g.t[2];
    g.cells = (long long)g.t[0] * g.t[1] * g.t[2];
    in.base = off;
    in.nint = (long long)g.n[0] * g.n[1] * g.n[2];
    in.gm = pp.gm;
    in.cfl_number = pp.cfl_number;
    in.ep = pp.ep;
    in.fh = pp.fh;
    in.cs_fac = pp.cs_fac;
    in.ca_fac = pp.ca_fac;
    in.vv_fac = pp.vv_fac;
    const float m3 = fminf(fminf((float)ds[0], (float)ds[1]), (float)ds[2]);
    in.min_dxyz = (double)m3;
    in.cfl_dx = pp.cfl_number * (double)m3;
    // block-tile axes: R = last non-degenerate axis (unit stride), C the one
    // before it, P the first of three
    int nd[3], nnd = 0;
    for (int a = 0; a < 3; ++a)
      if (g.s[a]) nd[nnd++] = a;
    in.ax_r = nnd > 0 ? nd[nnd - 1] : 2;
    in.ax_c = nnd > 1 ? nd[nnd - 2] : -1;
    in.ax_p = nnd > 2 ? nd[0] : -1;
    // a 3-D split instance the pipelined kernels can take runs through a
    // view: the batch-wide lists leave it out
    in.view = b->split && g.s[0] && g.s[1] && g.s[2] && s32_tiled_supported(g) &&
              !getenv("MISO_B200_BATCH_BLOCKS");
    b->insts.push_back(in);
    if (in.view) {
      off += (g.cells + 63) / 64 * 64;
      if (g.cells > b->max_cells) b->max_cells = g.cells;
      continue;
    }
    for (long long s = 0; s < in.nint; s += BATCH_TILE) tiles.push_back(BatchTile{n, (int)s});
    {
      const int nr = g.n[in.ax_r];
      const int nc = in.ax_c >= 0 ? g.n[in.ax_c] : 1;
      const int np = in.ax_p >= 0 ? g.n[in.ax_p] : 1;
      if (in.ax_p >= 0) {
        // 3-D: block tiles
        for (int pp2 = 0; pp2 < np; ++pp2)
          for (int c0 = 0; c0 < nc; c0 += BATCH_TC)
            for (int r0 = 0; r0 < nr; r0 += BATCH_TR)
              btiles.push_back(make_tile_geo(in, n, BlockTile{n, pp2, c0, r0}));
      } else {
        // 1-D / 2-D: warp-per-row items
        const int cb = b32_row_combo(in.ax_r, in.ax_c);
        const int ch = in.ax_c >= 0 ? ROW_CHUNK : 1;
        for (int c0 = 0; c0 < nc; c0 += ch)
          for (int r0 = 0; r0 < nr; r0 += ROW_OUT)
            rows[cb].push_back(RowItem{n, c0, c0 + ch < nc ? c0 + ch : nc, r0});
        if (in.ax_c >= 0) {
          b->sweep_c[in.ax_c] = true;
          for (int c0 = 0; c0 < nc; c0 += ROW_CHUNK)
            for (int r0 = 0; r0 < nr; r0 += 32)
              rows_c.push_back(RowItem{n, c0, c0 + ROW_CHUNK < nc ? c0 + ROW_CHUNK : nc, r0});
        }
      }
      // near-boundary interior cells, whose ghost images the fills write
      auto nearb = [&](int a2, int x) { return g.s[a2] && (x < g.m[a2] || x >= g.n[a2] - g.m[a2]); };
      for (int x0 = 0; x0 < g.n[0]; ++x0)
        for (int x1 = 0; x1 < g.n[1]; ++x1) {
          const bool row = nearb(0, x0) || nearb(1, x1);
          for (int x2 = 0; x2 < g.n[2]; ++x2) {
            if (!row && !nearb(2, x2)) {
              if (g.n[2] > 2 * g.m[2] && x2 == g.m[2]) x2 = g.n[2] - g.m[2] - 1;  // skip the middle
              continue;
            }
            scells.push_back(make_int4(n, x0, x1, x2));
          }
        }
    }
    off += (g.cells + 63) / 64 * 64;  // instances start on 256-byte (FP32) boundaries
    if (g.cells > b->max_cells) b->max_cells = g.cells;
  }
  b->total = off;
  b->ntiles = (int)tiles.size();
  b->nbtiles = (int)btiles.size();
  std::vector<RowItem> rows_all;
  for (int cb = 0; cb < ROW_COMBOS; ++cb) {
    b->row_off[cb] = (int)rows_all.size();
    rows_all.insert(rows_all.end(), rows[cb].begin(), rows[cb].end());
  }
  b->row_off[ROW_COMBOS] = (int)rows_all.size();
  b->nrows = (int)rows_all.size();
  b->nrows_c = (int)rows_c.size();
  b->nscells = (int)scells.size();

  cudaError_t e = cudaSuccess;
  int dev = 0;
  e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) {
    delete b;
    return bad(MISO_B200_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
  }
  b->grid = b->sms * 8;
  b->bgrid = b32_block_grid(b->sms);
  b->rgrid = 8 * b->sms;  // 8 warps per CTA, one row item per warp at a time
  if (stream) {
    b->stream = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete b;
      return bad(MISO_B200_ERR_CUDA, "stream creation failed");
    }
    b->own_stream = true;
  }
  const size_t cells = (size_t)b->total;
  std::vector<std::pair<void **, size_t>> plan;
  size_t total = 0;
  auto add = [&](void **p, size_t bytes) {
    plan.emplace_back(p, bytes);
    total += round_up(bytes);
  };
  add((void **)&b->d_insts, sizeof(BatchInst) * count);
  add((void **)&b->d_tiles, sizeof(BatchTile) * tiles.size());
  add((void **)&b->d_btiles, sizeof(TileGeo) * (btiles.empty() ? 1 : btiles.size()));
  add((void **)&b->d_rows, sizeof(RowItem) * (rows_all.empty() ? 1 : rows_all.size()));
  add((void **)&b->d_rows_c, sizeof(RowItem) * (rows_c.empty() ? 1 : rows_c.size()));
  add((void **)&b->d_scells, sizeof(int4) * (scells.empty() ? 1 : scells.size()));
  add((void **)&b->d_sc, sizeof(StepScalars) * count);
  add((void **)&b->d_dtmin, sizeof(unsigned int) * count);
  add((void **)&b->d_dtinit, sizeof(unsigned int) * count);
  add((void **)&b->d_err, sizeof(unsigned int));
  if (!b->split) {
    for (int s = 0; s < 3; ++s)
      for (int f = 0; f < NF; ++f) add((void **)&b->q64[s][f], cells * sizeof(double));
    add((void **)&b->cc64, cells * sizeof(double));
  } else {
    for (int s = 0; s < 2; ++s) {
      for (int f = 0; f < NF; ++f) add((void **)&b->hi[s][f], cells * sizeof(float));
      for (int f = 0; f < NF; ++f) add((void **)&b->lo[s][f], cells * sizeof(float));
    }
    for (int s = 0; s < 2; ++s)
      for (int f = 0; f < NF; ++f) add((void **)&b->stg[s][f], cells * sizeof(float));
    add((void **)&b->cc32, cells * sizeof(float));
  }
  e = cudaMalloc(&b->block, total);
  if (e != cudaSuccess) {
    if (b->own_stream) cudaStreamDestroy(b->stream);
    delete b;
    return bad(MISO_B200_ERR_NOMEM, "device allocation of " + std::to_string(total) +
                                        " bytes failed");
  }
  b->bytes = total;
  size_t o = 0;
  for (auto &pb : plan) {
    *pb.first = (char *)b->block + o;
    o += round_up(pb.second);
  }
  if (b->split)  // FP64 staging of one instance over the stage arrays (no state between steps)
    for (int f = 0; f < NF; ++f) b->io64[f] = (double *)b->stg[0][0] + (size_t)f * b->max_cells;
  e = cudaMemsetAsync(b->block, 0, total, b->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_insts, b->insts.data(), sizeof(BatchInst) * count,
                        cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_tiles, tiles.data(), sizeof(BatchTile) * tiles.size(),
                        cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess && !btiles.empty())
    e = cudaMemcpyAsync(b->d_btiles, btiles.data(), sizeof(TileGeo) * btiles.size(),
                        cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess && !rows_all.empty())
    e = cudaMemcpyAsync(b->d_rows, rows_all.data(), sizeof(RowItem) * rows_all.size(),
                        cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess && !rows_c.empty())
    e = cudaMemcpyAsync(b->d_rows_c, rows_c.data(), sizeof(RowItem) * rows_c.size(),
                        cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess && !scells.empty())
    e = cudaMemcpyAsync(b->d_scells, scells.data(), sizeof(int4) * scells.size(),
                        cudaMemcpyHostToDevice, b->stream);
  std::vector<unsigned int> init(count);
  const float big = 1.e10f;
  unsigned int bits;
  memcpy(&bits, &big, sizeof bits);
  for (auto &v : init) v = bits;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_dtmin, init.data(), sizeof(unsigned int) * count,
                        cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_dtinit, init.data(), sizeof(unsigned int) * count,
                        cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) {
    cudaFree(b->block);
    if (b->own_stream) cudaStreamDestroy(b->stream);
    delete b;
    return bad(MISO_B200_ERR_CUDA, std::string("batch set-up: ") + cudaGetErrorString(e));
  }
  // the views of the 3-D split instances, over the batch's arrays
  b->view_at.assign(count, -1);
  int nviews = 0;
  for (int n = 0; n < count; ++n) nviews += b->insts[n].view ? 1 : 0;
  // A grid large enough to fill the GPU with its own persistent kernels
  // steps on the batch's stream, in turn with the rest (run beside other
  // work, its persistent CTAs would not all be resident, and their static
  // share of the work items would finish unevenly); smaller grids run
  // concurrently on the view streams.
  const long long whole_gpu = 1LL << 24;
  int nsmall = 0;
  for (int n = 0; n < count; ++n)
    nsmall += b->insts[n].view && b->insts[n].nint < whole_gpu ? 1 : 0;
  if (nviews) {
    const int ns = nsmall < miso_b200_batch::VIEW_STREAMS ? nsmall : miso_b200_batch::VIEW_STREAMS;
    bool ok = cudaEventCreateWithFlags(&b->vfork, cudaEventDisableTiming) == cudaSuccess;
    for (int s = 0; s < ns && ok; ++s) {
      cudaStream_t vs = nullptr;
      cudaEvent_t ve = nullptr;
      ok = cudaStreamCreateWithFlags(&vs, cudaStreamNonBlocking) == cudaSuccess &&
           cudaEventCreateWithFlags(&ve, cudaEventDisableTiming) == cudaSuccess;
      if (vs) b->vstreams.push_back(vs);
      if (ve) b->vdone.push_back(ve);
    }
    const size_t pitch = round_up(cells * sizeof(float));
    int rc = ok ? MISO_B200_OK : MISO_B200_ERR_CUDA;
    int nlane = 0;
    for (int n = 0; n < count && rc == MISO_B200_OK; ++n) {
      const BatchInst &in = b->insts[n];
      if (!in.view) continue;
      float *hi[2][NF], *lo[2][NF], *stg[2][NF];
      for (int s = 0; s < 2; ++s)
        for (int f = 0; f < NF; ++f) {
          hi[s][f] = b->hi[s][f] + in.base;
          lo[s][f] = b->lo[s][f] + in.base;
          stg[s][f] = b->stg[s][f] + in.base;
        }
      int lane = -1;
      if (in.nint < whole_gpu) {
        lane = nlane % ns;
        ++nlane;
      }
      miso_b200_handle *vh = nullptr;
      rc = b200_view_create(grids[n], params[n], lane >= 0 ? b->vstreams[lane] : b->stream, hi,
                            lo, stg, b->cc32 + in.base, pitch, b->d_sc + n, &vh);
      if (rc == MISO_B200_OK) {
        b->view_at[n] = (int)b->views.size();
        b->views.push_back({n, vh, lane});
      }
    }
    if (rc != MISO_B200_OK) {
      miso_b200_batch_destroy(b);
      return bad(rc, "view set-up of a 3-D instance failed");
    }
  }
  *out = b;
  return MISO_B200_OK;
}

int miso_b200_batch_destroy(miso_b200_batch *b) {
  if (!b) return MISO_B200_ERR_ARG;
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->graph_exec) cudaGraphExecDestroy(b->graph_exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (auto &v : b->views) miso_b200_destroy(v.h);
  for (cudaStream_t s : b->vstreams) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
  for (cudaEvent_t e : b->vdone) cudaEventDestroy(e);
  if (b->vfork) cudaEventDestroy(b->vfork);
  if (b->block) cudaFree(b->block);
  if (b->own_stream) cudaStreamDestroy(b->stream);
  delete b;
  return MISO_B200_OK;
}

int miso_b200_batch_upload(miso_b200_batch *b, int index, const double *const q[9]) {
  if (!b || !q || index < 0 || index >= b->count) return MISO_B200_ERR_ARG;
  b->cfl_valid = false;
  const BatchInst &in = b->insts[index];
  const size_t bytes = (size_t)in.g.cells * sizeof(double);
  int rc;
  for (int f = 0; f < NF; ++f) {
    if (!q[f]) return b->fail(MISO_B200_ERR_ARG, "null field pointer");
    double *dst = b->split ? b->io64[f] : b->q64[0][f] + in.base;
    if ((rc = b->cuda(cudaMemcpyAsync(dst, q[f], bytes, cudaMemcpyDefault, b->stream), "upload")))
      return rc;
  }
  // a view's state goes to the view's own set (with the fused y and z pass
  // its steps keep one set while the batch's other instances alternate)
  const bool is_view = b->view_at.size() && b->view_at[index] >= 0;
  const int set = is_view ? b200_view_cur(b->views[b->view_at[index]].h) : b->cur;
  if (b->split) {
    FieldPtrs<const double> src;
    FieldPtrs<float> h, l;
    for (int f = 0; f < NF; ++f) {
      src.f[f] = b->io64[f];
      h.f[f] = b->hi[set][f] + in.base;
      l.f[f] = b->lo[set][f] + in.base;
    }
    launch_s32_to_split(in.g.cells, src, h, l, b->sms, b->stream);
    if ((rc = b->cuda(cudaGetLastError(), "to_split"))) return rc;
  }
  if ((rc = b->cuda(cudaStreamSynchronize(b->stream), "upload synchronize"))) return rc;
  if (is_view) {
    // a view's ghost layers and CFL minima follow its new state
    const auto &v = b->views[b->view_at[index]];
    if ((rc = b200_view_fill(v.h, set))) return b->fail(rc, miso_b200_last_error(v.h));
    return b->cuda(cudaStreamSynchronize(v.lane >= 0 ? b->vstreams[v.lane] : b->stream),
                   "upload synchronize");
  }
  return MISO_B200_OK;
}

int miso_b200_batch_download(miso_b200_batch *b, int index, double *const q[9]) {
  if (!b || !q || index < 0 || index >= b->count) return MISO_B200_ERR_ARG;
  const BatchInst &in = b->insts[index];
  const size_t bytes = (size_t)in.g.cells * sizeof(double);
  int rc;
  int set = b->cur;  // a view's state sits in the view's own set
  if (b->view_at.size() && b->view_at[index] >= 0) {
    // the lo ghost images of a view lag its interior until a download
    const auto &v = b->views[b->view_at[index]];
    set = b200_view_cur(v.h);
    if ((rc = b->cuda(cudaStreamSynchronize(b->stream), "download synchronize"))) return rc;
    if ((rc = b200_view_fresh_lo(v.h, set))) return b->fail(rc, miso_b200_last_error(v.h));
    if ((rc = b->cuda(cudaStreamSynchronize(v.lane >= 0 ? b->vstreams[v.lane] : b->stream),
                      "download synchronize")))
      return rc;
  }
  if (b->split) {
    FieldPtrs<const float> h, l;
    FieldPtrs<double> dst;
    for (int f = 0; f < NF; ++f) {
      h.f[f] = b->hi[set][f] + in.base;
      l.f[f] = b->lo[set][f] + in.base;
      dst.f[f] = b->io64[f];
    }
    launch_s32_from_split(in.g.cells, h, l, dst, b->sms, b->stream);
    if ((rc = b->cuda(cudaGetLastError(), "from_split"))) return rc;
  }
  for (int f = 0; f < NF; ++f) {
    if (!q[f]) return b->fail(MISO_B200_ERR_ARG, "null field pointer");
    const double *src = b->split ? b->io64[f] : b->q64[0][f] + in.base;
    if ((rc = b->cuda(cudaMemcpyAsync(q[f], src, bytes, cudaMemcpyDefault, b->stream),
                      "download")))
      return rc;
  }
  return b->cuda(cudaStreamSynchronize(b->stream), "download synchronize");
}

int miso_b200_batch_fill_ghosts(miso_b200_batch *b) {
  if (!b) return MISO_B200_ERR_ARG;
  b->cfl_valid = false;
  const BatchArgs a = b->args();
  if (!b->split) {
    b64_fill(a, b->mut(b->q64[0]), b->grid, b->stream);
  } else {
    b32_fill(a, b->mut(b->hi[b->cur]), NF, b->grid, b->stream);
    b32_fill(a, b->mut(b->lo[b->cur]), NF, b->grid, b->stream);
    if (int rc = b->fill_views()) return rc;
  }
  return b->cuda(cudaGetLastError(), "fill_ghosts");
}

int miso_b200_batch_run(miso_b200_batch *b, int nsteps, int use_graph) {
  if (!b || nsteps < 0) return MISO_B200_ERR_ARG;
  int rc;
  if (!use_graph) {
    for (int n = 0; n < nsteps; ++n)
      if ((rc = b->enqueue_step())) return rc;
    return MISO_B200_OK;
  }
  // the captured step relies on the CFL minima folded in by the previous
  // step's last sweep: run one step eagerly first when they are missing
  if (b->split && !b->cfl_valid && nsteps > 0) {
    if ((rc = b->enqueue_step())) return rc;
    --nsteps;
  }
  if (b->graph_exec && b->graph_cur != b->cur) {
    cudaGraphExecDestroy(b->graph_exec);
    cudaGraphDestroy(b->graph);
    b->graph_exec = nullptr;
    b->graph = nullptr;
  }
  if (!b->graph_exec) {
    const int before = b->cur;
    std::vector<int> vbefore;  // the views' own sets (restored with the batch's)
    for (auto &v : b->views) vbefore.push_back(b200_view_cur(v.h));
    const long long l0 = b->launches;
    if ((rc = b->cuda(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal),
                      "begin capture")))
      return rc;
    int steps = 1;
    rc = b->enqueue_step();
    if (!rc && b->cur != before) {
      steps = 2;
      rc = b->enqueue_step();
    }
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    b->cur = before;
    for (size_t n = 0; n < b->views.size(); ++n) b200_view_set_cur(b->views[n].h, vbefore[n]);
    const long long kernels = b->launches - l0;
    b->launches = l0;
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if ((rc = b->cuda(e, "end capture"))) return rc;
    b->graph = g;
    if ((rc = b->cuda(cudaGraphInstantiate(&b->graph_exec, g, 0), "graph instantiate")))
      return rc;
    b->graph_steps = steps;
    b->graph_cur = before;
    b->graph_kernels = kernels;
  }
  const int reps = nsteps / b->graph_steps, rem = nsteps % b->graph_steps;
  for (int n = 0; n < reps; ++n) {
    if ((rc = b->cuda(cudaGraphLaunch(b->graph_exec, b->stream), "graph launch"))) return rc;
    b->launches += b->graph_kernels;
  }
  for (int n = 0; n < rem; ++n)
    if ((rc = b->enqueue_step())) return rc;
  return MISO_B200_OK;
}

int miso_b200_batch_set_chunks(miso_b200_batch *b, int rk_chunk, int av_chunk) {
  if (!b || rk_chunk < 1 || av_chunk < 1) return MISO_B200_ERR_ARG;
  for (auto &v : b->views) {
    const int rc = miso_b200_set_chunks(v.h, rk_chunk, av_chunk);
    if (rc) return b->fail(rc, miso_b200_last_error(v.h));
  }
  if (b->graph_exec) {  // the captured step holds the old work lists
    cudaGraphExecDestroy(b->graph_exec);
    cudaGraphDestroy(b->graph);
    b->graph_exec = nullptr;
    b->graph = nullptr;
  }
  return MISO_B200_OK;
}

int miso_b200_batch_set_variant(miso_b200_batch *b, int kernel_class, int variant) {
  if (!b) return MISO_B200_ERR_ARG;
  if (kernel_class == 0 && (variant < 0 || variant > 3)) return MISO_B200_ERR_ARG;
  // the 1-D / 2-D instances: RK variant 3 defers their last update into the
  // step's first sweep (with the same bits), any other keeps it in the stage
  if (kernel_class == 0) b->defer_rows = variant == 3;
  for (auto &v : b->views) {
    const int rc = miso_b200_set_variant(v.h, kernel_class, variant);
    if (rc) return b->fail(rc, miso_b200_last_error(v.h));
  }
  if (b->graph_exec) {
    cudaGraphExecDestroy(b->graph_exec);
    cudaGraphDestroy(b->graph);
    b->graph_exec = nullptr;
    b->graph = nullptr;
  }
  return MISO_B200_OK;
}

int miso_b200_batch_views(miso_b200_batch *b, int *views) {
  if (!b || !views) return MISO_B200_ERR_ARG;
  *views = (int)b->views.size();
  return MISO_B200_OK;
}

int miso_b200_batch_sync(miso_b200_batch *b) {
  if (!b) return MISO_B200_ERR_ARG;
  return b->read_err();
}

int miso_b200_batch_dt(miso_b200_batch *b, double *dt) {
  if (!b || !dt) return MISO_B200_ERR_ARG;
  std::vector<StepScalars> sc(b->count);
  int rc = b->cuda(cudaMemcpyAsync(sc.data(), b->d_sc, sizeof(StepScalars) * b->count,
                                   cudaMemcpyDeviceToHost, b->stream),
                   "read dt");
  if (rc) return rc;
  if ((rc = b->cuda(cudaStreamSynchronize(b->stream), "synchronize"))) return rc;
  for (int n = 0; n < b->count; ++n) dt[n] = sc[n].dt;
  return MISO_B200_OK;
}

int miso_b200_batch_info(miso_b200_batch *b, long long *interior_cells, int *tiles,
                         long long *launches) {
  if (!b) return MISO_B200_ERR_ARG;
  long long n = 0;
  for (auto &in : b->insts) n += in.nint;
  if (interior_cells) *interior_cells = n;
  if (tiles) *tiles = b->ntiles;
  if (launches) *launches = b->launches;
  return MISO_B200_OK;
}

const char *miso_b200_batch_last_error(miso_b200_batch *b) { return b ? b->err.c_str() : ""; }

}  // extern "C"
