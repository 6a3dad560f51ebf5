// Allocation-free CFL time step over caller-owned FP64 fields.
//
// Some callers cannot let a library call cudaMalloc: applications that
// hand every byte of device memory to their own pool or hold it to a fixed
// budget (a cudaMalloc behind their back can fail, or fragment the memory
// they plan for), and applications whose other streams must not be stalled
// (cudaMalloc and cudaFree can synchronise the whole device, while this call
// waits for its own stream only).  For them miso_b200_cfl_noalloc() computes
// the same float-rounded CFL time step as miso_b200_cfl() -- the minimum
// over interior cells of cfl * min(dx, dy, dz) / (cs + |v| + ca) -- on 9
// device arrays the caller passes, without allocating anything: its only
// scratch (per-block partial minima, the result and an error word) is the
// file-scope device array below, which every GPU that loads the library
// keeps until the process exits.  The call copies the result to the host
// and waits for `stream` before it returns.
//
// Compiled with --fmad=false like the FP64 step kernels, so the candidate
// time step of every cell rounds exactly as on the reference's host path
// (mhd_integrator_host.hpp:303-334, eos.hpp:36-42, utility.hpp:91-124).
#include <cuda.h>

#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/miso_b200.h"
#include "common.cuh"

void miso_b200_set_global_error(const std::string &msg);  // capi.cu

namespace miso_b200 {
namespace noalloc {

// Largest number of partial minima: one per 16384 interior cells, so grids
// of up to 16384 * 16384 = 268,435,456 interior cells (e.g. 640^3).
constexpr int MAX_PARTIALS = 16384;
constexpr long long CELLS_PER_PARTIAL = 16384;
constexpr int THREADS = 256;
constexpr int SLOT_DT = MAX_PARTIALS;       // float: the reduced time step
constexpr int SLOT_ERR = MAX_PARTIALS + 1;  // unsigned bits: ERRBIT_NONFINITE
constexpr int SLOTS = MAX_PARTIALS + 64;    // 65,792 bytes in total

static __device__ __align__(256) float g_scratch[SLOTS];

// Device address of g_scratch, fetched once per device (a host-side use of
// the symbol's name is a host stand-in, not a device address).
struct DeviceScratch {
  bool ready = false;
  float *ptr = nullptr;
};
constexpr int MAX_DEVICES = 64;
DeviceScratch g_dev[MAX_DEVICES];
std::mutex g_mu;

__global__ void __launch_bounds__(THREADS)
cfl_partial_kernel(Geom g, FieldPtrs<const double> q, float *scratch, double gm,
                   double cfl_dx) {
  const long long nint = (long long)g.n[0] * g.n[1] * g.n[2];
  const long long begin = (long long)blockIdx.x * CELLS_PER_PARTIAL;
  const long long end = begin + CELLS_PER_PARTIAL < nint ? begin + CELLS_PER_PARTIAL : nint;
  float best = 1.e10f;
  bool bad = false;
  for (long long lin = begin + threadIdx.x; lin < end; lin += THREADS) {
    const int k = (int)(lin % g.n[2]) + g.m[2];
    const long long r1 = lin / g.n[2];
    const int j = (int)(r1 % g.n[1]) + g.m[1];
    const int i = (int)(r1 / g.n[1]) + g.m[0];
    const long long c = i * g.st[0] + j * g.st[1] + k;
    const double ro = q.f[RO][c], vx = q.f[VX][c], vy = q.f[VY][c], vz = q.f[VZ][c];
    const double bx = q.f[BX][c], by = q.f[BY][c], bz = q.f[BZ][c], ei = q.f[EI][c];
    const double cs = sqrt(gm * (gm - 1.0) * ei);
    const double vv = sqrt(+vx * vx + vy * vy + vz * vz);
    const double ca = sqrt((+bx * bx + by * by + bz * bz) / ro * PII4);
    const double total_vel = cs + vv + ca;
    best = fminf(best, __double2float_rn(cfl_dx / total_vel));
    bad |= !(ro > 0.0) || !(ei >= 0.0) || !isfinite(total_vel);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) best = fminf(best, __shfl_xor_sync(0xffffffffu, best, o));
  __shared__ float red[THREADS / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = best;
  if (bad) atomicOr(reinterpret_cast<unsigned int *>(scratch + SLOT_ERR), ERRBIT_NONFINITE);
  __syncthreads();
  if (threadIdx.x == 0) {
    float b = red[0];
    for (int w = 1; w < THREADS / 32; ++w) b = fminf(b, red[w]);
    scratch[blockIdx.x] = b;
  }
}

__global__ void __launch_bounds__(1024) cfl_finalize_kernel(float *scratch, int nparts) {
  float best = 1.e10f;
  for (int n = threadIdx.x; n < nparts; n += blockDim.x) best = fminf(best, scratch[n]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) best = fminf(best, __shfl_xor_sync(0xffffffffu, best, o));
  __shared__ float red[32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    float b = red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) b = fminf(b, red[w]);
    scratch[SLOT_DT] = b;
  }
}

int fail(int code, const std::string &msg) {
  miso_b200_set_global_error("miso_b200_cfl_noalloc: " + msg);
  return code;
}

// cuMemGetAddressRange through the runtime's driver entry point (no link
// against libcuda); null when the driver does not provide it.
using AddressRangeFn = CUresult (*)(CUdeviceptr *, size_t *, CUdeviceptr);
AddressRangeFn address_range_fn() {
  static AddressRangeFn fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<AddressRangeFn>(p);
  }();
  return fn;
}

// The array [p, p + bytes) must be device (or managed) memory of device
// `dev`, inside one allocation.  Host pointers, pinned host memory and
// arrays shorter than the grid are refused before any launch.  Neither
// query allocates.
bool device_array_ok(const void *p, size_t bytes, int dev, std::string &why) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();  // the query's error is not sticky; clear it
    why = "field pointer is not known to CUDA";
    return false;
  }
  if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) {
    why = "field pointer is not device memory";
    return false;
  }
  if (at.device != dev) {
    why = "field array lives on another device";
    return false;
  }
  // fail closed: without the extent query nothing is launched
  AddressRangeFn fn = address_range_fn();
  if (!fn) {
    why = "the driver offers no cuMemGetAddressRange to check the field arrays";
    return false;
  }
  CUdeviceptr base = 0;
  size_t size = 0;
  if (fn(&base, &size, (CUdeviceptr)p) != CUDA_SUCCESS) {
    why = "field pointer is not inside a device allocation";
    return false;
  }
  if ((CUdeviceptr)p + bytes > base + size) {
    why = "field array is shorter than the grid (ghosts included)";
    return false;
  }
  return true;
}

}  // namespace noalloc
}  // namespace miso_b200

using namespace miso_b200;

extern "C" int miso_b200_cfl_noalloc(const miso_b200_grid_desc *gd, const miso_b200_params *pp,
                                     const double *const q[9], void *stream, double *dt_out) {
  using namespace noalloc;
  if (!gd || !pp || !q || !dt_out) return fail(MISO_B200_ERR_ARG, "null argument");
  for (int f = 0; f < NF; ++f)
    if (!q[f]) return fail(MISO_B200_ERR_ARG, "null field pointer");
  if (gd->margin < 2) return fail(MISO_B200_ERR_ARG, "margin must be >= 2");
  if (!(pp->gm > 1.0) || !(pp->cfl_number > 0.0))
    return fail(MISO_B200_ERR_ARG, "invalid physics parameters");
  const int sz[3] = {gd->i_size, gd->j_size, gd->k_size};
  const double lo[3] = {gd->x_min, gd->y_min, gd->z_min};
  const double hi[3] = {gd->x_max, gd->y_max, gd->z_max};
  Geom g{};
  double ds[3];
  for (int a = 0; a < 3; ++a) {
    if (sz[a] < 1 || (sz[a] > 1 && sz[a] < gd->margin) || !(lo[a] < hi[a]))
      return fail(MISO_B200_ERR_ARG, "invalid grid size or range");
    g.n[a] = sz[a];
    g.s[a] = sz[a] > 1 ? 1 : 0;
    g.m[a] = gd->margin * g.s[a];
    g.t[a] = sz[a] + 2 * g.m[a];
    const double sp = (hi[a] - lo[a]) / (double)sz[a];
    ds[a] = g.s[a] ? sp : 1.e30;  // grid.hpp:67-90
  }
  g.st[2] = 1;
  g.st[1] = g.t[2];
  g.st[0] = (long long)g.t[1] * g.t[2];
  g.cells = (long long)g.t[0] * g.t[1] * g.t[2];
  const long long nint = (long long)g.n[0] * g.n[1] * g.n[2];
  const long long nparts = (nint + CELLS_PER_PARTIAL - 1) / CELLS_PER_PARTIAL;
  if (nparts > MAX_PARTIALS)
    return fail(MISO_B200_ERR_ARG,
                "grid too large for miso_b200_cfl_noalloc: " + std::to_string(nint) +
                    " interior cells, at most " +
                    std::to_string((long long)MAX_PARTIALS * CELLS_PER_PARTIAL));
  // mhd_integrator_host.hpp:323-325: cfl * min3(dx, dy, dz) through float
  const float m3 = fminf(fminf((float)ds[0], (float)ds[1]), (float)ds[2]);
  const double cfl_dx = pp->cfl_number * (double)m3;

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(MISO_B200_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= MAX_DEVICES) return fail(MISO_B200_ERR_ARG, "device index out of range");
  for (int f = 0; f < NF; ++f) {
    std::string why;
    if (!device_array_ok(q[f], (size_t)g.cells * sizeof(double), dev, why))
      return fail(MISO_B200_ERR_ARG, why + " (field " + std::to_string(f) + ")");
  }
  float *scratch = nullptr;
  {
    // once per device, with that device current
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_dev[dev].ready) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_scratch);
      if (e != cudaSuccess) {
        miso_b200_set_global_error(std::string("miso_b200_cfl_noalloc: cudaGetSymbolAddress: ") +
                                   cudaGetErrorString(e));
        return MISO_B200_ERR_CUDA;
      }
      g_dev[dev].ptr = static_cast<float *>(p);
      g_dev[dev].ready = true;
    }
    scratch = g_dev[dev].ptr;
  }
  cudaStream_t st = (cudaStream_t)stream;
  FieldPtrs<const double> qp;
  for (int f = 0; f < NF; ++f) qp.f[f] = q[f];
  // the error word starts at zero for this call; the partial minima are
  // all rewritten by the partial kernel
  e = cudaMemsetAsync(scratch + SLOT_ERR, 0, sizeof(unsigned int), st);
  if (e != cudaSuccess) return fail(MISO_B200_ERR_CUDA, cudaGetErrorString(e));
  cfl_partial_kernel<<<(int)nparts, THREADS, 0, st>>>(g, qp, scratch, pp->gm, cfl_dx);
  cfl_finalize_kernel<<<1, 1024, 0, st>>>(scratch, (int)nparts);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(MISO_B200_ERR_CUDA, cudaGetErrorString(e));
  float out[2];
  e = cudaMemcpyAsync(out, scratch + SLOT_DT, sizeof out, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(MISO_B200_ERR_CUDA, cudaGetErrorString(e));
  unsigned int err_bits;
  memcpy(&err_bits, &out[1], sizeof err_bits);
  if (err_bits & ERRBIT_NONFINITE)
    return fail(MISO_B200_ERR_NONFINITE,
                "non-positive or non-finite density / internal energy in the CFL pass");
  *dt_out = (double)out[0];
  return MISO_B200_OK;
}
