// Gather and scatter of the j and k face halos of a grid in shards
// (internal to the library).  Along i a face's layers are whole planes,
// contiguous in memory, and travel in place; a j face is `margin` rows of
// every plane and a k face `margin` words of every row, so around the
// exchange callback the library copies the `margin` interior layers next to
// each shared face into contiguous buffers and, after the callback, the
// received layers into the ghost layers: the reference's pack_y_send /
// pack_z_send and unpack_y_recv / unpack_z_recv
// (miso/include/miso/mhd_halo_exchange.hpp:303-364, 395-450), here one launch
// for both faces and every array.  A face buffer holds one array's layers in
// the arrays' own memory order (i, then j, then k fastest) over the full
// extent of the two other axes, ghosts included, as the reference's buffers
// do (its edge and corner ghosts then come from the neighbour as well; no
// stencil reads them).
#include "kernels.h"

namespace miso_b200 {

template <typename T>
__global__ void __launch_bounds__(256) face_copy_kernel(const FaceArgs f) {
  const long long per_side = (long long)f.n * f.face;
  const long long total = 2 * per_side;
  for (long long lin = blockIdx.x * (long long)blockDim.x + threadIdx.x; lin < total;
       lin += (long long)gridDim.x * blockDim.x) {
    const int side = lin >= per_side ? 1 : 0;
    if (!f.ext[side]) continue;
    const long long r = lin - side * per_side;
    const int arr = (int)(r / f.face);
    const long long e = r - (long long)arr * f.face;
    // coordinates inside the face box (d0, d1, d2), k fastest
    const long long x2 = e % f.d[2];
    const long long q = e / f.d[2];
    const long long x1 = q % f.d[1];
    const long long x0 = q / f.d[1];
    const long long cell = (x0 + (f.axis == 0 ? f.start[side] : 0)) * f.st[0] +
                           (x1 + (f.axis == 1 ? f.start[side] : 0)) * f.st[1] +
                           (x2 + (f.axis == 2 ? f.start[side] : 0));
    T *a = static_cast<T *>(f.arr[arr]);
    T *b = static_cast<T *>(f.buf[side]) + (long long)arr * f.face + e;
    if (f.pack)
      *b = a[cell];
    else
      a[cell] = *b;
  }
}

void launch_face_copy(const FaceArgs &f, size_t elem, int sms, cudaStream_t st) {
  const long long total = 2LL * f.n * f.face;
  long long blocks = (total + 255) / 256;
  if (blocks > 8LL * sms) blocks = 8LL * sms;
  if (blocks < 1) blocks = 1;
  if (elem == sizeof(double))
    face_copy_kernel<double><<<(unsigned)blocks, 256, 0, st>>>(f);
  else
    face_copy_kernel<float><<<(unsigned)blocks, 256, 0, st>>>(f);
}

}  // namespace miso_b200
