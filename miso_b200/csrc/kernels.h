// Host-side launch entry points of the device kernels (internal to the
// library; the public interface is include/miso_b200.h).
#pragma once

#include "common.cuh"

namespace miso_b200 {

// ---- FP64 form (bit-faithful to the reference's double host path) ----
void launch_fp64_rhs_stage(const Geom &g, const FieldPtrs<const double> &o,
                           const FieldPtrs<const double> &a, const FieldPtrs<double> &r,
                           const StepScalars *sc, int stage, double gm, const Source &src,
                           int sms, cudaStream_t st);
void launch_fp64_char_velocity(const Geom &g, const FieldPtrs<const double> &q, double *cc,
                               double gm, double cs_fac, double vv_fac, double ca_fac, int sms,
                               cudaStream_t st);
void launch_fp64_av_sweep(const Geom &g, const FieldPtrs<const double> &q,
                          const FieldPtrs<double> &r, const double *cc, const StepScalars *sc,
                          int dir, double ep, double fh, int sms, cudaStream_t st);
int cfl_partial_blocks(int sms);
void launch_fp64_cfl(const Geom &g, const FieldPtrs<const double> &q, float *partial,
                     StepScalars *sc, double gm, double cfl_number, double cfl_dx,
                     double min_dxyz, const Magneto &mg, int sms, cudaStream_t st);
void launch_cfl_finalize(const float *partial, int nparts, StepScalars *sc, double cfl_number,
                         double min_dxyz, cudaStream_t st);
// the magnetosphere demo's boundary after a mirror fill (FP64 state)
void launch_magneto_bc(const Geom &g, const FieldPtrs<double> &q, const Magneto &mg, double gm,
                       int sms, cudaStream_t st);
template <typename T>
void launch_fill_ghosts(const Geom &g, const FieldPtrs<T> &q, int nfields, int sms,
                        cudaStream_t st);

// The j or k face halo of a grid in shards (face_pack.cu): pack = 1 copies
// the `margin` interior layers next to each shared face (ext[side]) of n
// arrays into buf[side]; pack = 0 copies buf[side] into the ghost layers.
// A face of one array is the box d0 x d1 x d2 (the margin on `axis`, the
// full extent elsewhere) starting at layer start[side] of `axis`.
struct FaceArgs {
  void *arr[2 * NF + 1];
  int n;
  int axis;
  int pack;
  int ext[2];
  int start[2];
  long long d[3];
  long long st[3];
  long long face;  // elements of one array's face
  void *buf[2];
};
void launch_face_copy(const FaceArgs &f, size_t elem, int sms, cudaStream_t st);

}  // namespace miso_b200
