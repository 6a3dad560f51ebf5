// Host-side launch entry points of the FP32 split-precision kernels
// (internal to the library).
#pragma once

#include "common.cuh"

namespace miso_b200 {

void launch_s32_rk_stage(const Geom &g, const FieldPtrs<const float> &prev,
                         const FieldPtrs<float> &hi, const FieldPtrs<float> &lo,
                         const FieldPtrs<float> &out, const StepScalars *sc, int stage, double gm,
                         const Source &src, int sms, cudaStream_t st);
void launch_s32_char_velocity(const Geom &g, const FieldPtrs<const float> &u, float *cc,
                              double gm, double cs_fac, double vv_fac, double ca_fac, int sms,
                              cudaStream_t st);
void launch_s32_av_sweep(const Geom &g, const FieldPtrs<const float> &hi,
                         const FieldPtrs<const float> &lo, const FieldPtrs<float> &hi2,
                         const FieldPtrs<float> &lo2, const float *cc, const StepScalars *sc,
                         int dir, double ep, double fh, int sms, cudaStream_t st);
// the magnetosphere demo's boundary on the split state: hi + lo (pair) or
// a stage buffer's single words (hi), every cell
void launch_s32_magneto(const Geom &g, const FieldPtrs<float> &hi, const FieldPtrs<float> &lo,
                        bool pair, const Magneto &mg, double gm, int sms, cudaStream_t st);
void launch_s32_cfl_partial(const Geom &g, const FieldPtrs<const float> &u, float *partial,
                            int nparts, StepScalars *sc, double gm, double cfl_dx,
                            cudaStream_t st, const Magneto &mg = Magneto{},
                            const FieldPtrs<const float> &lo = FieldPtrs<const float>{});
void launch_s32_to_split(long long cells, const FieldPtrs<const double> &q,
                         const FieldPtrs<float> &hi, const FieldPtrs<float> &lo, int sms,
                         cudaStream_t st);
void launch_s32_from_split(long long cells, const FieldPtrs<const float> &hi,
                           const FieldPtrs<const float> &lo, const FieldPtrs<double> &q, int sms,
                           cudaStream_t st);

}  // namespace miso_b200
