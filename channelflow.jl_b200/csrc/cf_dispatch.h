// cf_dispatch.h -- kernel tables of the engine.  The kernels of one size (the
// Chebyshev length P of the column kernels, the padded length L of the
// periodic transforms) are instantiated in their own translation unit
// (cf_inst_col.cu, cf_inst_fft.cu, compiled once per size with CF_INST_P or
// CF_INST_L defined), so the library builds in parallel; the host code in
// cf_engine.cu picks a size's table through these declarations.
#pragma once
#include "cf_fftkernels.cuh"
#include "cf_kernels.cuh"

#ifndef CF_NCOL
#define CF_NCOL 2
#endif
static_assert(CF_NCOL == 1 || CF_NCOL == 2, "column teams use named barriers 1 and 2");

// Column-kernel lengths P and periodic lengths L with compile-time
// instantiations; other sizes use the run-time-sized one (argument 0).
#define CF_COL_LENGTHS(X) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384)

__host__ __device__ constexpr bool col_static_length(int P) {
#define CF_CASE(N) P == N ||
    return CF_COL_LENGTHS(CF_CASE) false;
#undef CF_CASE
}
// Threads per column of the column kernels of length P: one warp (a half warp
// per parity) for the compile-time lengths up to 64, two warps otherwise (the
// CF_TEAM of the length's translation unit).
__host__ __device__ constexpr int col_team_threads(int P) {
    return (col_static_length(P) && P <= CF_COL_TW_MAXP) ? 32 : 64;
}

typedef void (*ColKernel)(ColParams);
typedef void (*FftKernel)(FftParams);
typedef void (*DiagKernel)(ColParams, double*, double*);
typedef void (*ColBatchKernel)(const ColParams*, int, int, unsigned*);
// Variants of the batched column kernel the ensemble autotuner chooses from:
// (columns per block, blocks per SM of the register bound, for two-warp
// teams; 3/2 as many blocks for one-warp teams).  Variant 0 is the
// single-instance kernel's shape; 1-5 exist for P <= 128 (fewer registers,
// more blocks per SM).
#define CF_COL_BATCH_VARIANTS 6
static constexpr int kColBatchNcol[CF_COL_BATCH_VARIANTS] = {CF_NCOL, 2, 2, 1, 1, 1};
static constexpr int kColBatchMinb[CF_COL_BATCH_VARIANTS] = {0, 6, 8, 8, 12, 16};
__host__ __device__ constexpr bool col_batch_variants(int P) { return P != 0 && P <= 128; }
// blocks per SM of variant v at length P (the CF_MINB of cf_inst_col.cu)
static inline int col_batch_minb(int P, int v) {
    return col_team_threads(P) == 64 ? kColBatchMinb[v] : 3 * kColBatchMinb[v] / 2;
}
typedef void (*FftBatchKernel)(const FftParams*);
typedef void (*FftTmaKernel)(FftParams, FftMaps);

enum {
    KC_STAGE, KC_PREP, KC_NLOUT, KC_PROJECT, KC_PRESSURE, KC_STAGE_MX, KC_PREP_MX,
    KC_STAGE_CONV, KC_PREP_CONV, KC_STAGE_DIV, KC_PREP_DIV, KC_DIV, KC_PRESSURE_COEF,
    KC_STAGE_MXD, KC_PREP_MXD, KC_STAGE_MXS, KC_PREP_MXS, KC_COUNT
};
enum { KF_ZINV, KF_ZFWD, KF_XPASS, KF_XPASS_CONV, KF_XPASS_DIV, KF_XPASS2, KF_XPASS_IP, KF_XPASS_CONV_IP, KF_XPASS_DIV_IP, KF_COUNT };
// rows per block of the batched x-pass variants (KF_XPASS: 2; the others for
// short rows, chosen by the ensemble autotuner)
enum { KF_XPASS_R4 = KF_COUNT, KF_XPASS_R8, KF_XPASS_R16 };

// defined for P in CF_COL_LENGTHS and 0 (cf_inst_col.cu)
template <int P>
ColKernel col_kernel_for(int which);
template <int P>
DiagKernel diag_kernel_for();
template <int P>
ColBatchKernel col_batch_kernel_for(int variant);
// defined for L in CF_STATIC_FFT_LENGTHS and 0 (cf_inst_fft.cu); f32: the
// FP32 transforms of the mixed-precision form
template <int L>
FftKernel fft_kernel_for(int which, bool f32);
template <int L>
FftBatchKernel fft_batch_kernel_for(int which);
// the z kernels with TMA row transfers (which: KF_ZINV or KF_ZFWD)
template <int L>
FftTmaKernel fft_tma_kernel_for(int which, bool f32);
