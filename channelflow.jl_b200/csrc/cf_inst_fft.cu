// cf_inst_fft.cu -- the periodic-transform kernels of one padded length
// L = CF_INST_L (0: the run-time-sized instantiation); compiled once per length.
#include "cf_dispatch.h"

#ifndef CF_INST_L
#error "compile with -DCF_INST_L=<length>"
#endif

template <int L>
FftKernel fft_kernel_for(int which, bool f32) {
    switch (which) {
        case KF_ZINV: return f32 ? k_zinv<L, zf> : k_zinv<L, zd>;
        case KF_ZFWD: return f32 ? k_zfwd<L, zf> : k_zfwd<L, zd>;
        case KF_XPASS_CONV: return k_xpass_conv<L>;
        case KF_XPASS_DIV: return k_xpass_div<L>;
        case KF_XPASS2: return k_xpass2<L>;
        case KF_XPASS_IP: return f32 ? k_xpass_ip32<L> : k_xpass_ip<L>;
        case KF_XPASS_CONV_IP: return k_xpass_conv_ip<L>;
        case KF_XPASS_DIV_IP: return k_xpass_div_ip<L>;
        default: return f32 ? k_xpass<L, zf> : k_xpass<L, zd>;
    }
}
template <int L>
FftBatchKernel fft_batch_kernel_for(int which) {
    switch (which) {
        case KF_ZINV: return k_zinv_batch<L>;
        case KF_ZFWD: return k_zfwd_batch<L>;
        case KF_XPASS_R4: return k_xpass_rows_batch<L, 4>;
        case KF_XPASS_R8: return k_xpass_rows_batch<L, 8>;
        case KF_XPASS_R16: return k_xpass_rows_batch<L, 16>;
        default: return k_xpass_batch<L>;
    }
}

template <int L>
FftTmaKernel fft_tma_kernel_for(int which, bool f32) {
    if (which == KF_ZINV) return f32 ? k_zinv_tma<L, zf> : k_zinv_tma<L, zd>;
    return f32 ? k_zfwd_tma<L, zf> : k_zfwd_tma<L, zd>;
}

template FftKernel fft_kernel_for<CF_INST_L>(int, bool);
template FftTmaKernel fft_tma_kernel_for<CF_INST_L>(int, bool);
template FftBatchKernel fft_batch_kernel_for<CF_INST_L>(int);
