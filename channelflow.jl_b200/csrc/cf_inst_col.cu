// cf_inst_col.cu -- the column kernels of one Chebyshev length P = CF_INST_P
// (0: the run-time-sized instantiation); compiled once per length.
#include "cf_dispatch.h"

#ifndef CF_INST_P
#error "compile with -DCF_INST_P=<length>"
#endif
static_assert(CF_TEAM == col_team_threads(CF_INST_P), "the unit's team size is the host's");
// blocks per SM of a batched variant: n for two-warp teams, 3n/2 for one-warp
// teams (a register bound between the two-warp variants' and twice as many
// columns per SM)
#define CF_MINB(n) (CF_TEAM == 64 ? (n) : 3 * (n) / 2)

template <int P>
ColKernel col_kernel_for(int which) {
    switch (which) {
        case KC_STAGE: return k_column_stage<CF_NCOL, P>;
        case KC_PREP: return k_column_prep<CF_NCOL, P>;
        case KC_NLOUT: return k_column_nlout<CF_NCOL, P>;
        case KC_PROJECT: return k_column_project<CF_NCOL, P>;
        case KC_STAGE_MX: return k_column_stage_mx<CF_NCOL, P, 1>;
        case KC_PREP_MX: return k_column_prep<CF_NCOL, P, 1>;
        case KC_STAGE_MXD: return k_column_stage_mx<CF_NCOL, P, 2>;
        case KC_PREP_MXD: return k_column_prep<CF_NCOL, P, 2>;
        case KC_STAGE_MXS: return k_column_stage_mx<CF_NCOL, P, 3>;
        case KC_PREP_MXS: return k_column_prep<CF_NCOL, P, 3>;
        case KC_STAGE_CONV: return k_column_stage<CF_NCOL, P, NL_CONV>;
        case KC_PREP_CONV: return k_column_prep<CF_NCOL, P, 0, NL_CONV>;
        case KC_STAGE_DIV: return k_column_stage<CF_NCOL, P, NL_DIV>;
        case KC_PREP_DIV: return k_column_prep<CF_NCOL, P, 0, NL_DIV>;
        case KC_DIV: return k_column_div<CF_NCOL, P>;
        case KC_PRESSURE_COEF: return k_column_pressure<CF_NCOL, P, true>;
        default: return k_column_pressure<CF_NCOL, P>;
    }
}
template <int P>
DiagKernel diag_kernel_for() {
    return k_column_diag<CF_NCOL, P>;
}
template <int P>
ColBatchKernel col_batch_kernel_for(int variant) {
    if constexpr (col_batch_variants(P)) {
        switch (variant) {
            case 1: return k_column_stage_batch<2, P, CF_MINB(6)>;
            case 2: return k_column_stage_batch<2, P, CF_MINB(8)>;
            case 3: return k_column_stage_batch<1, P, CF_MINB(8)>;
            case 4: return k_column_stage_batch<1, P, CF_MINB(12)>;
            case 5: return k_column_stage_batch<1, P, CF_MINB(16)>;
            default: break;
        }
    }
    return k_column_stage_batch<CF_NCOL, P, col_minblocks<CF_NCOL, P>()>;
}

template ColKernel col_kernel_for<CF_INST_P>(int);
template DiagKernel diag_kernel_for<CF_INST_P>();
template ColBatchKernel col_batch_kernel_for<CF_INST_P>(int);
