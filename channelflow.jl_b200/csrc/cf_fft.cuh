// cf_fft.cuh -- in-shared-memory complex FFTs (Stockham autosort) for
// batches of transforms owned by a thread group (one warp or one block).
//
// A pass of radix R with Ns = product of the previous radices maps
//   in  x[j + r*L/R]           (j in [0, L/R), r in [0, R))
//   out y[(j/Ns)*Ns*R + j%Ns + r*Ns] = DFT_R(w^(r*(j%Ns)*L/(Ns*R)) x[...])_r
// and after all passes the buffer holds the DFT in natural order.  Each pass
// is done in place: every thread first loads the inputs of all butterflies
// it owns into registers, the group synchronises, then results are stored.
// tw[k] = exp(-2 pi i k / L); sgn = -1 forward, +1 backward (unnormalised).
#pragma once
#include "cf_common.cuh"

#define CF_FFT_MAXPASS 16

struct FftPlan {
    int L;
    int np;
    int R[CF_FFT_MAXPASS];
    const zd* tw;
};

template <bool BLOCK>
CF_DEV void group_sync() {
    if (BLOCK) __syncthreads();
    else __syncwarp();
}

CF_DEV zd tw_get(const zd* tw, int k, int sgn) {
    zd w = __ldg(tw + k);
    return sgn > 0 ? zconj(w) : w;
}

// radix-R DFT of v[0..R) in registers; sgn selects the exponent sign
template <int R>
CF_DEV void dft_small(zd* v, int sgn);

template <>
CF_DEV void dft_small<2>(zd* v, int) {
    zd a = v[0], b = v[1];
    v[0] = zadd(a, b);
    v[1] = zsub(a, b);
}
template <>
CF_DEV void dft_small<3>(zd* v, int sgn) {
    const double h = 0.86602540378443864676;  // sqrt(3)/2
    zd a = v[0], t1 = zadd(v[1], v[2]);
    zd t2 = zaxpy(a, -0.5, t1);
    zd t3 = zscale(zmuli(zsub(v[1], v[2])), h * sgn);
    v[0] = zadd(a, t1);
    v[1] = zadd(t2, t3);
    v[2] = zsub(t2, t3);
}
template <>
CF_DEV void dft_small<4>(zd* v, int sgn) {
    zd a0 = zadd(v[0], v[2]), a1 = zsub(v[0], v[2]);
    zd a2 = zadd(v[1], v[3]), a3 = zscale(zmuli(zsub(v[1], v[3])), (double)sgn);
    v[0] = zadd(a0, a2);
    v[2] = zsub(a0, a2);
    v[1] = zadd(a1, a3);
    v[3] = zsub(a1, a3);
}
template <>
CF_DEV void dft_small<5>(zd* v, int sgn) {
    const double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;
    const double s1 = 0.95105651629515357212, s2 = 0.58778525229247312917;
    zd a0 = v[0];
    zd p14 = zadd(v[1], v[4]), m14 = zsub(v[1], v[4]);
    zd p23 = zadd(v[2], v[3]), m23 = zsub(v[2], v[3]);
    zd r1 = zaxpy(zaxpy(a0, c1, p14), c2, p23);
    zd r2 = zaxpy(zaxpy(a0, c2, p14), c1, p23);
    zd i1 = zscale(zmuli(zaxpy(zscale(m14, s1), s2, m23)), (double)sgn);
    zd i2 = zscale(zmuli(zaxpy(zscale(m14, s2), -s1, m23)), (double)sgn);
    v[0] = zadd(a0, zadd(p14, p23));
    v[1] = zadd(r1, i1);
    v[4] = zsub(r1, i1);
    v[2] = zadd(r2, i2);
    v[3] = zsub(r2, i2);
}
template <>
CF_DEV void dft_small<8>(zd* v, int sgn) {
    const double h = 0.70710678118654752440;
    zd e[4] = {v[0], v[2], v[4], v[6]};
    zd o[4] = {v[1], v[3], v[5], v[7]};
    dft_small<4>(e, sgn);
    dft_small<4>(o, sgn);
    // w = exp(sgn i pi/4)
    zd w1o = zmake(h * (o[1].x - sgn * o[1].y), h * (o[1].y + sgn * o[1].x));
    zd w2o = zscale(zmuli(o[2]), (double)sgn);
    zd w3o = zmake(h * (-o[3].x - sgn * o[3].y), h * (-o[3].y + sgn * o[3].x));
    v[0] = zadd(e[0], o[0]);
    v[4] = zsub(e[0], o[0]);
    v[1] = zadd(e[1], w1o);
    v[5] = zsub(e[1], w1o);
    v[2] = zadd(e[2], w2o);
    v[6] = zsub(e[2], w2o);
    v[3] = zadd(e[3], w3o);
    v[7] = zsub(e[3], w3o);
}

// One in-place pass of compile-time radix R over nb transforms of length L
// (transform b starts at buf + b*bs).  MAXE bounds the complex registers per
// thread: the caller guarantees ceil(nb*L/R / nth) * R <= MAXE.
template <bool BLOCK, int R, int MAXE>
CF_DEV void fft_pass_t(zd* buf, int nb, int bs, int L, int Ns, const zd* tw, int sgn, int tid, int nth) {
    constexpr int MB = MAXE / R;
    const int NBf = L / R;
    const int total = nb * NBf;
    const int step = L / (Ns * R);
    zd v[MB > 0 ? MB : 1][R];
#pragma unroll
    for (int t = 0; t < MB; ++t) {
        int q = tid + t * nth;
        if (q < total) {
            int b = q / NBf, j = q - b * NBf;
            int k = j % Ns;
            const zd* src = buf + (long)b * bs;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                zd x = src[j + r * NBf];
                v[t][r] = (r == 0 || k == 0) ? x : zmul(x, tw_get(tw, k * r * step, sgn));
            }
        }
    }
    group_sync<BLOCK>();
#pragma unroll
    for (int t = 0; t < MB; ++t) {
        int q = tid + t * nth;
        if (q < total) {
            int b = q / NBf, j = q - b * NBf;
            int k = j % Ns;
            dft_small<R>(v[t], sgn);
            zd* dst = buf + (long)b * bs + (j / Ns) * Ns * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) dst[r * Ns] = v[t][r];
        }
    }
    group_sync<BLOCK>();
}

// Generic odd prime radix (R <= 31): direct DFT; used only for sizes with
// uncommon prime factors.  Same in-place protocol, registers in local memory.
template <bool BLOCK, int MAXE>
CF_DEV void fft_pass_generic(zd* buf, int nb, int bs, int L, int R, int Ns, const zd* tw, int sgn, int tid,
                             int nth) {
    const int NBf = L / R;
    const int total = nb * NBf;
    const int step = L / (Ns * R);
    const int mb = (total + nth - 1) / nth;
    zd v[MAXE];
    for (int t = 0; t < mb; ++t) {
        int q = tid + t * nth;
        if (q < total) {
            int b = q / NBf, j = q - b * NBf;
            int k = j % Ns;
            const zd* src = buf + (long)b * bs;
            for (int r = 0; r < R; ++r) {
                zd x = src[j + r * NBf];
                v[t * R + r] = (r == 0 || k == 0) ? x : zmul(x, tw_get(tw, k * r * step, sgn));
            }
        }
    }
    group_sync<BLOCK>();
    for (int t = 0; t < mb; ++t) {
        int q = tid + t * nth;
        if (q < total) {
            int b = q / NBf, j = q - b * NBf;
            int k = j % Ns;
            zd* dst = buf + (long)b * bs + (j / Ns) * Ns * R + k;
            for (int s = 0; s < R; ++s) {
                zd acc = v[t * R];
                for (int r = 1; r < R; ++r) acc = zadd(acc, zmul(v[t * R + r], tw_get(tw, ((s * r) % R) * NBf, sgn)));
                dst[s * Ns] = acc;
            }
        }
    }
    group_sync<BLOCK>();
}

// Full transform of nb batched sequences (length pl.L, batch stride bs).
template <bool BLOCK, int MAXE>
CF_DEV void group_fft(zd* buf, int nb, int bs, const FftPlan& pl, int sgn, int tid, int nth) {
    int Ns = 1;
    for (int p = 0; p < pl.np; ++p) {
        const int R = pl.R[p];
        switch (R) {
            case 2: fft_pass_t<BLOCK, 2, MAXE>(buf, nb, bs, pl.L, Ns, pl.tw, sgn, tid, nth); break;
            case 3: fft_pass_t<BLOCK, 3, MAXE>(buf, nb, bs, pl.L, Ns, pl.tw, sgn, tid, nth); break;
            case 4: fft_pass_t<BLOCK, 4, MAXE>(buf, nb, bs, pl.L, Ns, pl.tw, sgn, tid, nth); break;
            case 5: fft_pass_t<BLOCK, 5, MAXE>(buf, nb, bs, pl.L, Ns, pl.tw, sgn, tid, nth); break;
            case 8: fft_pass_t<BLOCK, 8, MAXE>(buf, nb, bs, pl.L, Ns, pl.tw, sgn, tid, nth); break;
            default: fft_pass_generic<BLOCK, MAXE>(buf, nb, bs, pl.L, R, Ns, pl.tw, sgn, tid, nth); break;
        }
        Ns *= R;
    }
}
