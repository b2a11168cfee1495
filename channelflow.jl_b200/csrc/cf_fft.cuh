// cf_fft.cuh -- in-shared-memory complex FFTs (Stockham autosort) for
// batches of transforms owned by a thread group (one warp or one block).
//
// A pass of radix R with Ns = product of the previous radices maps
//   in  x[j + r*L/R]           (j in [0, L/R), r in [0, R))
//   out y[(j/Ns)*Ns*R + j%Ns + r*Ns] = DFT_R(w^(r*(j%Ns)*L/(Ns*R)) x[...])_r
// and after all passes the buffer holds the DFT in natural order.  Each pass
// ping-pongs between two shared-memory buffers.
// tw[k] = exp(-2 pi i k / L); sgn = -1 forward, +1 backward (unnormalised).
#pragma once
#include "cf_common.cuh"

#define CF_FFT_MAXPASS 12

// radices packed 5 bits each (pass p: (rcode >> 5p) & 31), so kernels never
// index a parameter array at run time
struct FftPlan {
    int L;
    int np;
    unsigned long long rcode;
    const zd* tw;   // FP64 twiddles
    const zf* twf;  // FP32 twiddles (mixed-precision transforms)
};
template <class Z>
CF_DEV const Z* plan_tw(const FftPlan& pl);
template <>
CF_DEV const zd* plan_tw<zd>(const FftPlan& pl) { return pl.tw; }
template <>
CF_DEV const zf* plan_tw<zf>(const FftPlan& pl) { return pl.twf; }

// Barrier of the thread group: a warp, the whole block (bar == 0), or a
// column team on named barrier 1 or 2 (64 threads; a team of nth = 32 is one
// warp and syncs as one; literal ids: a run-time id makes the compiler
// reserve all sixteen barriers of the block).
template <bool BLOCK>
CF_DEV void group_sync(int bar, int nth) {
    if (!BLOCK || (bar != 0 && nth == 32)) __syncwarp();
    else if (bar == 1) asm volatile("bar.sync 1, 64;" ::: "memory");
    else if (bar == 2) asm volatile("bar.sync 2, 64;" ::: "memory");
    else __syncthreads();
}

// Shared-memory position of element e of a transform buffer: one pad slot
// after every 8 elements.  The stride-R stores of a Stockham pass then spread
// over the eight 16-byte bank groups, and an offset that is a multiple of 8
// elements is a constant position offset (9/8 of it), so the strided
// addresses of a butterfly cost one position computation.
CF_DEV int fpos(int e) { return e + (e >> 3); }
// complex slots a transform buffer of length L occupies (multiple of 8)
__host__ __device__ constexpr int fft_bufsz(int L) { return ((L + (L >> 3) + 1) + 7) & ~7; }
// Alternative layout without padding (buffers of round_up(L, 8) elements, for
// kernels whose shared memory is at an occupancy limit): the low three bits of
// e are XOR-ed with bits 3-5 and 6-8, spreading the strided stores over the
// bank groups as well, at a few more integer operations per access.
CF_DEV int swz(int e) { return e ^ (((e >> 3) ^ (e >> 6)) & 7); }
// The padded layout for 8-byte (complex float) elements: one pad slot after
// every 16 elements.  A warp's 8-byte accesses at a stride of 8 elements then
// fall on distinct bank pairs (the 1-in-8 padding leaves them 2-way
// conflicted for 8-byte elements).
CF_DEV int fpos16(int e) { return e + (e >> 4); }
// position of element e in a buffer of layout POS (0 padded 1 in 8, 1
// XOR-swizzled, 2 padded 1 in 16)
template <int POS>
CF_DEV int bpos(int e) {
    return POS == 1 ? swz(e) : (POS == 2 ? fpos16(e) : fpos(e));
}
// complex slots a transform buffer of length L occupies in layout POS
template <int POS>
__host__ __device__ constexpr int fft_bufsz_pos(int L) {
    return POS == 2 ? ((L + (L >> 4) + 1) + 7) & ~7 : (POS == 1 ? (L + 7) & ~7 : fft_bufsz(L));
}

template <class Z>
CF_DEV Z tw_get(const Z* tw, int k, int sgn) {
    Z w = __ldg(tw + k);
    return sgn > 0 ? zconj(w) : w;
}

// Twiddles w^r, r = 1..R-1, of one butterfly from the single table entry
// w = tw[t1] by complex products (w^r = w^(r/2) w^(r - r/2), depth <= 3 for
// R <= 9) instead of R-1 table loads: the loads share the L1/shared-memory
// pipe with the butterfly data, which bounds the transform kernels, while the
// FP64 pipe has room.  Each product adds about one rounding (a few 1e-16
// relative in FP64).
template <int R, class Z>
CF_DEV void tw_powers(const Z* tw, int t1, int sgn, Z* w) {
    w[1] = tw_get(tw, t1, sgn);
#pragma unroll
    for (int r = 2; r < R; ++r) w[r] = zmul(w[r >> 1], w[r - (r >> 1)]);
}

// a * (c + i sgn s): multiply by exp(sgn i theta) given (cos theta, sin theta)
template <class Z>
CF_DEV Z zrot(Z a, double c, double s, int sgn) {
    const double ss = sgn * s;
    return cmake<Z>(a.x * c - a.y * ss, a.x * ss + a.y * c);
}

// radix-R DFT of v[0..R) in registers (complex type Z); sgn selects the
// exponent sign.  R = 9 is computed as 3 x 3 and R = 16 as 4 x 4:
//   X[k1 + r1 k2] = sum_n2 w_r2^(n2 k2) w_R^(n2 k1) sum_n1 x[r2 n1 + n2] w_r1^(n1 k1)
template <int R, class Z>
CF_DEV void dft_small(Z* v, int sgn) {
    if constexpr (R == 2) {
        Z a = v[0], b = v[1];
        v[0] = zadd(a, b);
        v[1] = zsub(a, b);
    } else if constexpr (R == 3) {
        const double h = 0.86602540378443864676;  // sqrt(3)/2
        Z a = v[0], t1 = zadd(v[1], v[2]);
        Z t2 = zaxpy(a, -0.5, t1);
        Z t3 = zscale(zmuli(zsub(v[1], v[2])), h * sgn);
        v[0] = zadd(a, t1);
        v[1] = zadd(t2, t3);
        v[2] = zsub(t2, t3);
    } else if constexpr (R == 4) {
        Z a0 = zadd(v[0], v[2]), a1 = zsub(v[0], v[2]);
        Z a2 = zadd(v[1], v[3]), a3 = zscale(zmuli(zsub(v[1], v[3])), (double)sgn);
        v[0] = zadd(a0, a2);
        v[2] = zsub(a0, a2);
        v[1] = zadd(a1, a3);
        v[3] = zsub(a1, a3);
    } else if constexpr (R == 5) {
        const double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;
        const double s1 = 0.95105651629515357212, s2 = 0.58778525229247312917;
        Z a0 = v[0];
        Z p14 = zadd(v[1], v[4]), m14 = zsub(v[1], v[4]);
        Z p23 = zadd(v[2], v[3]), m23 = zsub(v[2], v[3]);
        Z r1 = zaxpy(zaxpy(a0, c1, p14), c2, p23);
        Z r2 = zaxpy(zaxpy(a0, c2, p14), c1, p23);
        Z i1 = zscale(zmuli(zaxpy(zscale(m14, s1), s2, m23)), (double)sgn);
        Z i2 = zscale(zmuli(zaxpy(zscale(m14, s2), -s1, m23)), (double)sgn);
        v[0] = zadd(a0, zadd(p14, p23));
        v[1] = zadd(r1, i1);
        v[4] = zsub(r1, i1);
        v[2] = zadd(r2, i2);
        v[3] = zsub(r2, i2);
    } else if constexpr (R == 8) {
        const double h = 0.70710678118654752440;
        Z e[4] = {v[0], v[2], v[4], v[6]};
        Z o[4] = {v[1], v[3], v[5], v[7]};
        dft_small<4>(e, sgn);
        dft_small<4>(o, sgn);
        // w = exp(sgn i pi/4)
        Z w1o = cmake<Z>(h * (o[1].x - sgn * o[1].y), h * (o[1].y + sgn * o[1].x));
        Z w2o = zscale(zmuli(o[2]), (double)sgn);
        Z w3o = cmake<Z>(h * (-o[3].x - sgn * o[3].y), h * (-o[3].y + sgn * o[3].x));
        v[0] = zadd(e[0], o[0]);
        v[4] = zsub(e[0], o[0]);
        v[1] = zadd(e[1], w1o);
        v[5] = zsub(e[1], w1o);
        v[2] = zadd(e[2], w2o);
        v[6] = zsub(e[2], w2o);
        v[3] = zadd(e[3], w3o);
        v[7] = zsub(e[3], w3o);
    } else if constexpr (R == 9) {
        // cos, sin of 2 pi m / 9 for m = 1, 2, 4
        const double c1 = 0.76604444311897803520, s1 = 0.64278760968653932632;
        const double c2 = 0.17364817766693034885, s2 = 0.98480775301220805936;
        const double c4 = -0.93969262078590838405, s4 = 0.34202014332566873304;
        Z y[3][3];
#pragma unroll
        for (int n2 = 0; n2 < 3; ++n2) {
            Z t[3] = {v[n2], v[3 + n2], v[6 + n2]};
            dft_small<3>(t, sgn);
            y[n2][0] = t[0];
            y[n2][1] = t[1];
            y[n2][2] = t[2];
        }
        // twiddles exp(sgn 2 pi i m / 9), m = n2 k1: (1,1) m=1, (1,2) m=2, (2,1) m=2, (2,2) m=4
        y[1][1] = zrot(y[1][1], c1, s1, sgn);
        y[1][2] = zrot(y[1][2], c2, s2, sgn);
        y[2][1] = zrot(y[2][1], c2, s2, sgn);
        y[2][2] = zrot(y[2][2], c4, s4, sgn);
#pragma unroll
        for (int k1 = 0; k1 < 3; ++k1) {
            Z t[3] = {y[0][k1], y[1][k1], y[2][k1]};
            dft_small<3>(t, sgn);
            v[k1] = t[0];
            v[k1 + 3] = t[1];
            v[k1 + 6] = t[2];
        }
    } else if constexpr (R == 16) {
        // cos, sin of 2 pi m / 16 for m = 1, 2, 3
        const double c1 = 0.92387953251128675613, s1 = 0.38268343236508977173;
        const double c2 = 0.70710678118654752440, s2 = 0.70710678118654752440;
        const double c3 = 0.38268343236508977173, s3 = 0.92387953251128675613;
        Z y[4][4];
#pragma unroll
        for (int n2 = 0; n2 < 4; ++n2) {
            Z t[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
            dft_small<4>(t, sgn);
#pragma unroll
            for (int k1 = 0; k1 < 4; ++k1) y[n2][k1] = t[k1];
        }
        // twiddles exp(sgn 2 pi i m / 16), m = n2 k1 in 1..9
        y[1][1] = zrot(y[1][1], c1, s1, sgn);
        y[1][2] = zrot(y[1][2], c2, s2, sgn);
        y[1][3] = zrot(y[1][3], c3, s3, sgn);
        y[2][1] = zrot(y[2][1], c2, s2, sgn);
        y[2][2] = zscale(zmuli(y[2][2]), (double)sgn);  // m = 4: exp(sgn i pi/2)
        y[2][3] = zrot(y[2][3], -c2, s2, sgn);          // m = 6: (cos, sin)(3pi/4) = (-c2, s2)
        y[3][1] = zrot(y[3][1], c3, s3, sgn);
        y[3][2] = zrot(y[3][2], -c2, s2, sgn);          // m = 6
        y[3][3] = zrot(y[3][3], -c1, -s1, sgn);         // m = 9: (cos, sin)(9pi/8) = (-c1, -s1)
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {
            Z t[4] = {y[0][k1], y[1][k1], y[2][k1], y[3][k1]};
            dft_small<4>(t, sgn);
            v[k1] = t[0];
            v[k1 + 4] = t[1];
            v[k1 + 8] = t[2];
            v[k1 + 12] = t[3];
        }
    }
}

// One out-of-place Stockham pass of compile-time radix R over nb transforms of
// length L (transform b at src + b*bs, written to dst + b*bs).  A thread keeps
// one butterfly in registers at a time.
template <bool BLOCK, int POS, int R, class Z>
CF_DEV void fft_pass_pp(const Z* __restrict__ src, Z* __restrict__ dst, int nb, int bs, int L, int Ns,
                        const Z* __restrict__ tw, int sgn, int tid, int nth, int bar) {
    const int NBf = L / R;
    const int total = nb * NBf;
    const int step = L / (Ns * R);
#pragma unroll 2
    for (int q = tid; q < total; q += nth) {
        const int b = q / NBf, j = q - b * NBf;
        const int k = j % Ns;
        const Z* s = src + (long)b * bs;
        Z v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            Z x = s[bpos<POS>(j + r * NBf)];
            v[r] = (r == 0 || k == 0) ? x : zmul(x, tw_get(tw, k * r * step, sgn));
        }
        dft_small<R>(v, sgn);
        Z* d = dst + (long)b * bs;
        const int o = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) d[bpos<POS>(o + r * Ns)] = v[r];
    }
    group_sync<BLOCK>(bar, nth);
}

// Generic prime radix (R <= 31) by a direct DFT; only sizes with uncommon
// prime factors take this path.
template <bool BLOCK, int POS, class Z>
CF_DEV void fft_pass_pp_generic(const Z* __restrict__ src, Z* __restrict__ dst, int nb, int bs, int L, int R,
                                int Ns, const Z* __restrict__ tw, int sgn, int tid, int nth, int bar) {
    const int NBf = L / R;
    const int total = nb * NBf;
    const int step = L / (Ns * R);
    for (int q = tid; q < total; q += nth) {
        const int b = q / NBf, j = q - b * NBf;
        const int k = j % Ns;
        const Z* s = src + (long)b * bs;
        Z* d = dst + (long)b * bs;
        const int ob = (j / Ns) * Ns * R + k;
        for (int o = 0; o < R; ++o) {
            Z acc = czero<Z>();
            for (int r = 0; r < R; ++r) {
                Z x = s[bpos<POS>(j + r * NBf)];
                if (r != 0 && k != 0) x = zmul(x, tw_get(tw, k * r * step, sgn));
                acc = zadd(acc, (r == 0) ? x : zmul(x, tw_get(tw, ((o * r) % R) * NBf, sgn)));
            }
            d[bpos<POS>(ob + o * Ns)] = acc;
        }
    }
    group_sync<BLOCK>(bar, nth);
}

// Compile-time-sized pass: L, Ns and R are constants, so the batch/butterfly
// index split and the twiddle indices need no run-time division, and the R
// strided positions are one fpos() plus constant offsets where the stride is a
// multiple of 8 (or the R outputs stay inside one group of 8).
template <bool BLOCK, int POS, int L, int Ns, int R, class Z>
CF_DEV void fft_pass_static(const Z* __restrict__ src, Z* __restrict__ dst, int nb, int bs,
                            const Z* __restrict__ tw, int sgn, int tid, int nth, int bar) {
    constexpr int NBf = L / R;
    constexpr int step = L / (Ns * R);
    constexpr bool LIN_LD = POS == 0 && (NBf % 8) == 0;
    constexpr bool LIN_ST = POS == 0 && ((Ns % 8) == 0 || (Ns == 1 && 8 % R == 0));
    constexpr int DLD = NBf + NBf / 8;
    constexpr int DST = (Ns == 1) ? 1 : Ns + Ns / 8;
    const int total = nb * NBf;
#pragma unroll 2
    for (int q = tid; q < total; q += nth) {
        const int b = q / NBf, j = q - b * NBf;
        const int k = j % Ns;
        const Z* s = src + (long)b * bs;
        const int pj = bpos<POS>(j);
        Z v[R], w[R];
        if constexpr (Ns > 1) tw_powers<R>(tw, k * step, sgn, w);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            Z x = s[LIN_LD ? pj + r * DLD : bpos<POS>(j + r * NBf)];
            if constexpr (Ns > 1) v[r] = (r == 0 || k == 0) ? x : zmul(x, w[r]);
            else v[r] = x;
        }
        dft_small<R>(v, sgn);
        Z* d = dst + (long)b * bs;
        const int o = (j / Ns) * Ns * R + k;
        const int po = bpos<POS>(o);
#pragma unroll
        for (int r = 0; r < R; ++r) d[LIN_ST ? po + r * DST : bpos<POS>(o + r * Ns)] = v[r];
    }
    group_sync<BLOCK>(bar, nth);
}
template <class Z, bool BLOCK, int POS, int L, int Ns, int R, int... Rest>
CF_DEV Z* fft_static(Z* src, Z* dst, int nb, int bs, const Z* tw, int sgn, int tid, int nth, int bar) {
    fft_pass_static<BLOCK, POS, L, Ns, R>(src, dst, nb, bs, tw, sgn, tid, nth, bar);
    if constexpr (sizeof...(Rest) == 0) {
        return dst;
    } else {
        return fft_static<Z, BLOCK, POS, L, Ns * R, Rest...>(dst, src, nb, bs, tw, sgn, tid, nth, bar);
    }
}

// In-place form of fft_pass_static for groups with a thread per butterfly
// (nb * L / R <= nth): a thread reads its butterfly's R inputs, the group
// synchronises, and the thread writes its R outputs over the same buffer.
// One buffer per transform instead of two (twice the transforms per shared
// memory) for one more barrier per pass.
template <bool BLOCK, int POS, int L, int Ns, int R, class Z>
CF_DEV void fft_pass_static_ip(Z* buf, int nb, int bs, const Z* __restrict__ tw, int sgn, int tid, int nth, int bar) {
    constexpr int NBf = L / R;
    constexpr int step = L / (Ns * R);
    constexpr bool LIN_LD = POS == 0 && (NBf % 8) == 0;
    constexpr bool LIN_ST = POS == 0 && ((Ns % 8) == 0 || (Ns == 1 && 8 % R == 0));
    constexpr int DLD = NBf + NBf / 8;
    constexpr int DST = (Ns == 1) ? 1 : Ns + Ns / 8;
    const bool act = tid < nb * NBf;
    const int b = act ? tid / NBf : 0, j = tid - b * NBf;
    const int k = j % Ns;
    Z v[R];
    if (act) {
        const Z* s = buf + (long)b * bs;
        const int pj = bpos<POS>(j);
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = s[LIN_LD ? pj + r * DLD : bpos<POS>(j + r * NBf)];
        if constexpr (Ns > 1) {
            Z w[R];
            tw_powers<R>(tw, k * step, sgn, w);
#pragma unroll
            for (int r = 1; r < R; ++r)
                if (k != 0) v[r] = zmul(v[r], w[r]);
        }
        dft_small<R>(v, sgn);
    }
    group_sync<BLOCK>(bar, nth);
    if (act) {
        Z* d = buf + (long)b * bs;
        const int o = (j / Ns) * Ns * R + k;
        const int po = bpos<POS>(o);
#pragma unroll
        for (int r = 0; r < R; ++r) d[LIN_ST ? po + r * DST : bpos<POS>(o + r * Ns)] = v[r];
    }
    group_sync<BLOCK>(bar, nth);
}
template <class Z, bool BLOCK, int POS, int L, int Ns, int R, int... Rest>
CF_DEV void fft_static_ip(Z* buf, int nb, int bs, const Z* tw, int sgn, int tid, int nth, int bar) {
    fft_pass_static_ip<BLOCK, POS, L, Ns, R>(buf, nb, bs, tw, sgn, tid, nth, bar);
    if constexpr (sizeof...(Rest) > 0) fft_static_ip<Z, BLOCK, POS, L, Ns * R, Rest...>(buf, nb, bs, tw, sgn, tid, nth, bar);
}
// First pass (Ns = 1) of an in-place transform whose inputs come from a
// functor instead of the buffer: thread (b, j), b < nb, j < L/R, takes
// get(b, j + r L/R) for r < R (from global memory, or computed from other
// buffers), and writes its R outputs to positions R j + r of transform b, as
// fft_pass_static_ip's first pass does after reading them from the buffer.
// The inputs never pass through shared memory: no staging pass, no barrier
// before the first pass.  read_buf: get reads the buffer itself, so a group
// barrier separates the reads from the writes.  Ends with a group barrier.
template <bool BLOCK, int POS, int L, int R, class Z, class Get>
CF_DEV void fft_pass_first_ip(Z* buf, int nb, int bs, int sgn, int tid, int nth, int bar, bool read_buf,
                              const Get& get) {
    constexpr int NBf = L / R;
    constexpr bool LIN_ST = POS == 0 && (8 % R == 0);
    const bool act = tid < nb * NBf;
    const int b = act ? tid / NBf : 0, j = tid - b * NBf;
    Z v[R];
    if (act) {
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = get(b, j + r * NBf);
        dft_small<R>(v, sgn);
    }
    if (read_buf) group_sync<BLOCK>(bar, nth);
    if (act) {
        Z* d = buf + (long)b * bs;
        const int po = bpos<POS>(R * j);
#pragma unroll
        for (int r = 0; r < R; ++r) d[LIN_ST ? po + r : bpos<POS>(R * j + r)] = v[r];
    }
    group_sync<BLOCK>(bar, nth);
}

// lengths with an in-place plan, and the most butterflies of one transform's
// passes (nb times it must not exceed the group's threads)
template <int L>
__host__ __device__ constexpr int fft_ip_butterflies() {
    return L == 512 ? 64 : (L == 576 ? 72 : 0);
}
// The passes after a first radix-8 pass (fft_pass_first_ip) of the in-place plans.
template <bool BLOCK, int L, int POS = 0, class Z>
CF_DEV void group_fft_ip_rest8(Z* a, int nb, int bs, const FftPlan& pl, int sgn, int tid, int nth, int bar) {
    static_assert(L == 512 || L == 576, "no in-place plan for this length");
    const Z* tw = plan_tw<Z>(pl);
    if constexpr (L == 512) fft_static_ip<Z, BLOCK, POS, 512, 8, 8, 8>(a, nb, bs, tw, sgn, tid, nth, bar);
    else fft_static_ip<Z, BLOCK, POS, 576, 8, 8, 9>(a, nb, bs, tw, sgn, tid, nth, bar);
}
template <bool BLOCK, int L, int POS = 0, class Z>
CF_DEV void group_fft_ip(Z* a, int nb, int bs, const FftPlan& pl, int sgn, int tid, int nth, int bar) {
    static_assert(fft_ip_butterflies<L>() > 0, "no in-place plan for this length");
    const Z* tw = plan_tw<Z>(pl);
    if constexpr (L == 512) fft_static_ip<Z, BLOCK, POS, 512, 1, 8, 8, 8>(a, nb, bs, tw, sgn, tid, nth, bar);
    else fft_static_ip<Z, BLOCK, POS, 576, 1, 8, 8, 9>(a, nb, bs, tw, sgn, tid, nth, bar);
}

// Full transform of nb sequences (length pl.L, element e of sequence b at
// b*bs + bpos<POS>(e), bs >= fft_bufsz(L) for the padded layout, >=
// round_up(L, 8) for the XOR layout) held in a; b is a scratch buffer of the
// same size.  Returns the buffer with the result.
template <bool BLOCK, int POS, class Z>
CF_DEV Z* group_fft(Z* a, Z* b, int nb, int bs, const FftPlan& pl, int sgn, int tid, int nth, int bar) {
    int Ns = 1;
    Z* src = a;
    Z* dst = b;
    const Z* tw = plan_tw<Z>(pl);
    for (int p = 0; p < pl.np; ++p) {
        const int R = (int)((pl.rcode >> (5 * p)) & 31ull);
        if (R == 8) fft_pass_pp<BLOCK, POS, 8>(src, dst, nb, bs, pl.L, Ns, tw, sgn, tid, nth, bar);
        else if (R == 4) fft_pass_pp<BLOCK, POS, 4>(src, dst, nb, bs, pl.L, Ns, tw, sgn, tid, nth, bar);
        else if (R == 2) fft_pass_pp<BLOCK, POS, 2>(src, dst, nb, bs, pl.L, Ns, tw, sgn, tid, nth, bar);
        else if (R == 3) fft_pass_pp<BLOCK, POS, 3>(src, dst, nb, bs, pl.L, Ns, tw, sgn, tid, nth, bar);
        else if (R == 5) fft_pass_pp<BLOCK, POS, 5>(src, dst, nb, bs, pl.L, Ns, tw, sgn, tid, nth, bar);
        else fft_pass_pp_generic<BLOCK, POS>(src, dst, nb, bs, pl.L, R, Ns, tw, sgn, tid, nth, bar);
        Ns *= R;
        Z* t = src;
        src = dst;
        dst = t;
    }
    return src;
}

// Transform of compile-time length L (the sizes of the supported grids);
// L == 0 selects the run-time plan.  The radix order of a static size need not
// match pl.R: any factorisation indexes the same twiddle table.
template <bool BLOCK, int L, int POS = 0, class Z>
CF_DEV Z* group_fft_L(Z* a, Z* b, int nb, int bs, const FftPlan& pl, int sgn, int tid, int nth, int bar) {
    const Z* tw = plan_tw<Z>(pl);
    if constexpr (L == 32) return fft_static<Z, BLOCK, POS, 32, 1, 8, 4>(a, b, nb, bs, tw, sgn, tid, nth, bar);
    else if constexpr (L == 48) return fft_static<Z, BLOCK, POS, 48, 1, 8, 2, 3>(a, b, nb, bs, tw, sgn, tid, nth, bar);
    else if constexpr (L == 64) return fft_static<Z, BLOCK, POS, 64, 1, 8, 8>(a, b, nb, bs, tw, sgn, tid, nth, bar);
    else if constexpr (L == 72) return fft_static<Z, BLOCK, POS, 72, 1, 8, 9>(a, b, nb, bs, tw, sgn, tid, nth, bar);
    else if constexpr (L == 96) return fft_static<Z, BLOCK, POS, 96, 1, 8, 4, 3>(a, b, nb, bs, tw, sgn, tid, nth, bar);
    else if constexpr (L == 128) return fft_static<Z, BLOCK, POS, 128, 1, 8, 8, 2>(a, b, nb, bs, tw, sgn, tid, nth, bar);
    else if constexpr (L == 192) return fft_static<Z, BLOCK, POS, 192, 1, 8, 8, 3>(a, b, nb, bs, tw, sgn, tid, nth, bar);
    else if constexpr (L == 256) return fft_static<Z, BLOCK, POS, 256, 1, 8, 8, 4>(a, b, nb, bs, tw, sgn, tid, nth, bar);
    else if constexpr (L == 384) return fft_static<Z, BLOCK, POS, 384, 1, 8, 8, 2, 3>(a, b, nb, bs, tw, sgn, tid, nth, bar);
    else if constexpr (L == 512) return fft_static<Z, BLOCK, POS, 512, 1, 8, 8, 8>(a, b, nb, bs, tw, sgn, tid, nth, bar);
    else if constexpr (L == 576) return fft_static<Z, BLOCK, POS, 576, 1, 8, 8, 9>(a, b, nb, bs, tw, sgn, tid, nth, bar);
    else if constexpr (L == 768) return fft_static<Z, BLOCK, POS, 768, 1, 8, 8, 4, 3>(a, b, nb, bs, tw, sgn, tid, nth, bar);
    else return group_fft<BLOCK, POS>(a, b, nb, bs, pl, sgn, tid, nth, bar);
}

// Lengths with a compile-time instantiation (others run the generic plan).
#define CF_STATIC_FFT_LENGTHS(X) X(32) X(48) X(64) X(72) X(96) X(128) X(192) X(256) X(384) X(512) X(576) X(768)
