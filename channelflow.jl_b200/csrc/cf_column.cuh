// cf_column.cuh -- per-column (one Fourier pair (k,l), all Chebyshev degrees)
// device building blocks.  A team owns one column: two parity groups of
// CF_COL_TW lanes (a warp each, or the two halves of one warp for the short
// columns), group q holding the degrees of parity q.  A column vector lives in shared memory split by
// parity, degree n at position (n & 1) * hs + (n >> 1) (hs = col_half_stride:
// P/2 + 1 rounded up to 4 mod 8), so each parity is a contiguous half and the
// recurrences below (which couple degrees of one parity only) run inside one
// parity group.
//
// Reference arithmetic restated here:
//  * Chebyshev derivative recurrence b_n = b_{n+2} + 2(n+1) a_{n+1}, b_0
//    halved (src/fields/operators.jl:38-61, solvers/batchedinfluence.jl:32-43),
//    evaluated as the equivalent suffix sums b_n = 2 sum_{m>n, m-n odd} m a_m.
//  * Tau Helmholtz solve of rows 0..P-2 of (th0 D^2 - th1) a = f plus wall rows
//    (docs/src/spatial.md:448-475), in its quasi-tridiagonal (spectral
//    integration) form: for n >= 2 of each parity
//       s_n a_{n-2} + d_n a_n + u_n a_{n+2} = g_n,
//    eliminated from the top degree downwards (a_n = alpha_n a_{n-2} + beta_n);
//    the two linear sweeps are prefix scans of affine maps and the wall row is
//    reduced with precomputed weights W_n (factors from the engine set-up).
//  * DCT-I (FFTW REDFT00, src/transforms/chebyshev.jl:45-66) of a complex
//    column of length P+1 through one complex FFT of length P.
//
// Chains of one parity are scanned in runs: each lane takes E consecutive
// chain elements (E odd, so the stride-E shared-memory accesses of a warp hit
// distinct bank groups) and the runs are combined by a scan over the group.
#pragma once
#include "cf_common.cuh"
#include "cf_fft.cuh"

// Lanes per parity group.  The short columns (compile-time P <= 64: at most
// 33 degrees per parity) give each parity half a warp, so that one warp owns
// a column and a column's instructions issue once, not once per parity warp;
// the others give each parity a warp.  The column kernels of one length are
// compiled in their own translation unit (CF_INST_P), so the width is a
// constant of the unit; the host takes a length's team size from
// col_team_threads (cf_dispatch.h).
#ifndef CF_COL_TW_MAXP
#define CF_COL_TW_MAXP 64  // longest compile-time length with one-warp teams
#endif
#if defined(CF_INST_P) && CF_INST_P != 0 && CF_INST_P <= CF_COL_TW_MAXP
#define CF_COL_TW 16
#define CF_COL_TW_LOG2 4
#else
#define CF_COL_TW 32
#define CF_COL_TW_LOG2 5
#endif
#define CF_TEAM (2 * CF_COL_TW)  // threads per column

// The long columns (P >= 192, and the run-time-sized kernels) call the
// repeated helpers below out of line (one copy each keeps those kernels'
// instructions within the instruction caches); the short ones inline them
// (the call costs more there than the fetch).
template <int PL>
__host__ __device__ constexpr bool col_ool() {
    return PL == 0 || PL >= 192;
}

// The two parity groups of one column.  Every routine below is called by all
// CF_TEAM threads of the team and ends with the team's barrier, after which
// all of its outputs are visible to both groups.
struct Team {
    int q;     // parity owned by this group (group index in the team)
    int lane;  // lane in the group (0 .. CF_COL_TW - 1)
    int tid;   // 0 .. CF_TEAM - 1
    int bar;   // named barrier of the team (1 or 2)
#if CF_COL_TW == 16
    unsigned gm;  // the group's lanes in its warp (the mask of its shuffles)
#endif
    int P;     // highest degree (even)
    int hs;    // half stride: col_half_stride(P)
    zd* xch;   // four complex of team scratch in shared memory
    double* sc;  // the column's Stokes-bank scalars (colsc 8, sa 4), staged by col_stage_scalars
};

// Team barrier (a team of one warp: the warp's).  The ids are literal (a
// run-time id makes the compiler reserve all sixteen barriers of the block,
// which limits blocks per SM).
CF_DEV void tsync(const Team& t) {
#if CF_COL_TW == 16
    __syncwarp();
#else
    if (t.bar == 1) asm volatile("bar.sync 1, 64;" ::: "memory");
    else asm volatile("bar.sync 2, 64;" ::: "memory");
#endif
}

// Collectives of one parity group (its lanes, width CF_COL_TW): the mask names
// the group's own lanes, so a group may call them in a branch the other group
// of its warp does not take (a whole warp: the constant full mask).
#if CF_COL_TW == 16
CF_DEV unsigned gmask(const Team& t) { return t.gm; }
#else
CF_DEV unsigned gmask(const Team&) { return 0xffffffffu; }
#endif
CF_DEV double gshfl_up_d(double v, int d, const Team& t) { return __shfl_up_sync(gmask(t), v, d, CF_COL_TW); }
CF_DEV double gshfl_xor_d(double v, int m, const Team& t) { return __shfl_xor_sync(gmask(t), v, m, CF_COL_TW); }
CF_DEV zd gshfl_up_z(zd v, int d, const Team& t) {
    return make_double2(gshfl_up_d(v.x, d, t), gshfl_up_d(v.y, d, t));
}
CF_DEV zd group_sum_z(zd v, const Team& t) {
#pragma unroll
    for (int m = CF_COL_TW / 2; m >= 1; m >>= 1) {
        v.x += gshfl_xor_d(v.x, m, t);
        v.y += gshfl_xor_d(v.y, m, t);
    }
    return v;
}
CF_DEV double group_sum_d(double v, const Team& t) {
#pragma unroll
    for (int m = CF_COL_TW / 2; m >= 1; m >>= 1) v += gshfl_xor_d(v, m, t);
    return v;
}
// inclusive additive scan in lane order
CF_DEV zd group_scan_z(zd v, const Team& t) {
#pragma unroll
    for (int d = 1; d < CF_COL_TW; d <<= 1) {
        zd o = gshfl_up_z(v, d, t);
        if (t.lane >= d) v = zadd(v, o);
    }
    return v;
}
// inclusive scan of affine maps f_i(x) = G_i + M_i x under composition in
// lane order: the result of lane j is f_j o ... o f_0
CF_DEV void group_scan_affine(double& M, zd& G, const Team& t) {
#pragma unroll
    for (int d = 1; d < CF_COL_TW; d <<= 1) {
        double Mo = gshfl_up_d(M, d, t);
        zd Go = gshfl_up_z(G, d, t);
        if (t.lane >= d) {
            G = zaxpy(G, M, Go);
            M = M * Mo;
        }
    }
}
// Offset of the odd half: P/2 + 1 (the even degrees) rounded up to 4 mod 8
// complex.  A loop over consecutive degrees puts the 8 threads of a 16-byte
// access phase on 4 even and 4 odd positions, which then fall in disjoint
// halves of the eight 16-byte bank groups (the column stride of the tiles,
// 2 hs + 2, is 2 mod 8 for the same reason with two columns per block).
__host__ __device__ constexpr int col_half_stride(int P) {
    return ((P >> 1) + 1) + ((4 - ((P >> 1) + 1)) & 7);
}
// shared-memory position of degree (or node) n
CF_DEV int ppos(int n, int hs) { return (n & 1) * hs + (n >> 1); }
// number of degrees of parity q in 0..P (P even)
CF_DEV int pcount(int q, int P) { return q ? (P >> 1) : (P >> 1) + 1; }

// Both groups obtain the group-uniform value v of each group: a from group 0,
// b from group 1.
CF_DEV void team_xchg(const Team& t, zd v, zd& a, zd& b) {
    if (t.lane == 0) t.xch[t.q] = v;
    tsync(t);
    a = t.xch[0];
    b = t.xch[1];
    tsync(t);
}

// Exclusive form of an inclusive group scan result.
CF_DEV zd group_excl_z(zd inc, const Team& t) {
    zd o = gshfl_up_z(inc, 1, t);
    return t.lane == 0 ? zzero() : o;
}

// Elements per lane of a chain of cnt elements scanned by one group (odd),
// and its largest value for the chains of a compile-time length PL (chains
// of at most (PL/2 + 1) elements): the loops over a lane's run are unrolled
// to that bound, so the run's loads issue together and its values stay in
// registers between the two passes of a scan.
CF_DEV int run_len(int cnt) { return ((cnt + CF_COL_TW - 1) >> CF_COL_TW_LOG2) | 1; }
template <int PL>
__host__ __device__ constexpr int run_max() {
    return PL ? ((((PL >> 1) + 1) + CF_COL_TW - 1) >> CF_COL_TW_LOG2) | 1 : 0;
}

// b = D a  (b != a).  Warp q writes the degrees of parity q of b from the
// degrees of parity 1-q of a; b_P = 0.  For a compile-time length, MODE 1
// computes it in place (b == a: every lane's run is read before the team
// barrier, written after it) and MODE 2 subtracts it (b -= D a, b != a).
#define CF_DIFF_SET 0
#define CF_DIFF_INPLACE 1
#define CF_DIFF_SUB 2
template <int PL, int MODE = CF_DIFF_SET>
CF_DEV void col_diff_body(const zd* a, zd* b, const Team& t) {
    static_assert(MODE == CF_DIFF_SET || PL != 0, "in-place and subtracting derivatives need a compile-time length");
    const int P = t.P, hs = t.hs, q = t.q, lane = t.lane;
    const int pin = 1 - q;                 // parity of the input chain
    const int top = pin ? P - 1 : P;       // m = top, top-2, ..., pin
    const int cnt = (top - pin) / 2 + 1;
    const zd* ah = a + pin * hs;           // a_m at ah[m >> 1]
    zd* bh = b + q * hs;                   // b_n at bh[n >> 1]
    const int E = run_len(cnt);
    const int i0 = lane * E;
    if constexpr (PL != 0) {
        constexpr int EM = run_max<PL>();
        zd v[EM];
#pragma unroll
        for (int s = 0; s < EM; ++s) {
            const int i = i0 + s, m = top - 2 * i;
            v[s] = (s < E && i < cnt && m >= 1) ? ah[m >> 1] : zzero();
        }
        zd tot = zzero();
#pragma unroll
        for (int s = 0; s < EM; ++s) {
            const int i = i0 + s, m = top - 2 * i;
            if (s < E && i < cnt && m >= 1) tot = zaxpy(tot, (double)m, v[s]);
        }
        zd run = group_excl_z(group_scan_z(tot, t), t);
        if (MODE == CF_DIFF_INPLACE) tsync(t);  // every input read before any output is written
#pragma unroll
        for (int s = 0; s < EM; ++s) {
            const int i = i0 + s, m = top - 2 * i;
            if (s < E && i < cnt && m >= 1) {
                run = zaxpy(run, (double)m, v[s]);
                const zd d = (m == 1) ? run : zscale(run, 2.0);
                zd& o = bh[(m - 1) >> 1];
                o = MODE == CF_DIFF_SUB ? zsub(o, d) : d;
            }
        }
    } else {
        zd tot = zzero();
        for (int s = 0; s < E; ++s) {
            const int i = i0 + s;
            const int m = top - 2 * i;
            if (i < cnt && m >= 1) tot = zaxpy(tot, (double)m, ah[m >> 1]);
        }
        zd run = group_excl_z(group_scan_z(tot, t), t);
        for (int s = 0; s < E; ++s) {
            const int i = i0 + s;
            const int m = top - 2 * i;
            if (i < cnt && m >= 1) {
                run = zaxpy(run, (double)m, ah[m >> 1]);
                bh[(m - 1) >> 1] = (m == 1) ? run : zscale(run, 2.0);
            }
        }
    }
    if (MODE != CF_DIFF_SUB && q == 0 && lane == 0) bh[P >> 1] = zzero();
    tsync(t);
}
template <int PL, int MODE = CF_DIFF_SET>
CF_DEV_NOINLINE void col_diff_ool(const zd* a, zd* b, const Team t) { col_diff_body<PL, MODE>(a, b, t); }
template <int PL, int MODE = CF_DIFF_SET>
CF_DEV void col_diff(const zd* a, zd* b, const Team& t) {
    if constexpr (col_ool<PL>()) col_diff_ool<PL, MODE>(a, b, t);
    else col_diff_body<PL, MODE>(a, b, t);
}

// The three elimination factor rows of a column (alpha, invden, W: src,
// src + Ny, src + 2 Ny; Ny doubles each, natural order) into shared memory in
// the parity layout: alpha and invden at fa and fa + 2 hs, W at fw.  Group q
// copies its parity; all loads of a lane are issued before its first store
// (one memory round trip for P <= 318).  Only group q reads them afterwards,
// so a warp barrier suffices.
CF_DEV void col_stage_factors(double* fa, double* fw, const double* __restrict__ src, const Team& t) {
    const int P = t.P, Ny = P + 1, hs = t.hs, q = t.q;
    const int nq = pcount(q, P);
    for (int base = t.lane; base < nq; base += 5 * CF_COL_TW) {
        double v[3][5];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int u = 0; u < 5; ++u) {
                const int j = base + CF_COL_TW * u;
                v[r][u] = j < nq ? __ldg(src + (long)r * Ny + 2 * j + q) : 0.0;
            }
#pragma unroll
        for (int u = 0; u < 5; ++u) {
            const int j = base + CF_COL_TW * u;
            if (j < nq) {
                fa[q * hs + j] = v[0][u];
                fa[2 * hs + q * hs + j] = v[1][u];
                fw[q * hs + j] = v[2][u];
            }
        }
    }
    __syncwarp();
}

// The same copies issued asynchronously (8-byte cp.async per value, one
// commit group): the caller works on while they land, then completes them
// with col_factors_wait before the solve reads them.
CF_DEV void col_stage_factors_async(double* fa, double* fw, const double* __restrict__ src, const Team& t) {
    const int P = t.P, Ny = P + 1, hs = t.hs, q = t.q;
    const int nq = pcount(q, P);
    for (int j = t.lane; j < nq; j += CF_COL_TW) {
        const double* s = src + 2 * j + q;
        cp_async_el<8>(fa + q * hs + j, s, true);
        cp_async_el<8>(fa + 2 * hs + q * hs + j, s + Ny, true);
        cp_async_el<8>(fw + q * hs + j, s + 2 * Ny, true);
    }
    cp_async_commit();
}
CF_DEV void col_factors_wait() {
    cp_async_wait<0>();
    __syncwarp();
}

// g_n of the integrated tau equation (n >= 2) from the right-hand side f
// (parity half fh, f_m at fh[m >> 1]).  gt holds the degree-only coefficients:
//   gt[n] = c_{n-2}/(4n(n-1)),  gt[Ny+n] = -[n<=P-2]/(2(n^2-1)),
//   gt[2Ny+n] = [n+2<=P-2]/(4n(n+1))   (c_0 = 2, c_m = 1 otherwise).
CF_DEV zd helm_g(const zd* fh, const double* __restrict__ gt, int n, int P) {
    const int Ny = P + 1, j = n >> 1;
    zd v = zscale(fh[j - 1], __ldg(gt + n));
    if (n <= P - 2) v = zaxpy(v, __ldg(gt + Ny + n), fh[j]);
    if (n + 2 <= P - 2) v = zaxpy(v, __ldg(gt + 2 * Ny + n), fh[j + 1]);
    return v;
}

// The tau Helmholtz solve below for a compile-time length: the same
// arithmetic in the same order, with each lane's run unrolled and its
// intermediate terms (g_n invden_n and the map factors of the backward sweep,
// beta and alpha of the forward sweep) kept in registers between the two
// passes of each sweep instead of being loaded again.  GF: the factors are
// read from their global rows in natural order (alpha = the row base,
// invden at + Ny, W at + 2 Ny; invden and W unused) instead of from the
// parity-layout copy in shared memory.
template <int PL, bool GF = false>
CF_DEV void col_helm_runs(zd* x, zd* scr, const double* alpha, const double* invden, const double* W,
                          const double* __restrict__ gt, double SA0, double SA1, double th1, zd bc0, zd bc1,
                          const Team& t, int top, int cnt, int E, int i0) {
    constexpr int EM = run_max<PL>();
    const int P = t.P, Ny = P + 1, q = t.q, lane = t.lane, hs = t.hs;
    zd* xh = x + q * hs;
    zd* sh = scr + q * hs;
    const double* ah = GF ? alpha : alpha + q * hs;
    const double* ih = GF ? alpha : invden + q * hs;
    const double* wh = GF ? alpha : W + q * hs;
    // factor of degree n (the parity-q half holds degree n at n >> 1)
    auto IH = [&](int n) { return GF ? __ldg(ih + Ny + n) : ih[n >> 1]; };
    auto WH = [&](int n) { return GF ? __ldg(wh + 2 * Ny + n) : wh[n >> 1]; };
    auto AH = [&](int j) { return GF ? __ldg(ah + 2 * j + q) : ah[j]; };
    // backward sweep beta_n = invden_n (g_n - u_n beta_{n+2}) as maps G + M x
    zd g[EM];
    double Ms[EM];
#pragma unroll
    for (int s = 0; s < EM; ++s) {
        const int i = i0 + s;
        g[s] = zzero();
        Ms[s] = 1.0;
        if (s < E && i < cnt) {
            const int n = top - 2 * i;
            const double id = IH(n);
            Ms[s] = th1 * __ldg(gt + 2 * Ny + n) * id;
            g[s] = zscale(helm_g(xh, gt, n, P), id);
        }
    }
    double Mc = 1.0;
    zd Gc = zzero();
#pragma unroll
    for (int s = 0; s < EM; ++s)
        if (s < E && i0 + s < cnt) {
            Gc = zaxpy(g[s], Ms[s], Gc);
            Mc *= Ms[s];
        }
    group_scan_affine(Mc, Gc, t);
    zd xv = group_excl_z(Gc, t);
    zd sw = zzero();
#pragma unroll
    for (int s = 0; s < EM; ++s) {
        const int i = i0 + s;
        if (s < E && i < cnt) {
            const int n = top - 2 * i;
            xv = zaxpy(g[s], Ms[s], xv);
            sh[n >> 1] = xv;
            sw = zaxpy(sw, WH(n), xv);
        }
    }
    sw = group_sum_z(sw, t);
    const zd a0 = zscale(zsub(q ? bc1 : bc0, sw), 1.0 / (q ? SA1 : SA0));
    __syncwarp();
    // forward sweep a_n = alpha_n a_{n-2} + beta_n, chain n = q+2, q+4, ..., top
    zd bv[EM];
    double av[EM];
#pragma unroll
    for (int s = 0; s < EM; ++s) {
        const int jj = i0 + s;
        bv[s] = zzero();
        av[s] = 1.0;
        if (s < E && jj < cnt) {
            bv[s] = sh[jj + 1];
            av[s] = AH(jj + 1);
        }
    }
    Mc = 1.0;
    Gc = zzero();
#pragma unroll
    for (int s = 0; s < EM; ++s)
        if (s < E && i0 + s < cnt) {
            Gc = zaxpy(bv[s], av[s], Gc);
            Mc *= av[s];
        }
    group_scan_affine(Mc, Gc, t);
    const double Me = gshfl_up_d(Mc, 1, t);
    const zd Ge = group_excl_z(Gc, t);
    xv = (lane == 0) ? a0 : zaxpy(Ge, Me, a0);
#pragma unroll
    for (int s = 0; s < EM; ++s) {
        const int jj = i0 + s;
        if (s < E && jj < cnt) {
            xv = zaxpy(bv[s], av[s], xv);
            xh[jj + 1] = xv;
        }
    }
    if (lane == 0) xh[0] = a0;
    tsync(t);
}

// Tau Helmholtz solve: x holds f on entry and a on exit; scr (distinct) holds
// the intermediate beta.  alpha, invden, W are the column's elimination
// factors in the parity layout (shared memory, staged by col_stage_factors);
// SA0/SA1 and bc0/bc1 are the wall-row sums and data of the two parities.
// Warp q solves the parity-q system alone.
template <int PL, bool GF = false>
CF_DEV void col_helm_body(zd* x, zd* scr, const double* alpha, const double* invden, const double* W,
                          const double* __restrict__ gt, double SA0, double SA1, double th1, zd bc0, zd bc1,
                          const Team& t) {
    static_assert(!GF || PL != 0, "factors from global memory need a compile-time length");
    const int P = t.P, Ny = P + 1, q = t.q, lane = t.lane, hs = t.hs;
    const int top = q ? P - 1 : P;
    const int cnt = (top - q) / 2;  // backward chain n = top, top-2, ..., q+2
    const int E = run_len(cnt);
    const int i0 = lane * E;
    if constexpr (PL != 0) {
        col_helm_runs<PL, GF>(x, scr, alpha, invden, W, gt, SA0, SA1, th1, bc0, bc1, t, top, cnt, E, i0);
        return;
    }
    zd* xh = x + q * hs;
    zd* sh = scr + q * hs;
    const double* ah = alpha + q * hs;
    const double* ih = invden + q * hs;
    const double* wh = W + q * hs;
    // backward sweep beta_n = invden_n (g_n - u_n beta_{n+2}) as maps G + M x
    double Mc = 1.0;
    zd Gc = zzero();
    for (int s = 0; s < E; ++s) {
        const int i = i0 + s;
        if (i < cnt) {
            const int n = top - 2 * i;
            const double id = ih[n >> 1];
            const double M = th1 * __ldg(gt + 2 * Ny + n) * id;
            Gc = zaxpy(zscale(helm_g(xh, gt, n, P), id), M, Gc);
            Mc *= M;
        }
    }
    group_scan_affine(Mc, Gc, t);
    zd xv = group_excl_z(Gc, t);
    zd sw = zzero();
    for (int s = 0; s < E; ++s) {
        const int i = i0 + s;
        if (i < cnt) {
            const int n = top - 2 * i;
            const double id = ih[n >> 1];
            const double M = th1 * __ldg(gt + 2 * Ny + n) * id;
            xv = zaxpy(zscale(helm_g(xh, gt, n, P), id), M, xv);
            sh[n >> 1] = xv;
            sw = zaxpy(sw, wh[n >> 1], xv);
        }
    }
    sw = group_sum_z(sw, t);
    const zd a0 = zscale(zsub(q ? bc1 : bc0, sw), 1.0 / (q ? SA1 : SA0));
    __syncwarp();
    // forward sweep a_n = alpha_n a_{n-2} + beta_n, chain n = q+2, q+4, ..., top
    Mc = 1.0;
    Gc = zzero();
    for (int s = 0; s < E; ++s) {
        const int jj = i0 + s;
        if (jj < cnt) {
            const int j = jj + 1;  // n = q + 2 j
            const double M = ah[j];
            Gc = zaxpy(sh[j], M, Gc);
            Mc *= M;
        }
    }
    group_scan_affine(Mc, Gc, t);
    const double Me = gshfl_up_d(Mc, 1, t);
    const zd Ge = group_excl_z(Gc, t);
    xv = (lane == 0) ? a0 : zaxpy(Ge, Me, a0);
    for (int s = 0; s < E; ++s) {
        const int jj = i0 + s;
        if (jj < cnt) {
            const int j = jj + 1;
            xv = zaxpy(sh[j], ah[j], xv);
            xh[j] = xv;
        }
    }
    if (lane == 0) xh[0] = a0;
    tsync(t);
}
template <int PL, bool GF = false>
CF_DEV_NOINLINE void col_helm_ool(zd* x, zd* scr, const double* alpha, const double* invden, const double* W,
                                  const double* __restrict__ gt, double SA0, double SA1, double th1, zd bc0,
                                  zd bc1, const Team t) {
    col_helm_body<PL, GF>(x, scr, alpha, invden, W, gt, SA0, SA1, th1, bc0, bc1, t);
}
template <int PL, bool GF = false>
CF_DEV void col_helm(zd* x, zd* scr, const double* alpha, const double* invden, const double* W,
                     const double* __restrict__ gt, double SA0, double SA1, double th1, zd bc0, zd bc1,
                     const Team& t) {
    if constexpr (col_ool<PL>()) col_helm_ool<PL, GF>(x, scr, alpha, invden, W, gt, SA0, SA1, th1, bc0, bc1, t);
    else col_helm_body<PL, GF>(x, scr, alpha, invden, W, gt, SA0, SA1, th1, bc0, bc1, t);
}

// DCT-I (REDFT00) of complex x[0..P] in place (parity layout).  z and z2 are
// transform buffers of fft_bufsz(P) complex (padded positions fpos).
// X_k = x_0 + (-1)^k x_P + 2 sum_{n=1}^{P-1} x_n cos(pi n k/P).  With
// z_n = (x_n + x_{P-n})/2 - sin(pi n/P)(x_n - x_{P-n}) and Z = FFT_P(z):
//   X_{2m} = Z_m + Z_{P-m},  X_1 = x_0 - x_P + 2 sum_{n=1}^{P-1} x_n cos(pi n/P),
//   X_{2m+1} = X_{2m-1} + i (Z_m - Z_{P-m}).
// cs[n] = (cos(pi n/P), sin(pi n/P)), n = 0..P.  P must be even.  After the
// FFT, group 0 writes the even outputs and group 1 scans the odd ones.
// MODE 1 (forward transform of nodal values, ffts.jl:65-82 with
// normalize_forward! :254-269): every output times `scale`, X_0 and X_P also
// halved.  MODE 2 (inverse, icheb with doubled endpoints and the 1/2 of
// copy_to_padded!, chebyshev.jl:58-66, ffts.jl:162): 0.5 * DCT of x with x_0, x_P doubled.
// Both are folded into the z staging (the transform is linear).
#define CF_DCT_FWD 1
#define CF_DCT_INV 2
// the team's complex FFT of length P (shared by both transform modes)
template <int PL>
CF_DEV_NOINLINE const zd* col_team_fft_ool(zd* z, zd* z2, const FftPlan pl, const Team t) {
    return group_fft_L<true, PL>(z, z2, 1, fft_bufsz(t.P), pl, -1, t.tid, CF_TEAM, t.bar);
}
template <int PL>
CF_DEV const zd* col_team_fft(zd* z, zd* z2, const FftPlan& pl, const Team& t) {
    if constexpr (col_ool<PL>()) return col_team_fft_ool<PL>(z, z2, pl, t);
    else return group_fft_L<true, PL>(z, z2, 1, fft_bufsz(t.P), pl, -1, t.tid, CF_TEAM, t.bar);
}
template <int PL, int MODE>
CF_DEV void col_redft00(zd* x, zd* z, zd* z2, const zd* __restrict__ cs, const FftPlan& pl, double scale,
                        const Team& t) {
    const int P = t.P, H = P >> 1, hs = t.hs;
    // weights of the end terms (n = 0) and of the interior terms
    const double we = (MODE == CF_DCT_FWD) ? scale : 1.0;
    const double wi = (MODE == CF_DCT_FWD) ? scale : (MODE == CF_DCT_INV ? 0.5 : 1.0);
    zd x1 = zzero();
    for (int n = t.tid; n <= H; n += CF_TEAM) {
        if (n == 0) {
            zd a = x[0], b = x[ppos(P, hs)];
            z[fpos(0)] = zscale(zadd(a, b), 0.5 * we);
            x1 = zaxpy(x1, we, zsub(a, b));
        } else if (n == H) {
            z[fpos(H)] = zscale(x[ppos(H, hs)], wi);
        } else {
            zd a = x[ppos(n, hs)], b = x[ppos(P - n, hs)];
            zd c = __ldg(cs + n);
            zd h = zscale(zadd(a, b), 0.5 * wi), d = zscale(zsub(a, b), wi);
            z[fpos(n)] = zaxpy(h, -c.y, d);
            z[fpos(P - n)] = zaxpy(h, c.y, d);
            x1 = zaxpy(x1, 2.0 * c.x, d);
        }
    }
    x1 = group_sum_z(x1, t);
    if (t.lane == 0) t.xch[t.q] = x1;
    tsync(t);
    x1 = zadd(t.xch[0], t.xch[1]);
    const zd* Z = col_team_fft<PL>(z, z2, pl, t);
    if (t.q == 1) {
        // odd outputs X_{2m+1}, m = 0..H-1: X_1 plus prefix sums of
        // i (Z_m - Z_{P-m}), in runs of E (odd) consecutive m per lane
        const int lane = t.lane;
        const int E = run_len(H);
        const int m0 = lane * E;
        zd* xo = x + hs;  // X_{2m+1} at xo[m]
        if constexpr (PL != 0) {
            constexpr int EM = run_max<PL>();
            zd d[EM];
#pragma unroll
            for (int s = 0; s < EM; ++s) {
                const int m = m0 + s;
                d[s] = (s < E && m >= 1 && m < H) ? zmuli(zsub(Z[fpos(m)], Z[fpos(P - m)])) : zzero();
            }
            zd tot = zzero();
#pragma unroll
            for (int s = 0; s < EM; ++s)
                if (s < E && m0 + s >= 1 && m0 + s < H) tot = zadd(tot, d[s]);
            zd run = zadd(x1, group_excl_z(group_scan_z(tot, t), t));
#pragma unroll
            for (int s = 0; s < EM; ++s) {
                const int m = m0 + s;
                if (s < E && m < H) {
                    if (m >= 1) run = zadd(run, d[s]);
                    xo[m] = run;
                }
            }
        } else {
            zd tot = zzero();
            for (int s = 0; s < E; ++s) {
                const int m = m0 + s;
                if (m >= 1 && m < H) tot = zadd(tot, zmuli(zsub(Z[fpos(m)], Z[fpos(P - m)])));
            }
            zd run = zadd(x1, group_excl_z(group_scan_z(tot, t), t));
            for (int s = 0; s < E; ++s) {
                const int m = m0 + s;
                if (m < H) {
                    if (m >= 1) run = zadd(run, zmuli(zsub(Z[fpos(m)], Z[fpos(P - m)])));
                    xo[m] = run;
                }
            }
        }
    } else {
        for (int m = t.lane; m <= H; m += CF_COL_TW)
            x[m] = (m == 0 || m == H) ? zscale(Z[fpos(m)], MODE == CF_DCT_FWD ? 1.0 : 2.0)
                                      : zadd(Z[fpos(m)], Z[fpos(P - m)]);
    }
    tsync(t);
}

// ---- two transforms at once: the team's FFT passes in place over both
// vectors (transform b at z + b*bs), so both fit the two transform buffers
// and the radix-8 passes keep all 64 threads busy (one butterfly per thread
// instead of 32 threads for one transform).
// In-place Stockham pass over NB transforms of length L (radix R, Ns = product
// of the earlier radices), each thread holding up to BPT butterflies: all
// reads, a team barrier, all writes, a team barrier.
template <int L, int Ns, int R, int NB>
CF_DEV void team_pass_ip(zd* buf, int bs, const zd* __restrict__ tw, int sgn, const Team& t) {
    constexpr int NBf = L / R, TOT = NB * NBf, BPT = (TOT + CF_TEAM - 1) / CF_TEAM;
    constexpr int step = L / (Ns * R);
    constexpr bool LIN_LD = (NBf % 8) == 0;
    constexpr bool LIN_ST = (Ns % 8) == 0 || (Ns == 1 && 8 % R == 0);
    constexpr int DLD = NBf + NBf / 8;
    constexpr int DST = (Ns == 1) ? 1 : Ns + Ns / 8;
    zd v[BPT][R];
#pragma unroll
    for (int u = 0; u < BPT; ++u) {
        const int q = t.tid + u * CF_TEAM;
        if (TOT % CF_TEAM == 0 || q < TOT) {
            const int b = q / NBf, j = q - b * NBf, k = j % Ns;
            const zd* s = buf + b * bs;
            const int pj = fpos(j);
#pragma unroll
            for (int r = 0; r < R; ++r) v[u][r] = s[LIN_LD ? pj + r * DLD : fpos(j + r * NBf)];
            if constexpr (Ns > 1) {
                zd w[R];
                tw_powers<R>(tw, k * step, sgn, w);
#pragma unroll
                for (int r = 1; r < R; ++r)
                    if (k != 0) v[u][r] = zmul(v[u][r], w[r]);
            }
            dft_small<R>(v[u], sgn);
        }
    }
    tsync(t);
#pragma unroll
    for (int u = 0; u < BPT; ++u) {
        const int q = t.tid + u * CF_TEAM;
        if (TOT % CF_TEAM == 0 || q < TOT) {
            const int b = q / NBf, j = q - b * NBf, k = j % Ns;
            zd* d = buf + b * bs;
            const int o = (j / Ns) * Ns * R + k;
            const int po = fpos(o);
#pragma unroll
            for (int r = 0; r < R; ++r) d[LIN_ST ? po + r * DST : fpos(o + r * Ns)] = v[u][r];
        }
    }
    tsync(t);
}
template <int L, int Ns, int NB, int R, int... Rest>
CF_DEV void team_fft_ip(zd* buf, int bs, const zd* tw, int sgn, const Team& t) {
    team_pass_ip<L, Ns, R, NB>(buf, bs, tw, sgn, t);
    if constexpr (sizeof...(Rest) > 0) team_fft_ip<L, Ns * R, NB, Rest...>(buf, bs, tw, sgn, t);
}
// forward FFT of length PL of the two transforms at z and z + bs (the
// factorisations of group_fft_L; PL = 192, 256, 384)
template <int PL>
CF_DEV void col_team_fft2_body(zd* z, int bs, const FftPlan& pl, const Team& t) {
    const zd* tw = pl.tw;
    if constexpr (PL == 192) team_fft_ip<192, 1, 2, 8, 8, 3>(z, bs, tw, -1, t);
    else if constexpr (PL == 256) team_fft_ip<256, 1, 2, 8, 8, 4>(z, bs, tw, -1, t);
    else team_fft_ip<384, 1, 2, 8, 8, 2, 3>(z, bs, tw, -1, t);
}
template <int PL>
CF_DEV_NOINLINE void col_team_fft2_ool(zd* z, int bs, const FftPlan pl, const Team t) {
    col_team_fft2_body<PL>(z, bs, pl, t);
}
// lengths that transform in pairs: the long compile-time lengths (measured:
// column kernel 6.06 -> 5.95 ms at P = 256; at P = 128, whose kernel is held
// by registers and whose radix-8 passes have 16 butterflies per transform,
// 0.399 -> 0.409 ms, so the shorter lengths keep single transforms)
template <int PL>
__host__ __device__ constexpr bool col_has_pair() {
    return PL == 192 || PL == 256 || PL == 384;
}
// col_redft00 of two vectors xa, xb (transform buffers z and z + bs): the
// same staging, transform and output steps, both vectors per step.
template <int PL, int MODE>
CF_DEV void col_redft00_pair(zd* xa, zd* xb, zd* z, int bs, const zd* __restrict__ cs, const FftPlan& pl,
                             double scale, const Team& t) {
    static_assert(col_has_pair<PL>(), "pair transforms need a compile-time length");
    const int P = t.P, H = P >> 1, hs = t.hs;
    const double we = (MODE == CF_DCT_FWD) ? scale : 1.0;
    const double wi = (MODE == CF_DCT_FWD) ? scale : (MODE == CF_DCT_INV ? 0.5 : 1.0);
    zd* const zb = z + bs;
    zd x1a = zzero(), x1b = zzero();
    for (int n = t.tid; n <= H; n += CF_TEAM) {
        if (n == 0) {
            const zd a = xa[0], b = xa[ppos(P, hs)], a2 = xb[0], b2 = xb[ppos(P, hs)];
            z[fpos(0)] = zscale(zadd(a, b), 0.5 * we);
            zb[fpos(0)] = zscale(zadd(a2, b2), 0.5 * we);
            x1a = zaxpy(x1a, we, zsub(a, b));
            x1b = zaxpy(x1b, we, zsub(a2, b2));
        } else if (n == H) {
            z[fpos(H)] = zscale(xa[ppos(H, hs)], wi);
            zb[fpos(H)] = zscale(xb[ppos(H, hs)], wi);
        } else {
            const zd a = xa[ppos(n, hs)], b = xa[ppos(P - n, hs)];
            const zd a2 = xb[ppos(n, hs)], b2 = xb[ppos(P - n, hs)];
            const zd c = __ldg(cs + n);
            const zd h = zscale(zadd(a, b), 0.5 * wi), d = zscale(zsub(a, b), wi);
            const zd h2 = zscale(zadd(a2, b2), 0.5 * wi), d2 = zscale(zsub(a2, b2), wi);
            z[fpos(n)] = zaxpy(h, -c.y, d);
            z[fpos(P - n)] = zaxpy(h, c.y, d);
            zb[fpos(n)] = zaxpy(h2, -c.y, d2);
            zb[fpos(P - n)] = zaxpy(h2, c.y, d2);
            x1a = zaxpy(x1a, 2.0 * c.x, d);
            x1b = zaxpy(x1b, 2.0 * c.x, d2);
        }
    }
    x1a = group_sum_z(x1a, t);
    x1b = group_sum_z(x1b, t);
    if (t.lane == 0) {
        t.xch[t.q] = x1a;
        t.xch[2 + t.q] = x1b;
    }
    tsync(t);
    x1a = zadd(t.xch[0], t.xch[1]);
    x1b = zadd(t.xch[2], t.xch[3]);
    if constexpr (col_ool<PL>()) col_team_fft2_ool<PL>(z, bs, pl, t);
    else col_team_fft2_body<PL>(z, bs, pl, t);
    if (t.q == 1) {
        const int lane = t.lane;
        const int E = run_len(H);
        const int m0 = lane * E;
        constexpr int EM = run_max<PL>();
        zd da[EM], db[EM];
#pragma unroll
        for (int s = 0; s < EM; ++s) {
            const int m = m0 + s;
            const bool in = s < E && m >= 1 && m < H;
            da[s] = in ? zmuli(zsub(z[fpos(m)], z[fpos(P - m)])) : zzero();
            db[s] = in ? zmuli(zsub(zb[fpos(m)], zb[fpos(P - m)])) : zzero();
        }
        zd ta = zzero(), tb = zzero();
#pragma unroll
        for (int s = 0; s < EM; ++s)
            if (s < E && m0 + s >= 1 && m0 + s < H) {
                ta = zadd(ta, da[s]);
                tb = zadd(tb, db[s]);
            }
        zd ra = zadd(x1a, group_excl_z(group_scan_z(ta, t), t));
        zd rb = zadd(x1b, group_excl_z(group_scan_z(tb, t), t));
        zd* xoa = xa + hs;
        zd* xob = xb + hs;
#pragma unroll
        for (int s = 0; s < EM; ++s) {
            const int m = m0 + s;
            if (s < E && m < H) {
                if (m >= 1) {
                    ra = zadd(ra, da[s]);
                    rb = zadd(rb, db[s]);
                }
                xoa[m] = ra;
                xob[m] = rb;
            }
        }
    } else {
        const double ew = MODE == CF_DCT_FWD ? 1.0 : 2.0;
        for (int m = t.lane; m <= H; m += CF_COL_TW) {
            const bool end = m == 0 || m == H;
            xa[m] = end ? zscale(z[fpos(m)], ew) : zadd(z[fpos(m)], z[fpos(P - m)]);
            xb[m] = end ? zscale(zb[fpos(m)], ew) : zadd(zb[fpos(m)], zb[fpos(P - m)]);
        }
    }
    tsync(t);
}

// Mean over y (meanmode.jl:13-19): a0 + sum_{even n >= 2} a_n / (1 - n^2),
// returned to both groups.
CF_DEV zd col_bulkmean(const zd* a, const Team& t) {
    zd s = zzero();
    if (t.q == 0) {
        for (int j = t.lane; j <= (t.P >> 1); j += CF_COL_TW) {
            const double n = 2.0 * j;
            s = (j == 0) ? zadd(s, a[0]) : zaxpy(s, 1.0 / (1.0 - n * n), a[j]);
        }
        s = group_sum_z(s, t);
    }
    zd m0, m1;
    team_xchg(t, s, m0, m1);
    return m0;
}
// a'(+1) = sum n^2 a_n ; a'(-1) = sum (-1)^(n+1) n^2 a_n, returned to both groups
CF_DEV void col_wallderiv(const zd* a, const Team& t, zd& right, zd& left) {
    const int q = t.q, nq = pcount(q, t.P);
    const zd* ah = a + q * t.hs;
    zd s = zzero();
    for (int j = t.lane; j < nq; j += CF_COL_TW) {
        const double n = 2.0 * j + q;
        s = zaxpy(s, n * n, ah[j]);
    }
    s = group_sum_z(s, t);
    zd s0, s1;
    team_xchg(t, s, s0, s1);
    right = zadd(s0, s1);
    left = zsub(s1, s0);
}
