// cf_kernels.cuh -- the CNRK2 stage kernels.
//
// Per stage (src/timesteppers/cnrk2.jl:170-205) the engine launches
//   k_zinv    nodal u, omega (6 fields)  -> z-padded, z-inverse FFT
//   k_xpass   x c2r of 6 rows, n = u x omega, x r2c of 3 rows, truncation
//   k_zfwd    z-forward FFT + z truncation -> n at Chebyshev nodes
//   k_column  forward DCT of n, Q update, RHS, Stokes solve (influence and tau
//             corrections, mean mode, flux constraint), curl and inverse DCT
//             of the new velocity and vorticity for the next stage.
// (rotational form; the convective form sends u and du/dy to the nodes and the
// divergence form u alone, and the latter's products pass through
// k_column_div, which returns N as coefficients, before k_column.)
// Field storage: complex (Ny, Nz, Nxh), k fastest; z-padded (Ny, Nzp, Nxh).
//
// Column kernels: a block holds NCOL columns, one team of two warps each
// (cf_column.cuh).  Shared memory: 6 vector regions x NCOL columns x cs
// complex (parity layout, cs = P + 2), 2 transform-buffer regions x NCOL x zs
// complex (zs >= fft_bufsz(P)), then 2 complex of team scratch per column.
#pragma once
#include "cf_column.cuh"

// Stokes bank of one implicit shift (per column data are column-contiguous)
struct BankDev {
    const double* fac_p;   // [B][3][Ny] alpha, invden, W (pressure, th0=1, th1=kappa^2)
    const double* fac_v;   // [B][3][Ny] velocity (th0=nu, th1=shift)
    const double* resp;    // [B][6][Ny] p+, p-, v+, v-, p0, v0
    const double* colsc;   // [B][8] inf00 inf01 inf10 inf11 sigma1 sigma2 shift kappa2p
    const double* sa;      // [B][4] SA_even/odd pressure, SA_even/odd velocity
    const double* meanc;   // [Ny] unit-gradient response of the mean mode
    double meanc_mean;
};

struct ColParams {
    int Nx, Nz, Nxh, Ny, P, B;
    int cs;  // stride of the vector regions 0-5 in shared memory (complex)
    int zs;  // stride of the transform-buffer regions 6-7 (>= fft_bufsz(P))
    double ax, bz;  // 2 pi / Lx, 2 pi / Lz
    double nu;
    // stage constants
    double lambda, weight, Acoef;
    int stage;  // 0, 1, 2
    int store_q;
    // state and work buffers
    zd* U[3];
    zd* Pf;
    zd* Q[3];
    zd* nod[6];  // nodal outputs (u, v, w, omega_x, omega_y, omega_z)
    const zd* Nn[3];  // nonlinear term at Chebyshev nodes (from k_zfwd)
    zd* Nout[3];      // optional: coefficient output of the nonlinear term
    BankDev bank;
    const double* base;      // Chebyshev coefficients of Ub
    const double* basecurv;  // of Ub''
    double nu_bm_curv;       // nu * bulkmean(Ub'')
    int cmode;               // 0 prescribed gradient, 1 bulk velocity
    double c1, c2;           // gradients, or perturbation bulk targets
    double* grad_out;        // [2]
    double* status;          // [4] diagnostics scratch (unused by the hot path)
    int* flags;              // status word set to 1 when the mean mode goes non-finite
    FftPlan plP;
    int bofs;        // first column block of the launch (a launch over part of the columns)
    int skip_nodal;  // stage kernels: end after storing the state (no nodal fields for a next stage)
    const zd* cs_tab;  // (cos, sin)(pi n / P)
    const double* helm_tab;  // [3][Ny] degree coefficients of the integrated tau rows
    double fnorm;  // 1 / (Nxp Nzp (Ny-1))
    // FP32 state (column_stage_body MIX 3): the mean-flow mode (column 0)
    // kept in FP64, [7][Ny]: U0, U1, U2, P, Q0, Q1, Q2
    zd* mean64;
};

// one of three pointers without indexing an array at run time
template <class T>
CF_DEV T* sel3(T* a, T* b, T* c, int i) {
    return i == 0 ? a : (i == 1 ? b : c);
}

// Blocks per SM the column kernels are compiled for (bounds their registers):
// at P = 256 shared memory allows 6 columns per SM, so 168 registers; at P =
// 384 it allows 4, so the full 255 (at 168 the paired transforms spilled); the
// smaller sizes are held to 128 registers (8 or more columns per SM).  One-warp
// teams: 16 columns per SM at P <= 64 (128 registers), 12 for the longer ones
// (170 registers).
template <int NCOL, int PL>
constexpr int col_minblocks() {
    if constexpr (CF_TEAM == 32) return (PL <= 64 ? 16 : 12) / NCOL;  // one-warp teams: 16 or 12 columns
    if constexpr (PL >= 384) return 4 / NCOL;
    return (PL == 0 || PL >= 256) ? 6 / NCOL : 8 / NCOL;
}

// Team scratch per column in shared memory (complex units): four for the
// team's exchanges, six holding the column's 12 Stokes-bank scalars.
#define CF_TEAM_SCRATCH 10

// Common set-up of a column kernel: the calling thread's team and column.
template <int NCOL, int PL>
struct ColCtx {
    Team t;
    int c0, c, ix, iz;
    bool valid;
    zd* smem;
    int cs, zs;
    CF_DEV ColCtx(zd* sm, const ColParams& p, int bx) {
        smem = sm;
        cs = p.cs;
        zs = p.zs;
        const int tm = threadIdx.x / CF_TEAM;
        t.tid = threadIdx.x - tm * CF_TEAM;
        t.q = t.tid >> CF_COL_TW_LOG2;
        t.lane = t.tid & (CF_COL_TW - 1);
#if CF_COL_TW == 16
        t.gm = 0xffffu << (threadIdx.x & 16);
#endif
        t.bar = 1 + tm;
        t.P = PL ? PL : p.P;
        t.hs = col_half_stride(t.P);
        t.xch = sm + (long)NCOL * (6 * cs + 2 * zs) + CF_TEAM_SCRATCH * tm;
        t.sc = reinterpret_cast<double*>(t.xch + 4);
        c0 = (bx + p.bofs) * NCOL;
        c = c0 + tm;
        valid = c < p.B;
        ix = c % p.Nxh;
        iz = c / p.Nxh;
    }
    // region r of the whole block / of this column
    CF_DEV zd* reg(int r) const {
        return r < 6 ? smem + (long)r * NCOL * cs : smem + (long)NCOL * (6 * cs + (r - 6) * zs);
    }
    CF_DEV zd* col(int r) const { return reg(r) + (threadIdx.x / CF_TEAM) * (r < 6 ? cs : zs); }
};

// The column's Stokes-bank scalars (colsc: inf00 inf01 inf10 inf11 sigma1
// sigma2 shift kappa2p; sa: SA_even/odd pressure, SA_even/odd velocity)
// copied asynchronously into the team scratch (t.sc[0..7], t.sc[8..11]) at the
// start of a kernel, so that the Stokes solve reads them from shared memory
// instead of waiting on a global load at each use.  Completed by the
// kernel's first tile_wait and block barrier.
template <class Ctx>
CF_DEV void col_stage_scalars(const Ctx& X, const BankDev& bk) {
    const Team& t = X.t;
    if (X.valid && t.tid < 12) {
        const double* src = t.tid < 8 ? bk.colsc + (long)X.c * 8 + t.tid : bk.sa + (long)X.c * 4 + (t.tid - 8);
        cp_async_el<8>(t.sc + t.tid, src, true);
    }
    cp_async_commit();
}

// Tile of NCOL adjacent columns x Ny degrees into shared memory (column t at
// sm + t*cs, parity layout).  Each thread issues up to 8 loads before storing
// any of them, so the block keeps many requests in flight.
// global element of type G (zd, or zf for the mixed-precision coefficients)
template <class G>
CF_DEV G from_zd(zd a);
template <>
CF_DEV zd from_zd<zd>(zd a) { return a; }
template <>
CF_DEV zf from_zd<zf>(zd a) { return to_zf(a); }

template <int NCOL, class G>
CF_DEV void tile_load_body(zd* sm, int cs, int hs, const G* g, int c0, int Ny, int B) {
    constexpr int NT = NCOL * CF_TEAM, K = 8;
    const int tot = Ny * NCOL;
    for (int base = threadIdx.x; base < tot; base += NT * K) {
        zd v[K];
#pragma unroll
        for (int u = 0; u < K; ++u) {
            const int e = base + u * NT;
            const int n = e / NCOL, t = e - n * NCOL;
            const int c = c0 + t;
            v[u] = (e < tot && c < B) ? to_zd(g[(long)n * B + c]) : zzero();
        }
#pragma unroll
        for (int u = 0; u < K; ++u) {
            const int e = base + u * NT;
            const int n = e / NCOL, t = e - n * NCOL;
            if (e < tot) sm[t * cs + ppos(n, hs)] = v[u];
        }
    }
}
template <int NCOL, class G>
CF_DEV_NOINLINE void tile_load_ool(zd* sm, int cs, int hs, const G* g, int c0, int Ny, int B) {
    tile_load_body<NCOL, G>(sm, cs, hs, g, c0, Ny, B);
}
template <int NCOL, int PL, class G>
CF_DEV void tile_load(zd* sm, int cs, int hs, const G* g, int c0, int Ny, int B) {
    if constexpr (col_ool<PL>()) tile_load_ool<NCOL, G>(sm, cs, hs, g, c0, Ny, B);
    else tile_load_body<NCOL, G>(sm, cs, hs, g, c0, Ny, B);
}
// The same tile of FP64 coefficients copied asynchronously (16-byte cp.async
// per complex, zero fill outside the grid): the call only issues the copies,
// so several tiles are in flight together; tile_wait() completes all of a
// thread's issued copies (a __syncthreads must follow before other threads
// read them).
template <int NCOL>
CF_DEV void tile_load_async_body(zd* sm, int cs, int hs, const zd* g, int c0, int Ny, int B) {
    constexpr int NT = NCOL * CF_TEAM;
    const int tot = Ny * NCOL;
    for (int e = threadIdx.x; e < tot; e += NT) {
        const int n = e / NCOL, t = e - n * NCOL;
        const int c = c0 + t;
        const bool ok = c < B;
        cp_async_el<16>(sm + t * cs + ppos(n, hs), ok ? g + (long)n * B + c : g, ok);
    }
    cp_async_commit();
}
template <int NCOL>
CF_DEV_NOINLINE void tile_load_async_ool(zd* sm, int cs, int hs, const zd* g, int c0, int Ny, int B) {
    tile_load_async_body<NCOL>(sm, cs, hs, g, c0, Ny, B);
}
template <int NCOL, int PL>
CF_DEV void tile_load_async(zd* sm, int cs, int hs, const zd* g, int c0, int Ny, int B) {
    if constexpr (col_ool<PL>()) tile_load_async_ool<NCOL>(sm, cs, hs, g, c0, Ny, B);
    else tile_load_async_body<NCOL>(sm, cs, hs, g, c0, Ny, B);
}
CF_DEV void tile_wait() { cp_async_wait<0>(); }
// FP32 tile of NCOL adjacent columns copied asynchronously into a dense
// staging run (element n NCOL + t; 8-byte cp.async per complex float, zero
// fill outside the grid); the caller commits and waits.  tile_widen then
// moves a staged tile into the parity layout as FP64 (the caller separates
// the two with a __syncthreads); where the tile holds column 0 (c0 == 0) and
// m64 is given, that column comes from m64 (the FP64 mean-flow mode) instead.
template <int NCOL>
CF_DEV void tile_stage32(zf* st, const zf* g, int c0, int Ny, int B) {
    const int tot = Ny * NCOL;
    for (int e = threadIdx.x; e < tot; e += NCOL * CF_TEAM) {
        const int n = e / NCOL, t = e - n * NCOL;
        const int c = c0 + t;
        const bool ok = c < B;
        cp_async_el<8>(st + e, ok ? g + (long)n * B + c : g, ok);
    }
}
template <int NCOL>
CF_DEV void tile_widen(zd* sm, int cs, int hs, const zf* st, int Ny, int c0, const zd* m64) {
    const int tot = Ny * NCOL;
    const bool mean = c0 == 0 && m64 != nullptr;
    for (int e = threadIdx.x; e < tot; e += NCOL * CF_TEAM) {
        const int n = e / NCOL, t = e - n * NCOL;
        sm[t * cs + ppos(n, hs)] = (mean && t == 0) ? m64[n] : to_zd(st[e]);
    }
}
// The same with the staged tile inside the destination region (its upper
// half): every thread reads its elements into registers, the block
// synchronises, then the FP64 values are written (for kernels without a free
// transform buffer to stage in).  PL: a compile-time length.
template <int NCOL, int PL>
CF_DEV void tile_widen_inplace(zd* sm, int cs, int hs, const zf* st, int Ny) {
    constexpr int NT = NCOL * CF_TEAM, K = (NCOL * (PL + 1) + NT - 1) / NT;
    const int tot = Ny * NCOL;
    zf v[K];
#pragma unroll
    for (int u = 0; u < K; ++u) {
        const int e = threadIdx.x + u * NT;
        v[u] = e < tot ? st[e] : make_float2(0.f, 0.f);
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < K; ++u) {
        const int e = threadIdx.x + u * NT;
        if (e < tot) {
            const int n = e / NCOL, t = e - n * NCOL;
            sm[t * cs + ppos(n, hs)] = to_zd(v[u]);
        }
    }
}
// column 0 of a tile (c0 == 0) written in FP64 to m64 (the mean-flow mode
// of an FP32 state)
template <int NCOL>
CF_DEV void tile_store_mean(const zd* sm, int hs, zd* m64, int Ny, int c0) {
    if (c0 != 0) return;
    for (int n = threadIdx.x; n < Ny; n += NCOL * CF_TEAM) m64[n] = sm[ppos(n, hs)];
}

template <int NCOL, class G>
CF_DEV void tile_store_body(const zd* sm, int cs, int hs, G* __restrict__ g, int c0, int Ny, int B) {
    const int tot = Ny * NCOL;
    for (int e = threadIdx.x; e < tot; e += NCOL * CF_TEAM) {
        const int n = e / NCOL, t = e - n * NCOL;
        const int c = c0 + t;
        if (c < B) g[(long)n * B + c] = from_zd<G>(sm[t * cs + ppos(n, hs)]);
    }
}
template <int NCOL, class G>
CF_DEV_NOINLINE void tile_store_ool(const zd* sm, int cs, int hs, G* __restrict__ g, int c0, int Ny, int B) {
    tile_store_body<NCOL, G>(sm, cs, hs, g, c0, Ny, B);
}
template <int NCOL, int PL, class G>
CF_DEV void tile_store(const zd* sm, int cs, int hs, G* __restrict__ g, int c0, int Ny, int B) {
    if constexpr (col_ool<PL>()) tile_store_ool<NCOL, G>(sm, cs, hs, g, c0, Ny, B);
    else tile_store_body<NCOL, G>(sm, cs, hs, g, c0, Ny, B);
}

CF_DEV bool col_nyquist(const ColParams& p, int ix, int iz) {
    return ((p.Nx % 2 == 0) && ix == p.Nx / 2) || ((p.Nz % 2 == 0) && iz == p.Nz / 2);
}

// zero the column vector x (both parities)
CF_DEV void col_zero(zd* x, const Team& t) {
    for (int n = t.tid; n < 2 * t.hs; n += CF_TEAM) x[n] = zzero();
}

// forward DCT of nodal values in x with normalisation, endpoint weights and
// Nyquist filter (ffts.jl:65-82, normalize_forward! :254-269)
template <int PL>
CF_DEV void col_forward_y(zd* x, zd* z, zd* z2, const ColParams& p, bool nyq, const Team& t) {
    if (nyq) {
        col_zero(x, t);
        tsync(t);
    } else {
        col_redft00<PL, CF_DCT_FWD>(x, z, z2, p.cs_tab, p.plP, p.fnorm, t);
    }
}
// inverse DCT: nodal values of the series (icheb with doubled endpoints, the
// 1/2 of copy_to_padded!, chebyshev.jl:58-66, ffts.jl:162)
template <int PL>
CF_DEV void col_inverse_y(zd* x, zd* z, zd* z2, const ColParams& p, const Team& t) {
    col_redft00<PL, CF_DCT_INV>(x, z, z2, p.cs_tab, p.plP, 1.0, t);
}
// the same for two vectors at once (transform buffers z and z2, in place)
template <int PL>
CF_DEV void col_inverse_y2(zd* xa, zd* xb, zd* z, zd* z2, const ColParams& p, const Team& t) {
    col_redft00_pair<PL, CF_DCT_INV>(xa, xb, z, (int)(z2 - z), p.cs_tab, p.plP, 1.0, t);
}

// Solve the Stokes problem of one column.  In: R0,R1,R2 (= Rx,Ry,Rz).
// Out: u in R0, v in V, w in R2, p in PT.  A is scratch; F0, F1 hold the
// staged elimination factors (GF: the solves read the factors from global
// memory and F0, F1 are not used).  Returns the mean gradients for the (0,0)
// column.
template <int PL, bool GF = false>
CF_DEV void col_stokes(zd* R0, zd* R1, zd* R2, zd* PT, zd* V, zd* A, zd* F0, zd* F1, const ColParams& p, int c,
                       int ix, int iz, const Team& t, double* gout) {
    const int P = t.P, Ny = P + 1, q = t.q, lane = t.lane, hs = t.hs;
    const int nq = pcount(q, P);
    const int qo = q * hs;  // offset of this warp's half
    const BankDev& bk = p.bank;
    const double k = p.ax * ix;
    const double l = p.bz * (iz <= (p.Nz >> 1) ? iz : iz - p.Nz);
    const double* sc = t.sc;  // colsc[0..7], sa at sc + 8
    const double* sa = sc + 8;
    const double shift = sc[6];
    const double* fv = bk.fac_v + (long)c * 3 * Ny;
    // elimination factors staged in shared memory (parity layout): alpha,
    // invden in F0, W in F1
    double* fa = reinterpret_cast<double*>(F0);
    double* fi = fa + 2 * hs;
    double* fw = reinterpret_cast<double*>(F1);
    if (c != 0) {
        // it = 0: pressure with zero wall values, (D^2 - kappa^2) p = D Ry + i k Rx + i l Rz
        // it = 1: normal velocity, (nu D^2 - shift) v = D p - Ry
        // (the solve's factors are copied into F0, F1 while the derivative
        // of its right-hand side is formed)
#pragma unroll 1
        for (int it = 0; it < 2; ++it) {
            const double* fsrc = it ? fv : bk.fac_p + (long)c * 3 * Ny;
            zd* x = it ? V : PT;
            if (!GF) col_stage_factors_async(fa, fw, fsrc, t);
            col_diff<PL>(it ? PT : R1, x, t);
            for (int j = lane; j < nq; j += CF_COL_TW) {
                const int o = qo + j;
                x[o] = it ? zsub(x[o], R1[o]) : zadd(x[o], zadd(zmulis(R0[o], k), zmulis(R2[o], l)));
            }
            if constexpr (GF) {
                __syncwarp();
                col_helm<PL, true>(x, A, fsrc, nullptr, nullptr, p.helm_tab, sa[2 * it], sa[2 * it + 1],
                                   it ? shift : sc[7], zzero(), zzero(), t);
            } else {
                col_factors_wait();
                col_helm<PL>(x, A, fa, fi, fw, p.helm_tab, sa[2 * it], sa[2 * it + 1], it ? shift : sc[7], zzero(),
                             zzero(), t);
            }
        }
        // influence and tau corrections (batchedinfluence.jl:101-120, 148-160):
        // this lane's response entries are requested first, so the loads
        // overlap the reductions below (one memory round trip, not one per
        // element)
        const double* __restrict__ rs = bk.resp + (long)c * 6 * Ny;
        constexpr int NIT = PL ? ((PL >> 1) + 1 + CF_COL_TW - 1) / CF_COL_TW : 1;
        double rv[6][NIT];
        if constexpr (PL != 0) {
#pragma unroll
            for (int u = 0; u < NIT; ++u) {
                const int j = lane + CF_COL_TW * u, n = 2 * j + q;
#pragma unroll
                for (int a = 0; a < 6; ++a) rv[a][u] = j < nq ? __ldg(rs + a * Ny + n) : 0.0;
            }
        }
        zd s = zzero();
        for (int j = lane; j < nq; j += CF_COL_TW) {
            const double n = 2.0 * j + q;
            s = zaxpy(s, n * n, V[qo + j]);
        }
        zd s0, s1;
        team_xchg(t, group_sum_z(s, t), s0, s1);
        // upper = -sum n^2 v_n, lower = sum (-1)^n n^2 v_n
        const zd up = zscale(zadd(s0, s1), -1.0), lo = zsub(s0, s1);
        const double i00 = sc[0], i01 = sc[1], i10 = sc[2], i11 = sc[3];
        const zd dp = zaxpy(zscale(up, i00), i01, lo);
        const zd dm = zaxpy(zscale(up, i10), i11, lo);
        if constexpr (PL != 0) {
#pragma unroll
            for (int u = 0; u < NIT; ++u) {
                const int j = lane + CF_COL_TW * u, o = qo + j;
                if (j < nq) {
                    PT[o] = zaxpy(zaxpy(PT[o], rv[0][u], dp), rv[1][u], dm);
                    V[o] = zaxpy(zaxpy(V[o], rv[2][u], dp), rv[3][u], dm);
                }
            }
        } else {
            for (int j = lane; j < nq; j += CF_COL_TW) {
                const int n = 2 * j + q, o = qo + j;
                PT[o] = zaxpy(zaxpy(PT[o], __ldg(rs + n), dp), __ldg(rs + Ny + n), dm);
                V[o] = zaxpy(zaxpy(V[o], __ldg(rs + 2 * Ny + n), dp), __ldg(rs + 3 * Ny + n), dm);
            }
        }
        tsync(t);
        // tau correction (batchedinfluence.jl:148-160); (Dp)_{P-1} = 2P p_P, (Dp)_P = 0
        const zd vP1 = V[ppos(P - 1, hs)], vP = V[ppos(P, hs)], pP = PT[ppos(P, hs)];
        const zd rP1 = R1[ppos(P - 1, hs)], rP = R1[ppos(P, hs)];
        const zd ts1 = zscale(zsub(zaxpy(zscale(vP1, shift), 2.0 * P, pP), rP1), 1.0 / (1.0 - sc[4]));
        const zd ts2 = zscale(zsub(zscale(vP, shift), rP), 1.0 / (1.0 - sc[5]));
        tsync(t);
        const zd sp = q ? ts2 : ts1, sv = q ? ts1 : ts2;
        if constexpr (PL != 0) {
#pragma unroll
            for (int u = 0; u < NIT; ++u) {
                const int j = lane + CF_COL_TW * u, o = qo + j;
                if (j < nq) {
                    PT[o] = zaxpy(PT[o], rv[4][u], sp);
                    V[o] = zaxpy(V[o], rv[5][u], sv);
                }
            }
        } else {
            for (int j = lane; j < nq; j += CF_COL_TW) {
                const int n = 2 * j + q, o = qo + j;
                PT[o] = zaxpy(PT[o], __ldg(rs + 4 * Ny + n), sp);
                V[o] = zaxpy(V[o], __ldg(rs + 5 * Ny + n), sv);
            }
        }
        tsync(t);
    } else {
        // mean mode (meanmode.jl:103-150): integrate Ry through degree P-1, gauge
        for (int j = lane; j < nq; j += CF_COL_TW) {
            const int n = 2 * j + q, o = qo + j;
            zd v = zzero();
            if (n >= 1) {
                zd lower = (n == 1) ? R1[0] : zscale(R1[ppos(n - 1, hs)], 0.5);
                zd upper = (n + 1 < P) ? zscale(R1[ppos(n + 1, hs)], 0.5) : zzero();
                v = zscale(zsub(lower, upper), 1.0 / n);
            }
            PT[o] = v;
            V[o] = zzero();
        }
        tsync(t);
        zd m = col_bulkmean(PT, t);  // PT[0] is zero here
        if (t.tid == 0) PT[0] = zscale(m, -1.0);
        tsync(t);
    }
    // tangential velocities: (nu D^2 - shift) u = i k p - Rx, likewise w
    for (int j = lane; j < nq; j += CF_COL_TW) {
        const int o = qo + j;
        R0[o] = zsub(zmulis(PT[o], k), R0[o]);
        R2[o] = zsub(zmulis(PT[o], l), R2[o]);
    }
    __syncwarp();
    if (!GF && c == 0) col_stage_factors(fa, fw, fv, t);
#pragma unroll 1
    for (int j = 0; j < 2; ++j) {
        if constexpr (GF)
            col_helm<PL, true>(j ? R2 : R0, A, fv, nullptr, nullptr, p.helm_tab, sa[2], sa[3], shift, zzero(), zzero(),
                               t);
        else
            col_helm<PL>(j ? R2 : R0, A, fa, fi, fw, p.helm_tab, sa[2], sa[3], shift, zzero(), zzero(), t);
    }
    if (c == 0) {
        double gx, gz;
        if (p.cmode == 1) {
            zd mu = col_bulkmean(R0, t), mw = col_bulkmean(R2, t);
            gx = (p.c1 - mu.x) / bk.meanc_mean;
            gz = (p.c2 - mw.x) / bk.meanc_mean;
        } else {
            gx = p.c1;
            gz = p.c2;
        }
        for (int j = lane; j < nq; j += CF_COL_TW) {
            const int o = qo + j;
            const double r = __ldg(bk.meanc + 2 * j + q);
            R0[o] = zadd(R0[o], zmake(gx * r, 0.0));
            R2[o] = zadd(R2[o], zmake(gz * r, 0.0));
        }
        tsync(t);
        gout[0] = gx;
        gout[1] = gz;
    }
}

// Total velocity (the base profile added to mode (0,0) of u) and the fields
// the nonlinear form needs at the nodes, inverse DCT to the nodal buffers.
// u, v, w in U0, U1, U2 (modified); Z, Z2 are transform buffers.
//   NL_ROT  W0, W1, W2 receive the vorticity (nonlinear.jl:179-185,
//           operators.jl:172-190); six nodal fields
//   NL_CONV W0, W1, W2 receive du_i/dy (grad!, operators.jl:206-214; the x and
//           z derivatives are formed by the periodic transforms); six fields
//   NL_DIV  u, v, w alone (nonlinear.jl:153-156); three fields
// MX (mixed precision, rotational form): the six fields stay coefficients
// (the tensor-core transform takes them to the nodes).
template <int PL, bool MX = false, int FORM = NL_ROT>
CF_DEV void col_prep_nodal(zd* U0, zd* U1, zd* U2, zd* W0, zd* W1, zd* W2, zd* Z, zd* Z2, const ColParams& p, int c,
                           int ix, int iz, const Team& t) {
    const int q = t.q, lane = t.lane, qo = q * t.hs, nq = pcount(q, t.P);
    const double k = p.ax * ix;
    const double l = p.bz * (iz <= (p.Nz >> 1) ? iz : iz - p.Nz);
    if (c == 0) {
        for (int j = lane; j < nq; j += CF_COL_TW) U0[qo + j] = zadd(U0[qo + j], zmake(__ldg(p.base + 2 * j + q), 0.0));
        tsync(t);
    }
    if (FORM == NL_ROT) {
        col_diff<PL>(U2, W0, t);  // omega_x = D w - i l v
        col_diff<PL>(U0, W2, t);  // omega_z = i k v - D u
        for (int j = lane; j < nq; j += CF_COL_TW) {
            const int o = qo + j;
            W0[o] = zsub(W0[o], zmulis(U1[o], l));
            if (MX) W1[o] = zmuli(zsub(zscale(U0[o], l), zscale(U2[o], k)));
            W2[o] = zsub(zmulis(U1[o], k), W2[o]);
        }
        tsync(t);
    } else if (FORM == NL_CONV) {
#pragma unroll 1
        for (int i = 0; i < 3; ++i) col_diff<PL>(sel3(U0, U1, U2, i), sel3(W0, W1, W2, i), t);
    }
    if (MX) return;
    // omega_y = i (l u - k w) is formed from the nodal u and w below (the
    // transform is linear): five transforms for the rotational form, in pairs
    // where the length has a pair transform
    if constexpr (col_has_pair<PL>()) {
        col_inverse_y2<PL>(U0, U1, Z, Z2, p, t);
        if (FORM == NL_DIV) {
            col_inverse_y<PL>(U2, Z, Z2, p, t);
        } else {
            col_inverse_y2<PL>(U2, W0, Z, Z2, p, t);
            if (FORM == NL_ROT) col_inverse_y<PL>(W2, Z, Z2, p, t);
            else col_inverse_y2<PL>(W1, W2, Z, Z2, p, t);
        }
    } else {
        constexpr int NF = FORM == NL_DIV ? 3 : 6;
#pragma unroll 1
        for (int i = 0; i < NF; ++i) {
            if (FORM == NL_ROT && i == 4) continue;
            zd* x = i < 3 ? sel3(U0, U1, U2, i) : sel3(W0, W1, W2, i - 3);
            col_inverse_y<PL>(x, Z, Z2, p, t);
        }
    }
    if (FORM == NL_ROT) {
        for (int j = lane; j < nq; j += CF_COL_TW) {
            const int o = qo + j;
            W1[o] = zmuli(zsub(zscale(U0[o], l), zscale(U2[o], k)));
        }
        tsync(t);
    }
}

// Full CNRK2 stage for NCOL columns per block (one team per column); bx is
// the block's index among the instance's column blocks.
// Regions: 0 R0, 1 R1, 2 R2, 3 PT, 4 A, 5 Bw, 6 Z, 7 Z2 (6, 7: transform buffers).
// The six nodal (or coefficient) fields u, v, w, omega from regions r0..r5
// to p.nod (MX: as complex float).
template <int NCOL, int PL, bool MX, class Ctx>
CF_DEV void store_six(const Ctx& X, const ColParams& p, int r0, int r1, int r2, int r3, int r4, int r5) {
    const int cs = X.cs, hs = X.t.hs, c0 = X.c0;
    const int rr[6] = {r0, r1, r2, r3, r4, r5};
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        if (MX) tile_store<NCOL, PL>(X.reg(rr[i]), cs, hs, reinterpret_cast<zf*>(p.nod[i]), c0, p.Ny, p.B);
        else tile_store<NCOL, PL>(X.reg(rr[i]), cs, hs, p.nod[i], c0, p.Ny, p.B);
    }
}

// the three nodal fields u, v, w from regions r0..r2 to p.nod (divergence form)
template <int NCOL, int PL, class Ctx>
CF_DEV void store_three(const Ctx& X, const ColParams& p, int r0, int r1, int r2) {
    tile_store<NCOL, PL>(X.reg(r0), X.cs, X.t.hs, p.nod[0], X.c0, p.Ny, p.B);
    tile_store<NCOL, PL>(X.reg(r1), X.cs, X.t.hs, p.nod[1], X.c0, p.Ny, p.B);
    tile_store<NCOL, PL>(X.reg(r2), X.cs, X.t.hs, p.nod[2], X.c0, p.Ny, p.B);
}

// MIX (mixed-precision forms; the arithmetic of the stage stays FP64):
//   0  FP64: the nonlinear term at the nodes in, nodal fields out (complex double)
//   1  tensor-core Chebyshev transforms outside: the term arrives as FP32
//      coefficients (normalised by the transform; p.Nn holds zf arrays) and
//      the new velocity and vorticity leave as FP32 coefficients in p.nod
//   2  FP32 nodal fields in and out, Chebyshev transforms here in FP64
//   3  as 2, with the state (U, P and the history Q) stored in FP32 in
//      global memory: p.U, p.Pf and p.Q hold zf arrays, widened to FP64 in
//      shared memory, and the stage's arithmetic stays FP64
// FORM: the nonlinear form; the divergence form's term arrives as FP64
// coefficients (from k_column_div), the others' at the nodes.
template <int NCOL, int PL, int MIX = 0, int FORM = NL_ROT>
CF_DEV void column_stage_body(const ColParams& p, int bx) {
    constexpr bool NCOEF = MIX == 1 || FORM == NL_DIV;  // N arrives as coefficients
    constexpr bool F32 = MIX != 0;                       // FP32 N in, FP32 fields out
    constexpr bool S32 = MIX == 3;                       // FP32 state in global memory
    // tensor-core forms at a compile-time length: no transform buffers (the
    // DCTs run outside; D^2 U in place, D P subtracted as it is formed, the
    // Stokes factors read from L2), six regions per column
    constexpr bool NOZ = MIX == 1 && PL != 0;
    extern __shared__ zd smem[];
    const ColCtx<NCOL, PL> X(smem, p, bx);
    const Team& t = X.t;
    const int cs = X.cs, hs = t.hs, c0 = X.c0, c = X.c, q = t.q, lane = t.lane;
    const int qo = q * hs, nq = pcount(q, t.P);
    const bool valid = X.valid;
    const bool nyq = valid ? col_nyquist(p, X.ix, X.iz) : true;
    const double k = p.ax * X.ix;
    const double l = p.bz * (X.iz <= (p.Nz >> 1) ? X.iz : X.iz - p.Nz);
    const double kap2 = k * k + l * l;

    // ---------------- Phase A: nonlinear term, history, right-hand side
    // The three components run through one copy of the loop body (pointers
    // selected, not indexed): the kernel's issue rate is limited by its
    // instruction footprint, so the body is not unrolled.  The tiles of
    // component i (N_i, Q_i, U_i) are requested together: U_i goes to a
    // right-hand-side region not yet written (1, then 2), and for i = 2, whose
    // right-hand side takes region 2, Q_2 goes there (consumed before the
    // right-hand side is formed) and U_2 to region 5.
    col_stage_scalars(X, p.bank);
    if (!S32) tile_load_async<NCOL, PL>(X.reg(3), cs, hs, p.Pf, c0, p.Ny, p.B);  // completed with N_0
    // The block's Stokes-bank data (read in Phase B) start on their way to
    // L2 now, so that Phase B's reads of them wait on L2, not on DRAM.
    if (threadIdx.x == 0 && c0 < p.B) {
        const long nc = min(NCOL, p.B - c0), Ny = p.Ny;
        const BankDev& bk = p.bank;
        l2_prefetch(bk.fac_p + c0 * 3 * Ny, nc * 3 * Ny * sizeof(double));
        l2_prefetch(bk.fac_v + c0 * 3 * Ny, nc * 3 * Ny * sizeof(double));
        l2_prefetch(bk.resp + c0 * 6 * Ny, nc * 6 * Ny * sizeof(double));
        l2_prefetch(bk.colsc + c0 * 8, nc * 8 * sizeof(double));
        l2_prefetch(bk.sa + c0 * 4, nc * 4 * sizeof(double));
    }
    double gold[2] = {p.c1, p.c2};
    zd bulkN0 = zzero(), bulkN2 = zzero(), wR0 = zzero(), wL0 = zzero(), wR2 = zzero(), wL2 = zzero();
#pragma unroll 1
    for (int i = 0; i < 3; ++i) {
        const zd* Nn_i = sel3(p.Nn[0], p.Nn[1], p.Nn[2], i);
        zd* Q_i = sel3(p.Q[0], p.Q[1], p.Q[2], i);
        zd* U_i = sel3(p.U[0], p.U[1], p.U[2], i);
        const int qreg = (i == 2) ? 2 : 5, ureg = (i == 2) ? 5 : i + 1;
        if constexpr (S32) {
            // the component's FP32 tiles (and P with the first) copied into
            // the transform buffers, free until the forward transform, then
            // widened into their regions
            zf* st = reinterpret_cast<zf*>(X.reg(6));
            const int T = NCOL * p.Ny;
            tile_stage32<NCOL>(st, reinterpret_cast<const zf*>(U_i), c0, p.Ny, p.B);
            tile_stage32<NCOL>(st + T, reinterpret_cast<const zf*>(Nn_i), c0, p.Ny, p.B);
            if (p.stage > 0) tile_stage32<NCOL>(st + 2 * T, reinterpret_cast<const zf*>(Q_i), c0, p.Ny, p.B);
            if (i == 0) tile_stage32<NCOL>(st + 3 * T, reinterpret_cast<const zf*>(p.Pf), c0, p.Ny, p.B);
            cp_async_commit();
            tile_wait();
            __syncthreads();
            const long ny = p.Ny;
            tile_widen<NCOL>(X.reg(ureg), cs, hs, st, p.Ny, c0, p.mean64 + i * ny);
            tile_widen<NCOL>(X.reg(4), cs, hs, st + T, p.Ny, c0, nullptr);
            if (p.stage > 0) tile_widen<NCOL>(X.reg(qreg), cs, hs, st + 2 * T, p.Ny, c0, p.mean64 + (4 + i) * ny);
            if (i == 0) tile_widen<NCOL>(X.reg(3), cs, hs, st + 3 * T, p.Ny, c0, p.mean64 + 3 * ny);
        } else {
            if (p.stage > 0) tile_load_async<NCOL, PL>(X.reg(qreg), cs, hs, Q_i, c0, p.Ny, p.B);
            tile_load_async<NCOL, PL>(X.reg(ureg), cs, hs, U_i, c0, p.Ny, p.B);
            if (NOZ) {
                // the FP32 term staged in the upper half of region 4 and widened in place
                zf* st = reinterpret_cast<zf*>(X.reg(4)) + (long)NCOL * cs;
                tile_stage32<NCOL>(st, reinterpret_cast<const zf*>(Nn_i), c0, p.Ny, p.B);
                cp_async_commit();
                tile_wait();
                __syncthreads();
                tile_widen_inplace<NCOL, PL>(X.reg(4), cs, hs, st, p.Ny);
            } else if (F32) {
                // the FP32 term copied into the (still free) transform
                // buffers beside the FP64 tiles, then widened into region 4
                zf* st = reinterpret_cast<zf*>(X.reg(6));
                tile_stage32<NCOL>(st, reinterpret_cast<const zf*>(Nn_i), c0, p.Ny, p.B);
                cp_async_commit();
                tile_wait();
                __syncthreads();
                tile_widen<NCOL>(X.reg(4), cs, hs, st, p.Ny, c0, nullptr);
            } else {
                tile_load_async<NCOL, PL>(X.reg(4), cs, hs, Nn_i, c0, p.Ny, p.B);
                tile_wait();
            }
        }
        __syncthreads();
        if (valid) {
            if (!NCOEF) {
                col_forward_y<PL>(X.col(4), X.col(6), X.col(7), p, nyq, t);
            } else if (nyq) {
                col_zero(X.col(4), t);
                tsync(t);
            }
            if (c == 0) {
                const zd bm = col_bulkmean(X.col(4), t);
                if (i == 0) bulkN0 = bm;
                if (i == 2) bulkN2 = bm;
            }
            if (p.stage > 0) {
                zd* A = X.col(4);
                const zd* Qo = X.col(qreg);
                for (int j = lane; j < nq; j += CF_COL_TW) A[qo + j] = zaxpy(A[qo + j], p.Acoef, Qo[qo + j]);
            }
        }
        __syncthreads();
        if (p.store_q) {
            if (S32) {
                tile_store<NCOL, PL>(X.reg(4), cs, hs, reinterpret_cast<zf*>(Q_i), c0, p.Ny, p.B);
                tile_store_mean<NCOL>(X.reg(4), hs, p.mean64 + (4 + i) * (long)p.Ny, p.Ny, c0);
            } else {
                tile_store<NCOL, PL>(X.reg(4), cs, hs, Q_i, c0, p.Ny, p.B);
            }
        }
        if (valid) {
            zd* U = X.col(ureg);
            zd* Qn = X.col(4);
            zd* Z = X.col(6);
            zd* R = X.col(i);
            if (c == 0) {
                zd wr, wl;
                col_wallderiv(U, t, wr, wl);
                if (i == 0) {
                    wR0 = wr;
                    wL0 = wl;
                }
                if (i == 2) {
                    wR2 = wr;
                    wL2 = wl;
                }
            }
            if constexpr (NOZ) {
                // R = lambda U + nu (D^2 U - kappa^2 U) - d_i P + (B/C) Q, the
                // y derivative of P subtracted last
                col_diff<PL>(U, R, t);
                col_diff<PL, CF_DIFF_INPLACE>(R, R, t);
                const zd* PT = X.col(3);
                const double kl = (i == 0) ? k : l;
                for (int j = lane; j < nq; j += CF_COL_TW) {
                    const int o = qo + j;
                    zd lap = zaxpy(R[o], -kap2, U[o]);
                    zd r = zaxpy(zscale(U[o], p.lambda), p.nu, lap);
                    if (i != 1) r = zsub(r, zmulis(PT[o], kl));
                    r = zaxpy(r, p.weight, Qn[o]);
                    R[o] = r;
                }
                __syncwarp();
                if (i == 1) col_diff<PL, CF_DIFF_SUB>(PT, R, t);
            } else {
                col_diff<PL>(U, Z, t);
                col_diff<PL>(Z, R, t);
                // R = lambda U + nu (D^2 U - kappa^2 U) - d_i P + (B/C) Q
                if (i == 1) col_diff<PL>(X.col(3), Z, t);
                const zd* PT = X.col(3);
                const double kl = (i == 0) ? k : l;
                for (int j = lane; j < nq; j += CF_COL_TW) {
                    const int o = qo + j;
                    zd lap = zaxpy(R[o], -kap2, U[o]);
                    zd r = zaxpy(zscale(U[o], p.lambda), p.nu, lap);
                    zd dP = (i == 1) ? Z[o] : zmulis(PT[o], kl);
                    r = zsub(r, dP);
                    r = zaxpy(r, p.weight, Qn[o]);
                    R[o] = r;
                }
            }
        }
        __syncthreads();
    }
    if (valid && c == 0) {
        zd* R0 = X.col(0);
        // A NaN or Inf anywhere in the state reaches every Fourier mode of the
        // nonlinear term within one stage (the periodic transforms mix all
        // modes), so the (0,0) team's bulk means and wall derivatives see it.
        if (t.tid == 0 && p.flags &&
            !isfinite(bulkN0.x + bulkN0.y + bulkN2.x + bulkN2.y + wR0.x + wL0.x + wR2.x + wL2.x))
            atomicExch(p.flags, 1);
        if (p.cmode == 1) {
            gold[0] = p.nu * (wR0.x - wL0.x) / 2 + p.nu_bm_curv + bulkN0.x;
            gold[1] = p.nu * (wR2.x - wL2.x) / 2 + bulkN2.x;
        }
        for (int j = lane; j < nq; j += CF_COL_TW)
            R0[qo + j] = zadd(R0[qo + j], zmake(2.0 * p.nu * __ldg(p.basecurv + 2 * j + q), 0.0));
        tsync(t);
        if (t.tid == 0) {
            R0[0].x -= gold[0];
            zd* R2 = X.col(2);
            R2[0].x -= gold[1];
        }
        tsync(t);
    }
    // ---------------- Phase B: Stokes solve
    if (valid) {
        if (nyq) {
            for (int r = 0; r < 6; ++r)
                if (r != 1) col_zero(X.col(r), t);
            tsync(t);
        } else {
            double g2[2];
            col_stokes<PL, NOZ>(X.col(0), X.col(1), X.col(2), X.col(3), X.col(4), X.col(5), X.col(6), X.col(7), p,
                                c, X.ix, X.iz, t, g2);
            if (c == 0 && t.tid == 0) {
                p.grad_out[0] = g2[0];
                p.grad_out[1] = g2[1];
            }
        }
    }
    __syncthreads();
    if constexpr (S32) {
        tile_store<NCOL, PL>(X.reg(0), cs, hs, reinterpret_cast<zf*>(p.U[0]), c0, p.Ny, p.B);
        tile_store<NCOL, PL>(X.reg(4), cs, hs, reinterpret_cast<zf*>(p.U[1]), c0, p.Ny, p.B);
        tile_store<NCOL, PL>(X.reg(2), cs, hs, reinterpret_cast<zf*>(p.U[2]), c0, p.Ny, p.B);
        tile_store<NCOL, PL>(X.reg(3), cs, hs, reinterpret_cast<zf*>(p.Pf), c0, p.Ny, p.B);
        const long ny = p.Ny;
        tile_store_mean<NCOL>(X.reg(0), hs, p.mean64, p.Ny, c0);
        tile_store_mean<NCOL>(X.reg(4), hs, p.mean64 + ny, p.Ny, c0);
        tile_store_mean<NCOL>(X.reg(2), hs, p.mean64 + 2 * ny, p.Ny, c0);
        tile_store_mean<NCOL>(X.reg(3), hs, p.mean64 + 3 * ny, p.Ny, c0);
    } else {
        tile_store<NCOL, PL>(X.reg(0), cs, hs, p.U[0], c0, p.Ny, p.B);
        tile_store<NCOL, PL>(X.reg(4), cs, hs, p.U[1], c0, p.Ny, p.B);
        tile_store<NCOL, PL>(X.reg(2), cs, hs, p.U[2], c0, p.Ny, p.B);
        tile_store<NCOL, PL>(X.reg(3), cs, hs, p.Pf, c0, p.Ny, p.B);
    }
    if (p.skip_nodal) return;
    __syncthreads();
    // ---------------- Phase C: total velocity, vorticity, nodal values
    if (valid)
        col_prep_nodal<PL, MIX == 1, FORM>(X.col(0), X.col(4), X.col(2), X.col(1), X.col(3), X.col(5), X.col(6),
                                           X.col(7), p, c, X.ix, X.iz, t);
    __syncthreads();
    if (FORM == NL_DIV) store_three<NCOL, PL>(X, p, 0, 4, 2);
    else store_six<NCOL, PL, F32>(X, p, 0, 4, 2, 1, 3, 5);
}

template <int NCOL, int PL, int FORM = NL_ROT>
__global__ void __launch_bounds__(NCOL * CF_TEAM, (col_minblocks<NCOL, PL>())) k_column_stage(ColParams p) {
    column_stage_body<NCOL, PL, 0, FORM>(p, blockIdx.x);
}
// Batched stage over the instances of a size class: item (instance i,
// column block bx), the instance's parameters staged in shared memory.
// counter == null: one item per block, (bx, i) = (blockIdx.x, blockIdx.y).
// Otherwise the launch is persistent: its blocks claim items in order
// (instance-major, it = i * nblk + bx) from the counter, zeroed before the
// launch, until all nitems are done.  MINB: blocks per SM the registers are
// bounded for (the ensemble autotuner's choice).
template <int NCOL, int PL, int MINB>
__global__ void __launch_bounds__(NCOL * CF_TEAM, MINB)
    k_column_stage_batch(const ColParams* __restrict__ pl, int nblk, int nitems, unsigned* counter) {
    __shared__ ColParams ps;
    if (!counter) {
        stage_params(&ps, pl + blockIdx.y);
        column_stage_body<NCOL, PL>(ps, blockIdx.x);
        return;
    }
    __shared__ int item;
    for (;;) {
        __syncthreads();  // every thread is done with the previous item
        if (threadIdx.x == 0) item = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int it = item;
        if (it >= nitems) return;
        const int inst = it / nblk;
        stage_params(&ps, pl + inst);
        column_stage_body<NCOL, PL>(ps, it - inst * nblk);
    }
}

// Mixed-precision stages (MIX 1, 2 and 3 of column_stage_body).  MIX 1 at a
// compile-time length takes six regions per column (no transform buffers),
// so four blocks fit per SM at P = 256 and the registers are bounded for them.
template <int NCOL, int PL, int MIX>
constexpr int col_minblocks_mx() {
    return (MIX == 1 && PL != 0) ? 8 / NCOL : col_minblocks<NCOL, PL>();
}
template <int NCOL, int PL, int MIX>
__global__ void __launch_bounds__(NCOL * CF_TEAM, (col_minblocks_mx<NCOL, PL, MIX>())) k_column_stage_mx(ColParams p) {
    column_stage_body<NCOL, PL, MIX>(p, blockIdx.x);
}

// Nodal fields of the nonlinear form (velocity and vorticity for the
// rotational form) from the state U (used after set_state); MIX 1: their FP32
// Chebyshev coefficients instead; MIX 2: FP32 nodal values; MIX 3: as 2, from
// an FP32 state.
template <int NCOL, int PL, int MIX = 0, int FORM = NL_ROT>
__global__ void __launch_bounds__(NCOL * CF_TEAM, (col_minblocks<NCOL, PL>())) k_column_prep(ColParams p) {
    extern __shared__ zd smem[];
    const ColCtx<NCOL, PL> X(smem, p, blockIdx.x);
    const int cs = X.cs, hs = X.t.hs, c0 = X.c0;
    if constexpr (MIX == 3) {
        // FP32 state staged in the transform buffers and widened (column 0,
        // the mean-flow mode, from its FP64 copy)
        zf* st = reinterpret_cast<zf*>(X.reg(6));
        const int T = NCOL * p.Ny;
        for (int i = 0; i < 3; ++i)
            tile_stage32<NCOL>(st + i * T, reinterpret_cast<const zf*>(sel3(p.U[0], p.U[1], p.U[2], i)), c0, p.Ny,
                               p.B);
        cp_async_commit();
        tile_wait();
        __syncthreads();
        for (int i = 0; i < 3; ++i) tile_widen<NCOL>(X.reg(i), cs, hs, st + i * T, p.Ny, c0, p.mean64 + i * (long)p.Ny);
    } else {
        tile_load_async<NCOL, PL>(X.reg(0), cs, hs, p.U[0], c0, p.Ny, p.B);
        tile_load_async<NCOL, PL>(X.reg(1), cs, hs, p.U[1], c0, p.Ny, p.B);
        tile_load_async<NCOL, PL>(X.reg(2), cs, hs, p.U[2], c0, p.Ny, p.B);
        tile_wait();
    }
    __syncthreads();
    if (X.valid)
        col_prep_nodal<PL, MIX == 1, FORM>(X.col(0), X.col(1), X.col(2), X.col(3), X.col(4), X.col(5), X.col(6),
                                           X.col(7), p, X.c, X.ix, X.iz, X.t);
    __syncthreads();
    if (FORM == NL_DIV) store_three<NCOL, PL>(X, p, 0, 1, 2);
    else store_six<NCOL, PL, (MIX != 0)>(X, p, 0, 1, 2, 3, 4, 5);
}

// Divergence form, after the periodic transforms: forward DCT of the six
// negated products -u_i u_j at the nodes (p.nod, order 00 01 02 11 12 22) and
// div! of the rows in coefficient space (operators.jl:270-294):
//   N_i = i k (-uu_i0) + D (-uu_i1) + i l (-uu_i2)
// written as FP64 coefficients to p.Nout.  Regions 0-5 hold the six products,
// 6 and 7 the transform buffers (region 6 then takes the derivative).
template <int NCOL, int PL>
__global__ void __launch_bounds__(NCOL * CF_TEAM, (col_minblocks<NCOL, PL>())) k_column_div(ColParams p) {
    extern __shared__ zd smem[];
    const ColCtx<NCOL, PL> X(smem, p, blockIdx.x);
    const Team& t = X.t;
    const int cs = X.cs, hs = t.hs, c0 = X.c0, qo = t.q * hs, nq = pcount(t.q, t.P);
#pragma unroll
    for (int m = 0; m < 6; ++m) tile_load_async<NCOL, PL>(X.reg(m), cs, hs, p.nod[m], c0, p.Ny, p.B);
    tile_wait();
    __syncthreads();
    if (X.valid) {
        const bool nyq = col_nyquist(p, X.ix, X.iz);
#pragma unroll 1
        for (int m = 0; m < 6; ++m) col_forward_y<PL>(X.col(m), X.col(6), X.col(7), p, nyq, t);
        const double k = p.ax * X.ix;
        const double l = p.bz * (X.iz <= (p.Nz >> 1) ? X.iz : X.iz - p.Nz);
        // row i: (x, y, z) entries in regions (a, b, c), result into region a
        // of a product no later row reads: N2 -> 5 (02, 12, 22), N1 -> 3
        // (01, 11, 12), N0 -> 0 (00, 01, 02)
        const int ra[3] = {2, 1, 0}, rb[3] = {4, 3, 1}, rc[3] = {5, 4, 2}, ro[3] = {5, 3, 0};
        zd* D = X.col(6);
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            col_diff<PL>(X.col(rb[r]), D, t);
            const zd* a = X.col(ra[r]);
            const zd* cz = X.col(rc[r]);
            zd* o = X.col(ro[r]);
            for (int j = t.lane; j < nq; j += CF_COL_TW) {
                const int e = qo + j;
                o[e] = zadd(zadd(zmulis(a[e], k), D[e]), zmulis(cz[e], l));
            }
            tsync(t);
        }
    }
    __syncthreads();
    tile_store<NCOL, PL>(X.reg(0), cs, hs, p.Nout[0], c0, p.Ny, p.B);
    tile_store<NCOL, PL>(X.reg(3), cs, hs, p.Nout[1], c0, p.Ny, p.B);
    tile_store<NCOL, PL>(X.reg(5), cs, hs, p.Nout[2], c0, p.Ny, p.B);
}

// Forward DCT of the nonlinear term only: coefficients into p.Nout.
template <int NCOL, int PL>
__global__ void __launch_bounds__(NCOL * CF_TEAM, (col_minblocks<NCOL, PL>())) k_column_nlout(ColParams p) {
    extern __shared__ zd smem[];
    const ColCtx<NCOL, PL> X(smem, p, blockIdx.x);
    const int cs = X.cs, hs = X.t.hs, c0 = X.c0;
    const bool nyq = X.valid ? col_nyquist(p, X.ix, X.iz) : true;
#pragma unroll 1
    for (int i = 0; i < 3; ++i) {
        tile_load<NCOL, PL>(X.reg(0), cs, hs, sel3(p.Nn[0], p.Nn[1], p.Nn[2], i), c0, p.Ny, p.B);
        __syncthreads();
        if (X.valid) col_forward_y<PL>(X.col(0), X.col(6), X.col(7), p, nyq, X.t);
        __syncthreads();
        tile_store<NCOL, PL>(X.reg(0), cs, hs, sel3(p.Nout[0], p.Nout[1], p.Nout[2], i), c0, p.Ny, p.B);
        __syncthreads();
    }
}

// Stokes projection (pressure.jl:36-54): R = -Laplacian(U), solve with the
// (nu = 1, lambda = 0) bank, velocity overwritten.
template <int NCOL, int PL>
__global__ void __launch_bounds__(NCOL * CF_TEAM, (col_minblocks<NCOL, PL>())) k_column_project(ColParams p) {
    extern __shared__ zd smem[];
    const ColCtx<NCOL, PL> X(smem, p, blockIdx.x);
    const Team& t = X.t;
    const int cs = X.cs, hs = t.hs, c0 = X.c0, qo = t.q * hs, nq = pcount(t.q, t.P);
    const double k = p.ax * X.ix;
    const double l = p.bz * (X.iz <= (p.Nz >> 1) ? X.iz : X.iz - p.Nz);
    const double kap2 = k * k + l * l;
    col_stage_scalars(X, p.bank);
    tile_wait();  // visible to the team after the loop's first block barrier
#pragma unroll 1
    for (int i = 0; i < 3; ++i) {
        tile_load<NCOL, PL>(X.reg(5), cs, hs, sel3(p.U[0], p.U[1], p.U[2], i), c0, p.Ny, p.B);
        __syncthreads();
        if (X.valid) {
            zd* U = X.col(5);
            zd* Z = X.col(6);
            zd* R = X.col(i);
            col_diff<PL>(U, Z, t);
            col_diff<PL>(Z, R, t);
            for (int j = t.lane; j < nq; j += CF_COL_TW) R[qo + j] = zscale(zaxpy(R[qo + j], -kap2, U[qo + j]), -1.0);
        }
        __syncthreads();
    }
    if (X.valid) {
        if (col_nyquist(p, X.ix, X.iz)) {
            for (int r = 0; r < 6; ++r) col_zero(X.col(r), t);
            tsync(t);
        } else {
            double g2[2];
            col_stokes<PL>(X.col(0), X.col(1), X.col(2), X.col(3), X.col(4), X.col(5), X.col(6), X.col(7), p, X.c,
                           X.ix, X.iz, t, g2);
        }
    }
    __syncthreads();
    tile_store<NCOL, PL>(X.reg(0), cs, hs, p.U[0], c0, p.Ny, p.B);
    tile_store<NCOL, PL>(X.reg(4), cs, hs, p.U[1], c0, p.Ny, p.B);
    tile_store<NCOL, PL>(X.reg(2), cs, hs, p.U[2], c0, p.Ny, p.B);
}

// Pressure reconstruction (pressure.jl:115-204) from the nonlinear term at
// the nodes (p.Nn; NCOEF: as coefficients) and the normal velocity U[1]:
// Neumann Helmholtz per mode with the factors in p.bank.fac_p / sa[0..1]
// (Neumann weights).
template <int NCOL, int PL, bool NCOEF = false>
__global__ void __launch_bounds__(NCOL * CF_TEAM, (col_minblocks<NCOL, PL>())) k_column_pressure(ColParams p) {
    extern __shared__ zd smem[];
    const ColCtx<NCOL, PL> X(smem, p, blockIdx.x);
    const Team& t = X.t;
    const int cs = X.cs, hs = t.hs, c0 = X.c0, c = X.c, q = t.q, lane = t.lane;
    const int P = t.P, qo = q * hs, nq = pcount(q, P);
    const bool nyq = X.valid ? col_nyquist(p, X.ix, X.iz) : true;
#pragma unroll 1
    for (int i = 0; i < 3; ++i) {
        tile_load<NCOL, PL>(X.reg(i), cs, hs, sel3(p.Nn[0], p.Nn[1], p.Nn[2], i), c0, p.Ny, p.B);
        __syncthreads();
        if (X.valid && !NCOEF) col_forward_y<PL>(X.col(i), X.col(6), X.col(7), p, nyq, t);
        __syncthreads();
    }
    tile_load<NCOL, PL>(X.reg(4), cs, hs, p.U[1], c0, p.Ny, p.B);
    __syncthreads();
    if (X.valid) {
        const double k = p.ax * X.ix;
        const double l = p.bz * (X.iz <= (p.Nz >> 1) ? X.iz : X.iz - p.Nz);
        zd* A0 = X.col(0);
        zd* A1 = X.col(1);
        zd* A2 = X.col(2);
        zd* PT = X.col(3);
        zd* V = X.col(4);
        if (nyq) {
            col_zero(PT, t);
            tsync(t);
        } else if (c == 0) {
            for (int j = lane; j < nq; j += CF_COL_TW) {
                const int n = 2 * j + q;
                zd v = zzero();
                if (n >= 1) {
                    zd lower = (n == 1) ? A1[0] : zscale(A1[ppos(n - 1, hs)], 0.5);
                    zd upper = (n + 1 < P) ? zscale(A1[ppos(n + 1, hs)], 0.5) : zzero();
                    v = zscale(zsub(lower, upper), 1.0 / n);
                }
                PT[qo + j] = v;
            }
            tsync(t);
            zd m = col_bulkmean(PT, t);
            if (t.tid == 0) PT[0] = zscale(m, -1.0);
            tsync(t);
        } else {
            col_diff<PL>(A1, PT, t);
            zd su = zzero();
            for (int j = lane; j < nq; j += CF_COL_TW) {
                const int n = 2 * j + q, o = qo + j;
                PT[o] = zadd(PT[o], zadd(zmulis(A0[o], k), zmulis(A2[o], l)));
                su = zadd(su, A1[o]);
                if (n >= 2) {
                    const double dn = (double)n;
                    su = zaxpy(su, p.nu * (dn * dn * (dn * dn - 1.0) / 3.0), V[o]);
                }
            }
            zd s0, s1;
            team_xchg(t, group_sum_z(su, t), s0, s1);
            const zd up = zadd(s0, s1), lo = zsub(s0, s1);
            const double* sa = p.bank.sa + (long)c * 4;
            // Neumann parity data: even rows (up - lo)/2, odd rows (up + lo)/2
            const double* fpn = p.bank.fac_p + (long)c * 3 * p.Ny;
            double* fa = reinterpret_cast<double*>(X.col(6));
            double* fw = reinterpret_cast<double*>(X.col(7));
            col_stage_factors(fa, fw, fpn, t);
            col_helm<PL>(PT, X.col(5), fa, fa + 2 * hs, fw, p.helm_tab, __ldg(sa + 0), __ldg(sa + 1), k * k + l * l,
                     zscale(zsub(up, lo), 0.5), zscale(zadd(up, lo), 0.5), t);
        }
    }
    __syncthreads();
    tile_store<NCOL, PL>(X.reg(3), cs, hs, p.Pf, c0, p.Ny, p.B);
}

// Diagnostics of the perturbation velocity on the device (postprocessing.jl:
// 80-95), per block: part[3 b] = sum over its columns of <u_i, u_i>,
// part[3 b + 1] = of <omega_i, omega_i>, part[3 b + 2] = max |div u|
// coefficient (summed by k_diag_reduce into acc[0..2]); acc[3], acc[4] =
// u'(+1), u'(-1) of the (0,0) mode.  <a, b> = sum_{m,n} conj(a_m) b_n M_mn
// with M_mn = (mom(m+n) + mom(|m-n|))/2, mom(j) = 1/(1-j^2) for even j, 0 for
// odd j (the Chebyshev inner product on [-1, 1] divided by 2), weighted 1 for
// kx = 0 and 2 otherwise; Nyquist columns are skipped.  M couples degrees of
// equal parity only, so parity group q sums the parity-q part, and only the even
// moments occur (table mom[h] = mom(2h), h = 0..P).  Regions: 0-2 u, v, w;
// 3-5 omega; 6 the moment table (block); 7 D v.
CF_DEV double diag_form(const zd* a, const double* mom, const Team& t) {
    // M is symmetric: the terms n > m count twice, n = m once; four
    // independent accumulators keep several loads and FMAs in flight.  m and n
    // have equal parity, so only even moments occur: mom[h] = mom(2h).
    const int q = t.q, qo = q * t.hs, nq = pcount(q, t.P);
    double s = 0.0;
    for (int j = t.lane; j < nq; j += CF_COL_TW) {
        const int m = 2 * j + q;
        const zd am = a[qo + j];
        zd acc[4] = {zzero(), zzero(), zzero(), zzero()};
        int i = j + 1;
        for (; i + 3 < nq; i += 4) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                // m + n = 2 (j + i + u + q), n - m = 2 (i + u - j)
                acc[u] = zaxpy(acc[u], mom[j + i + u + q] + mom[i + u - j], a[qo + i + u]);
            }
        }
        for (; i < nq; ++i) acc[0] = zaxpy(acc[0], mom[j + i + q] + mom[i - j], a[qo + i]);
        const zd off = zadd(zadd(acc[0], acc[1]), zadd(acc[2], acc[3]));
        // diagonal M_mm = (mom(2m) + mom(0)) / 2; off-diagonal pairs 2 M_mn = mom(m+n) + mom(n-m)
        const double Mmm = 0.5 * (mom[m] + mom[0]);
        s += Mmm * (am.x * am.x + am.y * am.y) + (am.x * off.x + am.y * off.y);  // Re(conj(a_m) ...)
    }
    return group_sum_d(s, t);
}

// The same form for a compile-time length, register-tiled over the upper
// triangle of E x E blocks.  The nq indices of a parity form NB = ceil(nq/E)
// blocks; the NB (NB + 1) / 2 block pairs (b <= c) are dealt to the lanes in
// turn (pair k to lane k mod CF_COL_TW), so every lane does the same number of pairs
// and no lane walks a longer triangle row than another.  A pair needs its 2E
// coefficients, 2E - 1 Hankel moments mom[jb + ic + q + k] and 2E - 1
// Toeplitz moments mom[|ic - jb - (E-1) + k|] (k = 0 .. 2E-2) for its E x E
// terms (a moment load feeds E FMA pairs); an off-diagonal pair stands for
// its mirror image too (M is symmetric: weight 2).  Indices past the table
// are clamped to finite entries whose coefficients are zero.
template <int PL>
CF_DEV double diag_form_tiled(const zd* a, const double* mom, const Team& t) {
    constexpr int E = run_max<PL>();
    const int q = t.q, qo = q * t.hs, nq = pcount(q, t.P), P = t.P;
    const int NB = (nq + E - 1) / E, npair = NB * (NB + 1) / 2;
    double s = 0.0;
    for (int k = t.lane; k < npair; k += CF_COL_TW) {
        // row b of the triangle starts at pair b NB - b (b - 1) / 2
        const double w = 2.0 * NB + 1.0;
        int b = (int)((w - sqrt(w * w - 8.0 * k)) * 0.5);
        while (b > 0 && b * NB - b * (b - 1) / 2 > k) --b;
        while ((b + 1) * NB - (b + 1) * b / 2 <= k) ++b;
        const int c = b + (k - (b * NB - b * (b - 1) / 2));
        const int jb = b * E, ic = c * E;
        double H[2 * E - 1], T[2 * E - 1];
        zd aj[E], ai[E];
#pragma unroll
        for (int m = 0; m < 2 * E - 1; ++m) {
            H[m] = mom[min(jb + ic + q + m, P)];
            T[m] = mom[min(abs(ic - jb - (E - 1) + m), P)];
        }
#pragma unroll
        for (int u = 0; u < E; ++u) {
            aj[u] = (jb + u < nq) ? a[qo + jb + u] : zzero();
            ai[u] = (ic + u < nq) ? a[qo + ic + u] : zzero();
        }
        double ps = 0.0;
#pragma unroll
        for (int d = 0; d < E; ++d) {
            zd acc = zzero();
#pragma unroll
            for (int u = 0; u < E; ++u) acc = zaxpy(acc, H[d + u] + T[u - d + E - 1], ai[u]);
            ps += aj[d].x * acc.x + aj[d].y * acc.y;  // Re(conj(a_j) sum_i (2 M_ji) a_i)
        }
        s += (b < c ? 2.0 : 1.0) * ps;
    }
    return 0.5 * group_sum_d(s, t);
}

template <int NCOL, int PL>
__global__ void __launch_bounds__(NCOL * CF_TEAM, (col_minblocks<NCOL, PL>())) k_column_diag(ColParams p,
                                                                                             double* acc,
                                                                                             double* part) {
    extern __shared__ zd smem[];
    __shared__ double red[3][2 * NCOL];
    const ColCtx<NCOL, PL> X(smem, p, blockIdx.x);
    const Team& t = X.t;
    const int cs = X.cs, hs = t.hs, c0 = X.c0, q = t.q, lane = t.lane, P = t.P;
    const int qo = q * hs, nq = pcount(q, P);
    tile_load_async<NCOL, PL>(X.reg(0), cs, hs, p.U[0], c0, p.Ny, p.B);
    tile_load_async<NCOL, PL>(X.reg(1), cs, hs, p.U[1], c0, p.Ny, p.B);
    tile_load_async<NCOL, PL>(X.reg(2), cs, hs, p.U[2], c0, p.Ny, p.B);
    tile_wait();
    double* mom = reinterpret_cast<double*>(X.reg(6));
    for (int j = threadIdx.x; j <= P; j += NCOL * CF_TEAM) mom[j] = 1.0 / (1.0 - 4.0 * (double)j * j);
    __syncthreads();
    double e = 0.0, dis = 0.0, dmax = 0.0;
    if (X.valid) {
        const bool nyq = col_nyquist(p, X.ix, X.iz);
        const double k = p.ax * X.ix;
        const double l = p.bz * (X.iz <= (p.Nz >> 1) ? X.iz : X.iz - p.Nz);
        zd* U0 = X.col(0);
        zd* U1 = X.col(1);
        zd* U2 = X.col(2);
        zd* W0 = X.col(3);
        zd* W1 = X.col(4);
        zd* W2 = X.col(5);
        zd* DV = X.col(7);
        col_diff<PL>(U2, W0, t);
        col_diff<PL>(U0, W2, t);
        col_diff<PL>(U1, DV, t);
        for (int j = lane; j < nq; j += CF_COL_TW) {
            const int o = qo + j;
            W0[o] = zsub(W0[o], zmulis(U1[o], l));
            W1[o] = zmuli(zsub(zscale(U0[o], l), zscale(U2[o], k)));
            W2[o] = zsub(zmulis(U1[o], k), W2[o]);
            const zd d = zadd(zadd(zmulis(U0[o], k), DV[o]), zmulis(U2[o], l));
            dmax = fmax(dmax, sqrt(d.x * d.x + d.y * d.y));
        }
        tsync(t);
        if (X.c == 0) {
            zd wr, wl;
            col_wallderiv(U0, t, wr, wl);
            if (t.tid == 0) {
                acc[3] = wr.x;
                acc[4] = wl.x;
            }
        }
        for (int m = 16; m >= 1; m >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, m));
        if (!nyq) {
            const double w = X.ix == 0 ? 1.0 : 2.0;
#pragma unroll 1
            for (int f = 0; f < 3; ++f) {
                if constexpr (PL != 0) {
                    e += diag_form_tiled<PL>(sel3(U0, U1, U2, f), mom, t);
                    dis += diag_form_tiled<PL>(sel3(W0, W1, W2, f), mom, t);
                } else {
                    e += diag_form(sel3(U0, U1, U2, f), mom, t);
                    dis += diag_form(sel3(W0, W1, W2, f), mom, t);
                }
            }
            e *= w;
            dis *= w;
        }
    }
    // block partials, one per parity group (no same-address atomics: summed by
    // k_diag_reduce)
    const int wi = threadIdx.x / CF_COL_TW;
    if (lane == 0) {
        red[0][wi] = e;
        red[1][wi] = dis;
        red[2][wi] = dmax;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double se = 0.0, sd = 0.0, mx = 0.0;
        for (int i = 0; i < 2 * NCOL; ++i) {
            se += red[0][i];
            sd += red[1][i];
            mx = fmax(mx, red[2][i]);
        }
        part[3 * blockIdx.x + 0] = se;
        part[3 * blockIdx.x + 1] = sd;
        part[3 * blockIdx.x + 2] = mx;
    }
}

// Sum of the diagnostics' block partials (one block of 1024 threads, fixed
// order): acc[0], acc[1] sums, acc[2] max.
static __global__ void __launch_bounds__(1024) k_diag_reduce(const double* __restrict__ part, int nblk, double* acc) {
    __shared__ double s[3][32];
    double a = 0.0, b = 0.0, m = 0.0;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
        a += part[3 * i];
        b += part[3 * i + 1];
        m = fmax(m, part[3 * i + 2]);
    }
    a = warp_sum_d(a);
    b = warp_sum_d(b);
    for (int o = 16; o >= 1; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) {
        s[0][threadIdx.x >> 5] = a;
        s[1][threadIdx.x >> 5] = b;
        s[2][threadIdx.x >> 5] = m;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sa = 0.0, sb = 0.0, sm = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            sa += s[0][w];
            sb += s[1][w];
            sm = fmax(sm, s[2][w]);
        }
        acc[0] = sa;
        acc[1] = sb;
        acc[2] = sm;
    }
}

// Power input of the mean profile (src/postprocessing.jl:113-128): for the
// (0,0) columns of u and w (with the base profile's coefficients added to u
// when base != null), nu/2 [conj(a(+1)) a'(+1) - conj(a(-1)) a'(-1)] -
// gradient * bulkmean(a), summed over the two components.  One warp; the
// column (0,0) of the (Ny, Nz, Nxh) layout has stride Nz * Nxh.
static __global__ void __launch_bounds__(32) k_power_input(const zd* __restrict__ u, const zd* __restrict__ w,
                                                         const double* __restrict__ base, long stride, int Ny,
                                                         double nu, double gx, double gz, double* out,
                                                         const double* __restrict__ gdev = nullptr) {
    const int lane = threadIdx.x;
    if (gdev) {  // the gradients from device memory (the step's own, recorded without a host round trip)
        gx = gdev[0];
        gz = gdev[1];
    }
    double tot = 0.0;
#pragma unroll 1
    for (int i = 0; i < 2; ++i) {
        const zd* a = i ? w : u;
        zd up = zzero(), lo = zzero(), dr = zzero(), dl = zzero(), bm = zzero();
        for (int n = lane; n < Ny; n += 32) {
            zd v = a[(long)n * stride];
            if (i == 0 && base) v.x += base[n];
            const double sg = (n & 1) ? -1.0 : 1.0, n2 = (double)n * n;
            up = zadd(up, v);
            lo = zaxpy(lo, sg, v);
            dr = zaxpy(dr, n2, v);
            dl = zaxpy(dl, -sg * n2, v);
            if (!(n & 1)) bm = (n == 0) ? zadd(bm, v) : zaxpy(bm, 1.0 / (1.0 - n2), v);
        }
        up = warp_sum_z(up);
        lo = warp_sum_z(lo);
        dr = warp_sum_z(dr);
        dl = warp_sum_z(dl);
        bm = warp_sum_z(bm);
        // real(conj(x) y) = x.re y.re + x.im y.im
        tot += nu / 2 * ((up.x * dr.x + up.y * dr.y) - (lo.x * dl.x + lo.y * dl.y)) - (i ? gz : gx) * bm.x;
    }
    if (lane == 0) *out = tot;
}
