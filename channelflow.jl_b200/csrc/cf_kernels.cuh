// cf_kernels.cuh -- the CNRK2 stage kernels.
//
// Per stage (src/timesteppers/cnrk2.jl:588-623) the engine launches
//   k_zinv    nodal u, omega (6 fields)  -> z-padded, z-inverse FFT
//   k_xpass   x c2r of 6 rows, n = u x omega, x r2c of 3 rows, truncation
//   k_zfwd    z-forward FFT + z truncation -> n at Chebyshev nodes
//   k_column  forward DCT of n, Q update, RHS, Stokes solve (influence and tau
//             corrections, mean mode, flux constraint), curl and inverse DCT
//             of the new velocity and vorticity for the next stage.
// Field storage: complex (Ny, Nz, Nxh), k fastest; z-padded (Ny, Nzp, Nxh).
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
    FftPlan plP;
    const zd* cs;  // (cos, sin)(pi n / P)
    double fnorm;  // 1 / (Nxp Nzp (Ny-1))
};

template <int NCOL>
CF_DEV void tile_load(zd* sm, int cs, const zd* __restrict__ g, int c0, const ColParams& p) {
    const int tot = p.Ny * NCOL;
    for (int e = threadIdx.x; e < tot; e += NCOL * 32) {
        const int n = e / NCOL, t = e - n * NCOL;
        const int c = c0 + t;
        sm[t * cs + n] = (c < p.B) ? g[(long)n * p.B + c] : zzero();
    }
}
template <int NCOL>
CF_DEV void tile_store(const zd* sm, int cs, zd* __restrict__ g, int c0, const ColParams& p) {
    const int tot = p.Ny * NCOL;
    for (int e = threadIdx.x; e < tot; e += NCOL * 32) {
        const int n = e / NCOL, t = e - n * NCOL;
        const int c = c0 + t;
        if (c < p.B) g[(long)n * p.B + c] = sm[t * cs + n];
    }
}

CF_DEV bool col_nyquist(const ColParams& p, int ix, int iz) {
    return ((p.Nx % 2 == 0) && ix == p.Nx / 2) || ((p.Nz % 2 == 0) && iz == p.Nz / 2);
}

// forward DCT of nodal values in x, normalisation, endpoint weights and
// Nyquist filter (ffts.jl:189-206, normalize_forward! :378-393)
CF_DEV void col_forward_y(zd* x, zd* z, const ColParams& p, bool nyq, int lane) {
    col_redft00(x, z, p.cs, p.plP, p.P, lane);
    for (int n = lane; n <= p.P; n += 32) {
        const double e = (n == 0 || n == p.P) ? 0.5 : 1.0;
        x[n] = nyq ? zzero() : zscale(x[n], p.fnorm * e);
    }
    __syncwarp();
}
// inverse DCT: nodal values of the series (icheb with doubled endpoints, the
// 1/2 of copy_to_padded!, ffts.jl:282-287)
CF_DEV void col_inverse_y(zd* x, zd* z, const ColParams& p, int lane) {
    if (lane == 0) {
        x[0] = zscale(x[0], 2.0);
        x[p.P] = zscale(x[p.P], 2.0);
    }
    __syncwarp();
    col_redft00(x, z, p.cs, p.plP, p.P, lane);
    for (int n = lane; n <= p.P; n += 32) x[n] = zscale(x[n], 0.5);
    __syncwarp();
}

// Solve the Stokes problem of one column.  In: R0,R1,R2 (= Rx,Ry,Rz).
// Out: u in R0, v in V, w in R2, p in PT.  A is scratch.  Returns the mean
// gradients for the (0,0) column.
CF_DEV void col_stokes(zd* R0, zd* R1, zd* R2, zd* PT, zd* V, zd* A, const ColParams& p, int c, int ix, int iz,
                       int lane, double* gout) {
    const int P = p.P, Ny = p.Ny;
    const BankDev& bk = p.bank;
    const double k = p.ax * ix;
    const double l = p.bz * (iz <= (p.Nz >> 1) ? iz : iz - p.Nz);
    const double* csc = bk.colsc + (long)c * 8;
    const double* sa = bk.sa + (long)c * 4;
    const double shift = __ldg(csc + 6);
    const double* fv = bk.fac_v + (long)c * 3 * Ny;
    if (c != 0) {
        // r = D Ry + i k Rx + i l Rz ; pressure with zero wall values
        col_diff(R1, PT, P, lane);
        for (int n = lane; n <= P; n += 32) PT[n] = zadd(PT[n], zadd(zmulis(R0[n], k), zmulis(R2[n], l)));
        __syncwarp();
        col_helm(PT, bk.fac_p + (long)c * 3 * Ny, __ldg(sa + 0), __ldg(sa + 1), __ldg(csc + 7), P, zzero(), zzero(),
                 lane);
        // q = D p - Ry ; normal velocity
        col_diff(PT, V, P, lane);
        for (int n = lane; n <= P; n += 32) V[n] = zsub(V[n], R1[n]);
        __syncwarp();
        col_helm(V, fv, __ldg(sa + 2), __ldg(sa + 3), shift, P, zzero(), zzero(), lane);
        // influence correction (batchedinfluence.jl:101-120)
        zd up = zzero(), lo = zzero();
        for (int n = lane; n <= P; n += 32) {
            double t = (double)n * n;
            up = zaxpy(up, -t, V[n]);
            lo = zaxpy(lo, (n & 1) ? -t : t, V[n]);
        }
        up = warp_sum_z(up);
        lo = warp_sum_z(lo);
        const double i00 = __ldg(csc + 0), i01 = __ldg(csc + 1), i10 = __ldg(csc + 2), i11 = __ldg(csc + 3);
        const zd dp = zaxpy(zscale(up, i00), i01, lo);
        const zd dm = zaxpy(zscale(up, i10), i11, lo);
        const double* rs = bk.resp + (long)c * 6 * Ny;
        for (int n = lane; n <= P; n += 32) {
            PT[n] = zaxpy(zaxpy(PT[n], __ldg(rs + n), dp), __ldg(rs + Ny + n), dm);
            V[n] = zaxpy(zaxpy(V[n], __ldg(rs + 2 * Ny + n), dp), __ldg(rs + 3 * Ny + n), dm);
        }
        __syncwarp();
        // tau correction (batchedinfluence.jl:148-160); (Dp)_{P-1} = 2P p_P, (Dp)_P = 0
        const zd s1 = zscale(zsub(zaxpy(zscale(V[P - 1], shift), 2.0 * P, PT[P]), R1[P - 1]),
                             1.0 / (1.0 - __ldg(csc + 4)));
        const zd s2 = zscale(zsub(zscale(V[P], shift), R1[P]), 1.0 / (1.0 - __ldg(csc + 5)));
        __syncwarp();
        for (int n = lane; n <= P; n += 32) {
            const bool ev = (n & 1) == 0;
            PT[n] = zadd(PT[n], zscale(ev ? s1 : s2, __ldg(rs + 4 * Ny + n)));
            V[n] = zadd(V[n], zscale(ev ? s2 : s1, __ldg(rs + 5 * Ny + n)));
        }
        __syncwarp();
    } else {
        // mean mode (meanmode.jl:278-288): integrate Ry through degree P-1, gauge
        for (int n = lane; n <= P; n += 32) {
            zd v = zzero();
            if (n >= 1) {
                zd lower = (n == 1) ? R1[0] : zscale(R1[n - 1], 0.5);
                zd upper = (n + 1 < P) ? zscale(R1[n + 1], 0.5) : zzero();
                v = zscale(zsub(lower, upper), 1.0 / n);
            }
            PT[n] = v;
            V[n] = zzero();
        }
        __syncwarp();
        zd m = col_bulkmean(PT, P, lane);  // PT[0] is zero here
        if (lane == 0) PT[0] = zscale(m, -1.0);
        __syncwarp();
    }
    // tangential velocities: (nu D^2 - shift) u = i k p - Rx, likewise w
    for (int n = lane; n <= P; n += 32) {
        R0[n] = zsub(zmulis(PT[n], k), R0[n]);
        R2[n] = zsub(zmulis(PT[n], l), R2[n]);
    }
    __syncwarp();
    col_helm(R0, fv, __ldg(sa + 2), __ldg(sa + 3), shift, P, zzero(), zzero(), lane);
    col_helm(R2, fv, __ldg(sa + 2), __ldg(sa + 3), shift, P, zzero(), zzero(), lane);
    if (c == 0) {
        double gx, gz;
        if (p.cmode == 1) {
            zd mu = col_bulkmean(R0, P, lane), mw = col_bulkmean(R2, P, lane);
            gx = (p.c1 - mu.x) / bk.meanc_mean;
            gz = (p.c2 - mw.x) / bk.meanc_mean;
        } else {
            gx = p.c1;
            gz = p.c2;
        }
        for (int n = lane; n <= P; n += 32) {
            const double r = __ldg(bk.meanc + n);
            R0[n] = zadd(R0[n], zmake(gx * r, 0.0));
            R2[n] = zadd(R2[n], zmake(gz * r, 0.0));
        }
        __syncwarp();
        gout[0] = gx;
        gout[1] = gz;
    }
}

// curl of the total velocity and inverse DCT of all six fields to the nodal
// buffers (nonlinear.jl:179-185, operators.jl:380-398).  u, v, w in U0, U1, U2
// (modified); W0, W1, W2, Z scratch.
template <int NCOL>
CF_DEV void col_prep_nodal(zd* U0, zd* U1, zd* U2, zd* W0, zd* W1, zd* W2, zd* Z, const ColParams& p, int c, int ix,
                           int iz, int lane, int c0, int cs) {
    const int P = p.P;
    const double k = p.ax * ix;
    const double l = p.bz * (iz <= (p.Nz >> 1) ? iz : iz - p.Nz);
    if (c == 0)
        for (int n = lane; n <= P; n += 32) U0[n] = zadd(U0[n], zmake(__ldg(p.base + n), 0.0));
    __syncwarp();
    col_diff(U2, W0, P, lane);  // omega_x = D w - i l v
    col_diff(U0, W2, P, lane);  // omega_z = i k v - D u
    for (int n = lane; n <= P; n += 32) {
        W0[n] = zsub(W0[n], zmulis(U1[n], l));
        W1[n] = zmuli(zsub(zscale(U0[n], l), zscale(U2[n], k)));
        W2[n] = zsub(zmulis(U1[n], k), W2[n]);
    }
    __syncwarp();
    zd* f[6] = {U0, U1, U2, W0, W1, W2};
#pragma unroll 1
    for (int i = 0; i < 6; ++i) col_inverse_y(f[i], Z, p, lane);
}

// Full CNRK2 stage for NCOL columns per block (one warp per column).
// SMEM per column: 7 vectors of CS complex.
template <int NCOL>
__global__ void __launch_bounds__(NCOL * 32) k_column_stage(ColParams p) {
    extern __shared__ zd smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cs = p.Ny + 1;  // column stride (complex)
    const int c0 = blockIdx.x * NCOL;
    const int c = c0 + warp;
    const bool valid = c < p.B;
    const int ix = c % p.Nxh, iz = c / p.Nxh;
    // regions: 0 R0, 1 R1, 2 R2, 3 PT, 4 A, 5 Bw, 6 Z
    zd* reg[7];
#pragma unroll
    for (int r = 0; r < 7; ++r) reg[r] = smem + (long)r * NCOL * cs;
    auto col = [&](int r) { return reg[r] + warp * cs; };
    const bool nyq = valid ? col_nyquist(p, ix, iz) : true;
    const double k = p.ax * ix;
    const double l = p.bz * (iz <= (p.Nz >> 1) ? iz : iz - p.Nz);
    const double kap2 = k * k + l * l;
    const int P = p.P;

    // ---------------- Phase A: nonlinear term, history, right-hand side
    tile_load<NCOL>(reg[3], cs, p.Pf, c0, p);
    double gold[2] = {p.c1, p.c2};
    zd bulkN[3], wallR[3], wallL[3];
#pragma unroll 1
    for (int i = 0; i < 3; ++i) {
        tile_load<NCOL>(reg[4], cs, p.Nn[i], c0, p);
        __syncthreads();
        if (valid) {
            col_forward_y(col(4), col(6), p, nyq, lane);
            if (c == 0) bulkN[i] = col_bulkmean(col(4), P, lane);
        }
        __syncthreads();
        if (p.stage > 0) tile_load<NCOL>(reg[5], cs, p.Q[i], c0, p);
        __syncthreads();
        if (valid && p.stage > 0) {
            zd* A = col(4);
            const zd* Qo = col(5);
            for (int n = lane; n <= P; n += 32) A[n] = zaxpy(A[n], p.Acoef, Qo[n]);
        }
        __syncthreads();
        if (p.store_q) tile_store<NCOL>(reg[4], cs, p.Q[i], c0, p);
        tile_load<NCOL>(reg[5], cs, p.U[i], c0, p);
        __syncthreads();
        if (valid) {
            zd* U = col(5);
            zd* Qn = col(4);
            zd* Z = col(6);
            zd* R = col(i);
            if (c == 0) col_wallderiv(U, P, lane, wallR[i], wallL[i]);
            col_diff(U, Z, P, lane);
            col_diff(Z, R, P, lane);
            // R = lambda U + nu (D^2 U - kappa^2 U) - d_i P + (B/C) Q
            if (i == 1) col_diff(col(3), Z, P, lane);
            const zd* PT = col(3);
            for (int n = lane; n <= P; n += 32) {
                zd lap = zaxpy(R[n], -kap2, U[n]);
                zd r = zaxpy(zscale(U[n], p.lambda), p.nu, lap);
                zd dP = (i == 0) ? zmulis(PT[n], k) : (i == 1 ? Z[n] : zmulis(PT[n], l));
                r = zsub(r, dP);
                r = zaxpy(r, p.weight, Qn[n]);
                R[n] = r;
            }
            __syncwarp();
        }
        __syncthreads();
    }
    if (valid && c == 0) {
        zd* R0 = col(0);
        if (p.cmode == 1) {
            gold[0] = p.nu * (wallR[0].x - wallL[0].x) / 2 + p.nu_bm_curv + bulkN[0].x;
            gold[1] = p.nu * (wallR[2].x - wallL[2].x) / 2 + bulkN[2].x;
        }
        for (int n = lane; n <= P; n += 32) R0[n] = zadd(R0[n], zmake(2.0 * p.nu * __ldg(p.basecurv + n), 0.0));
        __syncwarp();
        if (lane == 0) {
            R0[0].x -= gold[0];
            zd* R2 = col(2);
            R2[0].x -= gold[1];
        }
        __syncwarp();
    }
    // ---------------- Phase B: Stokes solve
    if (valid) {
        if (nyq) {
            for (int r = 0; r < 6; ++r) {
                if (r == 1) continue;
                zd* x = col(r);
                for (int n = lane; n <= P; n += 32) x[n] = zzero();
            }
            __syncwarp();
        } else {
            double g2[2];
            col_stokes(col(0), col(1), col(2), col(3), col(4), col(5), p, c, ix, iz, lane, g2);
            if (c == 0 && lane == 0) {
                p.grad_out[0] = g2[0];
                p.grad_out[1] = g2[1];
            }
        }
    }
    __syncthreads();
    tile_store<NCOL>(reg[0], cs, p.U[0], c0, p);
    tile_store<NCOL>(reg[4], cs, p.U[1], c0, p);
    tile_store<NCOL>(reg[2], cs, p.U[2], c0, p);
    tile_store<NCOL>(reg[3], cs, p.Pf, c0, p);
    __syncthreads();
    // ---------------- Phase C: total velocity, vorticity, nodal values
    if (valid) col_prep_nodal<NCOL>(col(0), col(4), col(2), col(1), col(3), col(5), col(6), p, c, ix, iz, lane, c0, cs);
    __syncthreads();
    tile_store<NCOL>(reg[0], cs, p.nod[0], c0, p);
    tile_store<NCOL>(reg[4], cs, p.nod[1], c0, p);
    tile_store<NCOL>(reg[2], cs, p.nod[2], c0, p);
    tile_store<NCOL>(reg[1], cs, p.nod[3], c0, p);
    tile_store<NCOL>(reg[3], cs, p.nod[4], c0, p);
    tile_store<NCOL>(reg[5], cs, p.nod[5], c0, p);
}

// Nodal velocity and vorticity from the state U (used after set_state).
template <int NCOL>
__global__ void __launch_bounds__(NCOL * 32) k_column_prep(ColParams p) {
    extern __shared__ zd smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cs = p.Ny + 1;
    const int c0 = blockIdx.x * NCOL;
    const int c = c0 + warp;
    zd* reg[7];
#pragma unroll
    for (int r = 0; r < 7; ++r) reg[r] = smem + (long)r * NCOL * cs;
    auto col = [&](int r) { return reg[r] + warp * cs; };
    tile_load<NCOL>(reg[0], cs, p.U[0], c0, p);
    tile_load<NCOL>(reg[1], cs, p.U[1], c0, p);
    tile_load<NCOL>(reg[2], cs, p.U[2], c0, p);
    __syncthreads();
    if (c < p.B)
        col_prep_nodal<NCOL>(col(0), col(1), col(2), col(3), col(4), col(5), col(6), p, c, c % p.Nxh, c / p.Nxh,
                             lane, c0, cs);
    __syncthreads();
    for (int i = 0; i < 6; ++i) tile_store<NCOL>(reg[i], cs, p.nod[i], c0, p);
}

// Forward DCT of the nonlinear term only: coefficients into p.Nout.
template <int NCOL>
__global__ void __launch_bounds__(NCOL * 32) k_column_nlout(ColParams p) {
    extern __shared__ zd smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cs = p.Ny + 1;
    const int c0 = blockIdx.x * NCOL;
    const int c = c0 + warp;
    zd* reg[2] = {smem, smem + NCOL * cs};
    for (int i = 0; i < 3; ++i) {
        tile_load<NCOL>(reg[0], cs, p.Nn[i], c0, p);
        __syncthreads();
        if (c < p.B) col_forward_y(reg[0] + warp * cs, reg[1] + warp * cs, p, col_nyquist(p, c % p.Nxh, c / p.Nxh), lane);
        __syncthreads();
        tile_store<NCOL>(reg[0], cs, p.Nout[i], c0, p);
        __syncthreads();
    }
}

// Stokes projection (pressure.jl:36-54): R = -Laplacian(U), solve with the
// (nu = 1, lambda = 0) bank, velocity overwritten.
template <int NCOL>
__global__ void __launch_bounds__(NCOL * 32) k_column_project(ColParams p) {
    extern __shared__ zd smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cs = p.Ny + 1;
    const int c0 = blockIdx.x * NCOL;
    const int c = c0 + warp;
    const bool valid = c < p.B;
    const int ix = c % p.Nxh, iz = c / p.Nxh;
    zd* reg[7];
#pragma unroll
    for (int r = 0; r < 7; ++r) reg[r] = smem + (long)r * NCOL * cs;
    auto col = [&](int r) { return reg[r] + warp * cs; };
    const double k = p.ax * ix;
    const double l = p.bz * (iz <= (p.Nz >> 1) ? iz : iz - p.Nz);
    const double kap2 = k * k + l * l;
    for (int i = 0; i < 3; ++i) {
        tile_load<NCOL>(reg[5], cs, p.U[i], c0, p);
        __syncthreads();
        if (valid) {
            zd* U = col(5);
            zd* Z = col(6);
            zd* R = col(i);
            col_diff(U, Z, p.P, lane);
            col_diff(Z, R, p.P, lane);
            for (int n = lane; n <= p.P; n += 32) R[n] = zscale(zaxpy(R[n], -kap2, U[n]), -1.0);
            __syncwarp();
        }
        __syncthreads();
    }
    if (valid) {
        if (col_nyquist(p, ix, iz)) {
            for (int r = 0; r < 6; ++r) {
                zd* x = col(r);
                for (int n = lane; n <= p.P; n += 32) x[n] = zzero();
            }
            __syncwarp();
        } else {
            double g2[2];
            col_stokes(col(0), col(1), col(2), col(3), col(4), col(5), p, c, ix, iz, lane, g2);
        }
    }
    __syncthreads();
    tile_store<NCOL>(reg[0], cs, p.U[0], c0, p);
    tile_store<NCOL>(reg[4], cs, p.U[1], c0, p);
    tile_store<NCOL>(reg[2], cs, p.U[2], c0, p);
}

// Pressure reconstruction (pressure.jl:115-204) from the nonlinear term at
// the nodes (p.Nn) and the normal velocity U[1]: Neumann Helmholtz per mode
// with the factors in p.bank.fac_p / sa[0..1] (Neumann weights).
template <int NCOL>
__global__ void __launch_bounds__(NCOL * 32) k_column_pressure(ColParams p) {
    extern __shared__ zd smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cs = p.Ny + 1;
    const int c0 = blockIdx.x * NCOL;
    const int c = c0 + warp;
    const bool valid = c < p.B;
    const int ix = c % p.Nxh, iz = c / p.Nxh;
    const int P = p.P;
    zd* reg[7];
#pragma unroll
    for (int r = 0; r < 7; ++r) reg[r] = smem + (long)r * NCOL * cs;
    auto col = [&](int r) { return reg[r] + warp * cs; };
    const bool nyq = valid ? col_nyquist(p, ix, iz) : true;
    for (int i = 0; i < 3; ++i) {
        tile_load<NCOL>(reg[i], cs, p.Nn[i], c0, p);
        __syncthreads();
        if (valid) col_forward_y(col(i), col(6), p, nyq, lane);
        __syncthreads();
    }
    tile_load<NCOL>(reg[4], cs, p.U[1], c0, p);
    __syncthreads();
    if (valid) {
        const double k = p.ax * ix;
        const double l = p.bz * (iz <= (p.Nz >> 1) ? iz : iz - p.Nz);
        zd* A0 = col(0);
        zd* A1 = col(1);
        zd* A2 = col(2);
        zd* PT = col(3);
        zd* V = col(4);
        if (nyq) {
            for (int n = lane; n <= P; n += 32) PT[n] = zzero();
            __syncwarp();
        } else if (c == 0) {
            for (int n = lane; n <= P; n += 32) {
                zd v = zzero();
                if (n >= 1) {
                    zd lower = (n == 1) ? A1[0] : zscale(A1[n - 1], 0.5);
                    zd upper = (n + 1 < P) ? zscale(A1[n + 1], 0.5) : zzero();
                    v = zscale(zsub(lower, upper), 1.0 / n);
                }
                PT[n] = v;
            }
            __syncwarp();
            zd m = col_bulkmean(PT, P, lane);
            if (lane == 0) PT[0] = zscale(m, -1.0);
            __syncwarp();
        } else {
            col_diff(A1, PT, P, lane);
            for (int n = lane; n <= P; n += 32) PT[n] = zadd(PT[n], zadd(zmulis(A0[n], k), zmulis(A2[n], l)));
            zd up = zzero(), lo = zzero();
            for (int n = lane; n <= P; n += 32) {
                up = zadd(up, A1[n]);
                lo = zaxpy(lo, (n & 1) ? -1.0 : 1.0, A1[n]);
                if (n >= 2) {
                    const double wn = p.nu * ((double)n * n * ((double)n * n - 1.0) / 3.0);
                    up = zaxpy(up, wn, V[n]);
                    lo = zaxpy(lo, (n & 1) ? -wn : wn, V[n]);
                }
            }
            up = warp_sum_z(up);
            lo = warp_sum_z(lo);
            __syncwarp();
            const double* sa = p.bank.sa + (long)c * 4;
            // Neumann parity data: even rows (up - lo)/2, odd rows (up + lo)/2
            col_helm(PT, p.bank.fac_p + (long)c * 3 * p.Ny, __ldg(sa + 0), __ldg(sa + 1), k * k + l * l, P,
                     zscale(zsub(up, lo), 0.5), zscale(zadd(up, lo), 0.5), lane);
        }
    }
    __syncthreads();
    tile_store<NCOL>(reg[3], cs, p.Pf, c0, p);
}
