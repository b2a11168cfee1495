// cf_column.cuh -- per-column (one Fourier pair (k,l), all Chebyshev degrees)
// device building blocks.  One warp owns one column; the column's vectors
// live in shared memory.  All routines are warp-synchronous.
//
// Reference arithmetic restated here:
//  * Chebyshev derivative recurrence b_n = b_{n+2} + 2(n+1) a_{n+1}, b_0
//    halved (src/fields/operators.jl:38-61, solvers/batchedinfluence.jl:32-43),
//    evaluated as the equivalent suffix sums b_n = 2 sum_{m>n, m-n odd} m a_m.
//  * Tau Helmholtz solve of rows 0..P-2 of (th0 D^2 - th1) a = f plus wall rows
//    (docs/src/spatial.md:448-475), in its quasi-tridiagonal (spectral
//    integration) form: for n >= 2 of each parity
//       s_n a_{n-2} + d_n a_n + u_n a_{n+2} = g_n,
//    eliminated from the top degree downwards.  The two linear sweeps are
//    parallel prefix scans of affine maps; the wall row is reduced with the
//    precomputed weights W (see cf_setup.cpp).
//  * DCT-I (FFTW REDFT00, src/transforms/chebyshev.jl:481-502) of a complex
//    column of length P+1 through one complex FFT of length P.
#pragma once
#include "cf_common.cuh"
#include "cf_fft.cuh"

#define CF_WARP_FFT_MAXE 16
#define CF_HELM_MAXR 8  // chain rounds of 32: supports P <= 510

// b = D a  (b != a), column of Ny = P+1 complex coefficients
CF_DEV void col_diff(const zd* a, zd* b, int P, int lane) {
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int top = ((P & 1) == q) ? P : P - 1;
        const int cnt = (top - q) / 2 + 1;  // m = top, top-2, ..., q
        zd carry = zzero();
        for (int base = 0; base < cnt; base += 32) {
            const int i = base + lane;
            const int m = top - 2 * i;
            zd val = zzero();
            if (i < cnt && m >= 1) val = zscale(a[m], (double)m);
            zd s = zadd(warp_scan_z(val, lane), carry);
            if (i < cnt && m >= 1) b[m - 1] = (m == 1) ? s : zscale(s, 2.0);
            carry = shfl_z(s, 31);
        }
    }
    if (lane == 0) b[P] = zzero();
    __syncwarp();
}

// In-place tau Helmholtz solve on x (input f, output a).  fac points at the
// column's factors: alpha[Ny], invden[Ny], W[Ny]; SA0/SA1 are the wall-row
// sums of the even/odd parity; bc0/bc1 the parity wall data.
CF_DEV void col_helm(zd* x, const double* __restrict__ fac, double SA0, double SA1, double th1, int P, zd bc0,
                     zd bc1, int lane) {
    const int Ny = P + 1;
    const double* alpha = fac;
    const double* invden = fac + Ny;
    const double* W = fac + 2 * Ny;
#pragma unroll 1
    for (int par = 0; par < 2; ++par) {
        const int top = ((P & 1) == par) ? P : P - 1;
        const int cnt = (top - par) / 2;  // chain n = top, top-2, ..., par+2
        // g_n from f (all values read before any write)
        zd g[CF_HELM_MAXR];
#pragma unroll
        for (int r = 0; r < CF_HELM_MAXR; ++r) {
            const int i = r * 32 + lane;
            g[r] = zzero();
            if (i < cnt) {
                const int n = top - 2 * i;
                const double cm = (n - 2 == 0) ? 2.0 : 1.0;
                zd v = zscale(x[n - 2], cm / (4.0 * n * (n - 1)));
                if (n <= P - 2) v = zaxpy(v, -1.0 / (2.0 * ((double)n * n - 1.0)), x[n]);
                if (n + 2 <= P - 2) v = zaxpy(v, 1.0 / (4.0 * n * (n + 1)), x[n + 2]);
                g[r] = v;
            }
        }
        __syncwarp();
        // backward sweep beta_n = invden_n (g_n - u_n beta_{n+2}), u_n = -th1/(4n(n+1))
        zd carry = zzero();
        zd sw = zzero();
#pragma unroll
        for (int r = 0; r < CF_HELM_MAXR; ++r) {
            const int base = r * 32;
            if (base >= cnt) break;
            const int i = base + lane;
            double M = 1.0;
            zd G = zzero();
            int n = 0;
            if (i < cnt) {
                n = top - 2 * i;
                const double id = __ldg(invden + n);
                G = zscale(g[r], id);
                M = (n + 2 <= P - 2) ? th1 / (4.0 * n * (n + 1)) * id : 0.0;
            }
            warp_scan_affine(M, G, lane);
            zd beta = zaxpy(G, M, carry);
            if (i < cnt) {
                x[n] = beta;
                sw = zaxpy(sw, __ldg(W + n), beta);
            }
            carry = shfl_z(beta, 31);
        }
        sw = warp_sum_z(sw);
        const double SA = par ? SA1 : SA0;
        const zd bc = par ? bc1 : bc0;
        const zd a0 = zscale(zsub(bc, sw), 1.0 / SA);
        __syncwarp();
        // forward sweep a_n = alpha_n a_{n-2} + beta_n
        carry = a0;
#pragma unroll
        for (int r = 0; r < CF_HELM_MAXR; ++r) {
            const int base = r * 32;
            if (base >= cnt) break;
            const int j = base + lane;
            double M = 1.0;
            zd G = zzero();
            int n = 0;
            if (j < cnt) {
                n = par + 2 + 2 * j;
                M = __ldg(alpha + n);
                G = x[n];
            }
            warp_scan_affine(M, G, lane);
            zd a = zaxpy(G, M, carry);
            __syncwarp();
            if (j < cnt) x[n] = a;
            carry = shfl_z(a, 31);
        }
        if (lane == 0) x[par] = a0;
        __syncwarp();
    }
}

// DCT-I (REDFT00, unnormalised) of complex x[0..P] in place; z is P complex
// of scratch.  X_k = x_0 + (-1)^k x_P + 2 sum_{n=1}^{P-1} x_n cos(pi n k/P).
// With z_n = (x_n + x_{P-n})/2 - sin(pi n/P)(x_n - x_{P-n}) and Z = FFT_P(z):
//   X_{2m} = Z_m + Z_{P-m},  X_1 = x_0 - x_P + 2 sum_{n=1}^{P-1} x_n cos(pi n/P),
//   X_{2m+1} = X_{2m-1} + i (Z_m - Z_{P-m}).
// cs[n] = (cos(pi n/P), sin(pi n/P)), n = 0..P.  P must be even.
CF_DEV void col_redft00(zd* x, zd* z, const zd* __restrict__ cs, const FftPlan& pl, int P, int lane) {
    const int H = P >> 1;
    zd x1 = zzero();
    for (int n = lane; n <= H; n += 32) {
        if (n == 0) {
            zd a = x[0], b = x[P];
            z[0] = zscale(zadd(a, b), 0.5);
            x1 = zadd(x1, zsub(a, b));
        } else if (n == H) {
            z[H] = x[H];
        } else {
            zd a = x[n], b = x[P - n];
            zd c = __ldg(cs + n);
            zd h = zscale(zadd(a, b), 0.5), d = zsub(a, b);
            z[n] = zaxpy(h, -c.y, d);
            z[P - n] = zaxpy(h, c.y, d);
            x1 = zaxpy(x1, 2.0 * c.x, d);
        }
    }
    x1 = warp_sum_z(x1);
    __syncwarp();
    group_fft<false, CF_WARP_FFT_MAXE>(z, 1, P, pl, -1, lane, 32);
    // odd outputs: prefix sums of i (Z_m - Z_{P-m}), m = 1..H-1
    zd carry = x1;
    for (int base = 0; base < H; base += 32) {
        const int m = base + lane;
        zd o = zzero();
        if (m >= 1 && m < H) o = zmuli(zsub(z[m], z[P - m]));
        zd s = zadd(warp_scan_z(o, lane), carry);
        if (m < H) x[2 * m + 1] = s;
        carry = shfl_z(s, 31);
    }
    for (int m = lane; m <= H; m += 32) {
        x[2 * m] = (m == 0 || m == H) ? zscale(z[m], 2.0) : zadd(z[m], z[P - m]);
    }
    __syncwarp();
}

// Mean over y (meanmode.jl:173-179): a0 + sum_{even n >= 2} a_n / (1 - n^2)
CF_DEV zd col_bulkmean(const zd* a, int P, int lane) {
    zd s = zzero();
    for (int n = lane; n <= P; n += 32) {
        if (n == 0) s = zadd(s, a[0]);
        else if ((n & 1) == 0) s = zaxpy(s, 1.0 / (1.0 - (double)n * n), a[n]);
    }
    return warp_sum_z(s);
}
// a'(+1) = sum n^2 a_n ; a'(-1) = sum (-1)^(n+1) n^2 a_n
CF_DEV void col_wallderiv(const zd* a, int P, int lane, zd& right, zd& left) {
    zd r = zzero(), l = zzero();
    for (int n = lane; n <= P; n += 32) {
        double w = (double)n * n;
        r = zaxpy(r, w, a[n]);
        l = zaxpy(l, (n & 1) ? w : -w, a[n]);
    }
    right = warp_sum_z(r);
    left = warp_sum_z(l);
}
