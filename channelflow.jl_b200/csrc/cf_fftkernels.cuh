// cf_fftkernels.cuh -- periodic-direction transforms of the rotational
// nonlinear term (src/ffts.jl:189-206 and 275-290, src/nonlinear.jl:184-191).
//
// k_zinv : nodal (Ny,Nz,Nxh) -> z-padded spectrum (copy_to_padded!, Nyquist
//          filter) -> backward z FFT of length Nzp   (Ny,Nzp,Nxh)
// k_xpass: backward x c2r of the six rows (pairs packed as one complex FFT),
//          n = u x omega at the padded points, forward x r2c, x truncation
// k_zfwd : forward z FFT of the three products, z truncation (copy_from_padded!)
// Shared-memory transform buffers use the swizzled positions of cf_fft.cuh.
#pragma once
#include "cf_fft.cuh"

struct FftParams {
    int Nx, Nz, Nxh, Ny, Nzp, Nxp;
    int tkz;       // columns per block in the z kernels
    int bsz, bsx;  // transform buffer strides: Nzp, Nxp rounded up to 8
    zd *nod0, *nod1, *nod2, *nod3, *nod4, *nod5;  // nodal fields
    zd *zp0, *zp1, *zp2, *zp3, *zp4, *zp5;        // z-padded fields
    FftPlan plZ, plX;
};

CF_DEV zd* sel6(zd* a0, zd* a1, zd* a2, zd* a3, zd* a4, zd* a5, int i) {
    switch (i) {
        case 0: return a0;
        case 1: return a1;
        case 2: return a2;
        case 3: return a3;
        case 4: return a4;
        default: return a5;
    }
}
CF_DEV zd* nod_of(const FftParams& p, int i) { return sel6(p.nod0, p.nod1, p.nod2, p.nod3, p.nod4, p.nod5, i); }
CF_DEV zd* zp_of(const FftParams& p, int i) { return sel6(p.zp0, p.zp1, p.zp2, p.zp3, p.zp4, p.zp5, i); }

CF_DEV int zpad_index(int iz, int Nz, int Nzp) { return iz <= (Nz >> 1) ? iz : Nzp - (Nz - iz); }

// grid: (ceil(Nxh/tkz), Ny, nfields); block 256; smem 2*tkz*bsz complex
template <int LZ>
__global__ void __launch_bounds__(256) k_zinv(FftParams p) {
    extern __shared__ zd sm[];
    const int f = blockIdx.z, n = blockIdx.y, k0 = blockIdx.x * p.tkz;
    const int tkz = p.tkz, Nz = p.Nz, Nzp = p.Nzp, Nxh = p.Nxh, bs = p.bsz;
    zd* bufB = sm + tkz * bs;
    const zd* src = nod_of(p, f) + (long)n * Nz * Nxh;
    zd* dst = zp_of(p, f) + (long)n * Nzp * Nxh;
    // zero the padding gap
    const int gap0 = (Nz >> 1) + 1, gap1 = Nzp - (Nz - gap0);
    for (int e = threadIdx.x; e < tkz * (gap1 - gap0); e += blockDim.x) {
        int t = e % tkz, z = gap0 + e / tkz;
        sm[t * bs + swz(z)] = zzero();
    }
    // loads batched 8 per thread before their stores (requests in flight)
    for (int base = threadIdx.x; base < tkz * Nz; base += 8 * 256) {
        zd v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = base + u * 256;
            const int t = e % tkz, iz = e / tkz, k = k0 + t;
            const bool nyq = ((p.Nz % 2 == 0) && iz == Nz / 2) || ((p.Nx % 2 == 0) && k == p.Nx / 2);
            v[u] = (e < tkz * Nz && k < Nxh && !nyq) ? src[(long)iz * Nxh + k] : zzero();
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = base + u * 256;
            if (e < tkz * Nz) sm[(e % tkz) * bs + swz(zpad_index(e / tkz, Nz, Nzp))] = v[u];
        }
    }
    __syncthreads();
    const zd* res = group_fft_L<true, LZ>(sm, bufB, tkz, bs, p.plZ, +1, threadIdx.x, blockDim.x, 0);
    for (int e = threadIdx.x; e < tkz * Nzp; e += blockDim.x) {
        int t = e % tkz, z = e / tkz;
        int k = k0 + t;
        if (k < Nxh) dst[(long)z * Nxh + k] = res[t * bs + swz(z)];
    }
}

// grid: (ceil(Nxh/tkz), Ny, 3); forward z FFT and truncation to Nz
template <int LZ>
__global__ void __launch_bounds__(256) k_zfwd(FftParams p) {
    extern __shared__ zd sm[];
    const int f = blockIdx.z, n = blockIdx.y, k0 = blockIdx.x * p.tkz;
    const int tkz = p.tkz, Nz = p.Nz, Nzp = p.Nzp, Nxh = p.Nxh, bs = p.bsz;
    zd* bufB = sm + tkz * bs;
    const zd* src = zp_of(p, f) + (long)n * Nzp * Nxh;
    zd* dst = nod_of(p, f) + (long)n * Nz * Nxh;
    for (int base = threadIdx.x; base < tkz * Nzp; base += 8 * 256) {
        zd v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = base + u * 256;
            const int k = k0 + e % tkz;
            v[u] = (e < tkz * Nzp && k < Nxh) ? src[(long)(e / tkz) * Nxh + k] : zzero();
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = base + u * 256;
            if (e < tkz * Nzp) sm[(e % tkz) * bs + swz(e / tkz)] = v[u];
        }
    }
    __syncthreads();
    const zd* res = group_fft_L<true, LZ>(sm, bufB, tkz, bs, p.plZ, -1, threadIdx.x, blockDim.x, 0);
    for (int e = threadIdx.x; e < tkz * Nz; e += blockDim.x) {
        int t = e % tkz, iz = e / tkz;
        int k = k0 + t;
        if (k < Nxh) dst[(long)iz * Nxh + k] = res[t * bs + swz(zpad_index(iz, Nz, Nzp))];
    }
}

// grid: (ceil(Nzp/2), Ny); block 256; smem 12*bsx complex (6 slots + scratch).
// Rows zA = 2*bx and zB = 2*bx+1 of plane n.  Slots 0..5 hold
// (u0+iu1, u2+iw0, w1+iw2) of row A at 0,2,4 and of row B at 1,3,5.
template <int LX>
__global__ void __launch_bounds__(256) k_xpass(FftParams p) {
    extern __shared__ zd sm[];
    const int n = blockIdx.y;
    const int zA = 2 * blockIdx.x, zB = zA + 1;
    const bool hasB = zB < p.Nzp;
    const int Nxp = p.Nxp, Nxh = p.Nxh, bs = p.bsx;
    const int Nxhp = Nxp / 2 + 1;
    const long rowA = ((long)n * p.Nzp + zA) * Nxh;
    const long rowB = ((long)n * p.Nzp + zB) * Nxh;
    const int xnyq = (p.Nx % 2 == 0) ? p.Nx / 2 : -1;
    zd* scr = sm + 6 * bs;
    // pack Hermitian pairs: Z_k = X_k + i Y_k, Z_{Nxp-k} = conj(X_k) + i conj(Y_k);
    // every position 0..Nxp-1 of the six slots is written (zeros for a missing
    // row B and for k >= Nxh)
    for (int base = threadIdx.x; base < 6 * Nxhp; base += 4 * 256) {
        zd X[4], Y[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = base + u * 256;
            const int slot = e / Nxhp, k = e - slot * Nxhp;
            const int pair = slot >> 1;
            const bool isB = slot & 1;
            const long row = isB ? rowB : rowA;
            X[u] = zzero();
            Y[u] = zzero();
            if (e < 6 * Nxhp && !(isB && !hasB) && k < Nxh && k != xnyq) {
                X[u] = zp_of(p, 2 * pair)[row + k];
                Y[u] = zp_of(p, 2 * pair + 1)[row + k];
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = base + u * 256;
            if (e >= 6 * Nxhp) continue;
            const int slot = e / Nxhp, k = e - slot * Nxhp;
            zd* s = sm + slot * bs;
            if (k == 0) {
                s[swz(0)] = zmake(X[u].x, Y[u].x);
            } else if (2 * k == Nxp) {
                s[swz(k)] = zmake(X[u].x, Y[u].x);
            } else {
                s[swz(k)] = zmake(X[u].x - Y[u].y, X[u].y + Y[u].x);
                s[swz(Nxp - k)] = zmake(X[u].x + Y[u].y, Y[u].x - X[u].y);
            }
        }
    }
    __syncthreads();
    zd* A = group_fft_L<true, LX>(sm, scr, 6, bs, p.plX, +1, threadIdx.x, blockDim.x, 0);
    zd* Bf = (A == sm) ? scr : sm;
    // rotational product n = u x omega at every padded x point of both rows
    for (int j = threadIdx.x; j < Nxp; j += blockDim.x) {
        const int sj = swz(j);
        zd a0 = A[0 * bs + sj], a1 = A[2 * bs + sj], a2 = A[4 * bs + sj];
        zd b0 = A[1 * bs + sj], b1 = A[3 * bs + sj], b2 = A[5 * bs + sj];
        // row A: u=(a0.x,a0.y,a1.x), w=(a1.y,a2.x,a2.y)
        double nA0 = a0.y * a2.y - a1.x * a2.x;
        double nA1 = a1.x * a1.y - a0.x * a2.y;
        double nA2 = a0.x * a2.x - a0.y * a1.y;
        double nB0 = b0.y * b2.y - b1.x * b2.x;
        double nB1 = b1.x * b1.y - b0.x * b2.y;
        double nB2 = b0.x * b2.x - b0.y * b1.y;
        Bf[0 * bs + sj] = zmake(nA0, nA1);
        Bf[1 * bs + sj] = zmake(nB0, nB1);
        Bf[2 * bs + sj] = zmake(nA2, nB2);
    }
    __syncthreads();
    const zd* F = group_fft_L<true, LX>(Bf, A, 3, bs, p.plX, -1, threadIdx.x, blockDim.x, 0);
    // separate the packed real transforms and keep k < Nxh
    for (int e = threadIdx.x; e < 3 * Nxh; e += blockDim.x) {
        const int slot = e / Nxh, k = e - slot * Nxh;
        const zd* s = F + slot * bs;
        zd Zk = s[swz(k)], Zm = s[swz((Nxp - k) % Nxp)];
        // X = (Z_k + conj Z_-k)/2 ; Y = (Z_k - conj Z_-k)/(2i)
        zd X = zmake(0.5 * (Zk.x + Zm.x), 0.5 * (Zk.y - Zm.y));
        zd Y = zmake(0.5 * (Zk.y + Zm.y), 0.5 * (Zm.x - Zk.x));
        if (slot == 0) {
            p.zp0[rowA + k] = X;
            p.zp1[rowA + k] = Y;
        } else if (slot == 1) {
            if (hasB) {
                p.zp0[rowB + k] = X;
                p.zp1[rowB + k] = Y;
            }
        } else {
            p.zp2[rowA + k] = X;
            if (hasB) p.zp2[rowB + k] = Y;
        }
    }
}
