// cf_fftkernels.cuh -- periodic-direction transforms of the rotational
// nonlinear term (src/ffts.jl:189-206 and 275-290, src/nonlinear.jl:184-191).
//
// k_zinv : nodal (Ny,Nz,Nxh) -> z-padded spectrum (copy_to_padded!, Nyquist
//          filter) -> backward z FFT of length Nzp   (Ny,Nzp,Nxh)
// k_xpass: backward x c2r of the six rows (pairs packed as one complex FFT),
//          n = u x omega at the padded points, forward x r2c, x truncation
// k_zfwd : forward z FFT of the three products, z truncation (copy_from_padded!)
#pragma once
#include "cf_fft.cuh"

#define CF_BLOCK_FFT_MAXE 24

struct FftParams {
    int Nx, Nz, Nxh, Ny, Nzp, Nxp;
    int tkz;          // columns per block in the z kernels
    zd* nod[6];       // nodal fields
    zd* zp[6];        // z-padded fields
    FftPlan plZ, plX;
};

CF_DEV int zpad_index(int iz, int Nz, int Nzp) { return iz <= (Nz >> 1) ? iz : Nzp - (Nz - iz); }

// grid: (ceil(Nxh/tkz), Ny, nfields); block 256; smem tkz*Nzp complex
__global__ void __launch_bounds__(256) k_zinv(FftParams p) {
    extern __shared__ zd sm[];
    const int f = blockIdx.z, n = blockIdx.y, k0 = blockIdx.x * p.tkz;
    const int tkz = p.tkz, Nz = p.Nz, Nzp = p.Nzp, Nxh = p.Nxh;
    const zd* src = p.nod[f] + (long)n * Nz * Nxh;
    zd* dst = p.zp[f] + (long)n * Nzp * Nxh;
    // zero the padding gap
    const int gap0 = (Nz >> 1) + 1, gap1 = Nzp - (Nz - gap0);
    for (int e = threadIdx.x; e < tkz * (gap1 - gap0); e += blockDim.x) {
        int t = e % tkz, z = gap0 + e / tkz;
        sm[t * Nzp + z] = zzero();
    }
    for (int e = threadIdx.x; e < tkz * Nz; e += blockDim.x) {
        int t = e % tkz, iz = e / tkz;
        int k = k0 + t;
        zd v = zzero();
        bool nyq = ((p.Nz % 2 == 0) && iz == Nz / 2) || ((p.Nx % 2 == 0) && k == p.Nx / 2);
        if (k < Nxh && !nyq) v = src[(long)iz * Nxh + k];
        sm[t * Nzp + zpad_index(iz, Nz, Nzp)] = v;
    }
    __syncthreads();
    group_fft<true, CF_BLOCK_FFT_MAXE>(sm, tkz, Nzp, p.plZ, +1, threadIdx.x, blockDim.x);
    for (int e = threadIdx.x; e < tkz * Nzp; e += blockDim.x) {
        int t = e % tkz, z = e / tkz;
        int k = k0 + t;
        if (k < Nxh) dst[(long)z * Nxh + k] = sm[t * Nzp + z];
    }
}

// grid: (ceil(Nxh/tkz), Ny, 3); forward z FFT and truncation to Nz
__global__ void __launch_bounds__(256) k_zfwd(FftParams p) {
    extern __shared__ zd sm[];
    const int f = blockIdx.z, n = blockIdx.y, k0 = blockIdx.x * p.tkz;
    const int tkz = p.tkz, Nz = p.Nz, Nzp = p.Nzp, Nxh = p.Nxh;
    const zd* src = p.zp[f] + (long)n * Nzp * Nxh;
    zd* dst = p.nod[f] + (long)n * Nz * Nxh;
    for (int e = threadIdx.x; e < tkz * Nzp; e += blockDim.x) {
        int t = e % tkz, z = e / tkz;
        int k = k0 + t;
        sm[t * Nzp + z] = (k < Nxh) ? src[(long)z * Nxh + k] : zzero();
    }
    __syncthreads();
    group_fft<true, CF_BLOCK_FFT_MAXE>(sm, tkz, Nzp, p.plZ, -1, threadIdx.x, blockDim.x);
    for (int e = threadIdx.x; e < tkz * Nz; e += blockDim.x) {
        int t = e % tkz, iz = e / tkz;
        int k = k0 + t;
        if (k < Nxh) dst[(long)iz * Nxh + k] = sm[t * Nzp + zpad_index(iz, Nz, Nzp)];
    }
}

// grid: (ceil(Nzp/2), Ny); block 256; smem 6*Nxp complex.  Rows zA = 2*bx and
// zB = 2*bx+1 of plane n.  Slots 0..5 hold (u0+iu1, u2+iw0, w1+iw2) of row A
// at 0,2,4 and of row B at 1,3,5.
__global__ void __launch_bounds__(256) k_xpass(FftParams p) {
    extern __shared__ zd sm[];
    const int n = blockIdx.y;
    const int zA = 2 * blockIdx.x, zB = zA + 1;
    const bool hasB = zB < p.Nzp;
    const int Nxp = p.Nxp, Nxh = p.Nxh;
    const int Nxhp = Nxp / 2 + 1;
    const long rowA = ((long)n * p.Nzp + zA) * Nxh;
    const long rowB = ((long)n * p.Nzp + zB) * Nxh;
    const int xnyq = (p.Nx % 2 == 0) ? p.Nx / 2 : -1;
    // pack Hermitian pairs: Z_k = X_k + i Y_k, Z_{Nxp-k} = conj(X_k) + i conj(Y_k)
    for (int e = threadIdx.x; e < 6 * Nxp; e += blockDim.x) sm[e] = zzero();
    __syncthreads();
    for (int e = threadIdx.x; e < 6 * Nxhp; e += blockDim.x) {
        const int slot = e / Nxhp, k = e - slot * Nxhp;
        const int pair = slot >> 1;
        const bool isB = slot & 1;
        if (isB && !hasB) continue;
        const long row = isB ? rowB : rowA;
        zd X = zzero(), Y = zzero();
        if (k < Nxh && k != xnyq) {
            X = p.zp[2 * pair][row + k];
            Y = p.zp[2 * pair + 1][row + k];
        }
        zd* s = sm + slot * Nxp;
        if (k == 0) {
            s[0] = zmake(X.x, Y.x);
        } else if (2 * k == Nxp) {
            s[k] = zmake(X.x, Y.x);
        } else {
            s[k] = zmake(X.x - Y.y, X.y + Y.x);
            s[Nxp - k] = zmake(X.x + Y.y, Y.x - X.y);
        }
    }
    __syncthreads();
    group_fft<true, CF_BLOCK_FFT_MAXE>(sm, 6, Nxp, p.plX, +1, threadIdx.x, blockDim.x);
    // rotational product n = u x omega at every padded x point of both rows
    for (int j = threadIdx.x; j < Nxp; j += blockDim.x) {
        zd a0 = sm[0 * Nxp + j], a1 = sm[2 * Nxp + j], a2 = sm[4 * Nxp + j];
        zd b0 = sm[1 * Nxp + j], b1 = sm[3 * Nxp + j], b2 = sm[5 * Nxp + j];
        // row A: u=(a0.x,a0.y,a1.x), w=(a1.y,a2.x,a2.y)
        double nA0 = a0.y * a2.y - a1.x * a2.x;
        double nA1 = a1.x * a1.y - a0.x * a2.y;
        double nA2 = a0.x * a2.x - a0.y * a1.y;
        double nB0 = b0.y * b2.y - b1.x * b2.x;
        double nB1 = b1.x * b1.y - b0.x * b2.y;
        double nB2 = b0.x * b2.x - b0.y * b1.y;
        sm[0 * Nxp + j] = zmake(nA0, nA1);
        sm[1 * Nxp + j] = zmake(nB0, nB1);
        sm[2 * Nxp + j] = zmake(nA2, nB2);
    }
    __syncthreads();
    group_fft<true, CF_BLOCK_FFT_MAXE>(sm, 3, Nxp, p.plX, -1, threadIdx.x, blockDim.x);
    // separate the packed real transforms and keep k < Nxh
    for (int e = threadIdx.x; e < 3 * Nxh; e += blockDim.x) {
        const int slot = e / Nxh, k = e - slot * Nxh;
        const zd* s = sm + slot * Nxp;
        zd Zk = s[k], Zm = s[(Nxp - k) % Nxp];
        // X = (Z_k + conj Z_-k)/2 ; Y = (Z_k - conj Z_-k)/(2i)
        zd X = zmake(0.5 * (Zk.x + Zm.x), 0.5 * (Zk.y - Zm.y));
        zd Y = zmake(0.5 * (Zk.y + Zm.y), 0.5 * (Zm.x - Zk.x));
        if (slot == 0) {
            p.zp[0][rowA + k] = X;
            p.zp[1][rowA + k] = Y;
        } else if (slot == 1) {
            if (hasB) {
                p.zp[0][rowB + k] = X;
                p.zp[1][rowB + k] = Y;
            }
        } else {
            p.zp[2][rowA + k] = X;
            if (hasB) p.zp[2][rowB + k] = Y;
        }
    }
}
