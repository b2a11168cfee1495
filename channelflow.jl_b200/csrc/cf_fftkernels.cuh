// cf_fftkernels.cuh -- periodic-direction transforms of the rotational
// nonlinear term (src/ffts.jl:189-206 and 275-290, src/nonlinear.jl:184-191).
//
// k_zinv : nodal (Ny,Nz,Nxh) -> z-padded spectrum (copy_to_padded!, Nyquist
//          filter) -> backward z FFT of length Nzp   (Ny,Nzp,Nxh)
// k_xpass: backward x c2r of the six rows (pairs packed as one complex FFT),
//          n = u x omega at the padded points, forward x r2c, x truncation
// k_zfwd : forward z FFT of the three products, z truncation (copy_from_padded!)
// Shared-memory transform buffers use the padded positions (fpos) of cf_fft.cuh.
#pragma once
#include "cf_fft.cuh"

struct FftParams {
    int Nx, Nz, Nxh, Ny, Nzp, Nxp;
    int tks;       // log2 of the columns per block in the z kernels
    int bsz, bsx;  // transform buffer strides: fft_bufsz(Nzp) + 1 (odd, padded layout),
                   // round_up(Nxp, 8) (XOR-swizzled layout: 12 buffers of the x-pass)
    // nodal and z-padded fields: complex double (FP64 path) or complex float
    // (FP32 transforms of the mixed-precision path)
    void *nod0, *nod1, *nod2, *nod3, *nod4, *nod5;
    void *zp0, *zp1, *zp2, *zp3, *zp4, *zp5;
    FftPlan plZ, plX;
};

CF_DEV void* sel6(void* a0, void* a1, void* a2, void* a3, void* a4, void* a5, int i) {
    switch (i) {
        case 0: return a0;
        case 1: return a1;
        case 2: return a2;
        case 3: return a3;
        case 4: return a4;
        default: return a5;
    }
}
template <class Z>
CF_DEV Z* nod_of(const FftParams& p, int i) {
    return static_cast<Z*>(sel6(p.nod0, p.nod1, p.nod2, p.nod3, p.nod4, p.nod5, i));
}
template <class Z>
CF_DEV Z* zp_of(const FftParams& p, int i) {
    return static_cast<Z*>(sel6(p.zp0, p.zp1, p.zp2, p.zp3, p.zp4, p.zp5, i));
}

CF_DEV int zpad_index(int iz, int Nz, int Nzp) { return iz <= (Nz >> 1) ? iz : Nzp - (Nz - iz); }

// grid: (ceil(Nxh/tkz), Ny, nfields); block 256; smem 2*tkz*bsz complex.
// Column t of the block's tkz columns is transform t (stride bsz, odd, so the
// column-interleaved staging stores hit distinct bank groups).
template <int LZ, class Z>
CF_DEV void zinv_body(const FftParams& p, int bx, int n, int f) {
    extern __shared__ __align__(16) unsigned char fsm_raw[];
    Z* sm = reinterpret_cast<Z*>(fsm_raw);
    const int tks = p.tks, tkz = 1 << tks, tm = tkz - 1;
    const int k0 = bx << tks;
    const int Nz = p.Nz, Nzp = LZ ? LZ : p.Nzp, Nxh = p.Nxh, bs = p.bsz;
    Z* bufB = sm + tkz * bs;
    const Z* src = nod_of<Z>(p, f) + (long)n * Nz * Nxh;
    Z* dst = zp_of<Z>(p, f) + (long)n * Nzp * Nxh;
    const int xnyq = (p.Nx % 2 == 0) ? p.Nx / 2 : -1, znyq = (Nz % 2 == 0) ? Nz / 2 : -1;
    // zero the padding gap
    const int gap0 = (Nz >> 1) + 1, gap1 = Nzp - (Nz - gap0);
    for (int e = threadIdx.x; e < ((gap1 - gap0) << tks); e += blockDim.x)
        sm[(e & tm) * bs + fpos(gap0 + (e >> tks))] = czero<Z>();
    // loads batched 8 per thread before their stores (requests in flight)
    const int ntot = Nz << tks;
    for (int base = threadIdx.x; base < ntot; base += 8 * 256) {
        Z v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = base + u * 256;
            const int iz = e >> tks, k = k0 + (e & tm);
            v[u] = (e < ntot && k < Nxh && iz != znyq && k != xnyq) ? src[(long)iz * Nxh + k] : czero<Z>();
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = base + u * 256;
            if (e < ntot) sm[(e & tm) * bs + fpos(zpad_index(e >> tks, Nz, Nzp))] = v[u];
        }
    }
    __syncthreads();
    const Z* res = group_fft_L<true, LZ>(sm, bufB, tkz, bs, p.plZ, +1, threadIdx.x, blockDim.x, 0);
    for (int e = threadIdx.x; e < (Nzp << tks); e += blockDim.x) {
        const int t = e & tm, z = e >> tks, k = k0 + t;
        if (k < Nxh) dst[(long)z * Nxh + k] = res[t * bs + fpos(z)];
    }
}

// grid: (ceil(Nxh/tkz), Ny, 3); forward z FFT and truncation to Nz
template <int LZ, class Z>
CF_DEV void zfwd_body(const FftParams& p, int bx, int n, int f) {
    extern __shared__ __align__(16) unsigned char fsm_raw[];
    Z* sm = reinterpret_cast<Z*>(fsm_raw);
    const int tks = p.tks, tkz = 1 << tks, tm = tkz - 1;
    const int k0 = bx << tks;
    const int Nz = p.Nz, Nzp = LZ ? LZ : p.Nzp, Nxh = p.Nxh, bs = p.bsz;
    Z* bufB = sm + tkz * bs;
    const Z* src = zp_of<Z>(p, f) + (long)n * Nzp * Nxh;
    Z* dst = nod_of<Z>(p, f) + (long)n * Nz * Nxh;
    const int ntot = Nzp << tks;
    for (int base = threadIdx.x; base < ntot; base += 8 * 256) {
        Z v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = base + u * 256;
            const int k = k0 + (e & tm);
            v[u] = (e < ntot && k < Nxh) ? src[(long)(e >> tks) * Nxh + k] : czero<Z>();
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = base + u * 256;
            if (e < ntot) sm[(e & tm) * bs + fpos(e >> tks)] = v[u];
        }
    }
    __syncthreads();
    const Z* res = group_fft_L<true, LZ>(sm, bufB, tkz, bs, p.plZ, -1, threadIdx.x, blockDim.x, 0);
    for (int e = threadIdx.x; e < (Nz << tks); e += blockDim.x) {
        const int t = e & tm, iz = e >> tks, k = k0 + t;
        if (k < Nxh) dst[(long)iz * Nxh + k] = res[t * bs + fpos(zpad_index(iz, Nz, Nzp))];
    }
}

// grid: (ceil(Nzp/2), Ny); block 256; smem 12*bsx complex (6 slots + scratch).
// Rows zA = 2*bx and zB = 2*bx+1 of plane n.  Slots 0..5 hold
// (u0+iu1, u2+iw0, w1+iw2) of row A at 0,2,4 and of row B at 1,3,5.
template <int LX, class Z>
CF_DEV void xpass_body(const FftParams& p, int bx, int n) {
    extern __shared__ __align__(16) unsigned char fsm_raw[];
    Z* sm = reinterpret_cast<Z*>(fsm_raw);
    const int zA = 2 * bx, zB = zA + 1;
    const bool hasB = zB < p.Nzp;
    const int Nxp = LX ? LX : p.Nxp, Nxh = p.Nxh, bs = p.bsx;
    const int Nxhp = Nxp / 2 + 1;
    const long rowA = ((long)n * p.Nzp + zA) * Nxh;
    const long rowB = ((long)n * p.Nzp + zB) * Nxh;
    const int xnyq = (p.Nx % 2 == 0) ? p.Nx / 2 : -1;
    Z* scr = sm + 6 * bs;
    // pack Hermitian pairs: Z_k = X_k + i Y_k, Z_{Nxp-k} = conj(X_k) + i conj(Y_k);
    // every position 0..Nxp-1 of the six slots is written (zeros for a missing
    // row B and for k >= Nxh)
    for (int base = threadIdx.x; base < 6 * Nxhp; base += 4 * 256) {
        Z X[4], Y[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = base + u * 256;
            const int slot = e / Nxhp, k = e - slot * Nxhp;
            const int pair = slot >> 1;
            const bool isB = slot & 1;
            const long row = isB ? rowB : rowA;
            X[u] = czero<Z>();
            Y[u] = czero<Z>();
            if (e < 6 * Nxhp && !(isB && !hasB) && k < Nxh && k != xnyq) {
                X[u] = zp_of<Z>(p, 2 * pair)[row + k];
                Y[u] = zp_of<Z>(p, 2 * pair + 1)[row + k];
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = base + u * 256;
            if (e >= 6 * Nxhp) continue;
            const int slot = e / Nxhp, k = e - slot * Nxhp;
            Z* s = sm + slot * bs;
            if (k == 0) {
                s[swz(0)] = cmake<Z>(X[u].x, Y[u].x);
            } else if (2 * k == Nxp) {
                s[swz(k)] = cmake<Z>(X[u].x, Y[u].x);
            } else {
                s[swz(k)] = cmake<Z>(X[u].x - Y[u].y, X[u].y + Y[u].x);
                s[swz(Nxp - k)] = cmake<Z>(X[u].x + Y[u].y, Y[u].x - X[u].y);
            }
        }
    }
    __syncthreads();
    Z* A = group_fft_L<true, LX, 1>(sm, scr, 6, bs, p.plX, +1, threadIdx.x, blockDim.x, 0);
    Z* Bf = (A == sm) ? scr : sm;
    // rotational product n = u x omega at every padded x point of both rows
    for (int j = threadIdx.x; j < Nxp; j += blockDim.x) {
        const int sj = swz(j);
        Z a0 = A[0 * bs + sj], a1 = A[2 * bs + sj], a2 = A[4 * bs + sj];
        Z b0 = A[1 * bs + sj], b1 = A[3 * bs + sj], b2 = A[5 * bs + sj];
        // row A: u=(a0.x,a0.y,a1.x), w=(a1.y,a2.x,a2.y)
        double nA0 = a0.y * a2.y - a1.x * a2.x;
        double nA1 = a1.x * a1.y - a0.x * a2.y;
        double nA2 = a0.x * a2.x - a0.y * a1.y;
        double nB0 = b0.y * b2.y - b1.x * b2.x;
        double nB1 = b1.x * b1.y - b0.x * b2.y;
        double nB2 = b0.x * b2.x - b0.y * b1.y;
        Bf[0 * bs + sj] = cmake<Z>(nA0, nA1);
        Bf[1 * bs + sj] = cmake<Z>(nB0, nB1);
        Bf[2 * bs + sj] = cmake<Z>(nA2, nB2);
    }
    __syncthreads();
    const Z* F = group_fft_L<true, LX, 1>(Bf, A, 3, bs, p.plX, -1, threadIdx.x, blockDim.x, 0);
    // separate the packed real transforms and keep k < Nxh
    for (int e = threadIdx.x; e < 3 * Nxh; e += blockDim.x) {
        const int slot = e / Nxh, k = e - slot * Nxh;
        const Z* s = F + slot * bs;
        Z Zk = s[swz(k)], Zm = s[swz((Nxp - k) % Nxp)];
        // X = (Z_k + conj Z_-k)/2 ; Y = (Z_k - conj Z_-k)/(2i)
        Z X = cmake<Z>(0.5 * (Zk.x + Zm.x), 0.5 * (Zk.y - Zm.y));
        Z Y = cmake<Z>(0.5 * (Zk.y + Zm.y), 0.5 * (Zm.x - Zk.x));
        if (slot == 0) {
            zp_of<Z>(p, 0)[rowA + k] = X;
            zp_of<Z>(p, 1)[rowA + k] = Y;
        } else if (slot == 1) {
            if (hasB) {
                zp_of<Z>(p, 0)[rowB + k] = X;
                zp_of<Z>(p, 1)[rowB + k] = Y;
            }
        } else {
            zp_of<Z>(p, 2)[rowA + k] = X;
            if (hasB) zp_of<Z>(p, 2)[rowB + k] = Y;
        }
    }
}

// Single-instance kernels and their batched forms (one launch per size class;
// blockIdx.z also selects the instance).
template <int LZ, class Z = zd>
__global__ void __launch_bounds__(256) k_zinv(FftParams p) {
    zinv_body<LZ, Z>(p, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <int LZ, class Z = zd>
__global__ void __launch_bounds__(256) k_zfwd(FftParams p) {
    zfwd_body<LZ, Z>(p, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <int LX, class Z = zd>
__global__ void __launch_bounds__(256) k_xpass(FftParams p) {
    xpass_body<LX, Z>(p, blockIdx.x, blockIdx.y);
}
// grid z = 6 * instances
template <int LZ>
__global__ void __launch_bounds__(256) k_zinv_batch(const FftParams* __restrict__ pl) {
    __shared__ FftParams ps;
    const int inst = blockIdx.z / 6;
    stage_params(&ps, pl + inst);
    zinv_body<LZ, zd>(ps, blockIdx.x, blockIdx.y, blockIdx.z - 6 * inst);
}
// grid z = 3 * instances
template <int LZ>
__global__ void __launch_bounds__(256) k_zfwd_batch(const FftParams* __restrict__ pl) {
    __shared__ FftParams ps;
    const int inst = blockIdx.z / 3;
    stage_params(&ps, pl + inst);
    zfwd_body<LZ, zd>(ps, blockIdx.x, blockIdx.y, blockIdx.z - 3 * inst);
}
// grid z = instances
template <int LX>
__global__ void __launch_bounds__(256) k_xpass_batch(const FftParams* __restrict__ pl) {
    __shared__ FftParams ps;
    stage_params(&ps, pl + blockIdx.z);
    xpass_body<LX, zd>(ps, blockIdx.x, blockIdx.y);
}
