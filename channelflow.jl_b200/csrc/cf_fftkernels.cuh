// cf_fftkernels.cuh -- periodic-direction transforms of the nonlinear term
// (src/ffts.jl:65-82, 151-166, 242-312; src/nonlinear.jl:113-199).
//
// k_zinv : nodal (Ny,Nz,Nxh) -> z-padded spectrum (copy_to_padded!, Nyquist
//          filter) -> backward z FFT of length Nzp   (Ny,Nzp,Nxh)
// k_xpass: backward x c2r of the rows (pairs packed as one complex FFT), the
//          product of the nonlinear form at the padded points, forward x r2c,
//          x truncation
// k_zfwd : forward z FFT of the products, z truncation (copy_from_padded!)
// Shared-memory transform buffers use the padded positions (fpos) of cf_fft.cuh.
//
// Fields per form (NlForm):
//   rotational  nodal u, omega (6) -> z-padded 0-5 -> n = u x omega (3)
//   convective  nodal u, du/dy (6) -> z-padded 0-5 and du/dz (6-8, made by
//               k_zinv) -> n = -(u.grad)u (3; du/dx made by k_xpass)
//   divergence  nodal u (3) -> z-padded 0-2 -> -u_i u_j (6: 00 01 02 11 12 22)
#pragma once
#include <cuda.h>  // CUtensorMap

#include "cf_fft.cuh"

// blocks per SM of the in-place x-pass (bounds its registers), and the x
// positions per thread of its row loads: one (measured at 384x257x384: 2.21
// ms, against 2.28 with two positions, whose loads in flight spill at this
// register bound, and 2.27 at five blocks per SM)
#ifndef CF_XPASS_IP_BLOCKS
#define CF_XPASS_IP_BLOCKS 4
#endif
#ifndef CF_XPASS_IP_KPT
#define CF_XPASS_IP_KPT 1
#endif
#ifndef CF_XPASS_IP32_BLOCKS
#define CF_XPASS_IP32_BLOCKS 5
#endif


struct FftParams {
    int Nx, Nz, Nxh, Ny, Nzp, Nxp;
    int tks;       // log2 of the columns per block in the z kernels
    int bsz, bsx;  // transform buffer strides: fft_bufsz(Nzp) + 1 (odd, padded layout),
                   // round_up(Nxp, 8) (XOR-swizzled layout: 12 buffers of the x-pass)
    int bsxp;      // fft_bufsz(Nxp): padded layout of the one-row FP64 x-pass
    int zbox, zpbox;  // TMA z kernels: rows per box of the nodal (Nz) and z-padded (Nzp) fields
    int stoff;     // TMA z kernels: byte offset of the staging buffer in shared memory
    int* err;      // TMA z kernels: set to 1 when a wait gives up
    long spins;    // TMA z kernels: polls of the first wait for a tile (CF_WAIT_SPINS; shortened only by tests)
    double ax, bz;  // 2 pi / Lx, 2 pi / Lz (derivatives of the convective form)
    // nodal and z-padded fields: complex double (FP64 path) or complex float
    // (FP32 transforms of the mixed-precision path)
    void *nod0, *nod1, *nod2, *nod3, *nod4, *nod5;
    void *zp0, *zp1, *zp2, *zp3, *zp4, *zp5, *zp6, *zp7, *zp8;
    FftPlan plZ, plX;
};

// field i of the parameter block without indexing an array at run time
template <class Z>
CF_DEV Z* nod_of(const FftParams& p, int i) {
    void* a;
    switch (i) {
        case 0: a = p.nod0; break;
        case 1: a = p.nod1; break;
        case 2: a = p.nod2; break;
        case 3: a = p.nod3; break;
        case 4: a = p.nod4; break;
        default: a = p.nod5; break;
    }
    return static_cast<Z*>(a);
}
template <class Z>
CF_DEV Z* zp_of(const FftParams& p, int i) {
    void* a;
    switch (i) {
        case 0: a = p.zp0; break;
        case 1: a = p.zp1; break;
        case 2: a = p.zp2; break;
        case 3: a = p.zp3; break;
        case 4: a = p.zp4; break;
        case 5: a = p.zp5; break;
        case 6: a = p.zp6; break;
        case 7: a = p.zp7; break;
        default: a = p.zp8; break;
    }
    return static_cast<Z*>(a);
}

// TMA maps of the z kernels' fields, over the scalars of the complex type:
// nodal (2 Nxh, Nz, Ny) with box (2 tkz, zbox, 1), z-padded (2 Nxh, Nzp, Ny)
// with box (2 tkz, zpbox, 1).
struct FftMaps {
    CUtensorMap nod[6];
    CUtensorMap zp[9];
};

// i s a
template <class Z>
CF_DEV Z cmuli(Z a, double s) {
    return cmake<Z>(-s * a.y, s * a.x);
}

CF_DEV int zpad_index(int iz, int Nz, int Nzp) { return iz <= (Nz >> 1) ? iz : Nzp - (Nz - iz); }

// grid: (ceil(Nxh/tkz), Ny, nfields); block 256; smem 2*tkz*bsz complex.
// Column t of the block's tkz columns is transform t (stride bsz, chosen by
// the host so that the column-interleaved stores hit distinct bank groups).  Fields 6-8
// (convective form) are d/dz of nodal fields 0-2: i bz l times the nodal
// values (ddx3!, operators.jl:14-23, applied after the Chebyshev transform,
// with which it commutes).
template <int LZ, class Z>
CF_DEV void zinv_body(const FftParams& p, int bx, int n, int f) {
    extern __shared__ __align__(128) unsigned char fsm_raw[];
    Z* sm = reinterpret_cast<Z*>(fsm_raw);
    const int tks = p.tks, tkz = 1 << tks, tm = tkz - 1;
    const int k0 = bx << tks;
    const int Nz = p.Nz, Nzp = LZ ? LZ : p.Nzp, Nxh = p.Nxh, bs = p.bsz;
    Z* bufB = sm + tkz * bs;
    const bool dz = f >= 6;
    const Z* src = nod_of<Z>(p, dz ? f - 6 : f) + (long)n * Nz * Nxh;
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
            if (dz) v[u] = cmuli(v[u], p.bz * (double)(iz <= (Nz >> 1) ? iz : iz - Nz));
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

// The z kernels with their strided row gathers and scatters done by TMA:
// tkz columns x all rows of one plane move as boxes of (2 tkz scalars, zbox
// rows) between the global fields and a dense staging layout in shared memory
// (stage[row * tkz + t]), so the strided 32-byte row segments cost no L1
// wavefronts.  Rows past the end of a box load as zeros and are not stored.
// smem: two transform buffers of tkz*bsz elements, the second at byte p.stoff
// (128-aligned), which also stages the rows: the loaded rows are unpacked from
// it before the transform uses it, and the result is packed for the store into
// whichever buffer the last pass did not write (no third buffer, so four
// blocks fit per SM at Nzp = 576 in FP64).  One thread issues the copies;
// every wait is bounded (p.err set, the block returns).
template <class Z>
CF_DEV Z* zstage(const FftParams& p) {
    extern __shared__ __align__(128) unsigned char fsm_raw[];
    return reinterpret_cast<Z*>(fsm_raw + p.stoff);
}
template <class Z>
CF_DEV bool zload_tma(const FftParams& p, const CUtensorMap* map, int k0, int rows, int box, int n, Z* stage,
                      uint64_t* mbar) {
    const uint32_t mb = smem_u32(mbar);
    const int tkz = 1 << p.tks, nb = (rows + box - 1) / box;
    if (threadIdx.x == 0) {
        mbar_init(mb, 1);
        fence_mbar_init();
        mbar_expect_tx(mb, (uint32_t)(nb * box * tkz * sizeof(Z)));
        for (int b = 0; b < nb; ++b) tma_load_3d(stage + (long)b * box * tkz, map, 2 * k0, b * box, n, mb);
    }
    __syncthreads();
    const bool ok = __syncthreads_and(mbar_wait(mb, 0, p.spins));
    if (!ok) {
        // the boxes still in flight land before the block gives up its shared memory
        mbar_wait(mb, 0);
        __syncthreads();
        if (threadIdx.x == 0) atomicExch(p.err, 1);
    }
    return ok;
}
template <class Z>
CF_DEV void zstore_tma(const FftParams& p, const CUtensorMap* map, int k0, int rows, int box, int n,
                       const Z* stage) {
    fence_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
        const int tkz = 1 << p.tks;
        for (int b = 0; b * box < rows; ++b) tma_store_3d(map, 2 * k0, b * box, n, stage + (long)b * box * tkz);
        bulk_commit();
        bulk_wait_read();
    }
}

template <int LZ, class Z>
CF_DEV void zinv_tma_body(const FftParams& p, const FftMaps& m, int bx, int n, int f) {
    extern __shared__ __align__(128) unsigned char fsm_raw[];
    __shared__ __align__(8) uint64_t mbar;
    Z* sm = reinterpret_cast<Z*>(fsm_raw);
    Z* const bufB = zstage<Z>(p);
    const int tks = p.tks, tkz = 1 << tks, tm = tkz - 1;
    const int k0 = bx << tks;
    const int Nz = p.Nz, Nzp = LZ ? LZ : p.Nzp, Nxh = p.Nxh, bs = p.bsz;
    const bool dz = f >= 6;
    const int xnyq = (p.Nx % 2 == 0) ? p.Nx / 2 : -1, znyq = (Nz % 2 == 0) ? Nz / 2 : -1;
    // zero the padding gap while the rows arrive
    const int gap0 = (Nz >> 1) + 1, gap1 = Nzp - (Nz - gap0);
    for (int e = threadIdx.x; e < ((gap1 - gap0) << tks); e += blockDim.x)
        sm[(e & tm) * bs + fpos(gap0 + (e >> tks))] = czero<Z>();
    if (!zload_tma<Z>(p, &m.nod[dz ? f - 6 : f], k0, Nz, p.zbox, n, bufB, &mbar)) return;
    for (int e = threadIdx.x; e < (Nz << tks); e += blockDim.x) {
        const int iz = e >> tks, k = k0 + (e & tm);
        Z v = (k < Nxh && iz != znyq && k != xnyq) ? bufB[e] : czero<Z>();
        if (dz) v = cmuli(v, p.bz * (double)(iz <= (Nz >> 1) ? iz : iz - Nz));
        sm[(e & tm) * bs + fpos(zpad_index(iz, Nz, Nzp))] = v;
    }
    __syncthreads();
    const Z* res = group_fft_L<true, LZ>(sm, bufB, tkz, bs, p.plZ, +1, threadIdx.x, blockDim.x, 0);
    Z* stage = (res == sm) ? bufB : sm;
    for (int e = threadIdx.x; e < (Nzp << tks); e += blockDim.x) stage[e] = res[(e & tm) * bs + fpos(e >> tks)];
    zstore_tma<Z>(p, &m.zp[f], k0, Nzp, p.zpbox, n, stage);
}

template <int LZ, class Z>
CF_DEV void zfwd_tma_body(const FftParams& p, const FftMaps& m, int bx, int n, int f) {
    extern __shared__ __align__(128) unsigned char fsm_raw[];
    __shared__ __align__(8) uint64_t mbar;
    Z* sm = reinterpret_cast<Z*>(fsm_raw);
    Z* const bufB = zstage<Z>(p);
    const int tks = p.tks, tkz = 1 << tks, tm = tkz - 1;
    const int k0 = bx << tks;
    const int Nz = p.Nz, Nzp = LZ ? LZ : p.Nzp, bs = p.bsz;
    if (!zload_tma<Z>(p, &m.zp[f], k0, Nzp, p.zpbox, n, bufB, &mbar)) return;
    for (int e = threadIdx.x; e < (Nzp << tks); e += blockDim.x) sm[(e & tm) * bs + fpos(e >> tks)] = bufB[e];
    __syncthreads();
    const Z* res = group_fft_L<true, LZ>(sm, bufB, tkz, bs, p.plZ, -1, threadIdx.x, blockDim.x, 0);
    Z* stage = (res == sm) ? bufB : sm;
    for (int e = threadIdx.x; e < (Nz << tks); e += blockDim.x)
        stage[e] = res[(e & tm) * bs + fpos(zpad_index(e >> tks, Nz, Nzp))];
    zstore_tma<Z>(p, &m.nod[f], k0, Nz, p.zbox, n, stage);
}

// grid: (ceil(Nxh/tkz), Ny, 3); forward z FFT and truncation to Nz
template <int LZ, class Z>
CF_DEV void zfwd_body(const FftParams& p, int bx, int n, int f) {
    extern __shared__ __align__(128) unsigned char fsm_raw[];
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

// Pack NS transform slots from pairs of real rows given by their half
// spectra X, Y (get(slot, k, X, Y) for k < Nxh, Nyquist excluded; zero
// elsewhere): Z_k = X_k + i Y_k, Z_{Nxp-k} = conj(X_k) + i conj(Y_k).  Every
// position 0..Nxp-1 of the slots is written.  The slot loop is unrolled, so
// get() sees a constant slot (its source pointer is selected at compile
// time); each thread issues the loads of all slots (KPT positions each)
// before its first store.  POS: the slots' layout (cf_fft.cuh bpos: 0 padded,
// 1 XOR-swizzled).
// FLAT: the (slot, position) pairs spread over all threads instead, with the
// slot known at run time (more threads busy when rows are short).
template <class Z, int POS, int NS, bool FLAT, int KP = 0, class Get>
CF_DEV void xpack(Z* sm, int bs, int Nxh, int Nxp, int xnyq, const Get& get) {
    if constexpr (FLAT) {
        const int Nxhp = Nxp / 2 + 1, tot = NS * Nxhp, NT = blockDim.x;
        for (int base = threadIdx.x; base < tot; base += 4 * NT) {
            Z X[4], Y[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int e = base + u * NT;
                const int slot = e / Nxhp, k = e - slot * Nxhp;
                X[u] = czero<Z>();
                Y[u] = czero<Z>();
                if (e < tot && k < Nxh && k != xnyq) get(slot, k, X[u], Y[u]);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int e = base + u * NT;
                if (e >= tot) continue;
                const int slot = e / Nxhp, k = e - slot * Nxhp;
                Z* o = sm + slot * bs;
                if (k == 0 || 2 * k == Nxp) {
                    o[bpos<POS>(k)] = cmake<Z>(X[u].x, Y[u].x);
                } else {
                    o[bpos<POS>(k)] = cmake<Z>(X[u].x - Y[u].y, X[u].y + Y[u].x);
                    o[bpos<POS>(Nxp - k)] = cmake<Z>(X[u].x + Y[u].y, Y[u].x - X[u].y);
                }
            }
        }
    } else {
        constexpr int KPT = KP ? KP : (NS <= 3 ? 2 : 1);  // positions per thread (loads in flight)
        const int Nxhp = Nxp / 2 + 1, NT = blockDim.x;
        for (int k0 = threadIdx.x; k0 < Nxhp; k0 += KPT * NT) {
            Z X[NS][KPT], Y[NS][KPT];
#pragma unroll
            for (int s = 0; s < NS; ++s)
#pragma unroll
                for (int u = 0; u < KPT; ++u) {
                    const int k = k0 + u * NT;
                    X[s][u] = czero<Z>();
                    Y[s][u] = czero<Z>();
                    if (k < Nxh && k != xnyq) get(s, k, X[s][u], Y[s][u]);
                }
#pragma unroll
            for (int s = 0; s < NS; ++s)
#pragma unroll
                for (int u = 0; u < KPT; ++u) {
                    const int k = k0 + u * NT;
                    if (k >= Nxhp) continue;
                    Z* o = sm + s * bs;
                    const Z x = X[s][u], y = Y[s][u];
                    if (k == 0 || 2 * k == Nxp) {
                        o[bpos<POS>(k)] = cmake<Z>(x.x, y.x);
                    } else {
                        o[bpos<POS>(k)] = cmake<Z>(x.x - y.y, x.y + y.x);
                        o[bpos<POS>(Nxp - k)] = cmake<Z>(x.x + y.y, y.x - x.y);
                    }
                }
        }
    }
}

// Separate NS forward-transformed slots into the half spectra of their two
// real rows, X = (Z_k + conj Z_-k)/2, Y = (Z_k - conj Z_-k)/(2i), and hand
// them to put(slot, k, X, Y) for k < Nxh (the x truncation); constant slot
// per unrolled iteration.
template <class Z, int POS, int NS, bool FLAT, class Put>
CF_DEV void xunpack(const Z* F, int bs, int Nxh, int Nxp, const Put& put) {
    if constexpr (FLAT) {
        for (int e = threadIdx.x; e < NS * Nxh; e += blockDim.x) {
            const int slot = e / Nxh, k = e - slot * Nxh;
            const Z* o = F + slot * bs;
            const Z Zk = o[bpos<POS>(k)], Zm = o[bpos<POS>((Nxp - k) % Nxp)];
            put(slot, k, cmake<Z>(0.5 * (Zk.x + Zm.x), 0.5 * (Zk.y - Zm.y)),
                cmake<Z>(0.5 * (Zk.y + Zm.y), 0.5 * (Zm.x - Zk.x)));
        }
    } else {
        for (int k = threadIdx.x; k < Nxh; k += blockDim.x) {
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                const Z* o = F + s * bs;
                const Z Zk = o[bpos<POS>(k)], Zm = o[bpos<POS>((Nxp - k) % Nxp)];
                put(s, k, cmake<Z>(0.5 * (Zk.x + Zm.x), 0.5 * (Zk.y - Zm.y)),
                    cmake<Z>(0.5 * (Zk.y + Zm.y), 0.5 * (Zm.x - Zk.x)));
            }
        }
    }
}

// Rotational form, two rows per block (the FP32 transforms of the mixed
// form).  grid: (ceil(Nzp/2), Ny); block 256; smem 12*bsx complex (6 slots +
// scratch).  Rows zA = 2*bx and zB = 2*bx+1 of plane n.  Slots 0..5 hold
// (u0+iu1, u2+iw0, w1+iw2) of row A at 0,2,4 and of row B at 1,3,5.
template <int LX, class Z>
CF_DEV void xpass_body(const FftParams& p, int bx, int n) {
    extern __shared__ __align__(128) unsigned char fsm_raw[];
    Z* sm = reinterpret_cast<Z*>(fsm_raw);
    const int zA = 2 * bx, zB = zA + 1;
    const bool hasB = zB < p.Nzp;
    const int Nxp = LX ? LX : p.Nxp, Nxh = p.Nxh, bs = p.bsx;
    const long rowA = ((long)n * p.Nzp + zA) * Nxh;
    const long rowB = ((long)n * p.Nzp + zB) * Nxh;
    const int xnyq = (p.Nx % 2 == 0) ? p.Nx / 2 : -1;
    Z* scr = sm + 6 * bs;
    // zeros for a missing row B
    xpack<Z, 1, 6, true>(sm, bs, Nxh, Nxp, xnyq, [&](int slot, int k, Z& X, Z& Y) {
        const int pair = slot >> 1;
        const bool isB = slot & 1;
        if (isB && !hasB) return;
        const long row = isB ? rowB : rowA;
        X = zp_of<Z>(p, 2 * pair)[row + k];
        Y = zp_of<Z>(p, 2 * pair + 1)[row + k];
    });
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
    xunpack<Z, 1, 3, true>(F, bs, Nxh, Nxp, [&](int slot, int k, Z X, Z Y) {
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
    });
}

// Rotational form, one row per block (the FP64 path: half the shared memory
// of the two-row form, so more blocks per SM hide the FFT passes' latency, in
// the padded layout, whose strided butterfly positions are constant offsets).
// grid: (Nzp, Ny); block 256; smem 6*bsxp complex.  Slots 0..2 hold (u0+iu1,
// u2+iw0, w1+iw2) of row z = bx; the products leave in (n0+in1, n2).
template <int LX, class Z>
CF_DEV void xpass_row_body(const FftParams& p, int z, int n) {
    extern __shared__ __align__(128) unsigned char fsm_raw[];
    Z* sm = reinterpret_cast<Z*>(fsm_raw);
    const int Nxp = LX ? LX : p.Nxp, Nxh = p.Nxh, bs = p.bsxp;
    const long row = ((long)n * p.Nzp + z) * Nxh;
    const int xnyq = (p.Nx % 2 == 0) ? p.Nx / 2 : -1;
    Z* scr = sm + 3 * bs;
    xpack<Z, 0, 3, false>(sm, bs, Nxh, Nxp, xnyq, [&](int slot, int k, Z& X, Z& Y) {
        X = zp_of<Z>(p, 2 * slot)[row + k];
        Y = zp_of<Z>(p, 2 * slot + 1)[row + k];
    });
    __syncthreads();
    Z* A = group_fft_L<true, LX, 0>(sm, scr, 3, bs, p.plX, +1, threadIdx.x, blockDim.x, 0);
    Z* Bf = (A == sm) ? scr : sm;
    for (int j = threadIdx.x; j < Nxp; j += blockDim.x) {
        const int sj = fpos(j);
        const Z a0 = A[0 * bs + sj], a1 = A[1 * bs + sj], a2 = A[2 * bs + sj];
        // u = (a0.x, a0.y, a1.x), omega = (a1.y, a2.x, a2.y)
        Bf[0 * bs + sj] = cmake<Z>(a0.y * a2.y - a1.x * a2.x, a1.x * a1.y - a0.x * a2.y);
        Bf[1 * bs + sj] = cmake<Z>(a0.x * a2.x - a0.y * a1.y, 0.0);
    }
    __syncthreads();
    const Z* F = group_fft_L<true, LX, 0>(Bf, A, 2, bs, p.plX, -1, threadIdx.x, blockDim.x, 0);
    xunpack<Z, 0, 2, false>(F, bs, Nxh, Nxp, [&](int slot, int k, Z X, Z Y) {
        if (slot == 0) {
            zp_of<Z>(p, 0)[row + k] = X;
            zp_of<Z>(p, 1)[row + k] = Y;
        } else {
            zp_of<Z>(p, 2)[row + k] = X;
        }
    });
}

// The same with the transforms in place (lengths with an in-place plan, whose
// butterflies fit the block's threads: 3 x 72 at Nxp = 576): three slots of
// fft_bufsz(Nxp), half the shared memory, so more blocks fit per SM.  The
// products n = u x omega are formed inside the first forward pass, from the
// three inverse-transformed slots, instead of in a pass of their own (the
// same arithmetic, one read-write sweep and one barrier fewer: 2.21 -> 2.15
// ms at 384x257x384).  Loading the packed spectra straight into the first
// inverse pass as well was measured slower (2.44 ms: every mode is then
// loaded twice, for k and Nxp - k, and the loads in flight spill registers).
// Z = zd (FP64, layout POS 0) or zf (the mixed forms' FP32 transforms, layout
// POS 2: padded 1 in 16, conflict-free for 8-byte elements).
template <int LX, class Z = zd, int POS = 0>
CF_DEV void xpass_row_ip_body(const FftParams& p, int z, int n) {
    static_assert(3 * fft_ip_butterflies<LX>() <= 256, "one butterfly per thread");
    extern __shared__ __align__(128) unsigned char fsm_raw[];
    Z* sm = reinterpret_cast<Z*>(fsm_raw);
    constexpr int bs = fft_bufsz_pos<POS>(LX);
    const int Nxh = p.Nxh;
    const long row = ((long)n * p.Nzp + z) * Nxh;
    const int xnyq = (p.Nx % 2 == 0) ? p.Nx / 2 : -1;
    xpack<Z, POS, 3, false, CF_XPASS_IP_KPT>(sm, bs, Nxh, LX, xnyq, [&](int slot, int k, Z& X, Z& Y) {
        X = zp_of<Z>(p, 2 * slot)[row + k];
        Y = zp_of<Z>(p, 2 * slot + 1)[row + k];
    });
    __syncthreads();
    group_fft_ip<true, LX, POS>(sm, 3, bs, p.plX, +1, threadIdx.x, blockDim.x, 0);
    // u = (a0.x, a0.y, a1.x), omega = (a1.y, a2.x, a2.y); slots (n0 + i n1, n2)
    auto product = [&](int s, int x) -> Z {
        const int sx = bpos<POS>(x);
        const Z a0 = sm[sx], a1 = sm[bs + sx], a2 = sm[2 * bs + sx];
        if (s == 0) return cmake<Z>(a0.y * a2.y - a1.x * a2.x, a1.x * a1.y - a0.x * a2.y);
        return cmake<Z>(a0.x * a2.x - a0.y * a1.y, 0.0);
    };
    fft_pass_first_ip<true, POS, LX, 8>(sm, 2, bs, -1, threadIdx.x, blockDim.x, 0, true, product);
    group_fft_ip_rest8<true, LX, POS>(sm, 2, bs, p.plX, -1, threadIdx.x, blockDim.x, 0);
    xunpack<Z, POS, 2, false>(sm, bs, Nxh, LX, [&](int slot, int k, Z X, Z Y) {
        if (slot == 0) {
            zp_of<Z>(p, 0)[row + k] = X;
            zp_of<Z>(p, 1)[row + k] = Y;
        } else {
            zp_of<Z>(p, 2)[row + k] = X;
        }
    });
}

// Convective form (nonlinear.jl:113-140, dot! operators.jl:247-254).  grid:
// (Nzp, Ny); block 256; smem 12*bsx complex.  One row z = bx of plane n, twelve
// real rows packed in six slots: field codes 0-2 u (z-padded 0-2), 3-5 du/dx
// (i ax k times fields 0-2, ddx1!), 6-8 du/dy (z-padded 3-5), 9-11 du/dz
// (z-padded 6-8); slot s holds codes 2s, 2s+1.  Product n_i = -(u0 du_i/dx +
// u1 du_i/dy + u2 du_i/dz) (the sign of _store_rhs!, nonlinear.jl:139), in
// slots (n0 + i n1, n2), written to z-padded 0-2.
template <int LX, class Z>
CF_DEV void xpass_conv_body(const FftParams& p, int z, int n) {
    extern __shared__ __align__(128) unsigned char fsm_raw[];
    Z* sm = reinterpret_cast<Z*>(fsm_raw);
    const int Nxp = LX ? LX : p.Nxp, Nxh = p.Nxh, bs = p.bsx;
    const long row = ((long)n * p.Nzp + z) * Nxh;
    const int xnyq = (p.Nx % 2 == 0) ? p.Nx / 2 : -1;
    Z* scr = sm + 6 * bs;
    auto fetch = [&](int code, int k) -> Z {
        if (code < 3) return zp_of<Z>(p, code)[row + k];
        if (code < 6) return cmuli(zp_of<Z>(p, code - 3)[row + k], p.ax * k);
        return zp_of<Z>(p, code - 3)[row + k];
    };
    xpack<Z, 1, 6, true>(sm, bs, Nxh, Nxp, xnyq, [&](int slot, int k, Z& X, Z& Y) {
        X = fetch(2 * slot, k);
        Y = fetch(2 * slot + 1, k);
    });
    __syncthreads();
    Z* A = group_fft_L<true, LX, 1>(sm, scr, 6, bs, p.plX, +1, threadIdx.x, blockDim.x, 0);
    Z* Bf = (A == sm) ? scr : sm;
    for (int j = threadIdx.x; j < Nxp; j += blockDim.x) {
        const int sj = swz(j);
        const Z s0 = A[0 * bs + sj], s1 = A[1 * bs + sj], s2 = A[2 * bs + sj];
        const Z s3 = A[3 * bs + sj], s4 = A[4 * bs + sj], s5 = A[5 * bs + sj];
        const double u0 = s0.x, u1 = s0.y, u2 = s1.x;
        const double gx0 = s1.y, gx1 = s2.x, gx2 = s2.y;
        const double gy0 = s3.x, gy1 = s3.y, gy2 = s4.x;
        const double gz0 = s4.y, gz1 = s5.x, gz2 = s5.y;
        const double n0 = -(u0 * gx0 + u1 * gy0 + u2 * gz0);
        const double n1 = -(u0 * gx1 + u1 * gy1 + u2 * gz1);
        const double n2 = -(u0 * gx2 + u1 * gy2 + u2 * gz2);
        Bf[0 * bs + sj] = cmake<Z>(n0, n1);
        Bf[1 * bs + sj] = cmake<Z>(n2, 0.0);
    }
    __syncthreads();
    const Z* F = group_fft_L<true, LX, 1>(Bf, A, 2, bs, p.plX, -1, threadIdx.x, blockDim.x, 0);
    xunpack<Z, 1, 2, true>(F, bs, Nxh, Nxp, [&](int slot, int k, Z X, Z Y) {
        if (slot == 0) {
            zp_of<Z>(p, 0)[row + k] = X;
            zp_of<Z>(p, 1)[row + k] = Y;
        } else {
            zp_of<Z>(p, 2)[row + k] = X;
        }
    });
}

// The convective x-pass with the transforms in place (lengths with an
// in-place plan; 512 threads, one per butterfly of the six slots: 6 x 72 at
// Nxp = 576): six slots of fft_bufsz(Nxp), so two blocks of 16 warps fit per
// SM instead of two of 8.  Same packing, product and truncation as
// xpass_conv_body; the product at j rewrites slots 0-1 at j in place.
template <int LX>
CF_DEV void xpass_conv_ip_body(const FftParams& p, int z, int n) {
    static_assert(6 * fft_ip_butterflies<LX>() <= 512, "one butterfly per thread");
    extern __shared__ __align__(128) unsigned char fsm_raw[];
    zd* sm = reinterpret_cast<zd*>(fsm_raw);
    const int Nxh = p.Nxh, bs = p.bsxp;
    const long row = ((long)n * p.Nzp + z) * Nxh;
    const int xnyq = (p.Nx % 2 == 0) ? p.Nx / 2 : -1;
    auto fetch = [&](int code, int k) -> zd {
        if (code < 3) return zp_of<zd>(p, code)[row + k];
        if (code < 6) return cmuli(zp_of<zd>(p, code - 3)[row + k], p.ax * k);
        return zp_of<zd>(p, code - 3)[row + k];
    };
    xpack<zd, 0, 6, true>(sm, bs, Nxh, LX, xnyq, [&](int slot, int k, zd& X, zd& Y) {
        X = fetch(2 * slot, k);
        Y = fetch(2 * slot + 1, k);
    });
    __syncthreads();
    group_fft_ip<true, LX, 0>(sm, 6, bs, p.plX, +1, threadIdx.x, blockDim.x, 0);
    for (int j = threadIdx.x; j < LX; j += blockDim.x) {
        const int sj = fpos(j);
        const zd s0 = sm[sj], s1 = sm[bs + sj], s2 = sm[2 * bs + sj];
        const zd s3 = sm[3 * bs + sj], s4 = sm[4 * bs + sj], s5 = sm[5 * bs + sj];
        const double u0 = s0.x, u1 = s0.y, u2 = s1.x;
        const double gx0 = s1.y, gx1 = s2.x, gx2 = s2.y;
        const double gy0 = s3.x, gy1 = s3.y, gy2 = s4.x;
        const double gz0 = s4.y, gz1 = s5.x, gz2 = s5.y;
        sm[sj] = zmake(-(u0 * gx0 + u1 * gy0 + u2 * gz0), -(u0 * gx1 + u1 * gy1 + u2 * gz1));
        sm[bs + sj] = zmake(-(u0 * gx2 + u1 * gy2 + u2 * gz2), 0.0);
    }
    __syncthreads();
    group_fft_ip<true, LX, 0>(sm, 2, bs, p.plX, -1, threadIdx.x, blockDim.x, 0);
    xunpack<zd, 0, 2, true>(sm, bs, Nxh, LX, [&](int slot, int k, zd X, zd Y) {
        if (slot == 0) {
            zp_of<zd>(p, 0)[row + k] = X;
            zp_of<zd>(p, 1)[row + k] = Y;
        } else {
            zp_of<zd>(p, 2)[row + k] = X;
        }
    });
}

// Divergence form (nonlinear.jl:146-167, outer! operators.jl:227-234).  grid:
// (ceil(Nzp/2), Ny); block 256; smem 12*bsx complex.  Rows zA = 2*bx, zB =
// 2*bx+1 of plane n; slot f holds (u_f row A) + i (u_f row B).  The six
// distinct products (u_i u_j = u_j u_i exactly) are negated (the sign of
// _store_rhs!, nonlinear.jl:166, moved ahead of the linear transforms and
// div!) into slots m = 00 01 02 11 12 22 and written to z-padded 0-5.
template <int LX, class Z>
CF_DEV void xpass_div_body(const FftParams& p, int bx, int n) {
    extern __shared__ __align__(128) unsigned char fsm_raw[];
    Z* sm = reinterpret_cast<Z*>(fsm_raw);
    const int zA = 2 * bx, zB = zA + 1;
    const bool hasB = zB < p.Nzp;
    const int Nxp = LX ? LX : p.Nxp, Nxh = p.Nxh, bs = p.bsx;
    const long rowA = ((long)n * p.Nzp + zA) * Nxh;
    const long rowB = ((long)n * p.Nzp + zB) * Nxh;
    const int xnyq = (p.Nx % 2 == 0) ? p.Nx / 2 : -1;
    Z* scr = sm + 6 * bs;
    xpack<Z, 1, 3, true>(sm, bs, Nxh, Nxp, xnyq, [&](int slot, int k, Z& X, Z& Y) {
        const Z* src = zp_of<Z>(p, slot);
        X = src[rowA + k];
        if (hasB) Y = src[rowB + k];
    });
    __syncthreads();
    Z* A = group_fft_L<true, LX, 1>(sm, scr, 3, bs, p.plX, +1, threadIdx.x, blockDim.x, 0);
    Z* Bf = (A == sm) ? scr : sm;
    for (int j = threadIdx.x; j < Nxp; j += blockDim.x) {
        const int sj = swz(j);
        const Z a0 = A[0 * bs + sj], a1 = A[1 * bs + sj], a2 = A[2 * bs + sj];
        Bf[0 * bs + sj] = cmake<Z>(-(a0.x * a0.x), -(a0.y * a0.y));
        Bf[1 * bs + sj] = cmake<Z>(-(a0.x * a1.x), -(a0.y * a1.y));
        Bf[2 * bs + sj] = cmake<Z>(-(a0.x * a2.x), -(a0.y * a2.y));
        Bf[3 * bs + sj] = cmake<Z>(-(a1.x * a1.x), -(a1.y * a1.y));
        Bf[4 * bs + sj] = cmake<Z>(-(a1.x * a2.x), -(a1.y * a2.y));
        Bf[5 * bs + sj] = cmake<Z>(-(a2.x * a2.x), -(a2.y * a2.y));
    }
    __syncthreads();
    const Z* F = group_fft_L<true, LX, 1>(Bf, A, 6, bs, p.plX, -1, threadIdx.x, blockDim.x, 0);
    xunpack<Z, 1, 6, true>(F, bs, Nxh, Nxp, [&](int slot, int k, Z X, Z Y) {
        Z* dst = zp_of<Z>(p, slot);
        dst[rowA + k] = X;
        if (hasB) dst[rowB + k] = Y;
    });
}

// The divergence x-pass with the transforms in place (lengths with an in-place
// plan; 512 threads, one per butterfly of the six product slots): six slots
// of fft_bufsz(Nxp).  The three forward transforms run in slots 0-2; the
// product at j reads slots 0-2 at j and writes slots 0-5 at j (one thread per
// j, no barrier of its own).
template <int LX>
CF_DEV void xpass_div_ip_body(const FftParams& p, int bx, int n) {
    static_assert(6 * fft_ip_butterflies<LX>() <= 512, "one butterfly per thread");
    extern __shared__ __align__(128) unsigned char fsm_raw[];
    zd* sm = reinterpret_cast<zd*>(fsm_raw);
    const int zA = 2 * bx, zB = zA + 1;
    const bool hasB = zB < p.Nzp;
    const int Nxh = p.Nxh, bs = p.bsxp;
    const long rowA = ((long)n * p.Nzp + zA) * Nxh;
    const long rowB = ((long)n * p.Nzp + zB) * Nxh;
    const int xnyq = (p.Nx % 2 == 0) ? p.Nx / 2 : -1;
    xpack<zd, 0, 3, true>(sm, bs, Nxh, LX, xnyq, [&](int slot, int k, zd& X, zd& Y) {
        const zd* src = zp_of<zd>(p, slot);
        X = src[rowA + k];
        if (hasB) Y = src[rowB + k];
    });
    __syncthreads();
    group_fft_ip<true, LX, 0>(sm, 3, bs, p.plX, +1, threadIdx.x, blockDim.x, 0);
    for (int j = threadIdx.x; j < LX; j += blockDim.x) {
        const int sj = fpos(j);
        const zd a0 = sm[sj], a1 = sm[bs + sj], a2 = sm[2 * bs + sj];
        sm[sj] = zmake(-(a0.x * a0.x), -(a0.y * a0.y));
        sm[bs + sj] = zmake(-(a0.x * a1.x), -(a0.y * a1.y));
        sm[2 * bs + sj] = zmake(-(a0.x * a2.x), -(a0.y * a2.y));
        sm[3 * bs + sj] = zmake(-(a1.x * a1.x), -(a1.y * a1.y));
        sm[4 * bs + sj] = zmake(-(a1.x * a2.x), -(a1.y * a2.y));
        sm[5 * bs + sj] = zmake(-(a2.x * a2.x), -(a2.y * a2.y));
    }
    __syncthreads();
    group_fft_ip<true, LX, 0>(sm, 6, bs, p.plX, -1, threadIdx.x, blockDim.x, 0);
    xunpack<zd, 0, 6, true>(sm, bs, Nxh, LX, [&](int slot, int k, zd X, zd Y) {
        zd* dst = zp_of<zd>(p, slot);
        dst[rowA + k] = X;
        if (hasB) dst[rowB + k] = Y;
    });
}

// Single-instance kernels and their batched forms (one launch per size class;
// blockIdx.z also selects the instance).
template <int LZ, class Z = zd>
__global__ void __launch_bounds__(256) k_zinv(FftParams p) {
    zinv_body<LZ, Z>(p, blockIdx.x, blockIdx.y, blockIdx.z);
}
// five blocks per SM in FP64 (two transform buffers of 2 x 657 complex at
// Nzp = 576; the register cap spills a few words, measured faster than four:
// 1.27 against 1.35 ms for the z-inverse at 384x257x384), six in FP32 (the
// register count they take uncapped)
template <int LZ, class Z = zd>
__global__ void __launch_bounds__(256, (sizeof(Z) == 16 ? 5 : 6)) k_zinv_tma(FftParams p, const __grid_constant__ FftMaps m) {
    zinv_tma_body<LZ, Z>(p, m, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <int LZ, class Z = zd>
__global__ void __launch_bounds__(256, (sizeof(Z) == 16 ? 5 : 6)) k_zfwd_tma(FftParams p, const __grid_constant__ FftMaps m) {
    zfwd_tma_body<LZ, Z>(p, m, blockIdx.x, blockIdx.y, blockIdx.z);
}
template <int LZ, class Z = zd>
__global__ void __launch_bounds__(256) k_zfwd(FftParams p) {
    zfwd_body<LZ, Z>(p, blockIdx.x, blockIdx.y, blockIdx.z);
}
// FP64: one row per block; FP32 (mixed form): two rows per block
template <int LX, class Z = zd>
__global__ void __launch_bounds__(256, (sizeof(Z) == 16 ? 3 : 4)) k_xpass(FftParams p) {
    if constexpr (sizeof(Z) == 16) xpass_row_body<LX, Z>(p, blockIdx.x, blockIdx.y);
    else xpass_body<LX, Z>(p, blockIdx.x, blockIdx.y);
}
// FP64, two rows per block (padded lengths up to 256, where one row leaves
// most of the block idle in the FFT passes)
// in-place transforms (lengths with an in-place plan; other lengths compile an
// empty kernel that the engine never selects)
template <int LX>
__global__ void __launch_bounds__(256, CF_XPASS_IP_BLOCKS) k_xpass_ip(FftParams p) {
    if constexpr (fft_ip_butterflies<LX>() > 0) xpass_row_ip_body<LX>(p, blockIdx.x, blockIdx.y);
}
// the same in FP32 (mixed forms): 14.8 KB of shared memory at Nxp = 576
template <int LX>
__global__ void __launch_bounds__(256, CF_XPASS_IP32_BLOCKS) k_xpass_ip32(FftParams p) {
    if constexpr (fft_ip_butterflies<LX>() > 0) xpass_row_ip_body<LX, zf, 2>(p, blockIdx.x, blockIdx.y);
}
template <int LX>
__global__ void __launch_bounds__(256) k_xpass2(FftParams p) {
    xpass_body<LX, zd>(p, blockIdx.x, blockIdx.y);
}
// in-place convective x-pass, 512 threads (lengths with an in-place plan;
// other lengths compile an empty kernel that the engine never selects)
template <int LX>
__global__ void __launch_bounds__(512, 2) k_xpass_conv_ip(FftParams p) {
    if constexpr (fft_ip_butterflies<LX>() > 0) xpass_conv_ip_body<LX>(p, blockIdx.x, blockIdx.y);
}
template <int LX>
__global__ void __launch_bounds__(256) k_xpass_conv(FftParams p) {
    xpass_conv_body<LX, zd>(p, blockIdx.x, blockIdx.y);
}
// in-place divergence x-pass, 512 threads (lengths with an in-place plan)
template <int LX>
__global__ void __launch_bounds__(512, 2) k_xpass_div_ip(FftParams p) {
    if constexpr (fft_ip_butterflies<LX>() > 0) xpass_div_ip_body<LX>(p, blockIdx.x, blockIdx.y);
}
template <int LX>
__global__ void __launch_bounds__(256) k_xpass_div(FftParams p) {
    xpass_div_body<LX, zd>(p, blockIdx.x, blockIdx.y);
}
// The z kernels of the ensembles' small grids, with the block's tkz
// transforms taken from consecutive (y, kx) pairs (pair y Nxh + kx) rather
// than from one plane: a plane of Nxh = 17, 25 or 33 columns would otherwise
// leave most of its last column group empty.  The transforms and their
// arithmetic are those of zinv_body / zfwd_body.  A thread's transform t =
// threadIdx.x & (tkz - 1) is the same in every loop below (the loops step by
// the block size, a multiple of tkz), so its pair is found once.
// grid: (ceil(Ny Nxh / tkz), 1, nfields).
CF_DEV void zflat_pair(const FftParams& p, int bx, int& y, int& k, bool& ok) {
    const int pair = (bx << p.tks) + (threadIdx.x & ((1 << p.tks) - 1));
    ok = pair < p.Ny * p.Nxh;
    y = ok ? pair / p.Nxh : 0;
    k = pair - y * p.Nxh;
}
template <int LZ>
CF_DEV void zinv_flat_body(const FftParams& p, int bx, int f) {
    extern __shared__ __align__(128) unsigned char fsm_raw[];
    zd* sm = reinterpret_cast<zd*>(fsm_raw);
    const int tks = p.tks, tkz = 1 << tks, tm = tkz - 1;
    const int Nz = p.Nz, Nzp = LZ ? LZ : p.Nzp, Nxh = p.Nxh, bs = p.bsz;
    zd* bufB = sm + tkz * bs;
    const bool dz = f >= 6;
    int y, k;
    bool ok;
    zflat_pair(p, bx, y, k, ok);
    const zd* src = nod_of<zd>(p, dz ? f - 6 : f) + (long)y * Nz * Nxh + k;
    zd* dst = zp_of<zd>(p, f) + (long)y * Nzp * Nxh + k;
    const int xnyq = (p.Nx % 2 == 0) ? p.Nx / 2 : -1, znyq = (Nz % 2 == 0) ? Nz / 2 : -1;
    const bool live = ok && k != xnyq;
    const int gap0 = (Nz >> 1) + 1, gap1 = Nzp - (Nz - gap0);
    for (int e = threadIdx.x; e < ((gap1 - gap0) << tks); e += blockDim.x)
        sm[(e & tm) * bs + fpos(gap0 + (e >> tks))] = czero<zd>();
    const int ntot = Nz << tks;
    for (int base = threadIdx.x; base < ntot; base += 8 * 256) {
        zd v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = base + u * 256;
            const int iz = e >> tks;
            v[u] = (e < ntot && live && iz != znyq) ? src[(long)iz * Nxh] : czero<zd>();
            if (dz) v[u] = cmuli(v[u], p.bz * (double)(iz <= (Nz >> 1) ? iz : iz - Nz));
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = base + u * 256;
            if (e < ntot) sm[(e & tm) * bs + fpos(zpad_index(e >> tks, Nz, Nzp))] = v[u];
        }
    }
    __syncthreads();
    const zd* res = group_fft_L<true, LZ>(sm, bufB, tkz, bs, p.plZ, +1, threadIdx.x, blockDim.x, 0);
    for (int e = threadIdx.x; e < (Nzp << tks); e += blockDim.x)
        if (ok) dst[(long)(e >> tks) * Nxh] = res[(e & tm) * bs + fpos(e >> tks)];
}
template <int LZ>
CF_DEV void zfwd_flat_body(const FftParams& p, int bx, int f) {
    extern __shared__ __align__(128) unsigned char fsm_raw[];
    zd* sm = reinterpret_cast<zd*>(fsm_raw);
    const int tks = p.tks, tkz = 1 << tks, tm = tkz - 1;
    const int Nz = p.Nz, Nzp = LZ ? LZ : p.Nzp, Nxh = p.Nxh, bs = p.bsz;
    zd* bufB = sm + tkz * bs;
    int y, k;
    bool ok;
    zflat_pair(p, bx, y, k, ok);
    const zd* src = zp_of<zd>(p, f) + (long)y * Nzp * Nxh + k;
    zd* dst = nod_of<zd>(p, f) + (long)y * Nz * Nxh + k;
    const int ntot = Nzp << tks;
    for (int base = threadIdx.x; base < ntot; base += 8 * 256) {
        zd v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = base + u * 256;
            v[u] = (e < ntot && ok) ? src[(long)(e >> tks) * Nxh] : czero<zd>();
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = base + u * 256;
            if (e < ntot) sm[(e & tm) * bs + fpos(e >> tks)] = v[u];
        }
    }
    __syncthreads();
    const zd* res = group_fft_L<true, LZ>(sm, bufB, tkz, bs, p.plZ, -1, threadIdx.x, blockDim.x, 0);
    for (int e = threadIdx.x; e < (Nz << tks); e += blockDim.x)
        if (ok) dst[(long)(e >> tks) * Nxh] = res[(e & tm) * bs + fpos(zpad_index(e >> tks, Nz, Nzp))];
}
// grid (ceil(Ny Nxh / tkz), 1, 6 * instances)
template <int LZ>
__global__ void __launch_bounds__(256) k_zinv_batch(const FftParams* __restrict__ pl) {
    __shared__ FftParams ps;
    const int inst = blockIdx.z / 6;
    stage_params(&ps, pl + inst);
    zinv_flat_body<LZ>(ps, blockIdx.x, blockIdx.z - 6 * inst);
}
// grid (ceil(Ny Nxh / tkz), 1, 3 * instances)
template <int LZ>
__global__ void __launch_bounds__(256) k_zfwd_batch(const FftParams* __restrict__ pl) {
    __shared__ FftParams ps;
    const int inst = blockIdx.z / 3;
    stage_params(&ps, pl + inst);
    zfwd_flat_body<LZ>(ps, blockIdx.x, blockIdx.z - 3 * inst);
}
// grid (ceil(Nzp/2), Ny, instances): two rows per block (the ensembles' grids
// are small)
template <int LX>
__global__ void __launch_bounds__(256) k_xpass_batch(const FftParams* __restrict__ pl) {
    __shared__ FftParams ps;
    stage_params(&ps, pl + blockIdx.z);
    xpass_body<LX, zd>(ps, blockIdx.x, blockIdx.y);
}

// Rotational x-pass of R rows per block (R even), for short rows: two rows
// leave most of a block's threads idle in the FFT passes (3 x 72 butterflies
// of 256 at Nxp = 48), R rows keep them busy.  The same arithmetic per row as
// xpass_body.  Slots 3r .. 3r+2 hold (u0+iu1, u2+iw0, w1+iw2) of row r; the
// products of rows 2q, 2q+1 leave in slots 3q (n0+in1 of 2q), 3q+1 (of 2q+1)
// and 3q+2 (n2 of 2q + i n2 of 2q+1).  smem 6 R bsx complex (XOR layout).
template <int LX, int R>
CF_DEV void xpass_rows_body(const FftParams& p, int bx, int n) {
    static_assert(R % 2 == 0, "rows are paired in the forward transform");
    extern __shared__ __align__(128) unsigned char fsm_raw[];
    zd* sm = reinterpret_cast<zd*>(fsm_raw);
    const int z0 = R * bx;
    const int nrow = min(R, p.Nzp - z0);
    const int Nxp = LX ? LX : p.Nxp, Nxh = p.Nxh, bs = p.bsx;
    const long row0 = ((long)n * p.Nzp + z0) * Nxh;
    const int xnyq = (p.Nx % 2 == 0) ? p.Nx / 2 : -1;
    zd* scr = sm + 3 * R * bs;
    xpack<zd, 1, 3 * R, true>(sm, bs, Nxh, Nxp, xnyq, [&](int slot, int k, zd& X, zd& Y) {
        const int r = slot / 3, f = slot - 3 * r;
        if (r >= nrow) return;  // zeros for rows past the end
        const long row = row0 + (long)r * Nxh;
        X = zp_of<zd>(p, 2 * f)[row + k];
        Y = zp_of<zd>(p, 2 * f + 1)[row + k];
    });
    __syncthreads();
    zd* A = group_fft_L<true, LX, 1>(sm, scr, 3 * R, bs, p.plX, +1, threadIdx.x, blockDim.x, 0);
    zd* Bf = (A == sm) ? scr : sm;
    for (int e = threadIdx.x; e < (R / 2) * Nxp; e += blockDim.x) {
        const int qd = e / Nxp, j = e - qd * Nxp, sj = swz(j);
        const zd* ra = A + 6 * qd * bs;
        const zd a0 = ra[0 * bs + sj], a1 = ra[1 * bs + sj], a2 = ra[2 * bs + sj];
        const zd b0 = ra[3 * bs + sj], b1 = ra[4 * bs + sj], b2 = ra[5 * bs + sj];
        // u = (a0.x, a0.y, a1.x), omega = (a1.y, a2.x, a2.y); likewise b
        const double nA0 = a0.y * a2.y - a1.x * a2.x;
        const double nA1 = a1.x * a1.y - a0.x * a2.y;
        const double nA2 = a0.x * a2.x - a0.y * a1.y;
        const double nB0 = b0.y * b2.y - b1.x * b2.x;
        const double nB1 = b1.x * b1.y - b0.x * b2.y;
        const double nB2 = b0.x * b2.x - b0.y * b1.y;
        zd* o = Bf + 3 * qd * bs;
        o[0 * bs + sj] = zmake(nA0, nA1);
        o[1 * bs + sj] = zmake(nB0, nB1);
        o[2 * bs + sj] = zmake(nA2, nB2);
    }
    __syncthreads();
    const zd* F = group_fft_L<true, LX, 1>(Bf, A, 3 * R / 2, bs, p.plX, -1, threadIdx.x, blockDim.x, 0);
    xunpack<zd, 1, 3 * R / 2, true>(F, bs, Nxh, Nxp, [&](int slot, int k, zd X, zd Y) {
        const int qd = slot / 3, w = slot - 3 * qd;
        const int rA = 2 * qd, rB = rA + 1;
        const long rowA = row0 + (long)rA * Nxh, rowB = rowA + Nxh;
        if (w == 0) {
            if (rA < nrow) {
                zp_of<zd>(p, 0)[rowA + k] = X;
                zp_of<zd>(p, 1)[rowA + k] = Y;
            }
        } else if (w == 1) {
            if (rB < nrow) {
                zp_of<zd>(p, 0)[rowB + k] = X;
                zp_of<zd>(p, 1)[rowB + k] = Y;
            }
        } else {
            if (rA < nrow) zp_of<zd>(p, 2)[rowA + k] = X;
            if (rB < nrow) zp_of<zd>(p, 2)[rowB + k] = Y;
        }
    });
}
// grid (ceil(Nzp/R), Ny, instances)
template <int LX, int R>
__global__ void __launch_bounds__(256) k_xpass_rows_batch(const FftParams* __restrict__ pl) {
    __shared__ FftParams ps;
    stage_params(&ps, pl + blockIdx.z);
    xpass_rows_body<LX, R>(ps, blockIdx.x, blockIdx.y);
}
