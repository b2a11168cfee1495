// cf_cheb.cuh -- Chebyshev transforms of many columns as tensor-core
// contractions (tcgen05, TF32 inputs, FP32 accumulation in tensor memory).
//
//   Y[f][n][c] = sum_k T[n][k] X[f][k][c],   n, k in [0, Ny), c in [0, C)
//
// for the fields f of one launch; X and Y are FP32 arrays (Ny rows of C
// floats: a complex (Ny, Nz, Nxh) field read as C = 2 Nxh Nz real columns, T
// being real).  T is the DCT-I of the forward transform (nodal values ->
// coefficients, with the reference's normalisation, ffts.jl:65-82 and
// :254-269) or of the inverse one (coefficients -> nodal values,
// chebyshev.jl:58-66 and ffts.jl:162), built by the engine.
//
// The contraction is computed transposed, D = X^T T^T: M = 128 columns of X per
// block (TMEM lane m = column), N = the output degrees (MMAs of at most 256),
// K = the input degrees in tiles of 16.  For more than 256 output degrees
// the degrees are split over two blocks (grid z), so that every block holds at
// most 256 TMEM columns and two blocks fit on an SM.  Both operands are K-major in shared
// memory, in the canonical no-swizzle layout of the tensor cores (core
// matrices of 8 rows x 16 bytes, rows 16 bytes apart, 8-row groups 128 bytes
// apart, 4-element K chunks LBO bytes apart):
//   A (X^T): element (m, k) of a K-tile at ((k/4)*128 + m)*16 + (k%4)*4 bytes
//            (LBO 2048 B); each thread stages one column m, four rows at a time,
//   B (T^T): element (n, k) of the block's output range at ((k/4)*NPs + n)*16
//            + (k%4)*4 bytes (LBO NPs*16 B), NPs = the range's size (a multiple
//            of 16); the engine stores T^T in global memory as K-tile images
//            [4-k chunk][NP rows][4 floats], NP = nsplit * NPs, from which a
//            block copies its NPs rows of each chunk.
// TF32 keeps 10 mantissa bits, so each operand is split into a TF32 head and
// the TF32 rounding of its remainder; hi*hi + hi*lo + lo*hi restores ~FP32
// accuracy (the three products accumulate in the same FP32 tensor memory).
// The BF16 split (SPLIT 1, kind::f16 with BF16 operands, K = 16 per MMA)
// writes each operand as three BF16 pieces x = b0 + b1 + b2 (8 significant
// bits each, 24 in all: the FP32 value), with b1 = bf16(x - b0) and
// b2 = bf16(x - b0 - b1), both differences exact in FP32, and accumulates the
// six products b_i c_j with i + j <= 2 (the dropped ones are below 2^-24 of
// the product): FP32-level accuracy from BF16 tensor cores.  Its chunks of 16
// bytes hold 8 K values, so a K-tile of 16 is two chunks and one MMA step;
// the images are [2 chunks][NP rows][8 bf16] per K-tile and piece.
#pragma once
#include <cuda_bf16.h>

#include "cf_common.cuh"

#define CF_CHEB_MT 128   // columns per block (MMA M)
#define CF_CHEB_KT 16    // input degrees per K-tile
#define CF_CHEB_MAXF 6   // fields per launch
#ifndef CF_CHEB_LOOKAHEAD
#define CF_CHEB_LOOKAHEAD 2  // K-steps of X in flight per producer thread (k_cheb_sym)
#endif

struct ChebParams {
    int Ny, NP, nkt;   // degrees, output rows of the images (nsplit * NPs), K-tiles
    int NPs;           // output rows per block (a multiple of 16, <= 256)
    int nst;           // shared-memory stages (1 or 2)
    long C;            // real columns per field
    const float* X[CF_CHEB_MAXF];
    float* Y[CF_CHEB_MAXF];
    // K-tile images of T^T, one per operand piece: TF32 [nkt][4 chunks][NP
    // rows][4 floats] (head, remainder); BF16 [nkt][2 chunks][NP rows][8
    // bf16] (three pieces)
    const void* B[3];
    int* err;          // set to 1 when a wait gives up
    long spins;        // polls of a wait for a free stage (CF_WAIT_SPINS; shortened only by tests)
};

// ---- PTX wrappers --------------------------------------------------------------

CF_DEV float tf32_round(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// shared-memory matrix descriptor, no swizzle (layout type 0), descriptor
// version 1; addresses and byte offsets in 16-byte units
CF_DEV uint64_t umma_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
// instruction descriptor: D F32, A and B TF32, both K-major, M x N
CF_DEV uint32_t umma_idesc_tf32(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
CF_DEV void umma_tf32(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
// instruction descriptor: D F32, A and B BF16 (kind::f16), both K-major, M x N
CF_DEV uint32_t umma_idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
CF_DEV void umma_f16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
// the three BF16 pieces of x (round to nearest even; the differences are exact)
CF_DEV void bf16_split3(float x, uint16_t& b0, uint16_t& b1, uint16_t& b2) {
    const __nv_bfloat16 h0 = __float2bfloat16_rn(x);
    const float r1 = x - __bfloat162float(h0);
    const __nv_bfloat16 h1 = __float2bfloat16_rn(r1);
    const __nv_bfloat16 h2 = __float2bfloat16_rn(r1 - __bfloat162float(h1));
    b0 = __bfloat16_as_ushort(h0);
    b1 = __bfloat16_as_ushort(h1);
    b2 = __bfloat16_as_ushort(h2);
}
// The same for a pair (x0, x1), packed as the operand words are: bf16 of x0
// in the low half, of x1 in the high half (cvt.rn.bf16x2.f32 rounds to
// nearest even, as __float2bfloat16_rn; the same pieces, two per instruction).
CF_DEV uint32_t bf16x2_rn(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}
CF_DEV void bf16x2_split3(float x0, float x1, uint32_t& w0, uint32_t& w1, uint32_t& w2) {
    w0 = bf16x2_rn(x0, x1);
    const float r0 = x0 - __uint_as_float(w0 << 16), r1 = x1 - __uint_as_float(w0 & 0xFFFF0000u);
    w1 = bf16x2_rn(r0, r1);
    const float s0 = r0 - __uint_as_float(w1 << 16), s1 = r1 - __uint_as_float(w1 & 0xFFFF0000u);
    w2 = bf16x2_rn(s0, s1);
}
CF_DEV void umma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}
CF_DEV void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
CF_DEV void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive TMEM columns of this warp's 32 lanes, one lane per thread
CF_DEV void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// ---- the kernel ------------------------------------------------------------------
// grid (ceil(C / 128), fields, nsplit); 128 threads.  Dynamic shared memory:
// nst stages of [A pieces, B pieces] (TF32: two pieces of 8 KB + NPs * 64 B;
// BF16: three of 4 KB + NPs * 32 B), then two mbarriers and the TMEM address.
// With two stages the loads of K-tile kt overlap the MMAs of K-tile kt - 1.
template <int SPLIT>
struct ChebSplit;
template <>
struct ChebSplit<0> {  // TF32 head and remainder, three products
    static constexpr int NPC = 2, ES = 4, CPK = 4, BQ = 5;
};
template <>
struct ChebSplit<1> {  // BF16 pieces b0 + b1 + b2, six products
    static constexpr int NPC = 3, ES = 2, CPK = 2, BQ = 4;
};
__host__ __device__ constexpr uint32_t cheb_stage_bytes(int NPs, int split) {
    return split ? 3u * CF_CHEB_MT * CF_CHEB_KT * 2 + 3u * NPs * CF_CHEB_KT * 2
                 : 2u * CF_CHEB_MT * CF_CHEB_KT * 4 + 2u * NPs * CF_CHEB_KT * 4;
}

template <int SPLIT>
__global__ void __launch_bounds__(128, 1) k_cheb_mma(ChebParams p) {
    using S = ChebSplit<SPLIT>;
    constexpr int NPC = S::NPC, CPK = S::CPK, BQ = S::BQ;
    constexpr uint32_t APB = CF_CHEB_MT * CF_CHEB_KT * S::ES;  // bytes of one A piece
    extern __shared__ __align__(1024) unsigned char csm[];
    const int f = blockIdx.y, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long c0 = (long)blockIdx.x * CF_CHEB_MT;
    const int NP = p.NP, NPs = p.NPs, nst = p.nst;
    const int nlo = blockIdx.z * NPs;  // first output row of this block
    const uint32_t sb = cheb_stage_bytes(NPs, SPLIT);
    const uint32_t BPB = (uint32_t)NPs * CF_CHEB_KT * S::ES;  // bytes of one B piece
    uint64_t* mbar = reinterpret_cast<uint64_t*>(csm + nst * sb);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 2);
    // TMEM columns: a power of two >= NP (and >= 32)
    const int ncols = NPs <= 32 ? 32 : (NPs <= 64 ? 64 : (NPs <= 128 ? 128 : 256));
    const float* X = p.X[f];
    float* Y = p.Y[f];

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        mbar_init(smem_u32(mbar), 1);
        mbar_init(smem_u32(mbar + 1), 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    bool ok = true;

    // Software pipeline: the X values of K-tile kt + 1 are requested into
    // registers before K-tile kt is written to shared memory and multiplied,
    // so their memory latency overlaps the staging and the MMAs.
    const long cm = c0 + tid;  // the column this thread stages
    const bool cin = cm < p.C;
    float xc[CF_CHEB_KT], xn[CF_CHEB_KT];
#pragma unroll
    for (int r = 0; r < CF_CHEB_KT; ++r) xc[r] = (cin && r < p.Ny) ? __ldg(X + (long)r * p.C + cm) : 0.0f;
    // 16-byte units of the B pieces per K-tile: NPs rows x CPK chunks
    const int nbu = NPs * CPK;
    int done = p.nkt;  // K-tiles whose MMAs were committed
    for (int kt = 0; kt < p.nkt; ++kt) {
        const int st = kt % nst;
        unsigned char* Ast = csm + st * sb;
        unsigned char* Bst = Ast + NPC * APB;
        const int k0 = kt * CF_CHEB_KT;
        // requests: X of the next K-tile, and this K-tile's rows of the images
        // (chunk ch, row n of the block's range; i = ch * NPs + n)
        if (kt + 1 < p.nkt) {
#pragma unroll
            for (int r = 0; r < CF_CHEB_KT; ++r) {
                const int k = k0 + CF_CHEB_KT + r;
                xn[r] = (cin && k < p.Ny) ? __ldg(X + (long)k * p.C + cm) : 0.0f;
            }
        }
        const uint4* bimg[NPC];
#pragma unroll
        for (int q = 0; q < NPC; ++q)
            bimg[q] = reinterpret_cast<const uint4*>(p.B[q]) + (long)kt * NP * CPK;
        uint4 vb[NPC][BQ];
        if (nbu <= BQ * 128) {
#pragma unroll
            for (int u = 0; u < BQ; ++u) {
                const int i = tid + 128 * u;
                if (i < nbu) {
                    const int ch = i / NPs, g = ch * NP + nlo + (i - ch * NPs);
#pragma unroll
                    for (int q = 0; q < NPC; ++q) vb[q][u] = __ldg(bimg[q] + g);
                }
            }
        }
        // the stage is free once the MMAs of K-tile kt - nst (its last user) are done
        if (kt >= nst) {
            ok = mbar_wait(smem_u32(mbar + st), (uint32_t)(((kt - nst) / nst) & 1), p.spins);
            tc_fence_after();
        }
        // A: column cm; chunk j (16 bytes) of K-tile values at (j * 128 + tid) * 16
        if constexpr (SPLIT == 0) {
#pragma unroll
            for (int j = 0; j < CF_CHEB_KT / 4; ++j) {
                float4 h = make_float4(tf32_round(xc[4 * j]), tf32_round(xc[4 * j + 1]), tf32_round(xc[4 * j + 2]),
                                       tf32_round(xc[4 * j + 3]));
                float4 l = make_float4(tf32_round(xc[4 * j] - h.x), tf32_round(xc[4 * j + 1] - h.y),
                                       tf32_round(xc[4 * j + 2] - h.z), tf32_round(xc[4 * j + 3] - h.w));
                const uint32_t o = (j * CF_CHEB_MT + tid) * 16;
                *reinterpret_cast<float4*>(Ast + o) = h;
                *reinterpret_cast<float4*>(Ast + APB + o) = l;
            }
        } else {
#pragma unroll
            for (int j = 0; j < CF_CHEB_KT / 8; ++j) {
                uint32_t w[3][4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    uint16_t a0, a1, a2, c0b, c1b, c2b;
                    bf16_split3(xc[8 * j + 2 * e], a0, a1, a2);
                    bf16_split3(xc[8 * j + 2 * e + 1], c0b, c1b, c2b);
                    w[0][e] = (uint32_t)a0 | ((uint32_t)c0b << 16);
                    w[1][e] = (uint32_t)a1 | ((uint32_t)c1b << 16);
                    w[2][e] = (uint32_t)a2 | ((uint32_t)c2b << 16);
                }
                const uint32_t o = (j * CF_CHEB_MT + tid) * 16;
#pragma unroll
                for (int q = 0; q < 3; ++q)
                    *reinterpret_cast<uint4*>(Ast + q * APB + o) = make_uint4(w[q][0], w[q][1], w[q][2], w[q][3]);
            }
        }
        // B: this block's NPs rows of each chunk of the K-tile's images
        if (nbu <= BQ * 128) {
#pragma unroll
            for (int u = 0; u < BQ; ++u) {
                const int i = tid + 128 * u;
                if (i < nbu) {
#pragma unroll
                    for (int q = 0; q < NPC; ++q) reinterpret_cast<uint4*>(Bst + q * BPB)[i] = vb[q][u];
                }
            }
        } else {
            for (int i = tid; i < nbu; i += 128) {
                const int ch = i / NPs, g = ch * NP + nlo + (i - ch * NPs);
#pragma unroll
                for (int q = 0; q < NPC; ++q) reinterpret_cast<uint4*>(Bst + q * BPB)[i] = __ldg(bimg[q] + g);
            }
        }
        fence_async_smem();
        // every thread stops here together if any wait gave up
        if (!__syncthreads_and(ok)) {
            ok = false;
            done = kt;
            break;
        }
        if (tid == 0) {
            tc_fence_after();
            // MMA steps of K (8 for TF32, 16 for BF16) that hold data
            const int kstep = SPLIT ? 16 : 8;
            const int ksteps = min(CF_CHEB_KT, p.Ny - k0 + kstep - 1) / kstep;
            for (int ks = 0; ks < ksteps; ++ks) {
                const uint32_t aoff = ks * 2 * CF_CHEB_MT * 16, boff = ks * 2 * NPs * 16;
                for (int n0 = 0; n0 < NPs; n0 += 256) {
                    const int N = min(256, NPs - n0);
                    const uint32_t d = tmem + (uint32_t)n0;
                    const uint32_t bo = boff + (n0 / 8) * 128;
                    uint64_t ad[NPC], bd[NPC];
#pragma unroll
                    for (int q = 0; q < NPC; ++q) {
                        ad[q] = umma_desc(smem_u32(Ast + q * APB) + aoff, CF_CHEB_MT * 16, 128);
                        bd[q] = umma_desc(smem_u32(Bst + q * BPB) + bo, NPs * 16, 128);
                    }
                    const uint32_t acc0 = (kt > 0 || ks > 0) ? 1u : 0u;
                    if constexpr (SPLIT == 0) {
                        const uint32_t idesc = umma_idesc_tf32(CF_CHEB_MT, N);
                        umma_tf32(d, ad[0], bd[0], idesc, acc0);
                        umma_tf32(d, ad[0], bd[1], idesc, 1u);
                        umma_tf32(d, ad[1], bd[0], idesc, 1u);
                    } else {
                        const uint32_t idesc = umma_idesc_bf16(CF_CHEB_MT, N);
                        umma_f16(d, ad[0], bd[0], idesc, acc0);
                        umma_f16(d, ad[0], bd[1], idesc, 1u);
                        umma_f16(d, ad[1], bd[0], idesc, 1u);
                        umma_f16(d, ad[0], bd[2], idesc, 1u);
                        umma_f16(d, ad[1], bd[1], idesc, 1u);
                        umma_f16(d, ad[2], bd[0], idesc, 1u);
                    }
                }
            }
            umma_commit(smem_u32(mbar + st));
        }
#pragma unroll
        for (int r = 0; r < CF_CHEB_KT; ++r) xc[r] = xn[r];
    }
    // drain: the last commit of every stage in use (also after a failed wait,
    // so no MMA is left running when TMEM is freed; all waits bounded)
    for (int kt = max(0, done - nst); kt < done; ++kt) {
        ok = mbar_wait(smem_u32(mbar + (kt % nst)), (uint32_t)((kt / nst) & 1)) && ok;
        tc_fence_after();
    }
    ok = __syncthreads_and(ok) != 0;
    if (!ok) {
        if (lane == 0) atomicExch(p.err, 1);
    } else {
        // epilogue: lane m of warp w holds column c0 + 32 w + m
        const long c = c0 + 32 * warp + lane;
        const uint32_t tw = tmem + ((uint32_t)(32 * warp) << 16);
        for (int n0 = 0; n0 < NPs; n0 += 16) {
            float v[16];
            tmem_ld16(tw + (uint32_t)n0, v);
            if (c < p.C) {
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    if (nlo + n0 + i < p.Ny) Y[(long)(nlo + n0 + i) * p.C + c] = v[i];
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

// ---- the transform folded by the symmetry of the DCT-I, persistent ------------
// T[n][P-k] = (-1)^n T[n][k] (the cosine's reflection; the endpoint weights
// are symmetric), so with S_k = X_k + X_{P-k} (k < P/2), S_{P/2} = X_{P/2},
// and D_k = X_k - X_{P-k} (k < P/2), H = P/2:
//   Y[2m]   = sum_{k=0}^{H}   T[2m][k]   S_k      (H + 1 outputs, H + 1 inputs)
//   Y[2m+1] = sum_{k=0}^{H-1} T[2m+1][k] D_k      (H outputs, H inputs)
// (T[2m+1][H] = cos(pi (2m+1) / 2) = 0): two products of half the size, half
// the MMAs of the full one.  Each CTA owns one parity q (its folded T^T
// resident in shared memory for the whole launch, loaded once) and walks the
// items (field, tile of 128 columns) of its pair of CTAs; the even and odd
// CTAs of a pair take the same items in the same order, so the second read of
// a tile's X rows comes from L2.
//   warps 0-7  producers: thread t takes column t % 128 of the tile and
//              half t / 128 of a K-step's 16 inputs (8 inputs and their
//              mirrors, so two threads per column keep twice the loads in
//              flight); forms S or D, splits the operand (TF32 head and
//              remainder, or three BF16 pieces), writes it into a stage of
//              the A ring and arrives on the stage's full barrier
//   warp 12    one thread issues the MMAs of a stage when it is full and
//              commits to its empty barrier; after an item's last K-step it
//              commits to the item's accumulator barrier.  Two accumulators
//              (TMEM columns 0 and 256) let an item's MMAs run while the
//              previous item is read out.  The warp also owns the TMEM
//              allocation (512 columns: one CTA per SM).
//   warps 8-11 epilogue: warp w reads TMEM lanes 32 (w - 8) .. +31 (its
//              columns of the tile), writes rows 2m + q of Y, and releases
//              the accumulator.
// Every wait is bounded: a wait that gives up sets p.err and the shared
// abort flag, every role leaves its loop, and the MMA thread waits for its
// MMAs in flight (one final commit) before the TMEM is freed.
struct ChebSymParams {
    int P;                 // Ny - 1 (even)
    int N[2], Npad[2];     // outputs per parity (H + 1, H) and the MMA N (multiple of 16, <= 256)
    int Kpad[2];           // inputs per parity padded to K-steps of 16
    int nst;               // A stages
    long C;                // real columns per field
    int nf, ntiles;        // fields, tiles of 128 columns per field
    const float* X[CF_CHEB_MAXF];
    float* Y[CF_CHEB_MAXF];
    const unsigned char* B[2];  // folded T^T images per parity: pieces back to back, bbytes[q] each
    unsigned bbytes[2];
    int* err;
    long spins;
};

template <int SPLIT>
__host__ __device__ constexpr unsigned cheb_sym_apiece() {
    return 128u * 16u * (SPLIT ? 2u : 4u);  // one A piece of a K-step (128 columns x 16 inputs)
}

template <int SPLIT>
__global__ void __launch_bounds__(416, 1) k_cheb_sym(ChebSymParams p) {
    using S = ChebSplit<SPLIT>;
    constexpr int NPC = S::NPC;
    constexpr int EPC = 16 / S::ES;  // inputs per 16-byte chunk
    constexpr unsigned APB = cheb_sym_apiece<SPLIT>();
    extern __shared__ __align__(1024) unsigned char csm[];
    const int q = blockIdx.x & 1, pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int P = p.P, H = P >> 1;
    const int Npad = p.Npad[q], Nq = p.N[q], nks = p.Kpad[q] / 16, nst = p.nst;
    const unsigned BPB = p.bbytes[q];
    const unsigned BPBmax = p.bbytes[0] > p.bbytes[1] ? p.bbytes[0] : p.bbytes[1];
    unsigned char* Bs = csm;
    unsigned char* As = csm + NPC * BPBmax;
    uint64_t* full = reinterpret_cast<uint64_t*>(As + (size_t)nst * NPC * APB);
    uint64_t* empty = full + nst;
    uint64_t* accf = empty + nst;
    uint64_t* acce = accf + 2;
    uint64_t* fin = acce + 2;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(fin + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
    const long C = p.C;
    const int nitems = p.nf * p.ntiles;

    if (warp == 12) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int s = 0; s < nst; ++s) {
            mbar_init(smem_u32(full + s), 256);
            mbar_init(smem_u32(empty + s), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(accf + b), 1);
            mbar_init(smem_u32(acce + b), 128);
        }
        mbar_init(smem_u32(fin), 1);
        *abort_flag = 0;
    }
    // the folded T^T of this parity, resident for the whole launch
    {
        const uint4* src = reinterpret_cast<const uint4*>(p.B[q]);
        uint4* dst = reinterpret_cast<uint4*>(Bs);
        const int n16 = (int)(NPC * BPB / 16);
        for (int i = tid; i < n16; i += blockDim.x) dst[i] = __ldg(src + i);
    }
    fence_async_smem();
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const long spins = p.spins;

    if (warp < 8) {
        // ---------------- producers
        // The items' K-steps form one sequence; the 16 X values of the step
        // LA ahead are requested into registers before the current one is
        // folded, split and written, so LA steps' loads are in flight while
        // a step is converted (measured at 384x257x384, inverse transform of
        // six fields: 1.02 ms with one step in flight, 0.88 with two, 0.91
        // with three and four, 1.77 with six).  Step, item and stage counters advance incrementally (no
        // divisions in the loop).
        const int col = tid & 127, half = tid >> 7;
        const int nitm = nitems > pair ? (nitems - pair + npairs - 1) / npairs : 0;
        const int nsteps = nitm * nks;
        // the step to load next: item itl, K-step ksl, its row pointer base and column
        int itl = pair, ksl = 0;
        const float* Xc = nullptr;  // column cl of the item's field (row 0)
        bool cinl = false;
        auto item_cols = [&](int it) {
            const int f = it / p.ntiles;
            const long cl = (long)(it - f * p.ntiles) * 128 + col;
            cinl = cl < C;
            Xc = p.X[f] + (cinl ? cl : 0);
        };
        auto load_next = [&](float* a, float* b) {
            if (ksl == 0) item_cols(itl);
            const int k0 = 16 * ksl + 8 * half;
            const float* pa = Xc + (long)k0 * C;        // rows k0 .. k0 + 7
            const float* pb = Xc + (long)(P - k0) * C;  // rows P - k0 .. P - k0 - 7
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const int k = k0 + r;
                a[r] = (cinl && k <= H) ? __ldg(pa) : 0.0f;
                b[r] = (cinl && k < H) ? __ldg(pb) : 0.0f;
                pa += C;
                pb -= C;
            }
            if (++ksl == nks) {
                ksl = 0;
                itl += npairs;
            }
        };
        // CF_CHEB_LOOKAHEAD + 1 steps in registers: the current one and the
        // next ones in flight
        constexpr int LA = CF_CHEB_LOOKAHEAD;
        float xa[LA + 1][8], xb[LA + 1][8];
#pragma unroll
        for (int d = 0; d < LA; ++d)
            if (d < nsteps) load_next(xa[d], xb[d]);
        int ks = 0, s = 0, u = 0;
        for (int g = 0; g < nsteps && !*abort_flag; ++g) {
            if (g + LA < nsteps) load_next(xa[LA], xb[LA]);
            const float* ca = xa[0];
            const float* cb = xb[0];
            float v[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const int k = 16 * ks + 8 * half + r;
                v[r] = q == 0 ? ca[r] + cb[r] : (k < H ? ca[r] - cb[r] : 0.0f);
            }
            if (u >= 1 && !mbar_wait(smem_u32(empty + s), (uint32_t)((u - 1) & 1), spins)) {
                *abort_flag = 1;
                atomicExch(p.err, 1);
                break;
            }
            unsigned char* Ast = As + (size_t)s * NPC * APB;
            if constexpr (SPLIT == 0) {
                // chunks 2 half, 2 half + 1 (four inputs each)
#pragma unroll
                for (int jj = 0; jj < 2; ++jj) {
                    const float* w = v + 4 * jj;
                    float4 h = make_float4(tf32_round(w[0]), tf32_round(w[1]), tf32_round(w[2]), tf32_round(w[3]));
                    float4 l = make_float4(tf32_round(w[0] - h.x), tf32_round(w[1] - h.y), tf32_round(w[2] - h.z),
                                           tf32_round(w[3] - h.w));
                    const unsigned o = ((2 * half + jj) * 128 + col) * 16;
                    *reinterpret_cast<float4*>(Ast + o) = h;
                    *reinterpret_cast<float4*>(Ast + APB + o) = l;
                }
            } else {
                // chunk half (eight inputs)
                uint32_t w[3][4];
#pragma unroll
                for (int e = 0; e < 4; ++e) bf16x2_split3(v[2 * e], v[2 * e + 1], w[0][e], w[1][e], w[2][e]);
                const unsigned o = (half * 128 + col) * 16;
#pragma unroll
                for (int pc = 0; pc < 3; ++pc)
                    *reinterpret_cast<uint4*>(Ast + pc * APB + o) = make_uint4(w[pc][0], w[pc][1], w[pc][2], w[pc][3]);
            }
            fence_async_smem();
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(full + s)) : "memory");
#pragma unroll
            for (int d = 0; d < LA; ++d)
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    xa[d][r] = xa[d + 1][r];
                    xb[d][r] = xb[d + 1][r];
                }
            if (++ks == nks) ks = 0;
            if (++s == nst) {
                s = 0;
                ++u;
            }
        }
    } else if (warp < 12) {
        // ---------------- epilogue
        const int ew = warp - 8;
        int li = 0;
        for (int it = pair; it < nitems && !*abort_flag; it += npairs, ++li) {
            const int bsel = li & 1;
            if (!mbar_wait(smem_u32(accf + bsel), (uint32_t)((li >> 1) & 1), spins)) {
                *abort_flag = 1;
                atomicExch(p.err, 1);
                break;
            }
            tc_fence_after();
            const int f = it / p.ntiles;
            const long c = (long)(it - f * p.ntiles) * 128 + 32 * ew + lane;
            const bool cin = c < C;
            float* yp = p.Y[f] + (long)q * C + (cin ? c : 0);  // row 2m + q, advanced by 2C per m
            const uint32_t ta = tmem + ((uint32_t)(32 * ew) << 16) + (uint32_t)(bsel * 256);
            for (int n0 = 0; n0 < Npad; n0 += 16) {
                float v[16];
                tmem_ld16(ta + (uint32_t)n0, v);
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    if (cin && n0 + i < Nq) *yp = v[i];
                    yp += 2 * C;
                }
            }
            tc_fence_before();
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(acce + bsel)) : "memory");
        }
    } else if (lane == 0) {
        // ---------------- MMA issue
        const int kstep = SPLIT ? 16 : 8;  // K per MMA
        const uint32_t idesc = SPLIT ? umma_idesc_bf16(128, Npad) : umma_idesc_tf32(128, Npad);
        int s = 0, u = 0;  // stage of the next fill consumed, and its use
        int li = 0;
        bool issued = false;
        for (int it = pair; it < nitems && !*abort_flag; it += npairs, ++li) {
            const int bsel = li & 1;
            if (li >= 2 && !mbar_wait(smem_u32(acce + bsel), (uint32_t)(((li >> 1) - 1) & 1), spins)) {
                *abort_flag = 1;
                atomicExch(p.err, 1);
                break;
            }
            tc_fence_after();
            const uint32_t d = tmem + (uint32_t)(bsel * 256);
            bool ok = true;
            for (int ks = 0; ks < nks; ++ks) {
                if (!mbar_wait(smem_u32(full + s), (uint32_t)(u & 1), spins)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t abase = smem_u32(As + (size_t)s * NPC * APB);
                for (int kk = 0; kk < 16 / kstep; ++kk) {
                    const uint32_t aoff = kk * (kstep / EPC) * 128 * 16;
                    const uint32_t boff = (uint32_t)((16 * ks + kk * kstep) / EPC) * Npad * 16;
                    uint64_t ad[NPC], bd[NPC];
#pragma unroll
                    for (int pc = 0; pc < NPC; ++pc) {
                        ad[pc] = umma_desc(abase + pc * APB + aoff, 128 * 16, 128);
                        bd[pc] = umma_desc(smem_u32(Bs + pc * BPB) + boff, Npad * 16, 128);
                    }
                    const uint32_t acc0 = (ks > 0 || kk > 0) ? 1u : 0u;
                    if constexpr (SPLIT == 0) {
                        umma_tf32(d, ad[0], bd[0], idesc, acc0);
                        umma_tf32(d, ad[0], bd[1], idesc, 1u);
                        umma_tf32(d, ad[1], bd[0], idesc, 1u);
                    } else {
                        umma_f16(d, ad[0], bd[0], idesc, acc0);
                        umma_f16(d, ad[0], bd[1], idesc, 1u);
                        umma_f16(d, ad[1], bd[0], idesc, 1u);
                        umma_f16(d, ad[0], bd[2], idesc, 1u);
                        umma_f16(d, ad[1], bd[1], idesc, 1u);
                        umma_f16(d, ad[2], bd[0], idesc, 1u);
                    }
                }
                issued = true;
                umma_commit(smem_u32(empty + s));
                if (++s == nst) {
                    s = 0;
                    ++u;
                }
            }
            if (!ok) {
                *abort_flag = 1;
                atomicExch(p.err, 1);
                break;
            }
            umma_commit(smem_u32(accf + bsel));
        }
        // every MMA issued by this thread is complete before the TMEM is freed
        if (issued) {
            umma_commit(smem_u32(fin));
            if (!mbar_wait(smem_u32(fin), 0)) atomicExch(p.err, 1);
        }
    }
    __syncwarp();  // warp 12 reconverges (lane 0 issued the MMAs)
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 12) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
}
