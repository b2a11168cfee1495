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
