// cf_common.cuh -- shared device helpers for the CNRK2 engine (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define CF_DEV __device__ __forceinline__
// Helpers called from many sites of the column kernels: one out-of-line copy
// each keeps a kernel's instructions within the instruction caches (inlined at
// every site, the column stage kernel stalled on instruction fetch).  Static:
// every translation unit keeps its own copy.
#define CF_DEV_NOINLINE static __device__ __noinline__

// Nonlinear forms of NonLinearTerm (src/nonlinear.jl:10-17); the values of
// cf_config.form.
enum NlForm { NL_ROT = 0, NL_CONV = 1, NL_DIV = 2 };

// ----------------------------------------------------------------- complex
typedef double2 zd;

CF_DEV zd zmake(double r, double i) { return make_double2(r, i); }
CF_DEV zd zadd(zd a, zd b) { return make_double2(a.x + b.x, a.y + b.y); }
CF_DEV zd zsub(zd a, zd b) { return make_double2(a.x - b.x, a.y - b.y); }
CF_DEV zd zscale(zd a, double s) { return make_double2(a.x * s, a.y * s); }
CF_DEV zd zmul(zd a, zd b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
CF_DEV zd zconj(zd a) { return make_double2(a.x, -a.y); }
// i * a
CF_DEV zd zmuli(zd a) { return make_double2(-a.y, a.x); }
// s * i * a  (real s)
CF_DEV zd zmulis(zd a, double s) { return make_double2(-a.y * s, a.x * s); }
// a + s * b
CF_DEV zd zaxpy(zd a, double s, zd b) { return make_double2(fma(s, b.x, a.x), fma(s, b.y, a.y)); }
CF_DEV zd zzero() { return make_double2(0.0, 0.0); }

// The same operations on single-precision complex values (the FP32 transforms
// of the mixed-precision path); real factors are rounded to float once.
typedef float2 zf;
CF_DEV zf zadd(zf a, zf b) { return make_float2(a.x + b.x, a.y + b.y); }
CF_DEV zf zsub(zf a, zf b) { return make_float2(a.x - b.x, a.y - b.y); }
CF_DEV zf zscale(zf a, double s) {
    const float f = (float)s;
    return make_float2(a.x * f, a.y * f);
}
CF_DEV zf zmul(zf a, zf b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
CF_DEV zf zconj(zf a) { return make_float2(a.x, -a.y); }
CF_DEV zf zmuli(zf a) { return make_float2(-a.y, a.x); }
CF_DEV zf zaxpy(zf a, double s, zf b) {
    const float f = (float)s;
    return make_float2(fmaf(f, b.x, a.x), fmaf(f, b.y, a.y));
}
// complex value of type Z (zd or zf) from real and imaginary parts
template <class Z>
CF_DEV Z cmake(double r, double i);
template <>
CF_DEV zd cmake<zd>(double r, double i) { return make_double2(r, i); }
template <>
CF_DEV zf cmake<zf>(double r, double i) { return make_float2((float)r, (float)i); }
template <class Z>
CF_DEV Z czero() { return cmake<Z>(0.0, 0.0); }
// conversions between the two precisions
CF_DEV zd to_zd(zd a) { return a; }
CF_DEV zd to_zd(zf a) { return make_double2((double)a.x, (double)a.y); }
CF_DEV zf to_zf(zd a) { return make_float2((float)a.x, (float)a.y); }

// ------------------------------------------------ asynchronous copies
// One element (8 or 16 bytes) copied global -> shared without passing through
// registers (zero fill when !ok; src must still be a valid address).  The
// copies of a thread complete in commit groups (cp_async_commit), waited for
// with cp_async_wait<N>() (all but the N most recent groups); a __syncthreads
// must follow before other threads read the copied data.
template <int BYTES>
CF_DEV void cp_async_el(void* sdst, const void* gsrc, bool ok) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(gsrc), "r"(ok ? 16 : 0)
                     : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(gsrc), "r"(ok ? 8 : 0)
                     : "memory");
}
CF_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
CF_DEV void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ------------------------------------------ mbarriers and bulk copies
CF_DEV uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
CF_DEV void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}
// Bounded wait for the completion of phase `parity`; false when it gave up
// after `limit` polls.  A kernel whose wait gave up still waits (with the
// default limit) for its own copies or MMAs in flight before it leaves, so no
// asynchronous write lands in shared memory that a later block owns.
#define CF_WAIT_SPINS (1L << 22)
CF_DEV bool mbar_wait(uint32_t mbar, uint32_t parity, long limit = CF_WAIT_SPINS) {
    for (long it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
// generic-proxy shared-memory writes made visible to the async proxy (TMA, tensor cores)
CF_DEV void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
CF_DEV void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
CF_DEV void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}
// TMA tile copies of a 3-D tensor map (no multicast): global -> shared
// completing on an mbarrier, shared -> global in a bulk group.  The
// innermost coordinate x times the element size is a multiple of 16 bytes at
// every call site.
CF_DEV void tma_load_3d(void* sdst, const void* map, int x, int y, int z, uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(sdst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(mbar)
        : "memory");
}
CF_DEV void tma_store_3d(const void* map, int x, int y, int z, const void* ssrc) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(map),
                 "r"(x), "r"(y), "r"(z), "r"(smem_u32(ssrc))
                 : "memory");
}
CF_DEV void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// until the bulk stores of this thread have read their shared memory (bounded
// by construction: the copies are in flight and complete)
CF_DEV void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// Hint: bring [p, p + bytes) into L2 (one bulk prefetch, no completion to
// wait for).  The range is narrowed to whole 16-byte granules inside it, so
// no byte outside the caller's range (inside one allocation) is named.
CF_DEV void l2_prefetch(const void* p, size_t bytes) {
    const uintptr_t a = ((uintptr_t)p + 15) & ~(uintptr_t)15, e = ((uintptr_t)p + bytes) & ~(uintptr_t)15;
    if (e > a)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((unsigned)(e - a)) : "memory");
}

// Copy of one instance's parameters into shared memory (batched launches:
// the block's instance is picked by a grid coordinate).
template <class T>
CF_DEV void stage_params(T* dst, const T* __restrict__ src) {
    static_assert(sizeof(T) % 8 == 0, "parameter blocks are copied as 8-byte words");
    const unsigned long long* s = reinterpret_cast<const unsigned long long*>(src);
    unsigned long long* d = reinterpret_cast<unsigned long long*>(dst);
    for (int i = threadIdx.x; i < (int)(sizeof(T) / 8); i += blockDim.x) d[i] = s[i];
    __syncthreads();
}

// ------------------------------------------------------------- warp utils
CF_DEV double shfl_up_d(double v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
CF_DEV double shfl_d(double v, int src) { return __shfl_sync(0xffffffffu, v, src); }
CF_DEV double shfl_xor_d(double v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }
CF_DEV zd shfl_up_z(zd v, int d) { return make_double2(shfl_up_d(v.x, d), shfl_up_d(v.y, d)); }
CF_DEV zd shfl_z(zd v, int src) { return make_double2(shfl_d(v.x, src), shfl_d(v.y, src)); }

CF_DEV zd warp_sum_z(zd v) {
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) {
        v.x += shfl_xor_d(v.x, m);
        v.y += shfl_xor_d(v.y, m);
    }
    return v;
}
CF_DEV double warp_sum_d(double v) {
#pragma unroll
    for (int m = 16; m >= 1; m >>= 1) v += shfl_xor_d(v, m);
    return v;
}

// Inclusive additive scan of complex values across the warp (lane order).
CF_DEV zd warp_scan_z(zd v, int lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        zd o = shfl_up_z(v, d);
        if (lane >= d) v = zadd(v, o);
    }
    return v;
}

// Inclusive scan of affine maps f_i(x) = G_i + M_i x under composition in
// lane order: the result of lane j is f_j o ... o f_0.
CF_DEV void warp_scan_affine(double& M, zd& G, int lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        double Mo = shfl_up_d(M, d);
        zd Go = shfl_up_z(G, d);
        if (lane >= d) {
            G = zaxpy(G, M, Go);
            M = M * Mo;
        }
    }
}
