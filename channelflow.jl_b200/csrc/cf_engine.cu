// cf_engine.cu -- host side of the B200 CNRK2 engine: set-up of the Stokes
// banks, transform plans, device buffers, the CUDA-graph step and the C ABI
// declared in include/cfb200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cfb200.h"
#include "cf_dispatch.h"
#include "cf_cheb.cuh"

// kz-plane chunks of the state in a host-buffer step (cf_step_host)
#define CF_HOST_CHUNKS 8

static_assert(CF_FORM_ROTATIONAL == NL_ROT && CF_FORM_CONVECTIVE == NL_CONV && CF_FORM_DIVERGENCE == NL_DIV,
              "cf_config.form values are the device form tags");

// Kernel of a size: the compile-time instantiation for the sizes of the
// supported workloads (index arithmetic by constants, unrolled runs), the
// run-time-sized one otherwise.
static ColKernel col_kernel(int which, int P) {
    switch (P) {
#define CF_CASE(N) \
    case N: return col_kernel_for<N>(which);
        CF_COL_LENGTHS(CF_CASE)
#undef CF_CASE
        default: return col_kernel_for<0>(which);
    }
}
static FftTmaKernel fft_tma_kernel(int which, int L, bool f32) {
    switch (L) {
#define CF_CASE(N) \
    case N: return fft_tma_kernel_for<N>(which, f32);
        CF_STATIC_FFT_LENGTHS(CF_CASE)
#undef CF_CASE
        default: return fft_tma_kernel_for<0>(which, f32);
    }
}
static FftKernel fft_kernel(int which, int L, bool f32 = false) {
    switch (L) {
#define CF_CASE(N) \
    case N: return fft_kernel_for<N>(which, f32);
        CF_STATIC_FFT_LENGTHS(CF_CASE)
#undef CF_CASE
        default: return fft_kernel_for<0>(which, f32);
    }
}

static thread_local std::string g_err;
static int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}
#define CU(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            return fail(e_ == cudaErrorMemoryAllocation ? CF_E_NOMEM : CF_E_CUDA,         \
                        std::string(#call) + " (cf_engine.cu:" + std::to_string(__LINE__) + \
                            "): " + cudaGetErrorString(e_));                              \
        }                                                                                 \
    } while (0)

// ===========================================================================
// Host numerics for the set-up (not timed): quasi-tridiagonal tau factors
// ===========================================================================
namespace setup {

static double cmul(int m) { return m == 0 ? 2.0 : 1.0; }

// Factors of the tau system rows 0..P-2 of (th0 D^2 - th1) a = f with wall
// rows (Dirichlet weights 1, Neumann weights n^2).  Equation n >= 2 of each
// parity (spectral integration of the tau rows):
//   s_n a_{n-2} + d_n a_n + u_n a_{n+2} = g_n
//   s_n = -c_{n-2} th1 / (4n(n-1)),  d_n = th0 + [n<=P-2] th1 / (2(n^2-1)),
//   u_n = -[n+2<=P-2] th1 / (4n(n+1)).
// Eliminated from the top: a_n = alpha_n a_{n-2} + beta_n.  W_n carries the
// wall row: sum_n w_n a_n = SA a_par + sum_{n>=par+2} W_n beta_n.
struct Helm {
    int P;
    double th0, th1;
    bool neumann;
    std::vector<double> alpha, invden, W;
    double SA[2];
    double w(int n) const { return neumann ? (double)n * n : 1.0; }
    double eq_s(int n) const { return -cmul(n - 2) * th1 / (4.0 * n * (n - 1)); }
    double eq_d(int n) const { return th0 + (n <= P - 2 ? th1 / (2.0 * ((double)n * n - 1.0)) : 0.0); }
    double eq_u(int n) const { return (n + 2 <= P - 2) ? -th1 / (4.0 * n * (n + 1)) : 0.0; }
    void init(int P_, double t0, double t1, bool neum) {
        P = P_; th0 = t0; th1 = t1; neumann = neum;
        alpha.assign(P + 1, 0.0); invden.assign(P + 1, 0.0); W.assign(P + 1, 0.0);
        for (int par = 0; par < 2; ++par) {
            const int top = ((P & 1) == par) ? P : P - 1;
            double anext = 0.0;
            for (int n = top; n >= par + 2; n -= 2) {
                double den = eq_d(n) + eq_u(n) * anext;
                invden[n] = 1.0 / den;
                alpha[n] = -eq_s(n) / den;
                anext = alpha[n];
            }
            double Wn = 0.0;
            for (int n = top; n >= par + 2; n -= 2) {
                Wn = (n == top) ? w(n) : w(n) + alpha[n + 2] * Wn;
                W[n] = Wn;
            }
            SA[par] = w(par) + (top >= par + 2 ? alpha[par + 2] * W[par + 2] : 0.0);
        }
    }
    // sequential solve (same algebra as the device scans)
    void solve(const double* f, double bp, double bm, double* a) const {
        double bc[2];
        if (!neumann) { bc[0] = 0.5 * (bp + bm); bc[1] = 0.5 * (bp - bm); }
        else { bc[0] = 0.5 * (bp - bm); bc[1] = 0.5 * (bp + bm); }
        std::vector<double> beta(P + 3, 0.0);
        for (int par = 0; par < 2; ++par) {
            const int top = ((P & 1) == par) ? P : P - 1;
            double bnext = 0.0, sw = 0.0;
            for (int n = top; n >= par + 2; n -= 2) {
                double g = cmul(n - 2) * f[n - 2] / (4.0 * n * (n - 1));
                if (n <= P - 2) g -= f[n] / (2.0 * ((double)n * n - 1.0));
                if (n + 2 <= P - 2) g += f[n + 2] / (4.0 * n * (n + 1));
                beta[n] = (g - eq_u(n) * bnext) * invden[n];
                bnext = beta[n];
                sw += W[n] * beta[n];
            }
            double prev = (bc[par] - sw) / SA[par];
            a[par] = prev;
            for (int n = par + 2; n <= top; n += 2) {
                prev = alpha[n] * prev + beta[n];
                a[n] = prev;
            }
        }
    }
};

static void diff(const double* a, double* b, int P) {
    std::vector<double> t(P + 1);
    t[P] = 0.0;
    if (P >= 1) t[P - 1] = 2.0 * P * a[P];
    for (int n = P - 2; n >= 0; --n) t[n] = t[n + 2] + 2.0 * (n + 1) * a[n + 1];
    t[0] *= 0.5;
    for (int n = 0; n <= P; ++n) b[n] = t[n];
}
static double wallderiv(const double* a, int P, bool right) {
    double s = 0.0;
    for (int n = 1; n <= P; ++n) {
        double w = (double)n * n;
        if (!right && (n % 2 == 0)) w = -w;
        s += w * a[n];
    }
    return s;
}
static double bulkmean(const double* a, int P) {
    double v = a[0];
    for (int n = 2; n <= P; n += 2) v += a[n] / (1.0 - (double)n * n);
    return v;
}

// Chebyshev coefficients of values at y_j = cos(pi j/P) (chebcoeffs): DCT-I
// evaluated directly in long double, divided by P, endpoints halved.
static void chebcoeffs(const double* vals, double* coef, int P) {
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k <= P; ++k) {
        long double s = 0.5L * vals[0] + 0.5L * ((k % 2) ? -1.0L : 1.0L) * vals[P];
        for (int n = 1; n < P; ++n) s += (long double)vals[n] * cosl(pi * (long double)((long long)n * k % (2 * P)) / P);
        long double c = 2.0L * s / P;
        if (k == 0 || k == P) c *= 0.5L;
        coef[k] = (double)c;
    }
}

template <class F>
static void parallel_for(long n, F f) {
    unsigned nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    if (n < 64) nt = 1;
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nt; ++t)
        th.emplace_back([=, &f] {
            for (long i = (long)t; i < n; i += nt) f(i);
        });
    for (auto& x : th) x.join();
}

}  // namespace setup

// ===========================================================================
// Engine
// ===========================================================================
// sizes of the folded tensor-core Chebyshev transform (cheb_sym_dims)
struct ChebSymDims {
    int N[2], Npad[2], Kpad[2], nst;
    unsigned bbytes[2];
    size_t smem;
};

struct DevBank {
    double *fac_p = nullptr, *fac_v = nullptr, *resp = nullptr, *colsc = nullptr, *sa = nullptr, *meanc = nullptr;
    double meanc_mean = 0.0, nu = 0.0, lambda = 0.0;
    bool ready = false;
    BankDev view() const {
        BankDev b;
        b.fac_p = fac_p; b.fac_v = fac_v; b.resp = resp; b.colsc = colsc; b.sa = sa; b.meanc = meanc;
        b.meanc_mean = meanc_mean;
        return b;
    }
};

struct cf_engine {
    int Nx, Ny, Nz, Nxh, Nxp, Nzp, P;
    long B, nr, nq;
    double Lx, Lz, nu, dt;
    int cmode;
    double c1, c2;  // as given (total bulk targets when cmode == 1)
    double basemean;
    std::vector<double> base, basecurv;
    int tkz;
    // TMA row transfers of the z kernels (maps of the FP64 and the FP32 fields)
    FftMaps maps64, maps32;
    bool tma64 = false, tma32 = false;
    // columns per block of the FP32 z-inverse without TMA: twice the FP64
    // groups' (rows of 8-byte elements gathered in segments as long as the
    // FP64 kernels'; measured 1.31 -> 1.02 ms at 384x257x384, while the
    // z-forward, whose stores are the strided side, is faster at tkz: 0.54
    // against 0.66 ms)
    int tkz32 = 0;
    int zbox = 0, zpbox = 0;  // rows per TMA box (nodal, z-padded)
    // status words written by the kernels, read and cleared by check_status:
    // [0] a TMA wait of a z kernel gave up, [1] a tensor-core wait gave up,
    // [2] the mean mode went non-finite (d_ffterr, d_cheberr point into it)
    int* d_status = nullptr;
    int* d_ffterr = nullptr;
    int device = 0;                  // the CUDA device the handle was created on
    long wait_spins = CF_WAIT_SPINS;  // polls of a kernel's first bounded wait (cf_set_wait_limit)
    size_t dev_bytes = 0;            // device memory the handle holds (cf_device_bytes)
    // device
    cudaStream_t stream = nullptr;
    int form = NL_ROT;  // nonlinear form (CF_FORM_*)
    // z-padded work fields: 6 (rotational, divergence) or 9 (convective)
    zd *U[3] = {}, *Pf = nullptr, *Q[3] = {}, *nod[6] = {}, *zp[9] = {};
    zd *tmpU = nullptr, *tmpP = nullptr;
    double *d_base = nullptr, *d_basecurv = nullptr, *d_grad = nullptr;
    zd *d_twP = nullptr, *d_twZ = nullptr, *d_twX = nullptr, *d_cs = nullptr;
    double* d_helmtab = nullptr;
    FftPlan plP, plZ, plX;
    DevBank bank[3], proj, neum;
    // factors of a step of another duration (the shortened final step of a
    // Flows interval): built on first use for tdt, kept for repeated calls
    DevBank tbank[3];
    double tdt = 0.0;
    bool nodal_valid = false;
    // mixed-precision form (CF_PRECISION_MIXED): FP32 nodal and z-padded
    // fields, FP32 twiddles, tensor-core Chebyshev transform images
    int mixed = 0;
    bool tc = false;  // mixed: Chebyshev transforms on the tensor cores (else FP64 in the column kernel)
    void *nod32[6] = {}, *zp32[6] = {};
    void* coef32[6] = {};  // FP32 Chebyshev coefficients (the transforms run out of place)
    zf *d_twZf = nullptr, *d_twXf = nullptr;
    unsigned char *d_chebF = nullptr, *d_chebI = nullptr;  // transform-matrix images, pieces back to back
    int split = 0;  // tensor-core operand split: 0 TF32 head and remainder, 1 three BF16 pieces
    int chebNP = 0, chebKT = 0;
    bool chebsym = false;  // the folded, persistent transform (k_cheb_sym) is used
    ChebSymDims symd;
    // CF_PRECISION_MIXED_F32STATE: the state the steps advance lives in
    // U32, P32, Q32 (complex float); U and Pf keep the FP64 copy that the
    // state entry points read and write.  valid64 / valid32: which copy is
    // current (converted on demand by state_to64 / state_to32).
    bool s32 = false;
    void *U32[3] = {}, *P32 = nullptr, *Q32[3] = {};
    zd* mean64 = nullptr;  // the mean-flow mode (column 0) of U, P, Q in FP64: [7][Ny]
    bool valid64 = true, valid32 = true;
    int* d_cheberr = nullptr;
    double* d_diag = nullptr;  // diagnostics accumulators
    double* d_rec = nullptr;   // rows of diagnostics recorded between steps (cf_step_record)
    int rec_cap = 0;           // rows d_rec holds
    double* d_diagpart = nullptr;  // diagnostics block partials (3 per column block)
    cudaGraphExec_t graph = nullptr;
    int last_launches = 0;
    // host-buffer steps (cf_step_host): the copy stream and the events that
    // order the kz-plane chunks of the state between it and the handle stream
    cudaStream_t cstream = nullptr;
    cudaEvent_t hev[2 * CF_HOST_CHUNKS + 2] = {};
    std::vector<void*> allocs;
};

static const double CA[3] = {0.0, -5.0 / 9.0, -153.0 / 128.0};
static const double CB[3] = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};
static const double CC[3] = {1.0 / 6.0, 5.0 / 24.0, 1.0 / 8.0};

static int dalloc(cf_engine* h, void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return fail(CF_E_NOMEM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
    h->allocs.push_back(*p);
    h->dev_bytes += bytes;
    return CF_OK;
}

// The handle's device is current for the duration of an entry point; the
// caller's current device is restored on return.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

static std::vector<int> fft_radices(int n) {
    std::vector<int> r;
    while (n % 8 == 0) { r.push_back(8); n /= 8; }
    while (n % 4 == 0) { r.push_back(4); n /= 4; }
    while (n % 2 == 0) { r.push_back(2); n /= 2; }
    while (n % 3 == 0) { r.push_back(3); n /= 3; }
    while (n % 5 == 0) { r.push_back(5); n /= 5; }
    for (int p = 7; p <= n; p += 2)
        while (n % p == 0) { r.push_back(p); n /= p; }
    return r;
}

static int rup8(int x) { return (x + 7) & ~7; }
// transform-buffer strides and shared memory of the periodic FFT kernels
// The z kernels' tkz transforms lie bs = fft_bufsz(Nzp) + (8 / tkz) % 8
// complex apart: an 8-thread phase of a 16-byte access touches 8/tkz rows of
// each of the tkz columns, and this offset puts the columns in disjoint
// 16-byte bank groups (tkz = 2: 4 groups apart; 4: 2; 8: 1), so the packing,
// unpacking and multi-transform FFT passes are free of bank conflicts
// (simulated: 1.22 wavefronts per ideal one at tkz = 2 with the odd stride).
static int zbs(const cf_engine* h) { return fft_bufsz(h->Nzp) + (8 / h->tkz) % 8; }
static int zbs_t(const cf_engine* h, int tkz) { return fft_bufsz(h->Nzp) + (8 / tkz) % 8; }
static size_t zsmem_t(const cf_engine* h, int tkz, size_t es) { return (size_t)2 * tkz * zbs_t(h, tkz) * es; }
static int xbs(const cf_engine* h) { return rup8(h->Nxp); }
static size_t zsmem(const cf_engine* h) { return (size_t)2 * h->tkz * zbs(h) * sizeof(zd); }
// TMA z kernels: the first transform buffer, then (128-aligned) the second,
// which also stages the rows of the nodal and z-padded transfers (boxes
// rounded up to whole boxes); es = bytes per complex element.  Either buffer
// stages the stored rows, so the rounded row counts must fit one buffer.
static int zstage_rows(const cf_engine* h) {
    const int rz = ((h->Nz + h->zbox - 1) / h->zbox) * h->zbox, rp = ((h->Nzp + h->zpbox - 1) / h->zpbox) * h->zpbox;
    return std::max(rz, rp);
}
static size_t zstage_off(const cf_engine* h, size_t es) {
    return ((size_t)h->tkz * zbs(h) * es + 127) & ~(size_t)127;
}
static size_t zsmem_tma(const cf_engine* h, size_t es) { return zstage_off(h, es) + (size_t)h->tkz * zbs(h) * es; }
// x-pass shared memory: 12 slots of round_up(Nxp, 8) (two rows of the FP32
// rotational form, the convective and divergence forms), or 6 slots of
// fft_bufsz(Nxp) (one row of the FP64 rotational form), 3 with the
// transforms in place
static size_t xsmem(const cf_engine* h, int slots = 12) {
    return (size_t)slots * (slots < 12 ? fft_bufsz(h->Nxp) : xbs(h)) * sizeof(zd);
}
static int ilog2(int v) {
    int r = 0;
    while ((1 << (r + 1)) <= v) ++r;
    return r;
}

// radices above 31 do not fit the packed plan (5 bits per pass)
static bool radices_ok(const std::vector<int>& rad) {
    for (int R : rad)
        if (R > 31) return false;
    return true;
}

static int make_plan(cf_engine* h, int L, FftPlan& pl, zd** dtw, zf** dtwf = nullptr) {
    std::vector<int> rad = fft_radices(L);
    if (rad.size() > CF_FFT_MAXPASS) return fail(CF_E_UNSUPPORTED, "FFT length has too many factors");
    pl.L = L;
    pl.np = (int)rad.size();
    pl.rcode = 0;
    for (int i = 0; i < pl.np; ++i) pl.rcode |= (unsigned long long)rad[i] << (5 * i);
    std::vector<zd> tw(L);
    const long double twopi = 6.283185307179586476925286766559005768L;
    for (int k = 0; k < L; ++k) {
        long double a = -twopi * (long double)k / (long double)L;
        tw[k] = make_double2((double)cosl(a), (double)sinl(a));
    }
    int rc = dalloc(h, (void**)dtw, sizeof(zd) * L);
    if (rc) return rc;
    CU(cudaMemcpy(*dtw, tw.data(), sizeof(zd) * L, cudaMemcpyHostToDevice));
    pl.tw = *dtw;
    pl.twf = nullptr;
    if (dtwf) {
        std::vector<zf> twf(L);
        for (int k = 0; k < L; ++k) twf[k] = make_float2((float)tw[k].x, (float)tw[k].y);
        if ((rc = dalloc(h, (void**)dtwf, sizeof(zf) * L))) return rc;
        CU(cudaMemcpy(*dtwf, twf.data(), sizeof(zf) * L, cudaMemcpyHostToDevice));
        pl.twf = *dtwf;
    }
    return CF_OK;
}

static double kx_of(const cf_engine* h, int ix) { return 2 * M_PI / h->Lx * ix; }
static double lz_of(const cf_engine* h, int iz) { return 2 * M_PI / h->Lz * (iz <= (h->Nz >> 1) ? iz : iz - h->Nz); }

// Stokes bank for (nu, lambda): batchedinfluence.jl:45-98, meanmode.jl:45-67
static int build_bank(cf_engine* h, DevBank& bk, double nu, double lambda) {
    const int P = h->P, Ny = h->Ny;
    const long B = h->B;
    std::vector<double> fac_p((size_t)B * 3 * Ny), fac_v((size_t)B * 3 * Ny), resp((size_t)B * 6 * Ny);
    std::vector<double> colsc((size_t)B * 8, 0.0), sa((size_t)B * 4, 0.0);
    std::vector<char> bad(B, 0);
    setup::parallel_for(B, [&](long c) {
        const int ix = (int)(c % h->Nxh), iz = (int)(c / h->Nxh);
        const double k = kx_of(h, ix), l = lz_of(h, iz);
        const double kap2 = k * k + l * l;
        const double kp = kap2 == 0.0 ? 1.0 : kap2;  // zero-mode placeholder
        const double shift = lambda + nu * kap2;
        setup::Helm ph, vh;
        ph.init(P, 1.0, kp, false);
        vh.init(P, nu, shift, false);
        std::vector<double> zero(Ny, 0.0), work(Ny), pp(Ny), pm(Ny), vp(Ny), vm(Ny), p0(Ny), v0(Ny);
        ph.solve(zero.data(), 1.0, 0.0, pp.data());
        setup::diff(pp.data(), work.data(), P);
        vh.solve(work.data(), 0.0, 0.0, vp.data());
        ph.solve(zero.data(), 0.0, 1.0, pm.data());
        setup::diff(pm.data(), work.data(), P);
        vh.solve(work.data(), 0.0, 0.0, vm.data());
        double a = setup::wallderiv(vp.data(), P, true), b = setup::wallderiv(vm.data(), P, true);
        double cc = setup::wallderiv(vp.data(), P, false), d = setup::wallderiv(vm.data(), P, false);
        double scale = std::max(std::max(std::fabs(a), std::fabs(b)), std::max(std::fabs(cc), std::fabs(d)));
        double inv[4] = {0, 0, 0, 0};
        if (!(std::isfinite(scale) && scale > 0)) {
            bad[c] = 1;
        } else {
            a /= scale; b /= scale; cc /= scale; d /= scale;
            double det = a * d - b * cc;
            if (!(std::isfinite(det) && std::fabs(det) > 2.220446049250313e-16 * std::max(std::fabs(a * d), std::fabs(b * cc)))) {
                bad[c] = 1;
            } else {
                inv[0] = d / (det * scale); inv[1] = -b / (det * scale);
                inv[2] = -cc / (det * scale); inv[3] = a / (det * scale);
            }
        }
        // auxiliary tau problem with source (T_{P-1} + T_P)'
        std::vector<double> src(Ny, 0.0), forcing(Ny);
        src[P - 1] = 1.0; src[P] = 1.0;
        setup::diff(src.data(), forcing.data(), P);
        ph.solve(forcing.data(), 0.0, 0.0, p0.data());
        setup::diff(p0.data(), forcing.data(), P);
        vh.solve(forcing.data(), 0.0, 0.0, v0.data());
        {
            double up = 0, lo = 0;
            for (int n = 1; n <= P; ++n) {
                double t = (double)n * n * v0[n];
                up -= t;
                lo -= (n % 2 == 1 ? 1.0 : -1.0) * t;
            }
            double dp = inv[0] * up + inv[1] * lo, dm = inv[2] * up + inv[3] * lo;
            for (int n = 0; n <= P; ++n) {
                p0[n] += dp * pp[n] + dm * pm[n];
                v0[n] += dp * vp[n] + dm * vm[n];
            }
        }
        setup::diff(p0.data(), forcing.data(), P);
        double* csc = &colsc[(size_t)c * 8];
        for (int i = 0; i < 4; ++i) csc[i] = inv[i];
        csc[4] = shift * v0[P - 1] + forcing[P - 1];
        csc[5] = shift * v0[P];
        csc[6] = shift;
        csc[7] = kp;
        double* fp = &fac_p[(size_t)c * 3 * Ny];
        double* fv = &fac_v[(size_t)c * 3 * Ny];
        for (int n = 0; n < Ny; ++n) {
            fp[n] = ph.alpha[n]; fp[Ny + n] = ph.invden[n]; fp[2 * Ny + n] = ph.W[n];
            fv[n] = vh.alpha[n]; fv[Ny + n] = vh.invden[n]; fv[2 * Ny + n] = vh.W[n];
        }
        double* s4 = &sa[(size_t)c * 4];
        s4[0] = ph.SA[0]; s4[1] = ph.SA[1]; s4[2] = vh.SA[0]; s4[3] = vh.SA[1];
        double* rs = &resp[(size_t)c * 6 * Ny];
        const std::vector<double>* v6[6] = {&pp, &pm, &vp, &vm, &p0, &v0};
        for (int i = 0; i < 6; ++i) std::memcpy(rs + (size_t)i * Ny, v6[i]->data(), sizeof(double) * Ny);
    });
    for (long c = 0; c < B; ++c)
        if (bad[c]) return fail(CF_E_SINGULAR, "singular influence matrix for system " + std::to_string(c + 1));
    // mean mode (nu D^2 - lambda) c = 1, c(+-1) = 0
    if (!(std::isfinite(nu) && nu > 0 && std::isfinite(lambda) && lambda >= 0))
        return fail(CF_E_ARG, "nu must be finite and positive, lambda finite and nonnegative");
    setup::Helm mh;
    mh.init(P, nu, lambda, false);
    std::vector<double> e0(Ny, 0.0), mc(Ny);
    e0[0] = 1.0;
    mh.solve(e0.data(), 0.0, 0.0, mc.data());
    bk.meanc_mean = setup::bulkmean(mc.data(), P);
    if (!(std::isfinite(bk.meanc_mean) && bk.meanc_mean != 0.0))
        return fail(CF_E_ARG, "the uniform-gradient response has no finite nonzero bulk mean");
    int rc;
    if (!bk.fac_p) {
        if ((rc = dalloc(h, (void**)&bk.fac_p, fac_p.size() * 8))) return rc;
        if ((rc = dalloc(h, (void**)&bk.fac_v, fac_v.size() * 8))) return rc;
        if ((rc = dalloc(h, (void**)&bk.resp, resp.size() * 8))) return rc;
        if ((rc = dalloc(h, (void**)&bk.colsc, colsc.size() * 8))) return rc;
        if ((rc = dalloc(h, (void**)&bk.sa, sa.size() * 8))) return rc;
        if ((rc = dalloc(h, (void**)&bk.meanc, Ny * 8))) return rc;
    }
    CU(cudaMemcpy(bk.fac_p, fac_p.data(), fac_p.size() * 8, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(bk.fac_v, fac_v.data(), fac_v.size() * 8, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(bk.resp, resp.data(), resp.size() * 8, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(bk.colsc, colsc.data(), colsc.size() * 8, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(bk.sa, sa.data(), sa.size() * 8, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(bk.meanc, mc.data(), Ny * 8, cudaMemcpyHostToDevice));
    bk.nu = nu;
    bk.lambda = lambda;
    bk.ready = true;
    return CF_OK;
}

// Neumann pressure factors (pressure.jl:131-177): th0 = 1, th1 = kappa^2
static int build_neumann(cf_engine* h) {
    DevBank& bk = h->neum;
    if (bk.ready) return CF_OK;
    const int P = h->P, Ny = h->Ny;
    const long B = h->B;
    std::vector<double> fac((size_t)B * 3 * Ny, 0.0), sa((size_t)B * 4, 1.0);
    setup::parallel_for(B, [&](long c) {
        const int ix = (int)(c % h->Nxh), iz = (int)(c / h->Nxh);
        const double k = kx_of(h, ix), l = lz_of(h, iz);
        const double kap2 = k * k + l * l;
        if (kap2 == 0.0) return;
        setup::Helm hn;
        hn.init(P, 1.0, kap2, true);
        double* f = &fac[(size_t)c * 3 * Ny];
        for (int n = 0; n < Ny; ++n) { f[n] = hn.alpha[n]; f[Ny + n] = hn.invden[n]; f[2 * Ny + n] = hn.W[n]; }
        sa[(size_t)c * 4 + 0] = hn.SA[0];
        sa[(size_t)c * 4 + 1] = hn.SA[1];
    });
    int rc;
    if ((rc = dalloc(h, (void**)&bk.fac_p, fac.size() * 8))) return rc;
    if ((rc = dalloc(h, (void**)&bk.sa, sa.size() * 8))) return rc;
    CU(cudaMemcpy(bk.fac_p, fac.data(), fac.size() * 8, cudaMemcpyHostToDevice));
    CU(cudaMemcpy(bk.sa, sa.data(), sa.size() * 8, cudaMemcpyHostToDevice));
    bk.ready = true;
    return CF_OK;
}

// column strides (complex) in shared memory: regions 0-5 hold parity-split
// vectors (2 (P/2 + 1) entries), regions 6-7 transform buffers (fft_bufsz(P))
// column vector regions: both parity halves (2 hs) and 2 more, so that the
// stride is 2 mod 8 complex (bank groups of the two-column tiles)
static int col_stride(const cf_engine* h) { return 2 * col_half_stride(h->P) + 2; }
static int col_zstride(const cf_engine* h) { return std::max(2 * col_half_stride(h->P), fft_bufsz(h->P)); }
// per column: 6 vectors, 2 transform buffers and CF_TEAM_SCRATCH complex of team scratch
static size_t col_smem(const cf_engine* h, int ncol = CF_NCOL) {
    return ((size_t)ncol * (6 * col_stride(h) + 2 * col_zstride(h)) + CF_TEAM_SCRATCH * ncol) * sizeof(zd);
}

// The tensor-core forms' stage kernel at a compile-time length keeps six
// regions per column and no transform buffers (its Chebyshev transforms run
// outside): launched with zs = 0 and this shared memory.
static bool stage_mx_noz(const cf_engine* h) { return h->tc && col_static_length(h->P); }
static size_t stage_mx_smem(const cf_engine* h) {
    if (!stage_mx_noz(h)) return col_smem(h);
    return ((size_t)CF_NCOL * 6 * col_stride(h) + CF_TEAM_SCRATCH * CF_NCOL) * sizeof(zd);
}

// threads per block of the handle's column kernels
static int col_threads(const cf_engine* h) { return CF_NCOL * col_team_threads(h->P); }

static ColParams col_params(const cf_engine* h) {
    ColParams p;
    std::memset(&p, 0, sizeof(p));
    p.Nx = h->Nx; p.Nz = h->Nz; p.Nxh = h->Nxh; p.Ny = h->Ny; p.P = h->P; p.B = (int)h->B;
    p.cs = col_stride(h);
    p.zs = col_zstride(h);
    p.ax = 2 * M_PI / h->Lx; p.bz = 2 * M_PI / h->Lz;
    p.nu = h->nu;
    for (int i = 0; i < 3; ++i) { p.U[i] = h->U[i]; p.Q[i] = h->Q[i]; p.Nn[i] = h->nod[i]; p.Nout[i] = nullptr; }
    p.Pf = h->Pf;
    for (int i = 0; i < 6; ++i) p.nod[i] = h->nod[i];
    p.base = h->d_base; p.basecurv = h->d_basecurv;
    double bmc = setup::bulkmean(h->basecurv.data(), h->P);
    p.nu_bm_curv = h->nu * bmc;
    p.cmode = h->cmode;
    if (h->cmode == 1) { p.c1 = h->c1 - h->basemean; p.c2 = h->c2; }
    else { p.c1 = h->c1; p.c2 = h->c2; }
    p.grad_out = h->d_grad;
    p.plP = h->plP;
    p.cs_tab = h->d_cs;
    p.helm_tab = h->d_helmtab;
    p.fnorm = 1.0 / ((double)h->Nxp * h->Nzp * (h->Ny - 1));
    p.flags = h->d_status + 2;
    return p;
}

static FftParams fft_params(const cf_engine* h) {
    FftParams f;
    f.Nx = h->Nx; f.Nz = h->Nz; f.Nxh = h->Nxh; f.Ny = h->Ny; f.Nzp = h->Nzp; f.Nxp = h->Nxp;
    f.tks = ilog2(h->tkz);
    f.bsz = zbs(h);
    f.bsx = xbs(h);
    f.bsxp = fft_bufsz(h->Nxp);
    f.ax = 2 * M_PI / h->Lx; f.bz = 2 * M_PI / h->Lz;
    f.nod0 = h->nod[0]; f.nod1 = h->nod[1]; f.nod2 = h->nod[2]; f.nod3 = h->nod[3]; f.nod4 = h->nod[4]; f.nod5 = h->nod[5];
    f.zp0 = h->zp[0]; f.zp1 = h->zp[1]; f.zp2 = h->zp[2]; f.zp3 = h->zp[3]; f.zp4 = h->zp[4]; f.zp5 = h->zp[5];
    f.zp6 = h->zp[6]; f.zp7 = h->zp[7]; f.zp8 = h->zp[8];
    f.plZ = h->plZ; f.plX = h->plX;
    f.zbox = h->zbox; f.zpbox = h->zpbox;
    f.stoff = (int)zstage_off(h, sizeof(zd));
    f.err = h->d_ffterr;
    f.spins = h->wait_spins;
    return f;
}

// z-inverse (nf fields) or z-forward of the FP64 (f32 false) or FP32 fields:
// the TMA kernels when the maps could be encoded, else the gather kernels
static void launch_z(cf_engine* h, int which, bool f32, int nf, const FftParams& f) {
    const dim3 g((unsigned)((h->Nxh + h->tkz - 1) / h->tkz), (unsigned)h->Ny, (unsigned)nf);
    if (f32 ? h->tma32 : h->tma64) {
        fft_tma_kernel(which, h->Nzp, f32)<<<g, 256, zsmem_tma(h, f32 ? sizeof(zf) : sizeof(zd)), h->stream>>>(
            f, f32 ? h->maps32 : h->maps64);
    } else if (f32) {
        const int t = which == KF_ZINV ? h->tkz32 : h->tkz;
        FftParams ft = f;
        ft.tks = ilog2(t);
        ft.bsz = zbs_t(h, t);
        const dim3 g32((unsigned)((h->Nxh + t - 1) / t), (unsigned)h->Ny, (unsigned)nf);
        fft_kernel(which, h->Nzp, true)<<<g32, 256, zsmem_t(h, t, sizeof(zf)), h->stream>>>(ft);
    } else {
        fft_kernel(which, h->Nzp, false)<<<g, 256, zsmem(h), h->stream>>>(f);
    }
}

// Launch shapes of the periodic transforms of the handle's nonlinear form:
// fields through the z-inverse and the z-forward, the x-pass kernel and its
// rows per block.
struct PeriodicShape {
    int nzinv, nzfwd, xkind, xrows, xthreads;
};
static PeriodicShape periodic_shape(const cf_engine* h) {
    // in-place transforms where the butterflies fit the block (half the shared
    // memory, more blocks per SM)
    const bool ip = h->Nxp == 512 || h->Nxp == 576;
    if (h->form == NL_CONV) return ip ? PeriodicShape{9, 3, KF_XPASS_CONV_IP, 1, 512} : PeriodicShape{9, 3, KF_XPASS_CONV, 1, 256};
    if (h->form == NL_DIV) return ip ? PeriodicShape{3, 6, KF_XPASS_DIV_IP, 2, 512} : PeriodicShape{3, 6, KF_XPASS_DIV, 2, 256};
    // one z-row per block from Nxp > 256 (measured: 2.94 against 3.16 ms at
    // Nxp = 576), two below (0.18 against 0.23 ms at Nxp = 192)
    if (h->Nxp <= 256) return {6, 3, KF_XPASS2, 2, 256};
    if (ip) return {6, 3, KF_XPASS_IP, 1, 256};
    return {6, 3, KF_XPASS, 1, 256};
}
// dynamic shared memory of the x-pass kind
static size_t xpass_smem(const cf_engine* h, int kind) {
    if (kind == KF_XPASS_IP) return xsmem(h, 3);
    if (kind == KF_XPASS || kind == KF_XPASS_CONV_IP || kind == KF_XPASS_DIV_IP) return xsmem(h, 6);
    return xsmem(h, 12);
}
static int launch_periodic_kernels(cf_engine* h, cudaEvent_t* ev) {
    FftParams f = fft_params(h);
    const PeriodicShape s = periodic_shape(h);
    const size_t smx = xpass_smem(h, s.xkind);
    launch_z(h, KF_ZINV, false, s.nzinv, f);
    if (ev) CU(cudaEventRecord(ev[0], h->stream));
    const dim3 gx((unsigned)((h->Nzp + s.xrows - 1) / s.xrows), (unsigned)h->Ny);
    fft_kernel(s.xkind, h->Nxp)<<<gx, s.xthreads, smx, h->stream>>>(f);
    if (ev) CU(cudaEventRecord(ev[1], h->stream));
    launch_z(h, KF_ZFWD, false, s.nzfwd, f);
    CU(cudaGetLastError());
    return CF_OK;
}

static unsigned col_blocks(const cf_engine* h) { return (unsigned)((h->B + CF_NCOL - 1) / CF_NCOL); }

// Nonlinear periodic transforms: nodal fields -> the nonlinear term at the
// nodes (nod[0..2]); for the divergence form the six products at the nodes,
// then k_column_div: N as coefficients into Nout (nod[0..2] when null).
static int launch_periodic(cf_engine* h, int* count, zd* const* Nout = nullptr) {
    int rc = launch_periodic_kernels(h, nullptr);
    if (rc) return rc;
    if (count) *count += 3;
    if (h->form == NL_DIV) {
        ColParams p = col_params(h);
        for (int i = 0; i < 3; ++i) p.Nout[i] = Nout ? Nout[i] : h->nod[i];
        col_kernel(KC_DIV, h->P)<<<col_blocks(h), col_threads(h), col_smem(h), h->stream>>>(p);
        if (count) *count += 1;
        CU(cudaGetLastError());
    }
    return CF_OK;
}
// kernel launches of one CNRK2 step (FP64 forms)
static int step_launches(const cf_engine* h) { return h->form == NL_DIV ? 15 : 12; }

static int launch_prep(cf_engine* h, zd* const Usrc[3], int* count) {
    ColParams p = col_params(h);
    for (int i = 0; i < 3; ++i) p.U[i] = Usrc[i];
    const int kc = h->form == NL_CONV ? KC_PREP_CONV : (h->form == NL_DIV ? KC_PREP_DIV : KC_PREP);
    col_kernel(kc, h->P)<<<col_blocks(h), col_threads(h), col_smem(h), h->stream>>>(p);
    if (count) *count += 1;
    CU(cudaGetLastError());
    return CF_OK;
}

// column-kernel parameters of CNRK2 stage j (cnrk2.jl:170-205)
static ColParams stage_col_params(const cf_engine* h, int j) {
    ColParams p = col_params(h);
    p.lambda = 1.0 / (CC[j] * h->dt);
    p.weight = CB[j] / CC[j];
    p.Acoef = CA[j];
    p.stage = j;
    p.store_q = (j < 2) ? 1 : 0;
    p.bank = h->bank[j].view();
    return p;
}
static int stage_kernel_kind(const cf_engine* h) {
    return h->form == NL_CONV ? KC_STAGE_CONV : (h->form == NL_DIV ? KC_STAGE_DIV : KC_STAGE);
}
static int launch_stage(cf_engine* h, int j, int* count) {
    int rc = launch_periodic(h, count);
    if (rc) return rc;
    ColParams p = stage_col_params(h, j);
    col_kernel(stage_kernel_kind(h), h->P)<<<col_blocks(h), col_threads(h), col_smem(h), h->stream>>>(p);
    if (count) *count += 1;
    CU(cudaGetLastError());
    return CF_OK;
}

// Same launches as one step, with events around every kernel class (zinv,
// xpass, zfwd, column; the divergence form's k_column_div counts with the
// column kernel) recorded on the handle's stream.
static int launch_step_profiled(cf_engine* h, cudaEvent_t* ev, double* acc) {
    for (int j = 0; j < 3; ++j) {
        ColParams p = stage_col_params(h, j);
        CU(cudaEventRecord(ev[0], h->stream));
        int rc = launch_periodic_kernels(h, ev + 1);
        if (rc) return rc;
        CU(cudaEventRecord(ev[3], h->stream));
        if (h->form == NL_DIV) {
            ColParams pd = col_params(h);
            for (int i = 0; i < 3; ++i) pd.Nout[i] = h->nod[i];
            col_kernel(KC_DIV, h->P)<<<col_blocks(h), col_threads(h), col_smem(h), h->stream>>>(pd);
        }
        col_kernel(stage_kernel_kind(h), h->P)<<<col_blocks(h), col_threads(h), col_smem(h), h->stream>>>(p);
        CU(cudaEventRecord(ev[4], h->stream));
        CU(cudaGetLastError());
        CU(cudaEventSynchronize(ev[4]));
        for (int k = 0; k < 4; ++k) {
            float ms = 0.f;
            CU(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
            acc[k] += ms;
        }
    }
    return CF_OK;
}

static int ensure_banks(cf_engine* h) {
    for (int j = 0; j < 3; ++j)
        if (!h->bank[j].ready) {
            int rc = build_bank(h, h->bank[j], h->nu, 1.0 / (CC[j] * h->dt));
            if (rc) return rc;
        }
    return CF_OK;
}

static void drop_graph(cf_engine* h) {
    if (h->graph) {
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
    }
}

// ---------------------------------------------------------------------------
// Mixed-precision form (CF_PRECISION_MIXED).  Per stage: FP32 z-inverse,
// x-pass (products in FP32) and z-forward transforms of the nonlinear term;
// the forward Chebyshev transform of N on the tensor cores; the FP64 column
// kernel without its DCTs (right-hand side, Stokes, influence and tau
// corrections, mean mode and flux constraint, curl in coefficient space); the
// inverse Chebyshev transform of the six fields on the tensor cores, in place.
// ---------------------------------------------------------------------------
typedef void (*ChebKernel)(ChebParams);
typedef void (*ChebSymKernel)(ChebSymParams);
static void cheb_images(int Ny, int inverse, double scale, int split, std::vector<unsigned char>& img, int& NP,
                        int& nkt);
static size_t cheb_smem(int NPs, int split);
static int cheb_stages(int NPs, int split);
static void cheb_dims(int Ny, int& NPs, int& nsplit, int& NP);
static int cheb_pieces(int split);
static size_t cheb_piece_bytes(int Ny, int split);
static ChebKernel cheb_kernel(int split);
static bool cheb_sym_dims(int Ny, int split, ChebSymDims& d);
static void cheb_sym_images(int Ny, int inverse, double scale, int split, const ChebSymDims& d,
                            std::vector<unsigned char>& img);
static ChebSymKernel cheb_sym_kernel(int split);
static int cheb_sym_grid(long C, int nf);

// ---- FP32 state (CF_PRECISION_MIXED_F32STATE): the FP64 copy of U and P
// and the FP32 state the steps advance, converted on demand.
// The mean-flow mode (column 0 of each field) stays FP64 in mean[f][n]:
// rounding copies it there, widening takes it from there.
struct StateCopy {
    const void* src[4];
    void* dst[4];
    zd* mean;
    long B;
};
static __global__ void __launch_bounds__(256) k_state_convert(StateCopy a, long n, int to32) {
    const long tot = 4 * n, stride = (long)gridDim.x * blockDim.x, ny = n / a.B;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < tot; i += stride) {
        const int f = (int)(i / n);
        const long e = i - f * n;
        const bool mean = e % a.B == 0;
        if (to32) {
            const zd v = static_cast<const zd*>(a.src[f])[e];
            static_cast<zf*>(a.dst[f])[e] = to_zf(v);
            if (mean) a.mean[f * ny + e / a.B] = v;
        } else {
            static_cast<zd*>(a.dst[f])[e] =
                mean ? a.mean[f * ny + e / a.B] : to_zd(static_cast<const zf*>(a.src[f])[e]);
        }
    }
}
static int state_convert(cf_engine* h, bool to32) {
    StateCopy a;
    for (int i = 0; i < 3; ++i) {
        a.src[i] = to32 ? (const void*)h->U[i] : h->U32[i];
        a.dst[i] = to32 ? h->U32[i] : (void*)h->U[i];
    }
    a.src[3] = to32 ? (const void*)h->Pf : h->P32;
    a.dst[3] = to32 ? h->P32 : (void*)h->Pf;
    a.mean = h->mean64;
    a.B = h->B;
    k_state_convert<<<4 * 148, 256, 0, h->stream>>>(a, h->nr, to32 ? 1 : 0);
    CU(cudaGetLastError());
    return CF_OK;
}
// the FP32 state made current before a step reads it (rounded from the FP64
// copy after a state entry point wrote that)
static int state_to32(cf_engine* h) {
    if (!h->s32 || h->valid32) return CF_OK;
    int rc = state_convert(h, true);
    if (rc) return rc;
    h->valid32 = true;
    return CF_OK;
}
// the FP64 copy made current before an entry point reads it
static int state_to64(cf_engine* h) {
    if (!h->s32 || h->valid64) return CF_OK;
    int rc = state_convert(h, false);
    if (rc) return rc;
    h->valid64 = true;
    return CF_OK;
}
// after an entry point wrote the FP64 copy / a step advanced the FP32 state
static void state_wrote64(cf_engine* h) {
    if (h->s32) h->valid64 = true, h->valid32 = false;
}
static void state_stepped(cf_engine* h) {
    if (h->s32) h->valid32 = true, h->valid64 = false;
}
// column-kernel parameters of the mixed form's own kernels: the FP32 state
// buffers in place of the FP64 ones (F32STATE)
static void mx_state(const cf_engine* h, ColParams& p) {
    if (!h->s32) return;
    for (int i = 0; i < 3; ++i) {
        p.U[i] = static_cast<zd*>(h->U32[i]);
        p.Q[i] = static_cast<zd*>(h->Q32[i]);
    }
    p.Pf = static_cast<zd*>(h->P32);
    p.mean64 = h->mean64;
}

static FftParams fft_params32(const cf_engine* h) {
    FftParams f = fft_params(h);
    f.nod0 = h->nod32[0]; f.nod1 = h->nod32[1]; f.nod2 = h->nod32[2];
    f.nod3 = h->nod32[3]; f.nod4 = h->nod32[4]; f.nod5 = h->nod32[5];
    f.zp0 = h->zp32[0]; f.zp1 = h->zp32[1]; f.zp2 = h->zp32[2];
    f.zp3 = h->zp32[3]; f.zp4 = h->zp32[4]; f.zp5 = h->zp32[5];
    f.stoff = (int)zstage_off(h, sizeof(zf));
    return f;
}
// FP32 x-pass: in place, one row per block, where the length has an in-place
// plan (Nxp = 512, 576); else two rows per block between ping-pong buffers
static void launch_xpass32(cf_engine* h, const FftParams& f) {
    if (h->Nxp == 512 || h->Nxp == 576) {
        const int bs = h->Nxp == 512 ? fft_bufsz_pos<2>(512) : fft_bufsz_pos<2>(576);
        fft_kernel(KF_XPASS_IP, h->Nxp, true)<<<dim3((unsigned)h->Nzp, (unsigned)h->Ny), 256,
                                                 3 * bs * sizeof(zf), h->stream>>>(f);
        return;
    }
    dim3 gx((unsigned)((h->Nzp + 1) / 2), (unsigned)h->Ny);
    fft_kernel(KF_XPASS, h->Nxp, true)<<<gx, 256, xsmem(h) / 2, h->stream>>>(f);
}
static int launch_periodic32(cf_engine* h, int* count) {
    FftParams f = fft_params32(h);
    launch_z(h, KF_ZINV, true, 6, f);
    launch_xpass32(h, f);
    launch_z(h, KF_ZFWD, true, 3, f);
    if (count) *count += 3;
    CU(cudaGetLastError());
    return CF_OK;
}
// Chebyshev transform of the first nf FP32 fields (forward: N at the nodes,
// nod32 -> normalised coefficients, coef32; inverse: coefficients, coef32 ->
// nodal values, nod32).  Out of place: the two blocks that share a column tile
// when the output degrees are split both read all of its input rows.
static int launch_cheb(cf_engine* h, int nf, bool inverse, int* count) {
    if (h->chebsym) {
        ChebSymParams q;
        std::memset(&q, 0, sizeof(q));
        const ChebSymDims& d = h->symd;
        q.P = h->P;
        for (int i = 0; i < 2; ++i) {
            q.N[i] = d.N[i];
            q.Npad[i] = d.Npad[i];
            q.Kpad[i] = d.Kpad[i];
            q.bbytes[i] = d.bbytes[i];
        }
        q.nst = d.nst;
        q.C = 2 * h->B;
        q.nf = nf;
        q.ntiles = (int)((q.C + 127) / 128);
        for (int f = 0; f < nf; ++f) {
            q.X[f] = static_cast<const float*>(inverse ? h->coef32[f] : h->nod32[f]);
            q.Y[f] = static_cast<float*>(inverse ? h->nod32[f] : h->coef32[f]);
        }
        const unsigned char* img = inverse ? h->d_chebI : h->d_chebF;
        q.B[0] = img;
        q.B[1] = img + (size_t)cheb_pieces(h->split) * d.bbytes[0];
        q.err = h->d_cheberr;
        q.spins = h->wait_spins;
        cheb_sym_kernel(h->split)<<<cheb_sym_grid(q.C, nf), 416, d.smem, h->stream>>>(q);
        if (count) *count += 1;
        CU(cudaGetLastError());
        return CF_OK;
    }
    ChebParams p;
    std::memset(&p, 0, sizeof(p));
    p.Ny = h->Ny;
    p.NP = h->chebNP;
    p.nkt = h->chebKT;
    int NPs, nsplit, NPt;
    cheb_dims(h->Ny, NPs, nsplit, NPt);
    p.NPs = NPs;
    p.nst = cheb_stages(NPs, h->split);
    p.C = 2 * h->B;
    for (int f = 0; f < nf; ++f) {
        p.X[f] = static_cast<const float*>(inverse ? h->coef32[f] : h->nod32[f]);
        p.Y[f] = static_cast<float*>(inverse ? h->nod32[f] : h->coef32[f]);
    }
    const unsigned char* img = inverse ? h->d_chebI : h->d_chebF;
    const size_t pb = cheb_piece_bytes(h->Ny, h->split);
    for (int q = 0; q < cheb_pieces(h->split); ++q) p.B[q] = img + q * pb;
    p.err = h->d_cheberr;
    p.spins = h->wait_spins;
    dim3 grid((unsigned)((p.C + CF_CHEB_MT - 1) / CF_CHEB_MT), (unsigned)nf, (unsigned)nsplit);
    cheb_kernel(h->split)<<<grid, 128, cheb_smem(NPs, h->split), h->stream>>>(p);
    if (count) *count += 1;
    CU(cudaGetLastError());
    return CF_OK;
}
static int launch_stage_mx(cf_engine* h, int j, int* count) {
    int rc;
    if ((rc = launch_periodic32(h, count))) return rc;
    if (!h->tc) {
        // FP32 nodal fields in and out, Chebyshev transforms in the column kernel
        ColParams p = stage_col_params(h, j);
        for (int i = 0; i < 3; ++i) p.Nn[i] = static_cast<const zd*>(h->nod32[i]);
        for (int i = 0; i < 6; ++i) p.nod[i] = static_cast<zd*>(h->nod32[i]);
        mx_state(h, p);
        col_kernel(h->s32 ? KC_STAGE_MXS : KC_STAGE_MXD, h->P)<<<col_blocks(h), col_threads(h), col_smem(h),
                                                                 h->stream>>>(p);
        if (count) *count += 1;
        CU(cudaGetLastError());
        return CF_OK;
    }
    if ((rc = launch_cheb(h, 3, false, count))) return rc;
    ColParams p = stage_col_params(h, j);
    for (int i = 0; i < 3; ++i) p.Nn[i] = static_cast<const zd*>(h->coef32[i]);
    for (int i = 0; i < 6; ++i) p.nod[i] = static_cast<zd*>(h->coef32[i]);
    if (stage_mx_noz(h)) p.zs = 0;
    col_kernel(KC_STAGE_MX, h->P)<<<col_blocks(h), col_threads(h), stage_mx_smem(h), h->stream>>>(p);
    if (count) *count += 1;
    CU(cudaGetLastError());
    return launch_cheb(h, 6, true, count);
}
static int launch_prep_mx(cf_engine* h, int* count) {
    ColParams p = col_params(h);
    if (!h->tc) {
        for (int i = 0; i < 6; ++i) p.nod[i] = static_cast<zd*>(h->nod32[i]);
        mx_state(h, p);
        col_kernel(h->s32 ? KC_PREP_MXS : KC_PREP_MXD, h->P)<<<col_blocks(h), col_threads(h), col_smem(h),
                                                               h->stream>>>(p);
        if (count) *count += 1;
        CU(cudaGetLastError());
        return CF_OK;
    }
    for (int i = 0; i < 6; ++i) p.nod[i] = static_cast<zd*>(h->coef32[i]);
    col_kernel(KC_PREP_MX, h->P)<<<col_blocks(h), col_threads(h), col_smem(h), h->stream>>>(p);
    if (count) *count += 1;
    CU(cudaGetLastError());
    return launch_cheb(h, 6, true, count);
}
// Wait for the handle's stream and report what its kernels flagged since the
// last check (each flag is reported once, then cleared): a bounded wait that
// gave up (CF_E_CUDA; the output of that launch is not valid) or a non-finite
// mean mode (CF_E_NONFINITE: a NaN or Inf anywhere in the state reaches the
// (0,0) mode through the nonlinear term within one stage).
// The calls that do not step (nonlinear term, projection, pressure,
// diagnostics) report the wait flags only and leave a non-finite flag of an
// earlier step for the next step-synchronising call (with_state false).
static int check_status(cf_engine* h, bool with_state = true) {
    int st[4];
    CU(cudaMemcpyAsync(st, h->d_status, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    const int n = with_state ? 3 : 2;
    if (!(st[0] | st[1] | (with_state ? st[2] : 0))) return CF_OK;
    CU(cudaMemsetAsync(h->d_status, 0, n * sizeof(int), h->stream));
    CU(cudaStreamSynchronize(h->stream));
    if (st[0]) return fail(CF_E_CUDA, "z transform kernel: a TMA wait timed out");
    if (st[1]) return fail(CF_E_CUDA, "Chebyshev transform kernel: a tensor-core wait timed out");
    return fail(CF_E_NONFINITE, "the state became non-finite (NaN or Inf in the mean mode)");
}
// mixed step with per-kernel event timing: kernel_ms = [z-inverse, x-pass,
// z-forward, column, forward Chebyshev, inverse Chebyshev] summed over steps
static int step_profiled_mx(cf_engine* h, double t, int nsteps, double* t_out, double* kernel_ms) {
    int rc = CF_OK, cnt = 0;
    if ((rc = state_to32(h))) return rc;
    if (!h->nodal_valid) {
        if ((rc = launch_prep_mx(h, &cnt))) return rc;
        h->nodal_valid = true;
    }
    cudaEvent_t ev[7];
    for (int k = 0; k < 7; ++k) CU(cudaEventCreate(&ev[k]));
    for (int k = 0; k < 6; ++k) kernel_ms[k] = 0.0;
    FftParams f = fft_params32(h);
    const int order[6] = {0, 1, 2, 4, 3, 5};  // launch order -> kernel_ms slot
    for (int s = 0; s < nsteps && rc == CF_OK; ++s)
        for (int j = 0; j < 3 && rc == CF_OK; ++j) {
            ColParams p = stage_col_params(h, j);
            void* const* io = h->tc ? h->coef32 : h->nod32;
            for (int i = 0; i < 3; ++i) p.Nn[i] = static_cast<const zd*>(io[i]);
            for (int i = 0; i < 6; ++i) p.nod[i] = static_cast<zd*>(io[i]);
            mx_state(h, p);
            if (stage_mx_noz(h)) p.zs = 0;
            cudaEventRecord(ev[0], h->stream);
            launch_z(h, KF_ZINV, true, 6, f);
            cudaEventRecord(ev[1], h->stream);
            launch_xpass32(h, f);
            cudaEventRecord(ev[2], h->stream);
            launch_z(h, KF_ZFWD, true, 3, f);
            cudaEventRecord(ev[3], h->stream);
            if (h->tc && (rc = launch_cheb(h, 3, false, nullptr))) break;
            cudaEventRecord(ev[4], h->stream);
            col_kernel(h->tc ? KC_STAGE_MX : (h->s32 ? KC_STAGE_MXS : KC_STAGE_MXD), h->P)<<<
                col_blocks(h), col_threads(h), h->tc ? stage_mx_smem(h) : col_smem(h), h->stream>>>(p);
            cudaEventRecord(ev[5], h->stream);
            if (h->tc && (rc = launch_cheb(h, 6, true, nullptr))) break;
            cudaEventRecord(ev[6], h->stream);
            if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(ev[6]) != cudaSuccess) {
                rc = fail(CF_E_CUDA, "mixed step failed");
                break;
            }
            for (int k = 0; k < 6; ++k) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
                kernel_ms[order[k]] += ms;
            }
        }
    for (int k = 0; k < 7; ++k) cudaEventDestroy(ev[k]);
    state_stepped(h);
    if (rc) return rc;
    if ((rc = check_status(h))) return rc;
    h->last_launches = cnt + (h->tc ? 18 : 12) * nsteps;
    if (t_out) *t_out = t + nsteps * h->dt;
    return CF_OK;
}

static int build_graph(cf_engine* h) {
    if (h->graph) return CF_OK;
    cudaGraph_t g;
    CU(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int cnt = 0, rc = CF_OK;
    for (int j = 0; j < 3 && rc == CF_OK; ++j) rc = h->mixed ? launch_stage_mx(h, j, &cnt) : launch_stage(h, j, &cnt);
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(CF_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&h->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(CF_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    return CF_OK;
}

// Tensor maps of the z kernels' TMA row transfers.  The encoder is the
// driver's cuTensorMapEncodeTiled, looked up through the runtime (no driver
// library link).  Returns false (the gather kernels are used) when a map
// cannot be encoded, e.g. a row stride that is not a multiple of 16 bytes.
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled_fn() {
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
        else
            cudaGetLastError();
    }
    return fn;
}
// one field: complex elements (2 scalars) of es bytes, (Nxh, rows, Ny), box (tkz, box rows, 1)
static bool encode_field(const cf_engine* h, CUtensorMap* m, void* base, int rows, int box, bool f32) {
    EncodeTiledFn fn = encode_tiled_fn();
    if (!fn || !base) return false;
    const size_t sc = f32 ? 4 : 8;
    const cuuint64_t dims[3] = {(cuuint64_t)2 * h->Nxh, (cuuint64_t)rows, (cuuint64_t)h->Ny};
    const cuuint64_t strides[2] = {(cuuint64_t)2 * h->Nxh * sc, (cuuint64_t)2 * h->Nxh * rows * sc};
    const cuuint32_t boxd[3] = {(cuuint32_t)(2 * h->tkz), (cuuint32_t)box, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    return fn(m, f32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims, strides,
              boxd, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
static void encode_maps(cf_engine* h) {
    std::memset(&h->maps64, 0, sizeof(FftMaps));
    std::memset(&h->maps32, 0, sizeof(FftMaps));
    // only for narrow column groups: with tkz >= 4 the gathered row segments
    // are 64 bytes or more and the plain loads cost less than the staging
    // (measured: TMA 1.71 against 1.79 ms for the z-inverse at tkz = 2,
    // 0.119 against 0.091 ms at tkz = 8)
    bool ok = h->d_ffterr != nullptr && h->tkz <= 2;
    for (int i = 0; i < 6 && ok; ++i)
        if (h->nod[i]) ok = encode_field(h, &h->maps64.nod[i], h->nod[i], h->Nz, h->zbox, false);
    for (int i = 0; i < 9 && ok; ++i)
        if (h->zp[i]) ok = encode_field(h, &h->maps64.zp[i], h->zp[i], h->Nzp, h->zpbox, false);
    ok = ok && zstage_rows(h) <= zbs(h);
    h->tma64 = ok && zsmem_tma(h, sizeof(zd)) <= (size_t)227 * 1024;
    if (h->mixed) {
        ok = h->d_ffterr != nullptr && h->tkz <= 2;
        for (int i = 0; i < 6 && ok; ++i) ok = encode_field(h, &h->maps32.nod[i], h->nod32[i], h->Nz, h->zbox, true);
        for (int i = 0; i < 6 && ok; ++i) ok = encode_field(h, &h->maps32.zp[i], h->zp32[i], h->Nzp, h->zpbox, true);
        h->tma32 = ok && zstage_rows(h) <= zbs(h) && zsmem_tma(h, sizeof(zf)) <= (size_t)227 * 1024;
    }
    h->tkz32 = h->tkz;
    if (h->mixed && !h->tma32) {
        const int t = std::min(2 * h->tkz, 32);
        if ((size_t)2 * t * zbs_t(h, t) * sizeof(zf) <= (size_t)74 * 1024) h->tkz32 = t;
    }
}

// Raise a kernel's dynamic shared-memory limit to at least `need`.  The limit
// belongs to the kernel, not to a handle: handles of different grids share the
// run-time-sized instantiations, so it is only ever raised.
static std::mutex g_attr_mu;
template <class K>
static int raise_smem_limit(K* fn, size_t need) {
    std::lock_guard<std::mutex> lock(g_attr_mu);
    cudaFuncAttributes a;
    CU(cudaFuncGetAttributes(&a, (const void*)fn));
    if ((size_t)a.maxDynamicSharedSizeBytes < need)
        CU(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need));
    return CF_OK;
}

static int set_attrs(cf_engine* h) {
    const int maxsm = 227 * 1024;
    size_t need[3] = {col_smem(h), zsmem(h), std::max(xsmem(h), xsmem(h, 6))};
    for (size_t x : need)
        if (x > (size_t)maxsm) return fail(CF_E_UNSUPPORTED, "grid too large for the shared-memory tiles");
    int rc;
    for (int w = 0; w < KC_COUNT; ++w)
        if ((rc = raise_smem_limit(col_kernel(w, h->P), need[0]))) return rc;
    if ((rc = raise_smem_limit(fft_kernel(KF_ZINV, h->Nzp), need[1]))) return rc;
    if ((rc = raise_smem_limit(fft_kernel(KF_ZFWD, h->Nzp), need[1]))) return rc;
    if ((rc = raise_smem_limit(fft_kernel(KF_XPASS, h->Nxp), need[2]))) return rc;
    if ((rc = raise_smem_limit(fft_kernel(KF_XPASS_CONV, h->Nxp), need[2]))) return rc;
    if ((rc = raise_smem_limit(fft_kernel(KF_XPASS_DIV, h->Nxp), need[2]))) return rc;
    if ((rc = raise_smem_limit(fft_kernel(KF_XPASS2, h->Nxp), need[2]))) return rc;
    if ((rc = raise_smem_limit(fft_kernel(KF_XPASS_IP, h->Nxp), xsmem(h, 3)))) return rc;
    if ((rc = raise_smem_limit(fft_kernel(KF_XPASS_CONV_IP, h->Nxp), xsmem(h, 6)))) return rc;
    if ((rc = raise_smem_limit(fft_kernel(KF_XPASS_DIV_IP, h->Nxp), xsmem(h, 6)))) return rc;
    if (h->tma64) {
        if ((rc = raise_smem_limit(fft_tma_kernel(KF_ZINV, h->Nzp, false), zsmem_tma(h, sizeof(zd))))) return rc;
        if ((rc = raise_smem_limit(fft_tma_kernel(KF_ZFWD, h->Nzp, false), zsmem_tma(h, sizeof(zd))))) return rc;
    }
    if (h->tma32) {
        if ((rc = raise_smem_limit(fft_tma_kernel(KF_ZINV, h->Nzp, true), zsmem_tma(h, sizeof(zf))))) return rc;
        if ((rc = raise_smem_limit(fft_tma_kernel(KF_ZFWD, h->Nzp, true), zsmem_tma(h, sizeof(zf))))) return rc;
    }
    if (h->mixed) {
        if ((rc = raise_smem_limit(fft_kernel(KF_ZINV, h->Nzp, true), zsmem_t(h, h->tkz32, sizeof(zf))))) return rc;
        if ((rc = raise_smem_limit(fft_kernel(KF_ZFWD, h->Nzp, true), zsmem_t(h, h->tkz, sizeof(zf))))) return rc;
        if ((rc = raise_smem_limit(fft_kernel(KF_XPASS, h->Nxp, true), need[2] / 2))) return rc;
    }
    if (h->mixed && h->tc) {
        int NPs, nsplit, NPt;
        cheb_dims(h->Ny, NPs, nsplit, NPt);
        if ((rc = raise_smem_limit(cheb_kernel(h->split), cheb_smem(NPs, h->split)))) return rc;
        if (h->chebsym && (rc = raise_smem_limit(cheb_sym_kernel(h->split), h->symd.smem))) return rc;
    }
    return CF_OK;
}

static int validate_and_size(cf_engine* h, const cf_config* c) {
    if (!(c->Ny >= 5 && c->Ny % 2 == 1)) return fail(CF_E_ARG, "Gibson's tau correction requires odd Ny >= 5");
    if (!(c->Nx > 0 && c->Nz > 0)) return fail(CF_E_ARG, "Nx and Nz must be positive");
    if (!(std::isfinite(c->Lx) && std::isfinite(c->Lz) && c->Lx > 0 && c->Lz > 0))
        return fail(CF_E_ARG, "Lx and Lz must be finite and positive");
    if (!(std::isfinite(c->dt) && c->dt > 0)) return fail(CF_E_ARG, "dt must be finite and positive");
    if (!(std::isfinite(c->nu) && c->nu > 0)) return fail(CF_E_ARG, "nu must be finite and positive");
    if (c->constraint != 0 && c->constraint != 1) return fail(CF_E_ARG, "unknown constraint kind");
    if (c->precision != CF_PRECISION_FP64 && c->precision != CF_PRECISION_MIXED &&
        c->precision != CF_PRECISION_MIXED_TC && c->precision != CF_PRECISION_MIXED_BF16 &&
        c->precision != CF_PRECISION_MIXED_F32STATE)
        return fail(CF_E_ARG, "unknown precision mode");
    if ((c->precision == CF_PRECISION_MIXED_TC || c->precision == CF_PRECISION_MIXED_BF16) && c->Ny > 512)
        return fail(CF_E_UNSUPPORTED, "the tensor-core Chebyshev transforms support Ny <= 512");
    h->mixed = c->precision != CF_PRECISION_FP64;
    h->tc = c->precision == CF_PRECISION_MIXED_TC || c->precision == CF_PRECISION_MIXED_BF16;
    h->split = c->precision == CF_PRECISION_MIXED_BF16 ? 1 : 0;
    h->s32 = c->precision == CF_PRECISION_MIXED_F32STATE;
    if (c->form != CF_FORM_ROTATIONAL && c->form != CF_FORM_CONVECTIVE && c->form != CF_FORM_DIVERGENCE)
        return fail(CF_E_ARG, "unknown nonlinear form");
    if (h->mixed && c->form != CF_FORM_ROTATIONAL)
        return fail(CF_E_UNSUPPORTED, "the mixed-precision form runs the rotational nonlinear term");
    h->form = c->form;
    if (!(std::isfinite(c->c1) && std::isfinite(c->c2))) return fail(CF_E_ARG, "mean-flow constraint values must be finite");
    h->Nx = c->Nx; h->Ny = c->Ny; h->Nz = c->Nz; h->Lx = c->Lx; h->Lz = c->Lz;
    h->nu = c->nu; h->dt = c->dt; h->cmode = c->constraint; h->c1 = c->c1; h->c2 = c->c2;
    h->P = h->Ny - 1;
    h->Nxh = h->Nx / 2 + 1;
    h->Nxp = (3 * h->Nx + 1) / 2;
    h->Nzp = (3 * h->Nz + 1) / 2;
    h->B = (long)h->Nxh * h->Nz;
    h->nr = h->B * h->Ny;
    h->nq = (long)h->Nxh * h->Nzp * h->Ny;
    if (col_smem(h) > (size_t)227 * 1024) return fail(CF_E_UNSUPPORTED, "Ny too large for the column kernel");
    std::vector<int> rP = fft_radices(h->P), rZ = fft_radices(h->Nzp), rX = fft_radices(h->Nxp);
    if (!radices_ok(rP) || rP.size() > CF_FFT_MAXPASS)
        return fail(CF_E_UNSUPPORTED, "Chebyshev transform length not supported (prime factors <= 31)");
    if (!radices_ok(rX) || rX.size() > CF_FFT_MAXPASS || (size_t)12 * rup8(h->Nxp) * 16 > 227 * 1024)
        return fail(CF_E_UNSUPPORTED, "padded x length not supported");
    if (!radices_ok(rZ) || rZ.size() > CF_FFT_MAXPASS)
        return fail(CF_E_UNSUPPORTED, "padded z length not supported");
    // z kernels: two tkz x Nzp buffers; keep them near 74 KB (three blocks per SM)
    h->tkz = 0;
    for (int t : {8, 4, 2, 1})
        if ((size_t)2 * t * (fft_bufsz(h->Nzp) + 1) * 16 <= 74 * 1024 || t == 1) { h->tkz = t; break; }
    if (zsmem(h) > (size_t)227 * 1024) return fail(CF_E_UNSUPPORTED, "padded z length not supported");
    // TMA boxes: at most 256 rows, a multiple of 8 rows (128-byte box strides
    // in the staging buffer for both element sizes)
    auto box_rows = [](int rows) {
        const int nb = (rows + 255) / 256;
        return ((rows + nb - 1) / nb + 7) & ~7;
    };
    h->zbox = box_rows(h->Nz);
    h->zpbox = box_rows(h->Nzp);
    return CF_OK;
}

// ---- host-buffer steps: the state crosses PCIe in kz-plane chunks that
// overlap the column kernels on either side of the step
//
// Chunk k holds the kz planes [zb[k], zb[k+1]) of every y plane: columns
// [zb[k] Nxh, zb[k+1] Nxh) (column c = kz Nxh + kx), whole column blocks when
// zb[k] Nxh is a multiple of CF_NCOL.  Returns the number of chunks.
static int host_chunks(const cf_engine* h, int* zb) {
    const int K = std::min(CF_HOST_CHUNKS, std::max(1, h->Nz / 2));
    zb[0] = 0;
    for (int k = 1; k < K; ++k) {
        int z = (int)((long)k * h->Nz / K);
        if (((long)z * h->Nxh) % CF_NCOL) z -= 1;  // Nxh odd: an even plane (Nz >= 2K keeps them increasing)
        zb[k] = z;
    }
    zb[K] = h->Nz;
    return K;
}
static unsigned chunk_block(const cf_engine* h, const int* zb, int K, int k) {
    return k >= K ? col_blocks(h) : (unsigned)(((long)zb[k] * h->Nxh) / CF_NCOL);
}
// copy kz planes [z0, z1) of every y plane of one field (pitched: a y plane
// is B = Nz Nxh complex, the chunk a contiguous run of it)
static int copy_planes(void* dst, const void* src, const cf_engine* h, int z0, int z1, cudaMemcpyKind kind,
                       cudaStream_t st) {
    const size_t pitch = sizeof(zd) * (size_t)h->B, off = sizeof(zd) * (size_t)z0 * h->Nxh;
    const size_t width = sizeof(zd) * (size_t)(z1 - z0) * h->Nxh;
    CU(cudaMemcpy2DAsync((char*)dst + off, pitch, (const char*)src + off, pitch, width, (size_t)h->Ny, kind, st));
    return CF_OK;
}
static int ensure_copy_stream(cf_engine* h) {
    if (h->cstream) return CF_OK;
    CU(cudaStreamCreateWithFlags(&h->cstream, cudaStreamNonBlocking));
    for (cudaEvent_t& e : h->hev) CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return CF_OK;
}
// column kernel over the blocks [b0, b1) of the columns
static int launch_cols(cf_engine* h, int kind, ColParams p, unsigned b0, unsigned b1, int* count) {
    if (b1 <= b0) return CF_OK;
    p.bofs = (int)b0;
    col_kernel(kind, h->P)<<<b1 - b0, col_threads(h), col_smem(h), h->stream>>>(p);
    if (count) *count += 1;
    CU(cudaGetLastError());
    return CF_OK;
}
// prep (nodal fields of the state) and stage-j column kernel of the FP64
// forms and of the mixed form with the Chebyshev transforms in the kernel
static int host_prep_kind(const cf_engine* h, ColParams& p) {
    p = col_params(h);
    if (h->mixed) {
        for (int i = 0; i < 6; ++i) p.nod[i] = static_cast<zd*>(h->nod32[i]);
        return KC_PREP_MXD;
    }
    return h->form == NL_CONV ? KC_PREP_CONV : (h->form == NL_DIV ? KC_PREP_DIV : KC_PREP);
}
static int host_stage_kind(const cf_engine* h, int j, ColParams& p) {
    p = stage_col_params(h, j);
    if (h->mixed) {
        for (int i = 0; i < 3; ++i) p.Nn[i] = static_cast<const zd*>(h->nod32[i]);
        for (int i = 0; i < 6; ++i) p.nod[i] = static_cast<zd*>(h->nod32[i]);
        return KC_STAGE_MXD;
    }
    return stage_kernel_kind(h);
}

static void host_synth(const cf_engine* h, uint64_t seed, double amp, int shape, double rho, std::vector<std::complex<double>>& U);

// Fixed scratch of cf_nonlinear_noalloc: one array per device (module
// scope, resident from module load until exit).  Host code names
// g_noalloc_scratch only through the device address that cudaGetSymbolAddress
// returns for the current device; cf_create looks it up with the handle's
// device current (every create refreshes it, so a context recreated after a
// device reset gets its own address; handles of the old context are invalid
// after such a reset anyway).
#define CF_MAX_DEVICES 64
static __device__ __align__(256) unsigned char g_noalloc_scratch[CF_NOALLOC_SCRATCH_BYTES];
static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[CF_MAX_DEVICES] = {};

static int noalloc_setup(int dev) {
    if (dev < 0 || dev >= CF_MAX_DEVICES) return fail(CF_E_UNSUPPORTED, "device ordinal out of range");
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return fail(CF_E_CUDA, std::string("scratch address: ") + cudaGetErrorString(e));
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    g_noalloc_addr[dev] = p;
    return CF_OK;
}
static void* noalloc_scratch(int dev) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    return (dev >= 0 && dev < CF_MAX_DEVICES) ? g_noalloc_addr[dev] : nullptr;
}

extern "C" {

const char* cf_last_error(void) { return g_err.c_str(); }

void cf_destroy(cf_handle* h) {
    if (!h) return;
    DeviceGuard dg_(h->device);
    drop_graph(h);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->cstream) cudaStreamSynchronize(h->cstream);
    for (void* p : h->allocs) cudaFree(p);
    for (cudaEvent_t e : h->hev)
        if (e) cudaEventDestroy(e);
    if (h->cstream) cudaStreamDestroy(h->cstream);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

int cf_create(const cf_config* cfg, cf_handle** out) {
    if (!cfg || !out) return fail(CF_E_ARG, "null argument");
    *out = nullptr;
    cf_engine* h = new cf_engine();
    int rc = validate_and_size(h, cfg);
    if (rc) { delete h; return rc; }
    // base profile at the nodes (problem.jl:92) and its coefficients (cnrk2.jl:58-82)
    std::vector<double> vals(h->Ny);
    for (int j = 0; j < h->Ny; ++j) {
        double y = (2 * j == h->P) ? 0.0 : std::cos(M_PI * j / h->P);
        if (cfg->profile == CF_PROFILE_COUETTE) vals[j] = y;
        else if (cfg->profile == CF_PROFILE_POISEUILLE) vals[j] = 1 - y * y;
        else if (cfg->profile == CF_PROFILE_VALUES && cfg->base_values) vals[j] = cfg->base_values[j];
        else { delete h; return fail(CF_E_ARG, "unknown base profile"); }
    }
    h->base.resize(h->Ny); h->basecurv.resize(h->Ny);
    setup::chebcoeffs(vals.data(), h->base.data(), h->P);
    std::vector<double> d1(h->Ny);
    setup::diff(h->base.data(), d1.data(), h->P);
    setup::diff(d1.data(), h->basecurv.data(), h->P);
    h->basemean = setup::bulkmean(h->base.data(), h->P);

    auto bail = [&](int code) { cf_destroy(h); return code; };
    if (cudaGetDevice(&h->device) != cudaSuccess) { delete h; return fail(CF_E_CUDA, "no CUDA device"); }
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(CF_E_CUDA, "cannot create stream (no CUDA device?)"));
    if ((rc = noalloc_setup(h->device))) return bail(rc);
    if ((rc = dalloc(h, (void**)&h->d_status, 4 * sizeof(int)))) return bail(rc);
    if (cudaMemset(h->d_status, 0, 4 * sizeof(int)) != cudaSuccess) return bail(fail(CF_E_CUDA, "upload failed"));
    h->d_ffterr = h->d_status;
    h->d_cheberr = h->d_status + 1;
    const size_t fr = sizeof(zd) * h->nr, fq = sizeof(zd) * h->nq;
    for (int i = 0; i < 3; ++i) {
        if ((rc = dalloc(h, (void**)&h->U[i], fr))) return bail(rc);
        if ((rc = dalloc(h, (void**)&h->Q[i], fr))) return bail(rc);
    }
    if ((rc = dalloc(h, (void**)&h->Pf, fr))) return bail(rc);
    for (int i = 0; i < 6; ++i)
        if ((rc = dalloc(h, (void**)&h->nod[i], fr))) return bail(rc);
    for (int i = 0; i < periodic_shape(h).nzinv || i < 6; ++i)
        if ((rc = dalloc(h, (void**)&h->zp[i], fq))) return bail(rc);
    if ((rc = dalloc(h, (void**)&h->d_base, 8 * h->Ny))) return bail(rc);
    if ((rc = dalloc(h, (void**)&h->d_basecurv, 8 * h->Ny))) return bail(rc);
    if ((rc = dalloc(h, (void**)&h->d_grad, 8 * 2))) return bail(rc);
    if (cudaMemcpy(h->d_base, h->base.data(), 8 * h->Ny, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(h->d_basecurv, h->basecurv.data(), 8 * h->Ny, cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(fail(CF_E_CUDA, "upload failed"));
    for (int i = 0; i < 3; ++i) cudaMemset(h->U[i], 0, fr), cudaMemset(h->Q[i], 0, fr);
    cudaMemset(h->Pf, 0, fr);
    cudaMemset(h->d_grad, 0, 16);
    if ((rc = make_plan(h, h->P, h->plP, &h->d_twP))) return bail(rc);
    if ((rc = make_plan(h, h->Nzp, h->plZ, &h->d_twZ, h->mixed ? &h->d_twZf : nullptr))) return bail(rc);
    if ((rc = make_plan(h, h->Nxp, h->plX, &h->d_twX, h->mixed ? &h->d_twXf : nullptr))) return bail(rc);
    if (h->mixed) {
        // FP32 work fields and (tensor-core transforms) the coefficient
        // fields and the two transform-matrix images
        for (int i = 0; i < 6; ++i) {
            if ((rc = dalloc(h, &h->nod32[i], sizeof(zf) * h->nr))) return bail(rc);
            if ((rc = dalloc(h, &h->zp32[i], sizeof(zf) * h->nq))) return bail(rc);
            if (h->tc && (rc = dalloc(h, &h->coef32[i], sizeof(zf) * h->nr))) return bail(rc);
        }
    }
    if (h->s32) {
        const size_t f32 = sizeof(zf) * h->nr;
        for (int i = 0; i < 3; ++i) {
            if ((rc = dalloc(h, &h->U32[i], f32))) return bail(rc);
            if ((rc = dalloc(h, &h->Q32[i], f32))) return bail(rc);
            cudaMemset(h->U32[i], 0, f32);
            cudaMemset(h->Q32[i], 0, f32);
        }
        if ((rc = dalloc(h, &h->P32, f32))) return bail(rc);
        cudaMemset(h->P32, 0, f32);
        if ((rc = dalloc(h, (void**)&h->mean64, sizeof(zd) * 7 * h->Ny))) return bail(rc);
        cudaMemset(h->mean64, 0, sizeof(zd) * 7 * h->Ny);
    }
    if (h->mixed && h->tc) {
        std::vector<unsigned char> fimg, iimg;
        const double fscale = 1.0 / ((double)h->Nxp * h->Nzp * (h->Ny - 1));
        h->chebsym = cheb_sym_dims(h->Ny, h->split, h->symd);
        if (h->chebsym) {
            cheb_sym_images(h->Ny, 0, fscale, h->split, h->symd, fimg);
            cheb_sym_images(h->Ny, 1, 1.0, h->split, h->symd, iimg);
        } else {
            cheb_images(h->Ny, 0, fscale, h->split, fimg, h->chebNP, h->chebKT);
            cheb_images(h->Ny, 1, 1.0, h->split, iimg, h->chebNP, h->chebKT);
        }
        if ((rc = dalloc(h, (void**)&h->d_chebF, fimg.size()))) return bail(rc);
        if ((rc = dalloc(h, (void**)&h->d_chebI, iimg.size()))) return bail(rc);
        if (cudaMemcpy(h->d_chebF, fimg.data(), fimg.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(h->d_chebI, iimg.data(), iimg.size(), cudaMemcpyHostToDevice) != cudaSuccess)
            return bail(fail(CF_E_CUDA, "upload failed"));
    }
    {
        std::vector<zd> cs(h->P + 1);
        const long double pi = 3.141592653589793238462643383279502884L;
        for (int n = 0; n <= h->P; ++n) {
            long double a = pi * (long double)n / (long double)h->P;
            cs[n] = make_double2((double)cosl(a), (double)sinl(a));
        }
        if ((rc = dalloc(h, (void**)&h->d_cs, sizeof(zd) * (h->P + 1)))) return bail(rc);
        cudaMemcpy(h->d_cs, cs.data(), sizeof(zd) * (h->P + 1), cudaMemcpyHostToDevice);
        // degree coefficients of the integrated tau rows (see helm_g)
        const int P = h->P, Ny = h->Ny;
        std::vector<double> gt((size_t)3 * Ny, 0.0);
        for (int n = 2; n <= P; ++n) {
            gt[n] = (n == 2 ? 2.0 : 1.0) / (4.0 * n * (n - 1));
            gt[Ny + n] = (n <= P - 2) ? -1.0 / (2.0 * ((double)n * n - 1.0)) : 0.0;
            gt[2 * Ny + n] = (n + 2 <= P - 2) ? 1.0 / (4.0 * n * (n + 1)) : 0.0;
        }
        if ((rc = dalloc(h, (void**)&h->d_helmtab, sizeof(double) * gt.size()))) return bail(rc);
        cudaMemcpy(h->d_helmtab, gt.data(), sizeof(double) * gt.size(), cudaMemcpyHostToDevice);
    }
    encode_maps(h);
    if ((rc = set_attrs(h))) return bail(rc);
    if ((rc = ensure_banks(h))) return bail(rc);
    if (cudaDeviceSynchronize() != cudaSuccess) return bail(fail(CF_E_CUDA, "set-up failed"));
    *out = h;
    return CF_OK;
}

int cf_set_constraint(cf_handle* h, int kind, double c1, double c2) {
    if (!h) return fail(CF_E_ARG, "null handle");
    if (kind != 0 && kind != 1) return fail(CF_E_ARG, "unknown constraint kind");
    if (!(std::isfinite(c1) && std::isfinite(c2))) return fail(CF_E_ARG, "mean-flow constraint values must be finite");
    h->cmode = kind; h->c1 = c1; h->c2 = c2;
    drop_graph(h);
    return CF_OK;
}

int cf_set_state(cf_handle* h, const double* U, const double* P) {
    if (!h || !U || !P) return fail(CF_E_ARG, "null argument");
    DeviceGuard dg_(h->device);
    const size_t fr = sizeof(zd) * h->nr;
    for (int i = 0; i < 3; ++i) CU(cudaMemcpyAsync(h->U[i], U + 2 * i * h->nr, fr, cudaMemcpyHostToDevice, h->stream));
    CU(cudaMemcpyAsync(h->Pf, P, fr, cudaMemcpyHostToDevice, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    h->nodal_valid = false;
    state_wrote64(h);
    return CF_OK;
}
int cf_get_state(cf_handle* h, double* U, double* P) {
    if (!h || !U) return fail(CF_E_ARG, "null argument");
    DeviceGuard dg_(h->device);
    int rc;
    if ((rc = state_to64(h))) return rc;
    const size_t fr = sizeof(zd) * h->nr;
    for (int i = 0; i < 3; ++i) CU(cudaMemcpyAsync(U + 2 * i * h->nr, h->U[i], fr, cudaMemcpyDeviceToHost, h->stream));
    if (P) CU(cudaMemcpyAsync(P, h->Pf, fr, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    return CF_OK;
}
int cf_set_state_device(cf_handle* h, const void* U, const void* P) {
    if (!h || !U || !P) return fail(CF_E_ARG, "null argument");
    DeviceGuard dg_(h->device);
    const size_t fr = sizeof(zd) * h->nr;
    for (int i = 0; i < 3; ++i)
        CU(cudaMemcpyAsync(h->U[i], (const char*)U + i * fr, fr, cudaMemcpyDeviceToDevice, h->stream));
    CU(cudaMemcpyAsync(h->Pf, P, fr, cudaMemcpyDeviceToDevice, h->stream));
    h->nodal_valid = false;
    state_wrote64(h);
    return CF_OK;
}
int cf_get_state_device(cf_handle* h, void* U, void* P) {
    if (!h || !U) return fail(CF_E_ARG, "null argument");
    DeviceGuard dg_(h->device);
    int rc;
    if ((rc = state_to64(h))) return rc;
    const size_t fr = sizeof(zd) * h->nr;
    for (int i = 0; i < 3; ++i)
        CU(cudaMemcpyAsync((char*)U + i * fr, h->U[i], fr, cudaMemcpyDeviceToDevice, h->stream));
    if (P) CU(cudaMemcpyAsync(P, h->Pf, fr, cudaMemcpyDeviceToDevice, h->stream));
    return CF_OK;
}

int cf_step(cf_handle* h, double t, int nsteps, double* t_out, double* grads_out) {
    if (!h) return fail(CF_E_ARG, "null handle");
    DeviceGuard dg_(h->device);
    if (nsteps < 0) return fail(CF_E_ARG, "nsteps must be nonnegative");
    int rc, cnt = 0;
    if ((rc = state_to32(h))) return rc;
    if (!h->nodal_valid) {
        if ((rc = h->mixed ? launch_prep_mx(h, &cnt) : launch_prep(h, h->U, &cnt))) return rc;
        h->nodal_valid = true;
    }
    if ((rc = build_graph(h))) return rc;
    for (int s = 0; s < nsteps; ++s) CU(cudaGraphLaunch(h->graph, h->stream));
    if (nsteps > 0) state_stepped(h);
    cnt += (h->mixed && h->tc ? 18 : step_launches(h)) * nsteps;
    h->last_launches = cnt;
    if (t_out) *t_out = t + nsteps * h->dt;
    if (grads_out && (rc = check_status(h))) return rc;
    if (grads_out) {
        double g[2];
        CU(cudaMemcpyAsync(g, h->d_grad, 16, cudaMemcpyDeviceToHost, h->stream));
        CU(cudaStreamSynchronize(h->stream));
        grads_out[0] = g[0];
        grads_out[1] = g[1];
    }
    return CF_OK;
}

int cf_step_dt(cf_handle* h, double t, double dt, double* t_out, double* grads_out) {
    if (!h) return fail(CF_E_ARG, "null handle");
    DeviceGuard dg_(h->device);
    if (!(std::isfinite(dt) && dt > 0)) return fail(CF_E_ARG, "dt must be finite and positive");
    if (dt == h->dt) return cf_step(h, t, 1, t_out, grads_out);
    if (h->s32) return fail(CF_E_UNSUPPORTED, "a step of another duration is not supported with the FP32 state");
    int rc, cnt = 0;
    if (h->tdt != dt) {
        // the factors may still be read by an earlier step of this kind
        CU(cudaStreamSynchronize(h->stream));
        h->tdt = 0.0;
        for (int j = 0; j < 3; ++j)
            if ((rc = build_bank(h, h->tbank[j], h->nu, 1.0 / (CC[j] * dt)))) return rc;
        h->tdt = dt;
    }
    if (!h->nodal_valid) {
        if ((rc = h->mixed ? launch_prep_mx(h, &cnt) : launch_prep(h, h->U, &cnt))) return rc;
        h->nodal_valid = true;
    }
    // the stage launches read dt and the banks from the handle: swap the
    // temporary ones in for three eager stages (the nominal step's graph holds
    // its own parameters)
    std::swap(h->bank, h->tbank);
    const double dt0 = h->dt;
    h->dt = dt;
    rc = CF_OK;
    for (int j = 0; j < 3 && rc == CF_OK; ++j) rc = h->mixed ? launch_stage_mx(h, j, &cnt) : launch_stage(h, j, &cnt);
    h->dt = dt0;
    std::swap(h->bank, h->tbank);
    if (rc) return rc;
    h->last_launches = cnt;
    if (t_out) *t_out = t + dt;
    if (grads_out && (rc = check_status(h))) return rc;
    if (grads_out) {
        double g[2];
        CU(cudaMemcpyAsync(g, h->d_grad, 16, cudaMemcpyDeviceToHost, h->stream));
        CU(cudaStreamSynchronize(h->stream));
        grads_out[0] = g[0];
        grads_out[1] = g[1];
    }
    return CF_OK;
}

// step! over host arrays (cnrk2.jl:149-207 with CPU fields): upload U and
// P, advance nsteps, download the new U and P.  The state crosses PCIe in
// kz-plane chunks on a copy stream: the nodal fields of chunk k are computed
// while chunk k+1 arrives; the pressure, first read by the first stage's
// column kernel, arrives during that stage's periodic transforms; the last
// stage's column kernel runs chunk by chunk, each chunk downloaded while the
// next is computed.  That kernel leaves out the nodal fields of a following
// stage (a host step's successor uploads a new state), so afterwards the
// handle's nodal fields are stale and a following cf_step recomputes them
// from the state, which gives the same values.
int cf_step_host(cf_handle* h, double* U, double* P, double t, int nsteps, double* t_out, double* grads_out) {
    if (!h || !U || !P) return fail(CF_E_ARG, "null argument");
    DeviceGuard dg_(h->device);
    if (nsteps < 0) return fail(CF_E_ARG, "nsteps must be nonnegative");
    int rc;
    if (nsteps == 0 || (h->mixed && h->tc) || h->s32) {
        // the tensor-core form transforms all columns in one launch: no chunks
        if ((rc = cf_set_state(h, U, P)) || (rc = cf_step(h, t, nsteps, t_out, grads_out))) return rc;
        return cf_get_state(h, U, P);
    }
    if ((rc = ensure_copy_stream(h))) return rc;
    if (nsteps > 2 && (rc = build_graph(h))) return rc;
    int zb[CF_HOST_CHUNKS + 1];
    const int K = host_chunks(h, zb);
    cudaEvent_t* up = h->hev + 1;                    // velocity chunks 0..K-1, then the pressure
    cudaEvent_t* dn = h->hev + CF_HOST_CHUNKS + 2;   // last-stage column chunks
    const size_t fd = 2 * (size_t)h->nr;  // doubles per field
    zd* dev[4] = {h->U[0], h->U[1], h->U[2], h->Pf};
    double* host[4] = {U, U + fd, U + 2 * fd, P};
    // the copies of the state follow the work already queued on the handle
    CU(cudaEventRecord(h->hev[0], h->stream));
    CU(cudaStreamWaitEvent(h->cstream, h->hev[0], 0));
    auto run = [&]() -> int {
        int r, cnt = 0;
        for (int k = 0; k < K; ++k) {
            for (int i = 0; i < 3; ++i)
                if ((r = copy_planes(dev[i], host[i], h, zb[k], zb[k + 1], cudaMemcpyHostToDevice, h->cstream)))
                    return r;
            CU(cudaEventRecord(up[k], h->cstream));
        }
        if ((r = copy_planes(dev[3], host[3], h, 0, h->Nz, cudaMemcpyHostToDevice, h->cstream))) return r;
        CU(cudaEventRecord(up[K], h->cstream));
        ColParams pp;
        const int kprep = host_prep_kind(h, pp);
        for (int k = 0; k < K; ++k) {
            CU(cudaStreamWaitEvent(h->stream, up[k], 0));
            if ((r = launch_cols(h, kprep, pp, chunk_block(h, zb, K, k), chunk_block(h, zb, K, k + 1), &cnt)))
                return r;
        }
        h->nodal_valid = true;
        for (int s = 0; s < nsteps; ++s) {
            const bool first = s == 0, last = s == nsteps - 1;
            if (!first && !last) {
                CU(cudaGraphLaunch(h->graph, h->stream));
                cnt += step_launches(h);
                continue;
            }
            for (int j = 0; j < 3; ++j) {
                if ((r = h->mixed ? launch_periodic32(h, &cnt) : launch_periodic(h, &cnt))) return r;
                if (first && j == 0) CU(cudaStreamWaitEvent(h->stream, up[K], 0));
                ColParams p;
                const int kind = host_stage_kind(h, j, p);
                if (!(last && j == 2)) {
                    if ((r = launch_cols(h, kind, p, 0, col_blocks(h), &cnt))) return r;
                    continue;
                }
                p.skip_nodal = 1;
                h->nodal_valid = false;
                for (int k = 0; k < K; ++k) {
                    if ((r = launch_cols(h, kind, p, chunk_block(h, zb, K, k), chunk_block(h, zb, K, k + 1), &cnt)))
                        return r;
                    CU(cudaEventRecord(dn[k], h->stream));
                    CU(cudaStreamWaitEvent(h->cstream, dn[k], 0));
                    for (int i = 0; i < 4; ++i)
                        if ((r = copy_planes(host[i], dev[i], h, zb[k], zb[k + 1], cudaMemcpyDeviceToHost, h->cstream)))
                            return r;
                }
            }
        }
        h->last_launches = cnt;
        return CF_OK;
    };
    rc = run();
    // no copy into or out of the caller's buffers outlives the call
    const cudaError_t e = cudaStreamSynchronize(h->cstream);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(CF_E_CUDA, std::string("host step copies: ") + cudaGetErrorString(e));
    if ((rc = check_status(h))) return rc;
    if (t_out) *t_out = t + nsteps * h->dt;
    if (grads_out) {
        double g[2];
        CU(cudaMemcpyAsync(g, h->d_grad, 16, cudaMemcpyDeviceToHost, h->stream));
        CU(cudaStreamSynchronize(h->stream));
        grads_out[0] = g[0];
        grads_out[1] = g[1];
    }
    return CF_OK;
}

static int ensure_tmp(cf_engine* h) {
    int rc;
    if (!h->tmpU) {
        if ((rc = dalloc(h, (void**)&h->tmpU, sizeof(zd) * h->nr * 3))) return rc;
        if ((rc = dalloc(h, (void**)&h->tmpP, sizeof(zd) * h->nr))) return rc;
    }
    return CF_OK;
}

// The nonlinear term of the velocity in Us as coefficients, overwriting Us
// (the velocity is consumed by the preparation kernel first).
static int launch_nonlinear(cf_engine* h, zd* const Us[3]) {
    int rc;
    if ((rc = launch_prep(h, Us, nullptr))) return rc;
    if (h->form == NL_DIV) return launch_periodic(h, nullptr, Us);
    if ((rc = launch_periodic(h, nullptr))) return rc;
    ColParams p = col_params(h);
    for (int i = 0; i < 3; ++i) p.Nout[i] = Us[i];
    col_kernel(KC_NLOUT, h->P)<<<col_blocks(h), col_threads(h), col_smem(h), h->stream>>>(p);
    CU(cudaGetLastError());
    return CF_OK;
}

int cf_nonlinear(cf_handle* h, const double* U, double* N) {
    if (!h || !U || !N) return fail(CF_E_ARG, "null argument");
    DeviceGuard dg_(h->device);
    int rc = ensure_tmp(h);
    if (rc) return rc;
    const size_t fr = sizeof(zd) * h->nr;
    CU(cudaMemcpyAsync(h->tmpU, U, 3 * fr, cudaMemcpyHostToDevice, h->stream));
    zd* Us[3] = {h->tmpU, h->tmpU + h->nr, h->tmpU + 2 * h->nr};
    if ((rc = launch_nonlinear(h, Us))) return rc;
    CU(cudaMemcpyAsync(N, h->tmpU, 3 * fr, cudaMemcpyDeviceToHost, h->stream));
    if ((rc = check_status(h, false))) return rc;
    h->nodal_valid = false;
    return CF_OK;
}

int cf_nonlinear_noalloc(cf_handle* h, const double* U, double* N) {
    if (!h || !U || !N) return fail(CF_E_ARG, "null argument");
    DeviceGuard dg_(h->device);
    const size_t fr = sizeof(zd) * h->nr;
    if (3 * fr > (size_t)CF_NOALLOC_SCRATCH_BYTES)
        return fail(CF_E_ARG, "grid too large for the fixed scratch (3 * Nr * 16 bytes > 16 MiB)");
    void* scr = noalloc_scratch(h->device);
    if (!scr) return fail(CF_E_CUDA, "fixed scratch address not set up for the handle's device");
    int rc;
    zd* base = static_cast<zd*>(scr);
    zd* Us[3] = {base, base + h->nr, base + 2 * h->nr};
    CU(cudaMemcpyAsync(base, U, 3 * fr, cudaMemcpyHostToDevice, h->stream));
    if ((rc = launch_nonlinear(h, Us))) return rc;
    CU(cudaMemcpyAsync(N, base, 3 * fr, cudaMemcpyDeviceToHost, h->stream));
    if ((rc = check_status(h, false))) return rc;
    h->nodal_valid = false;
    return CF_OK;
}

static int project_dev(cf_engine* h, zd* const Ud[3]) {
    int rc;
    if (!h->proj.ready && (rc = build_bank(h, h->proj, 1.0, 0.0))) return rc;
    ColParams p = col_params(h);
    for (int i = 0; i < 3; ++i) p.U[i] = Ud[i];
    p.bank = h->proj.view();
    if (h->cmode == 1) { p.cmode = 1; p.c1 = h->c1 - h->basemean; p.c2 = h->c2; }
    else { p.cmode = 0; p.c1 = 0.0; p.c2 = 0.0; }
    double* gtmp = h->d_grad;
    p.grad_out = gtmp;
    col_kernel(KC_PROJECT, h->P)<<<col_blocks(h), col_threads(h), col_smem(h), h->stream>>>(p);
    CU(cudaGetLastError());
    return CF_OK;
}

static int pressure_dev(cf_engine* h, zd* const Ud[3], zd* Pout) {
    int rc;
    if ((rc = build_neumann(h))) return rc;
    if ((rc = launch_prep(h, Ud, nullptr))) return rc;
    if ((rc = launch_periodic(h, nullptr))) return rc;
    ColParams p = col_params(h);
    for (int i = 0; i < 3; ++i) p.U[i] = Ud[i];
    p.Pf = Pout;
    p.bank = h->neum.view();
    // the divergence form's term arrives in nod[0..2] as coefficients
    col_kernel(h->form == NL_DIV ? KC_PRESSURE_COEF : KC_PRESSURE, h->P)<<<col_blocks(h), col_threads(h),
                                                                          col_smem(h), h->stream>>>(p);
    CU(cudaGetLastError());
    h->nodal_valid = false;
    return CF_OK;
}

int cf_project(cf_handle* h, double* U) {
    if (!h || !U) return fail(CF_E_ARG, "null argument");
    DeviceGuard dg_(h->device);
    int rc = ensure_tmp(h);
    if (rc) return rc;
    const size_t fr = sizeof(zd) * h->nr;
    CU(cudaMemcpyAsync(h->tmpU, U, 3 * fr, cudaMemcpyHostToDevice, h->stream));
    zd* Us[3] = {h->tmpU, h->tmpU + h->nr, h->tmpU + 2 * h->nr};
    if ((rc = project_dev(h, Us))) return rc;
    CU(cudaMemcpyAsync(U, h->tmpU, 3 * fr, cudaMemcpyDeviceToHost, h->stream));
    if ((rc = check_status(h, false))) return rc;
    return CF_OK;
}

int cf_pressure(cf_handle* h, const double* U, double* P) {
    if (!h || !U || !P) return fail(CF_E_ARG, "null argument");
    DeviceGuard dg_(h->device);
    int rc = ensure_tmp(h);
    if (rc) return rc;
    const size_t fr = sizeof(zd) * h->nr;
    CU(cudaMemcpyAsync(h->tmpU, U, 3 * fr, cudaMemcpyHostToDevice, h->stream));
    zd* Us[3] = {h->tmpU, h->tmpU + h->nr, h->tmpU + 2 * h->nr};
    if ((rc = pressure_dev(h, Us, h->tmpP))) return rc;
    CU(cudaMemcpyAsync(P, h->tmpP, fr, cudaMemcpyDeviceToHost, h->stream));
    if ((rc = check_status(h, false))) return rc;
    return CF_OK;
}

int cf_random_state(cf_handle* h, unsigned long long seed, double amp, int shape, double rho) {
    if (!h) return fail(CF_E_ARG, "null handle");
    DeviceGuard dg_(h->device);
    if (!(amp >= 0)) return fail(CF_E_ARG, "epsilon must be non-negative");
    std::vector<std::complex<double>> U;
    host_synth(h, seed, amp, shape, rho, U);
    const size_t fr = sizeof(zd) * h->nr;
    for (int i = 0; i < 3; ++i) CU(cudaMemcpyAsync(h->U[i], U.data() + i * h->nr, fr, cudaMemcpyHostToDevice, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    int rc;
    if ((rc = project_dev(h, h->U))) return rc;
    if ((rc = pressure_dev(h, h->U, h->Pf))) return rc;
    if ((rc = check_status(h, false))) return rc;
    h->nodal_valid = false;
    state_wrote64(h);
    return CF_OK;
}

static DiagKernel diag_kernel(int P) {
    switch (P) {
#define CF_CASE(N) \
    case N: return diag_kernel_for<N>();
        CF_COL_LENGTHS(CF_CASE)
#undef CF_CASE
        default: return diag_kernel_for<0>();
    }
}

static int ensure_diag(cf_engine* h) {
    int rc;
    if (!h->d_diag) {
        if ((rc = dalloc(h, (void**)&h->d_diag, 8 * sizeof(double)))) return rc;
        if ((rc = dalloc(h, (void**)&h->d_diagpart, 3 * sizeof(double) * col_blocks(h)))) return rc;
        if ((rc = raise_smem_limit(diag_kernel(h->P), col_smem(h)))) return rc;
    }
    return CF_OK;
}

// Diagnostics on the device: one column team per Fourier column (see
// k_column_diag); five doubles come back to the host.
int cf_diagnostics(cf_handle* h, double* out) {
    if (!h || !out) return fail(CF_E_ARG, "null argument");
    DeviceGuard dg_(h->device);
    int rc;
    if ((rc = ensure_diag(h)) || (rc = state_to64(h))) return rc;
    CU(cudaMemsetAsync(h->d_diag, 0, 8 * sizeof(double), h->stream));
    ColParams p = col_params(h);
    diag_kernel(h->P)<<<col_blocks(h), col_threads(h), col_smem(h), h->stream>>>(p, h->d_diag, h->d_diagpart);
    k_diag_reduce<<<1, 1024, 0, h->stream>>>(h->d_diagpart, (int)col_blocks(h), h->d_diag);
    CU(cudaGetLastError());
    double acc[5];
    CU(cudaMemcpyAsync(acc, h->d_diag, 5 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if ((rc = check_status(h, false))) return rc;
    out[0] = acc[0] / 2;
    out[1] = h->nu * acc[1];
    out[2] = acc[2];
    out[3] = h->nu * acc[3];
    out[4] = h->nu * acc[4];
    return CF_OK;
}

// One row of recorded diagnostics into acc[0..7] on the handle's stream, no
// host synchronisation: the block partials of k_column_diag summed by
// k_diag_reduce (acc[0..2]), the wall derivatives (acc[3..4]), the step's
// last gradients (acc[5..6]) and the total-flow power input with those
// gradients (acc[7]).
static int record_diag(cf_engine* h, double* acc, int* count) {
    int rc;
    if ((rc = state_to64(h))) return rc;
    ColParams p = col_params(h);
    diag_kernel(h->P)<<<col_blocks(h), col_threads(h), col_smem(h), h->stream>>>(p, acc, h->d_diagpart);
    k_diag_reduce<<<1, 1024, 0, h->stream>>>(h->d_diagpart, (int)col_blocks(h), acc);
    CU(cudaMemcpyAsync(acc + 5, h->d_grad, 2 * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    k_power_input<<<1, 32, 0, h->stream>>>(h->U[0], h->U[2], h->d_base, (long)h->Nz * h->Nxh, h->Ny, h->nu, 0.0,
                                           0.0, acc + 7, h->d_grad);
    CU(cudaGetLastError());
    *count += 3;
    return CF_OK;
}

int cf_step_record(cf_handle* h, double t, int nsteps, int every, double* series, double* t_out,
                   double* grads_out) {
    if (!h || !series) return fail(CF_E_ARG, "null argument");
    if (nsteps < 0 || every <= 0) return fail(CF_E_ARG, "nsteps must be nonnegative and every positive");
    DeviceGuard dg_(h->device);
    int rc;
    const int nrec = nsteps / every;
    if ((rc = ensure_diag(h))) return rc;
    if (nrec > h->rec_cap) {
        const int cap = std::max(nrec, 64);
        if ((rc = dalloc(h, (void**)&h->d_rec, (size_t)cap * 8 * sizeof(double)))) return rc;
        h->rec_cap = cap;
    }
    int cnt = 0;
    double tc = t;
    for (int r = 0; r < nrec; ++r) {
        if ((rc = cf_step(h, tc, every, &tc, nullptr))) return rc;
        cnt += h->last_launches;
        if ((rc = record_diag(h, h->d_rec + 8L * r, &cnt))) return rc;
    }
    if (nsteps > nrec * every) {
        if ((rc = cf_step(h, tc, nsteps - nrec * every, &tc, nullptr))) return rc;
        cnt += h->last_launches;
    }
    std::vector<double> acc((size_t)nrec * 8);
    if (nrec) CU(cudaMemcpyAsync(acc.data(), h->d_rec, acc.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    double g[2];
    CU(cudaMemcpyAsync(g, h->d_grad, 16, cudaMemcpyDeviceToHost, h->stream));
    if ((rc = check_status(h))) return rc;
    for (int r = 0; r < nrec; ++r) {
        const double* a = acc.data() + 8L * r;
        double* o = series + 9L * r;
        o[0] = t + (double)(r + 1) * every * h->dt;
        o[1] = a[0] / 2;
        o[2] = h->nu * a[1];
        o[3] = a[2];
        o[4] = h->nu * a[3];
        o[5] = h->nu * a[4];
        o[6] = a[5];
        o[7] = a[6];
        o[8] = a[7];
    }
    h->last_launches = cnt;
    if (t_out) *t_out = tc;
    if (grads_out) {
        grads_out[0] = g[0];
        grads_out[1] = g[1];
    }
    return CF_OK;
}

// Power input of the engine's mean profile (one warp over the (0,0) column;
// one double comes back).
int cf_power_input(cf_handle* h, int with_base, double dPdx, double dPdz, double* out) {
    if (!h || !out) return fail(CF_E_ARG, "null argument");
    if (!(std::isfinite(dPdx) && std::isfinite(dPdz))) return fail(CF_E_ARG, "pressure gradient must be finite");
    DeviceGuard dg_(h->device);
    int rc;
    if ((rc = ensure_diag(h)) || (rc = state_to64(h))) return rc;
    k_power_input<<<1, 32, 0, h->stream>>>(h->U[0], h->U[2], with_base ? h->d_base : nullptr, (long)h->Nz * h->Nxh,
                                           h->Ny, h->nu, dPdx, dPdz, h->d_diag + 6);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(out, h->d_diag + 6, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if ((rc = check_status(h, false))) return rc;
    return CF_OK;
}

int cf_step_profiled(cf_handle* h, double t, int nsteps, double* t_out, double* kernel_ms) {
    if (!h || !kernel_ms) return fail(CF_E_ARG, "null argument");
    DeviceGuard dg_(h->device);
    if (h->mixed) return step_profiled_mx(h, t, nsteps, t_out, kernel_ms);
    int rc = CF_OK, cnt = 0;
    if (!h->nodal_valid) {
        if ((rc = launch_prep(h, h->U, &cnt))) return rc;
        h->nodal_valid = true;
    }
    cudaEvent_t ev[5];
    for (int k = 0; k < 5; ++k) CU(cudaEventCreate(&ev[k]));
    for (int k = 0; k < 6; ++k) kernel_ms[k] = 0.0;
    for (int s = 0; s < nsteps && rc == CF_OK; ++s) rc = launch_step_profiled(h, ev, kernel_ms);
    for (int k = 0; k < 5; ++k) cudaEventDestroy(ev[k]);
    if (rc) return rc;
    if ((rc = check_status(h))) return rc;
    h->last_launches = cnt + step_launches(h) * nsteps;
    if (t_out) *t_out = t + nsteps * h->dt;
    return CF_OK;
}

int cf_sync(cf_handle* h) {
    if (!h) return fail(CF_E_ARG, "null handle");
    DeviceGuard dg_(h->device);
    int rc;
    if ((rc = check_status(h))) return rc;
    return CF_OK;
}
int cf_set_wait_limit(cf_handle* h, long spins) {
    if (!h) return fail(CF_E_ARG, "null handle");
    h->wait_spins = spins < 0 ? CF_WAIT_SPINS : spins;
    drop_graph(h);  // the step graph holds the launch parameters
    return CF_OK;
}
long long cf_device_bytes(cf_handle* h) { return h ? (long long)h->dev_bytes : 0; }
int cf_last_launch_count(cf_handle* h) { return h ? h->last_launches : 0; }
void* cf_stream(cf_handle* h) { return h ? (void*)h->stream : nullptr; }

}  // extern "C"

// Seeded synthetic coefficients: splitmix64 hash of (seed, component, ix, iz,
// n) -> two uniforms -> Box-Muller; amplitude shaped in (k, l, n).
static inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}
static inline double unit01(uint64_t v) { return ((v >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
static void host_synth(const cf_engine* h, uint64_t seed, double amp, int shape, double rho,
                       std::vector<std::complex<double>>& U) {
    const long S = h->B;
    U.assign((size_t)3 * h->nr, 0.0);
    for (int c = 0; c < 3; ++c)
        for (int n = 0; n < h->Ny; ++n)
            for (int iz = 0; iz < h->Nz; ++iz) {
                int l = iz <= (h->Nz >> 1) ? iz : iz - h->Nz;
                for (int ix = 0; ix < h->Nxh; ++ix) {
                    bool nyq = ((h->Nx % 2 == 0) && ix == h->Nx / 2) || ((h->Nz % 2 == 0) && iz == h->Nz / 2);
                    double s, r;
                    if (shape == 0) { s = std::exp(-(std::abs(ix) + std::abs(l)) / 4.0); r = std::exp(-n / 4.0); }
                    else { s = 1.0 / (1.0 + (double)ix * ix + (double)l * l); r = std::pow(rho, n); }
                    std::complex<double> v = 0;
                    if (!nyq) {
                        uint64_t key = splitmix64(seed ^ splitmix64(((uint64_t)c << 56) ^ ((uint64_t)ix << 36) ^
                                                                   ((uint64_t)iz << 16) ^ (uint64_t)n));
                        double a = unit01(splitmix64(key)), b = unit01(splitmix64(key ^ 0xD1B54A32D192ED03ULL));
                        double rr = std::sqrt(-2.0 * std::log(a));
                        v = amp * s * r * std::complex<double>(rr * std::cos(2 * M_PI * b), rr * std::sin(2 * M_PI * b));
                    }
                    U[(size_t)c * h->nr + n * S + (long)iz * h->Nxh + ix] = v;
                }
            }
    for (int c = 0; c < 3; ++c)
        for (int n = 0; n < h->Ny; ++n) {
            std::complex<double>* col = U.data() + (size_t)c * h->nr + n * S;
            col[0] = col[0].real();
            for (int iz = (h->Nz >> 1) + 1; iz < h->Nz; ++iz) col[(long)iz * h->Nxh] = std::conj(col[(long)(h->Nz - iz) * h->Nxh]);
        }
}

// ---------------------------------------------------------------------------
// Ensembles: independent channels (grids, Re, seeds) advanced together.
// Instances with the same grid form a size class.  Every stage launches each
// of the four kernels once per class over all of its instances (a grid
// coordinate selects the instance, whose parameters the block stages in
// shared memory), and the classes run as parallel branches of one CUDA graph
// per step: 12 launches per class per step, whatever the instance count.
// ---------------------------------------------------------------------------
static ColBatchKernel col_batch_kernel(int P, int variant) {
    switch (P) {
#define CF_CASE(N) \
    case N: return col_batch_kernel_for<N>(variant);
        CF_COL_LENGTHS(CF_CASE)
#undef CF_CASE
        default: return col_batch_kernel_for<0>(variant);
    }
}
// the variants that exist for a class's Chebyshev length (the compile-time
// lengths up to 128 have all of them)
static int col_batch_nvariants(int P) {
    switch (P) {
#define CF_CASE(N) \
    case N: return col_batch_variants(N) ? CF_COL_BATCH_VARIANTS : 1;
        CF_COL_LENGTHS(CF_CASE)
#undef CF_CASE
        default: return 1;
    }
}
static FftBatchKernel fft_batch_kernel(int which, int L) {
    switch (L) {
#define CF_CASE(N) \
    case N: return fft_batch_kernel_for<N>(which);
        CF_STATIC_FFT_LENGTHS(CF_CASE)
#undef CF_CASE
        default: return fft_batch_kernel_for<0>(which);
    }
}

struct BatchClass {
    int Nx = 0, Ny = 0, Nz = 0;
    std::vector<int> members;
    // the column kernel's schedule, chosen by autotune_batch: variant (columns
    // per block, register bound) and persistent launch (grid pgrid) or one
    // block per item; counters of the persistent launches (one per stage)
    int var = 0;
    bool persist = false;
    unsigned pgrid = 0;
    unsigned* d_counter = nullptr;
    double step_ms = 0.0;
    // the periodic kernels' shapes, also chosen by autotune_batch: columns
    // per z block (0: the instances' own) and rows per x-pass block
    int tkz = 0;
    int xkind = KF_XPASS;
    FftParams* d_fft = nullptr;
    ColParams* d_col[3] = {nullptr, nullptr, nullptr};
    std::vector<FftParams> h_fft;
    std::vector<ColParams> h_col[3];
    cudaStream_t side = nullptr;
    cudaEvent_t join = nullptr;
};

struct cf_batch {
    std::vector<cf_engine*> inst;
    std::vector<BatchClass> cls;
    std::string schedule;  // what the autotuner measured and chose
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr, done = nullptr;
    cudaGraphExec_t graph = nullptr;
    std::vector<void*> allocs;
    int last_launches = 0;
};

void cf_destroy_batch(cf_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (BatchClass& c : b->cls) {
        if (c.side) cudaStreamDestroy(c.side);
        if (c.join) cudaEventDestroy(c.join);
    }
    for (void* p : b->allocs) cudaFree(p);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->done) cudaEventDestroy(b->done);
    if (b->stream) cudaStreamDestroy(b->stream);
    for (cf_engine* h : b->inst) cf_destroy(h);
    delete b;
}

static int batch_alloc(cf_batch* b, void** p, size_t bytes) {
    if (cudaMalloc(p, bytes) != cudaSuccess) return fail(CF_E_NOMEM, "device allocation failed");
    b->allocs.push_back(*p);
    return CF_OK;
}

// The batched periodic kernels' shapes of a class: columns per z block
// (their transform stride and shared memory follow from it) and rows per
// x-pass block.
static int class_tkz(const cf_batch* b, const BatchClass& c) { return c.tkz ? c.tkz : b->inst[c.members[0]]->tkz; }
static int zbs_of(int Nzp, int tkz) { return fft_bufsz(Nzp) + (8 / tkz) % 8; }
static size_t class_zsmem(const cf_batch* b, const BatchClass& c) {
    const int tkz = class_tkz(b, c);
    return (size_t)2 * tkz * zbs_of(b->inst[c.members[0]]->Nzp, tkz) * sizeof(zd);
}
static int xpass_rows(int xkind) {
    return xkind == KF_XPASS_R4 ? 4 : (xkind == KF_XPASS_R8 ? 8 : (xkind == KF_XPASS_R16 ? 16 : 2));
}
static size_t class_xsmem(const cf_batch* b, const BatchClass& c) {
    return (size_t)6 * xpass_rows(c.xkind) * xbs(b->inst[c.members[0]]) * sizeof(zd);
}

// Parameters of every instance (host copies refreshed from the instances,
// so constraint changes made through an instance handle take effect).
static int batch_upload(cf_batch* b) {
    for (BatchClass& c : b->cls) {
        for (size_t k = 0; k < c.members.size(); ++k) {
            cf_engine* h = b->inst[c.members[k]];
            c.h_fft[k] = fft_params(h);
            const int tkz = class_tkz(b, c);
            c.h_fft[k].tks = ilog2(tkz);
            c.h_fft[k].bsz = zbs_of(h->Nzp, tkz);
            for (int j = 0; j < 3; ++j) c.h_col[j][k] = stage_col_params(h, j);
        }
        CU(cudaMemcpyAsync(c.d_fft, c.h_fft.data(), sizeof(FftParams) * c.h_fft.size(), cudaMemcpyHostToDevice,
                           b->stream));
        for (int j = 0; j < 3; ++j)
            CU(cudaMemcpyAsync(c.d_col[j], c.h_col[j].data(), sizeof(ColParams) * c.h_col[j].size(),
                               cudaMemcpyHostToDevice, b->stream));
    }
    CU(cudaStreamSynchronize(b->stream));
    return CF_OK;
}

static int autotune_batch(cf_batch* b);

int cf_create_batch(const cf_config* cfgs, int n, cf_batch** out) {
    if (!cfgs || n <= 0 || !out) return fail(CF_E_ARG, "null argument or empty ensemble");
    *out = nullptr;
    cf_batch* b = new cf_batch();
    auto bail = [&](int code) {
        cf_destroy_batch(b);
        return code;
    };
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) != cudaSuccess)
        return bail(fail(CF_E_CUDA, "cannot create stream (no CUDA device?)"));
    for (int i = 0; i < n; ++i) {
        cf_handle* h = nullptr;
        int rc = cf_create(cfgs + i, &h);
        if (rc) return bail(rc);
        b->inst.push_back(h);
        if (h->mixed) return bail(fail(CF_E_UNSUPPORTED, "ensembles run the FP64 plain form"));
        if (h->form != NL_ROT) return bail(fail(CF_E_UNSUPPORTED, "ensembles run the rotational nonlinear form"));
    }
    for (int i = 0; i < n; ++i) {
        cf_engine* h = b->inst[i];
        BatchClass* c = nullptr;
        for (BatchClass& x : b->cls)
            if (x.Nx == h->Nx && x.Ny == h->Ny && x.Nz == h->Nz) c = &x;
        if (!c) {
            b->cls.emplace_back();
            c = &b->cls.back();
            c->Nx = h->Nx;
            c->Ny = h->Ny;
            c->Nz = h->Nz;
        }
        c->members.push_back(i);
    }
    for (BatchClass& c : b->cls) {
        const int m = (int)c.members.size();
        cf_engine* r = b->inst[c.members[0]];
        if (6L * m > 65535) return bail(fail(CF_E_UNSUPPORTED, "more than 10922 instances of one grid"));
        if (col_smem(r) + sizeof(ColParams) > (size_t)227 * 1024)
            return bail(fail(CF_E_UNSUPPORTED, "Ny too large for the batched column kernel"));
        c.h_fft.resize(m);
        int rc;
        if ((rc = batch_alloc(b, (void**)&c.d_fft, sizeof(FftParams) * m))) return bail(rc);
        for (int j = 0; j < 3; ++j) {
            c.h_col[j].resize(m);
            if ((rc = batch_alloc(b, (void**)&c.d_col[j], sizeof(ColParams) * m))) return bail(rc);
        }
        const size_t smz = zsmem(r), smx = xsmem(r);
        for (int v = 0; v < col_batch_nvariants(r->P); ++v)
            if ((rc = raise_smem_limit(col_batch_kernel(r->P, v), col_smem(r, kColBatchNcol[v])))) return bail(rc);
        if ((rc = batch_alloc(b, (void**)&c.d_counter, 3 * sizeof(unsigned)))) return bail(rc);
        // the largest shapes the autotuner may choose
        const size_t smz_max = std::max(smz, (size_t)2 * 32 * zbs_of(r->Nzp, 32) * sizeof(zd));
        for (int xk : {KF_XPASS_R4, KF_XPASS_R8, KF_XPASS_R16}) {
            const size_t need = (size_t)6 * xpass_rows(xk) * xbs(r) * sizeof(zd);
            if (need <= (size_t)200 * 1024 && (rc = raise_smem_limit(fft_batch_kernel(xk, r->Nxp), need)))
                return bail(rc);
        }
        if ((rc = raise_smem_limit(fft_batch_kernel(KF_ZINV, r->Nzp), std::min(smz_max, (size_t)200 * 1024))) ||
            (rc = raise_smem_limit(fft_batch_kernel(KF_ZFWD, r->Nzp), std::min(smz_max, (size_t)200 * 1024))) ||
            (rc = raise_smem_limit(fft_batch_kernel(KF_XPASS, r->Nxp), smx)))
            return bail(rc);
        if (cudaStreamCreateWithFlags(&c.side, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&c.join, cudaEventDisableTiming) != cudaSuccess)
            return bail(fail(CF_E_CUDA, "cannot create stream"));
    }
    int rc = batch_upload(b);
    if (rc) return bail(rc);
    if ((rc = autotune_batch(b))) return bail(rc);
    *out = b;
    return CF_OK;
}

// The four launches of stage j for one size class on stream s.
// `which` selects the kernels (1 z-inverse, 2 x-pass, 4 z-forward, 8 column;
// 15: the whole stage, as the graph launches it).
static int launch_class_stage(const cf_batch* b, const BatchClass& c, int j, cudaStream_t s, int which = 15) {
    const cf_engine* r = b->inst[c.members[0]];
    const unsigned m = (unsigned)c.members.size();
    // z kernels: groups of tkz consecutive (y, kx) pairs
    const int tkz = class_tkz(b, c);
    const unsigned gzx = (unsigned)(((long)r->Ny * r->Nxh + tkz - 1) / tkz);
    if (which & 1)
        fft_batch_kernel(KF_ZINV, r->Nzp)<<<dim3(gzx, 1, 6 * m), 256, class_zsmem(b, c), s>>>(c.d_fft);
    if (which & 2) {
        const int rows = xpass_rows(c.xkind);
        fft_batch_kernel(c.xkind, r->Nxp)<<<dim3((r->Nzp + rows - 1) / rows, r->Ny, m), 256, class_xsmem(b, c), s>>>(
            c.d_fft);
    }
    if (which & 4)
        fft_batch_kernel(KF_ZFWD, r->Nzp)<<<dim3(gzx, 1, 3 * m), 256, class_zsmem(b, c), s>>>(c.d_fft);
    if (!(which & 8)) {
        CU(cudaGetLastError());
        return CF_OK;
    }
    const int ncol = kColBatchNcol[c.var];
    const int nblk = (int)((r->B + ncol - 1) / ncol);
    const ColBatchKernel ck = col_batch_kernel(r->P, c.var);
    if (c.persist) {
        CU(cudaMemsetAsync(c.d_counter + j, 0, sizeof(unsigned), s));
        ck<<<c.pgrid, ncol * col_team_threads(r->P), col_smem(r, ncol), s>>>(c.d_col[j], nblk, nblk * (int)m, c.d_counter + j);
    } else {
        ck<<<dim3((unsigned)nblk, m), ncol * col_team_threads(r->P), col_smem(r, ncol), s>>>(c.d_col[j], nblk, nblk * (int)m, nullptr);
    }
    CU(cudaGetLastError());
    return CF_OK;
}

// The ensemble autotuner.  For every size class, each kernel of the stage is
// timed alone over its candidate shapes (CUDA events around one launch per
// stage, after one untimed launch) and the fastest shape is kept for the
// ensemble's graph:
//   z kernels   columns per block tkz (the instances' own, then x2, x4 .. 32)
//   x-pass      rows per block 2, 4, 8, 16
//   column      each variant (columns per block, register bound) in both
//               schedules: one block per column block of every instance, or a
//               persistent grid of the blocks that fit at once claiming the
//               (instance, column block) items in order
// The arithmetic per column and per row is the same in every shape, so the
// choice changes no result.  It runs at creation on the zero state; the
// members' state is zeroed again afterwards.
static int autotune_batch(cf_batch* b) {
    int rc = CF_OK;
    for (cf_engine* h : b->inst) {
        if ((rc = launch_prep(h, h->U, nullptr))) return rc;
        CU(cudaStreamSynchronize(h->stream));
    }
    int dev = 0, nsm = 0, smax = 0;
    CU(cudaGetDevice(&dev));
    CU(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    CU(cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaEvent_t e0, e1;
    CU(cudaEventCreate(&e0));
    CU(cudaEventCreate(&e1));
    // device time of the kernels `which` of one step of class c (ms), or < 0
    auto time_class = [&](BatchClass& c, int which, float& ms) -> int {
        int r2 = batch_upload(b);
        for (int rep = 0; rep < 2 && !r2; ++rep) {
            if (rep == 1 && cudaEventRecord(e0, b->stream) != cudaSuccess) r2 = fail(CF_E_CUDA, "event");
            for (int j = 0; j < 3 && !r2; ++j) r2 = launch_class_stage(b, c, j, b->stream, which);
            if (rep == 1 && !r2 && cudaEventRecord(e1, b->stream) != cudaSuccess) r2 = fail(CF_E_CUDA, "event");
        }
        if (r2) return r2;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
            return fail(CF_E_CUDA, "autotuner timing failed");
        return CF_OK;
    };
    std::string out;
    for (BatchClass& c : b->cls) {
        const cf_engine* r = b->inst[c.members[0]];
        const int m = (int)c.members.size();
        char buf[1024];
        std::snprintf(buf, sizeof buf, "%dx%dx%d x%d:", c.Nx, c.Ny, c.Nz, m);
        std::string line = buf, cand;
        float ms = 0.f, total = 0.f;
        // z kernels
        {
            float best = 1e30f;
            int bt = r->tkz;
            cand.clear();
            for (int tkz = r->tkz; tkz <= 32 && !rc; tkz *= 2) {
                c.tkz = tkz;
                if (class_zsmem(b, c) > (size_t)std::min(smax, 200 * 1024)) break;
                if ((rc = time_class(c, 1 | 4, ms))) break;
                std::snprintf(buf, sizeof buf, "%s%d: %.3f", cand.empty() ? "" : ", ", tkz, ms);
                cand += buf;
                if (ms < best) best = ms, bt = tkz;
            }
            if (rc) break;
            c.tkz = bt;
            total += best;
            std::snprintf(buf, sizeof buf, " z kernels tkz=%d (%.3f ms; candidates %s)", bt, best, cand.c_str());
            line += buf;
        }
        // x-pass
        {
            float best = 1e30f;
            int bk = KF_XPASS;
            cand.clear();
            const int xkinds[] = {KF_XPASS, KF_XPASS_R4, KF_XPASS_R8, KF_XPASS_R16};
            for (int xk : xkinds) {
                c.xkind = xk;
                if (xk != KF_XPASS && class_xsmem(b, c) > (size_t)200 * 1024) continue;
                if ((rc = time_class(c, 2, ms))) break;
                std::snprintf(buf, sizeof buf, "%s%d rows: %.3f", cand.empty() ? "" : ", ", xpass_rows(xk), ms);
                cand += buf;
                if (ms < best) best = ms, bk = xk;
            }
            if (rc) break;
            c.xkind = bk;
            total += best;
            std::snprintf(buf, sizeof buf, "; x-pass %d rows per block (%.3f ms; candidates %s)", xpass_rows(bk), best,
                          cand.c_str());
            line += buf;
        }
        // column kernel
        {
            float best = 1e30f;
            int bv = 0;
            bool bp = false;
            unsigned bg = 0;
            cand.clear();
            for (int v = 0; v < col_batch_nvariants(r->P) && !rc; ++v)
                for (int pers = 0; pers < 2 && !rc; ++pers) {
                    const int ncol = kColBatchNcol[v];
                    const int nitems = (int)((r->B + ncol - 1) / ncol) * m;
                    int occ = 0;
                    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, col_batch_kernel(r->P, v), ncol * col_team_threads(r->P),
                                                                      col_smem(r, ncol)) != cudaSuccess || occ < 1) {
                        cudaGetLastError();
                        continue;
                    }
                    c.var = v;
                    c.persist = pers != 0;
                    c.pgrid = (unsigned)std::min<long>(nitems, (long)occ * nsm);
                    if (c.persist && (int)c.pgrid >= nitems) continue;  // one wave: the same as a block per item
                    if ((rc = time_class(c, 8, ms))) break;
                    std::snprintf(buf, sizeof buf, "%s(%d,%d,%s) %.3f", cand.empty() ? "" : ", ", ncol,
                                  v ? col_batch_minb(r->P, v) : 0, c.persist ? "persistent" : "grid", ms);
                    cand += buf;
                    if (ms < best) best = ms, bv = v, bp = c.persist, bg = c.pgrid;
                }
            if (rc) break;
            c.var = bv;
            c.persist = bp;
            c.pgrid = bg;
            total += best;
            std::snprintf(buf, sizeof buf, "; column kernel ncol=%d minb=%d %s (%.3f ms; candidates (ncol,minb,schedule) %s)",
                          kColBatchNcol[bv], bv ? col_batch_minb(r->P, bv) : 0,
                          bp ? ("persistent grid " + std::to_string(bg)).c_str() : "one block per item", best,
                          cand.c_str());
            line += buf;
        }
        c.step_ms = total;
        std::snprintf(buf, sizeof buf, "; %.3f ms per step of the class alone\n", total);
        out += line + buf;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if ((rc = batch_upload(b))) return rc;
    // back to the zero state the members were created with
    for (cf_engine* h : b->inst) {
        const size_t fr = sizeof(zd) * h->nr;
        for (int i = 0; i < 3; ++i) {
            CU(cudaMemsetAsync(h->U[i], 0, fr, b->stream));
            CU(cudaMemsetAsync(h->Q[i], 0, fr, b->stream));
        }
        CU(cudaMemsetAsync(h->Pf, 0, fr, b->stream));
        h->nodal_valid = false;
    }
    CU(cudaStreamSynchronize(b->stream));
    b->schedule = out;
    return CF_OK;
}

static int build_batch_graph(cf_batch* b) {
    if (b->graph) return CF_OK;
    cudaGraph_t g;
    CU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int rc = CF_OK;
    if (cudaEventRecord(b->fork, b->stream) != cudaSuccess) rc = fail(CF_E_CUDA, "event record");
    for (BatchClass& c : b->cls)
        if (!rc && cudaStreamWaitEvent(c.side, b->fork, 0) != cudaSuccess) rc = fail(CF_E_CUDA, "stream wait");
    for (int j = 0; j < 3 && !rc; ++j)
        for (BatchClass& c : b->cls)
            if (!rc) rc = launch_class_stage(b, c, j, c.side);
    for (BatchClass& c : b->cls) {
        if (!rc && cudaEventRecord(c.join, c.side) != cudaSuccess) rc = fail(CF_E_CUDA, "event record");
        if (!rc && cudaStreamWaitEvent(b->stream, c.join, 0) != cudaSuccess) rc = fail(CF_E_CUDA, "stream wait");
    }
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (rc) {
        if (e == cudaSuccess) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return fail(CF_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail(CF_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    return CF_OK;
}

int cf_batch_size(cf_batch* b) { return b ? (int)b->inst.size() : 0; }

cf_handle* cf_batch_instance(cf_batch* b, int i) {
    if (!b || i < 0 || i >= (int)b->inst.size()) {
        fail(CF_E_ARG, "instance index out of range");
        return nullptr;
    }
    return b->inst[i];
}

int cf_step_batch(cf_batch* b, int nsteps) {
    if (!b) return fail(CF_E_ARG, "null ensemble");
    if (nsteps < 0) return fail(CF_E_ARG, "nsteps must be nonnegative");
    int rc, cnt = 0;
    // instance streams: work queued through instance handles finishes first;
    // nodal fields of instances whose state was set are rebuilt
    for (cf_engine* h : b->inst) {
        if (!h->nodal_valid) {
            if ((rc = launch_prep(h, h->U, &cnt))) return rc;
            h->nodal_valid = true;
        }
        CU(cudaStreamSynchronize(h->stream));
    }
    if ((rc = batch_upload(b))) return rc;
    if ((rc = build_batch_graph(b))) return rc;
    for (int s = 0; s < nsteps; ++s) CU(cudaGraphLaunch(b->graph, b->stream));
    cnt += 12 * (int)b->cls.size() * nsteps;
    b->last_launches = cnt;
    // later work through an instance handle waits for the ensemble's steps
    CU(cudaEventRecord(b->done, b->stream));
    for (cf_engine* h : b->inst) CU(cudaStreamWaitEvent(h->stream, b->done, 0));
    return CF_OK;
}

int cf_batch_last_launch_count(cf_batch* b) { return b ? b->last_launches : 0; }
int cf_batch_schedule(cf_batch* b, char* buf, int cap) {
    if (!b || !buf || cap < 1) return fail(CF_E_ARG, "null argument");
    const int n = std::min((int)b->schedule.size(), cap - 1);
    std::memcpy(buf, b->schedule.data(), (size_t)n);
    buf[n] = 0;
    return n;
}
void* cf_batch_stream(cf_batch* b) { return b ? (void*)b->stream : nullptr; }

// ---------------------------------------------------------------------------
// Chebyshev transforms on the tensor cores (mixed-precision path)
// ---------------------------------------------------------------------------
// TF32 rounding of x (to nearest, ties away from zero), as cvt.rna.tf32.f32
static float host_tf32(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7F800000u) != 0x7F800000u) u = (u + 0x1000u) & ~0x1FFFu;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

// T^T K-tile images (TF32 heads and remainders, see cf_cheb.cuh) of
//   inverse:  y_n = sum_k a_k cos(pi n k / P)                 (chebyshev.jl:58-66, ffts.jl:162)
//   forward:  a_k = scale e_k sum_n w_n x_n cos(pi n k / P)   (ffts.jl:65-82,
//             e_k = 1/2 at k = 0, P; w_n = 1 at n = 0, P, else 2)
// Output rows per block: all of them (rounded up to 16) when at most 256,
// else split over two blocks so that each holds <= 256 TMEM columns.
static void cheb_dims(int Ny, int& NPs, int& nsplit, int& NP) {
    const int n16 = (Ny + 15) & ~15;
    nsplit = n16 <= 256 ? 1 : 2;
    NPs = nsplit == 1 ? n16 : (((n16 + 1) / 2 + 15) & ~15);
    NP = nsplit * NPs;
}
// BF16 rounding to nearest even of a finite float (the IEEE rule on the
// upper 16 bits of the FP32 pattern)
static uint16_t host_bf16(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}
static float bf16_value(uint16_t b) {
    const uint32_t u = (uint32_t)b << 16;
    float x;
    std::memcpy(&x, &u, 4);
    return x;
}
// Image bytes per piece and pieces of a split (0: TF32 head and remainder,
// 1: three BF16 pieces).
static int cheb_pieces(int split) { return split ? 3 : 2; }
static size_t cheb_piece_bytes(int Ny, int split) {
    int NPs, nsplit, NP;
    cheb_dims(Ny, NPs, nsplit, NP);
    const int nkt = (Ny + CF_CHEB_KT - 1) / CF_CHEB_KT;
    return (size_t)nkt * NP * CF_CHEB_KT * (split ? 2 : 4);
}
static void cheb_images(int Ny, int inverse, double scale, int split, std::vector<unsigned char>& img, int& NP,
                        int& nkt) {
    const int P = Ny - 1;
    int NPs, nsplit;
    cheb_dims(Ny, NPs, nsplit, NP);
    nkt = (Ny + CF_CHEB_KT - 1) / CF_CHEB_KT;
    const size_t pb = cheb_piece_bytes(Ny, split);
    img.assign(pb * cheb_pieces(split), 0);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int n = 0; n < Ny; ++n)        // output degree / node
        for (int k = 0; k < Ny; ++k) {  // input node / degree
            const long m = ((long)n * k) % (2L * P);
            const double c = (double)cosl(pi * (long double)m / (long double)P);
            double t;
            if (inverse) {
                t = c;
            } else {
                const double e = (n == 0 || n == P) ? 0.5 : 1.0, w = (k == 0 || k == P) ? 1.0 : 2.0;
                t = scale * e * w * c;
            }
            const int kt = k / CF_CHEB_KT, kl = k % CF_CHEB_KT;
            if (split == 0) {
                const float th = host_tf32((float)t);
                const float tl = host_tf32((float)(t - (double)th));
                const size_t idx = (size_t)kt * NP * CF_CHEB_KT + ((size_t)(kl / 4) * NP + n) * 4 + (kl % 4);
                std::memcpy(&img[4 * idx], &th, 4);
                std::memcpy(&img[pb + 4 * idx], &tl, 4);
            } else {
                const float tf = (float)t;
                const uint16_t b0 = host_bf16(tf);
                const float r1 = tf - bf16_value(b0);
                const uint16_t b1 = host_bf16(r1);
                const uint16_t b2 = host_bf16(r1 - bf16_value(b1));
                const size_t idx = (size_t)kt * NP * CF_CHEB_KT + ((size_t)(kl / 8) * NP + n) * 8 + (kl % 8);
                std::memcpy(&img[2 * idx], &b0, 2);
                std::memcpy(&img[pb + 2 * idx], &b1, 2);
                std::memcpy(&img[2 * pb + 2 * idx], &b2, 2);
            }
        }
}

// Shared-memory stages of k_cheb_mma (two when they fit) and its dynamic
// shared memory, padded so that the blocks that fit on an SM (228 KB, 1 KB
// reserved per block) also fit in its 512 TMEM columns, so no block ever waits
// in the TMEM allocation.
static int cheb_stages(int NPs, int split) {
    const size_t stage = cheb_stage_bytes(NPs, split);
    return 2 * stage + 64 <= (size_t)220 * 1024 ? 2 : 1;
}
static size_t cheb_smem(int NPs, int split) {
    const size_t stage = cheb_stage_bytes(NPs, split);
    const size_t tiles = cheb_stages(NPs, split) * stage + 64;
    const int ncols = NPs <= 32 ? 32 : (NPs <= 64 ? 64 : (NPs <= 128 ? 128 : 256));
    const size_t per_sm = 233472, maxb = 512 / ncols;
    const size_t floor_b = per_sm / (maxb + 1) - 1024 + 16;  // maxb + 1 blocks no longer fit
    return std::max(tiles, floor_b);
}
static ChebKernel cheb_kernel(int split) { return split ? k_cheb_mma<1> : k_cheb_mma<0>; }

// The folded transform (k_cheb_sym): per parity q the outputs n = 2m + q
// (N[0] = P/2 + 1, N[1] = P/2), the inputs (P/2 + 1 and P/2), both padded to
// 16; the folded T^T of each parity resident in shared memory with nst A
// stages (4 .. 2).  False when it does not fit (large Ny): the unfolded
// kernel runs.
static bool cheb_sym_dims(int Ny, int split, ChebSymDims& d) {
    const int P = Ny - 1, H = P / 2;
    if (P < 4 || P % 2) return false;
    d.N[0] = H + 1;
    d.N[1] = H;
    const int es = split ? 2 : 4, npc = cheb_pieces(split), epc = 16 / es;
    for (int q = 0; q < 2; ++q) {
        d.Npad[q] = (d.N[q] + 15) & ~15;
        d.Kpad[q] = (d.N[q] + 15) & ~15;
        d.bbytes[q] = (unsigned)((d.Kpad[q] / epc) * d.Npad[q] * 16);
    }
    if (d.Npad[0] > 256) return false;
    const size_t apb = (size_t)128 * 16 * es;
    for (int nst = 4; nst >= 2; --nst) {
        const size_t sm = (size_t)npc * std::max(d.bbytes[0], d.bbytes[1]) + (size_t)nst * npc * apb +
                          (size_t)(2 * nst + 5) * 8 + 16;
        if (sm <= (size_t)227 * 1024) {
            d.nst = nst;
            // at least half an SM's shared memory, so that one CTA runs per
            // SM and its 512 TMEM columns are never contended
            d.smem = std::max(sm, (size_t)116 * 1024);
            return true;
        }
    }
    return false;
}
// Folded T^T images: parity 0's pieces, then parity 1's, each piece
// [Kpad / EPC chunks][Npad rows][16 bytes] with input k of row m at chunk
// k / EPC, element k % EPC (the layout of cheb_images over all K at once);
// row m of parity q is output n = 2m + q, its inputs k < N[q] (parity 0: k =
// 0..P/2, the last multiplying X_{P/2} alone; parity 1: k = 0..P/2 - 1).
static void cheb_sym_images(int Ny, int inverse, double scale, int split, const ChebSymDims& d,
                            std::vector<unsigned char>& img) {
    const int P = Ny - 1, npc = cheb_pieces(split);
    img.assign((size_t)npc * (d.bbytes[0] + d.bbytes[1]), 0);
    const long double pi = 3.141592653589793238462643383279502884L;
    size_t base = 0;
    for (int q = 0; q < 2; ++q) {
        const size_t pb = d.bbytes[q];
        for (int m = 0; m < d.N[q]; ++m)
            for (int k = 0; k < d.N[q]; ++k) {
                const int n = 2 * m + q;
                const long mm = ((long)n * k) % (2L * P);
                const double c = (double)cosl(pi * (long double)mm / (long double)P);
                double t;
                if (inverse) {
                    t = c;
                } else {
                    const double e = (n == 0 || n == P) ? 0.5 : 1.0, w = (k == 0 || k == P) ? 1.0 : 2.0;
                    t = scale * e * w * c;
                }
                if (split == 0) {
                    const float th = host_tf32((float)t);
                    const float tl = host_tf32((float)(t - (double)th));
                    const size_t o = ((size_t)(k / 4) * d.Npad[q] + m) * 16 + (k % 4) * 4;
                    std::memcpy(&img[base + o], &th, 4);
                    std::memcpy(&img[base + pb + o], &tl, 4);
                } else {
                    const float tf = (float)t;
                    const uint16_t b0 = host_bf16(tf);
                    const float r1 = tf - bf16_value(b0);
                    const uint16_t b1 = host_bf16(r1);
                    const uint16_t b2 = host_bf16(r1 - bf16_value(b1));
                    const size_t o = ((size_t)(k / 8) * d.Npad[q] + m) * 16 + (k % 8) * 2;
                    std::memcpy(&img[base + o], &b0, 2);
                    std::memcpy(&img[base + pb + o], &b1, 2);
                    std::memcpy(&img[base + 2 * pb + o], &b2, 2);
                }
            }
        base += (size_t)npc * pb;
    }
}
static ChebSymKernel cheb_sym_kernel(int split) { return split ? k_cheb_sym<1> : k_cheb_sym<0>; }
// two CTAs (one per parity) per pair, a pair per two SMs, no more pairs than items
static int cheb_sym_grid(long C, int nf) {
    static int nsm = 0;
    if (!nsm) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm < 2) nsm = 2;
    }
    const long items = (long)nf * ((C + 127) / 128);
    return 2 * (int)std::max(1L, std::min((long)(nsm / 2), items));
}

int cf_cheb_transform_split(const float* X, float* Y, int Ny, long C, int nfields, int inverse, double scale,
                            int split) {
    if (!X || !Y) return fail(CF_E_ARG, "null argument");
    if (Ny < 2 || Ny > 512) return fail(CF_E_UNSUPPORTED, "Chebyshev transform needs 2 <= Ny <= 512");
    if (C < 1 || nfields < 1 || nfields > CF_CHEB_MAXF) return fail(CF_E_ARG, "need C >= 1 and 1..6 fields");
    if (split != 0 && split != 1) return fail(CF_E_ARG, "split must be 0 (TF32) or 1 (BF16)");
    std::vector<unsigned char> img;
    int NP = 0, nkt = 0;
    ChebSymDims sd;
    const bool sym = cheb_sym_dims(Ny, split, sd);
    if (sym) cheb_sym_images(Ny, inverse, scale, split, sd, img);
    else cheb_images(Ny, inverse, scale, split, img, NP, nkt);
    const size_t pb = cheb_piece_bytes(Ny, split);
    const size_t fb = sizeof(float) * (size_t)Ny * C;
    float *dX = nullptr, *dY = nullptr;
    unsigned char* dB = nullptr;
    int* derr = nullptr;
    int rc = CF_OK;
    auto cleanup = [&]() {
        cudaFree(dX);
        cudaFree(dY);
        cudaFree(dB);
        cudaFree(derr);
    };
    if (cudaMalloc(&dX, fb * nfields) != cudaSuccess || cudaMalloc(&dY, fb * nfields) != cudaSuccess ||
        cudaMalloc(&dB, img.size()) != cudaSuccess || cudaMalloc(&derr, sizeof(int)) != cudaSuccess) {
        cleanup();
        return fail(CF_E_NOMEM, "device allocation failed");
    }
    do {
        if (cudaMemcpy(dX, X, fb * nfields, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(dB, img.data(), img.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemset(derr, 0, sizeof(int)) != cudaSuccess || cudaMemset(dY, 0, fb * nfields) != cudaSuccess) {
            rc = fail(CF_E_CUDA, "upload failed");
            break;
        }
        if (sym) {
            if ((rc = raise_smem_limit(cheb_sym_kernel(split), sd.smem))) break;
            ChebSymParams q;
            std::memset(&q, 0, sizeof(q));
            q.P = Ny - 1;
            for (int i = 0; i < 2; ++i) {
                q.N[i] = sd.N[i];
                q.Npad[i] = sd.Npad[i];
                q.Kpad[i] = sd.Kpad[i];
                q.bbytes[i] = sd.bbytes[i];
            }
            q.nst = sd.nst;
            q.C = C;
            q.nf = nfields;
            q.ntiles = (int)((C + 127) / 128);
            for (int f = 0; f < nfields; ++f) {
                q.X[f] = dX + (size_t)f * Ny * C;
                q.Y[f] = dY + (size_t)f * Ny * C;
            }
            q.B[0] = dB;
            q.B[1] = dB + (size_t)cheb_pieces(split) * sd.bbytes[0];
            q.err = derr;
            q.spins = CF_WAIT_SPINS;
            cheb_sym_kernel(split)<<<cheb_sym_grid(C, nfields), 416, sd.smem>>>(q);
        }
        int NPs, nsplit, NPt;
        cheb_dims(Ny, NPs, nsplit, NPt);
        if (!sym && (rc = raise_smem_limit(cheb_kernel(split), cheb_smem(NPs, split)))) break;
        ChebParams p;
        std::memset(&p, 0, sizeof(p));
        p.Ny = Ny;
        p.NP = NP;
        p.nkt = nkt;
        p.NPs = NPs;
        p.nst = cheb_stages(NPs, split);
        p.C = C;
        for (int f = 0; f < nfields; ++f) {
            p.X[f] = dX + (size_t)f * Ny * C;
            p.Y[f] = dY + (size_t)f * Ny * C;
        }
        for (int q = 0; q < cheb_pieces(split); ++q) p.B[q] = dB + q * pb;
        p.err = derr;
        p.spins = CF_WAIT_SPINS;
        dim3 grid((unsigned)((C + CF_CHEB_MT - 1) / CF_CHEB_MT), (unsigned)nfields, (unsigned)nsplit);
        if (!sym) cheb_kernel(split)<<<grid, 128, cheb_smem(NPs, split)>>>(p);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) {
            rc = fail(CF_E_CUDA, std::string("Chebyshev transform kernel: ") + cudaGetErrorString(e));
            break;
        }
        int herr = 0;
        cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
        if (herr) {
            rc = fail(CF_E_CUDA, "Chebyshev transform kernel: a tensor-core wait timed out");
            break;
        }
        if (cudaMemcpy(Y, dY, fb * nfields, cudaMemcpyDeviceToHost) != cudaSuccess) rc = fail(CF_E_CUDA, "download failed");
    } while (0);
    cleanup();
    return rc;
}
int cf_cheb_transform(const float* X, float* Y, int Ny, long C, int nfields, int inverse, double scale) {
    return cf_cheb_transform_split(X, Y, Ny, C, nfields, inverse, scale, 0);
}
