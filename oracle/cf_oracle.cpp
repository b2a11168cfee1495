// cf_oracle.cpp -- CPU FP64 ORACLE for the CNRK2 step of ChannelFlow.jl.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker, never the product:
// only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg (and its
// `--impl reference` arm) may load the library built from it.  The product path
// (libcfb200) never links, loads or calls anything here.
//
// It restates, function by function, the reference algorithm (paths relative
// to the ChannelFlow.jl repository):
//   grids / storage      src/grids.jl:22-96, src/indexing.jl:14-28
//   transforms           src/ffts.jl:65-82, 151-166, 242-312
//   DCT-I (REDFT00)      src/transforms/chebyshev.jl:45-66
//   operators            src/fields/operators.jl:14-190, 270-294
//   nonlinear terms      src/nonlinear.jl:113-193 (rotational, convective,
//                        divergence forms)
//   influence solver     src/solvers/influence.jl:60-316
//   batched bank         src/solvers/batchedinfluence.jl:32-160
//   mean mode            src/solvers/meanmode.jl:13-150
//   Stokes wrapper       src/solvers/stokes.jl:23-108
//   CNRK2                src/timesteppers/cnrk2.jl:12-207
//   projection/pressure  src/pressure.jl:36-204
//   diagnostics          src/postprocessing.jl:21-128
// The tau Helmholtz solver of the un-vendored dependency
// ChebyshevHelmoltzSolvers.jl (v0.1.0, git-tree 27b8d9f9...) is restated from
// its defining tau system (docs/src/spatial.md:448-475): rows 0..P-2 of
// (theta0*D^2 - theta1*I) a = f plus two wall rows.  The default solver
// assembles that system explicitly (parity split) and factors it by dense LU
// with partial pivoting; for large Ny a quasi-tridiagonal elimination of the
// same system (spectral integration form) is available and is checked against
// the dense path by the tests.
//
// Storage: complex spectral fields are (Ny, Nz, Nxh) in C order, i.e. the
// reference's column-major (k, l, n) with k fastest; padded physical fields are
// (Ny, Nzp, Nxp) in C order.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cd;

static thread_local std::string g_error;
static void set_error(const std::string& s) { g_error = s; }

// ---------------------------------------------------------------------------
// Complex FFT: Stockham autosort, arbitrary length (radix 4, 2, 3, 5 and a
// generic prime butterfly).  Twiddles are computed in long double.
// ---------------------------------------------------------------------------
struct FFTPlan {
    int n = 0;
    std::vector<int> radices;
    std::vector<cd> tw;  // exp(-2 pi i k / n), k = 0..n-1
};

static std::vector<int> factorize(int n) {
    std::vector<int> r;
    while (n % 4 == 0) { r.push_back(4); n /= 4; }
    while (n % 2 == 0) { r.push_back(2); n /= 2; }
    while (n % 3 == 0) { r.push_back(3); n /= 3; }
    while (n % 5 == 0) { r.push_back(5); n /= 5; }
    for (int p = 7; p * p <= n; p += 2)
        while (n % p == 0) { r.push_back(p); n /= p; }
    if (n > 1) r.push_back(n);
    return r;
}

static const FFTPlan& get_plan(int n) {
    static std::mutex mu;
    static std::map<int, std::unique_ptr<FFTPlan>> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(n);
    if (it != cache.end()) return *it->second;
    auto p = std::make_unique<FFTPlan>();
    p->n = n;
    p->radices = factorize(n);
    p->tw.resize(n);
    const long double twopi = 6.283185307179586476925286766559005768L;
    for (int k = 0; k < n; ++k) {
        long double a = -twopi * (long double)k / (long double)n;
        p->tw[k] = cd((double)cosl(a), (double)sinl(a));
    }
    auto& ref = *p;
    cache[n] = std::move(p);
    return ref;
}

// In-place complex FFT of x (length n, contiguous); sign = -1 forward, +1 backward
// (unnormalised).  work must hold n elements.
static void fft_inplace(cd* x, cd* work, int n, int sign) {
    if (n == 1) return;
    const FFTPlan& p = get_plan(n);
    cd* src = x;
    cd* dst = work;
    int Ns = 1;
    cd v[64];
    std::vector<cd> vbig;
    for (int R : p.radices) {
        cd* vv = v;
        if (R > 64) { vbig.resize(R); vv = vbig.data(); }
        const int NR = n / R;
        const int step = n / (Ns * R);
        for (int j = 0; j < NR; ++j) {
            const int k = j % Ns;
            for (int r = 0; r < R; ++r) {
                cd w = p.tw[(size_t)((long long)k * r * step % n)];
                if (sign > 0) w = std::conj(w);
                vv[r] = src[j + r * NR] * w;
            }
            // radix-R DFT in place on vv
            if (R == 2) {
                cd a = vv[0], b = vv[1];
                vv[0] = a + b; vv[1] = a - b;
            } else if (R == 4) {
                cd a0 = vv[0] + vv[2], a1 = vv[0] - vv[2];
                cd a2 = vv[1] + vv[3], a3 = vv[1] - vv[3];
                // multiply a3 by -i (forward) or +i (backward)
                cd a3r = sign < 0 ? cd(a3.imag(), -a3.real()) : cd(-a3.imag(), a3.real());
                vv[0] = a0 + a2; vv[2] = a0 - a2;
                vv[1] = a1 + a3r; vv[3] = a1 - a3r;
            } else {
                cd out[64];
                std::vector<cd> outbig;
                cd* o = out;
                if (R > 64) { outbig.resize(R); o = outbig.data(); }
                const int stepR = n / R;  // exp(-2 pi i q r / R) = tw[(q r mod R) * n/R]
                for (int q = 0; q < R; ++q) {
                    cd s = 0;
                    for (int r = 0; r < R; ++r) {
                        cd w = p.tw[(size_t)(((long long)q * r) % R) * stepR];
                        if (sign > 0) w = std::conj(w);
                        s += vv[r] * w;
                    }
                    o[q] = s;
                }
                for (int q = 0; q < R; ++q) vv[q] = o[q];
            }
            const int idxD = (j / Ns) * Ns * R + k;
            for (int r = 0; r < R; ++r) dst[idxD + r * Ns] = vv[r];
        }
        std::swap(src, dst);
        Ns *= R;
    }
    if (src != x) std::memcpy(x, src, sizeof(cd) * n);
}

// REDFT00 (DCT-I, unnormalised) of a complex sequence of length P+1 with
// stride s, in place: Y_k = x_0 + (-1)^k x_P + 2 sum_{n=1}^{P-1} x_n cos(pi n k/P).
// Computed as the FFT of the even extension of length 2P.
static void redft00(cd* x, long s, int P, cd* buf /*2P*/, cd* work /*2P*/) {
    const int L = 2 * P;
    for (int n = 0; n <= P; ++n) buf[n] = x[n * s];
    for (int n = 1; n < P; ++n) buf[L - n] = x[n * s];
    fft_inplace(buf, work, L, -1);
    for (int k = 0; k <= P; ++k) x[k * s] = buf[k];
}

// ---------------------------------------------------------------------------
// Chebyshev coefficient utilities (ordinary coefficients, src/fields/operators.jl)
// ---------------------------------------------------------------------------
// Derivative recurrence of _batchdiff! (batchedinfluence.jl:32-43) for one
// column with stride s: b_P = 0, b_{P-1} = 2P a_P, b_n = b_{n+2} + 2(n+1) a_{n+1},
// b_0 halved.  Works for real or complex T.
template <class T>
static void cheb_diff(const T* a, long sa, T* b, long sb, int Ny) {
    const int P = Ny - 1;
    std::vector<T> tmp(Ny);
    tmp[P] = T(0);
    if (P >= 1) tmp[P - 1] = T(2.0 * P) * a[P * sa];
    for (int n = P - 2; n >= 0; --n) tmp[n] = tmp[n + 2] + T(2.0 * (n + 1)) * a[(n + 1) * sa];
    tmp[0] *= 0.5;
    for (int n = 0; n < Ny; ++n) b[n * sb] = tmp[n];
}

// Mean over y: a0 + sum_{even n>=2} a_n/(1-n^2)  (meanmode.jl:13-19)
template <class T>
static T bulkmean(const T* a, long s, int Ny) {
    T v = a[0];
    for (int n = 2; n <= Ny - 1; n += 2) v += a[n * s] / (1.0 - (double)n * n);
    return v;
}

// u'(+1) = sum n^2 a_n ; u'(-1) = sum (-1)^(n+1) n^2 a_n
template <class T>
static T wall_deriv(const T* a, long s, int Ny, bool right) {
    T v = T(0);
    for (int n = 1; n < Ny; ++n) {
        double w = (double)n * n;
        if (!right && (n % 2 == 0)) w = -w;
        v += w * a[n * s];
    }
    return v;
}

// Chebyshev coefficients from values at y_j = cos(pi j/P) (chebcoeffs)
static void cheb_coeffs(const double* vals, double* coef, int Ny) {
    const int P = Ny - 1;
    std::vector<cd> x(Ny), buf(2 * P), work(2 * P);
    for (int j = 0; j < Ny; ++j) x[j] = vals[j];
    redft00(x.data(), 1, P, buf.data(), work.data());
    for (int n = 0; n < Ny; ++n) {
        double c = x[n].real() / P;
        if (n == 0 || n == P) c *= 0.5;
        coef[n] = c;
    }
}

// ---------------------------------------------------------------------------
// Tau Helmholtz solver: rows 0..P-2 of (th0*D^2 - th1) a = f, plus wall rows.
// Dirichlet: a(+1) = bp, a(-1) = bm.  Neumann: a'(+1) = bp, a'(-1) = bm.
// ---------------------------------------------------------------------------
// Timing samples only: when > 1, every independent loop of a stage (columns,
// planes, rows, points) runs over 1/g_sample_div of its range, so a bounded
// fraction of one stage can be timed.  Results are then not meaningful.
static long g_sample_div = 1;
static inline long sampled(long n) { return g_sample_div > 1 ? std::max(1L, n / g_sample_div) : n; }
static int g_helm_method = 0;       // 0 auto, 1 dense, 2 quasi-tridiagonal
static int g_dense_max_ny = 65;     // auto: dense LU up to this Ny

struct Helm {
    int Ny = 0, P = 0;
    bool neumann = false;
    double th0 = 1, th1 = 0;
    bool dense = true;
    // dense parity blocks
    int M[2] = {0, 0};
    std::vector<double> LU[2];
    std::vector<int> piv[2];
    // quasi-tridiagonal factors (index by n)
    std::vector<double> alpha, invden;
    double SA[2] = {0, 0};

    static double cm(int m) { return m == 0 ? 2.0 : 1.0; }

    void init(int Ny_, double t0, double t1, bool neum) {
        Ny = Ny_; P = Ny - 1; th0 = t0; th1 = t1; neumann = neum;
        dense = g_helm_method == 1 || (g_helm_method == 0 && Ny <= g_dense_max_ny);
        if (dense) init_dense(); else init_qt();
    }
    // number of unknowns of parity par: n = par, par+2, ... <= P
    int count(int par) const { return par > P ? 0 : (P - par) / 2 + 1; }

    void init_dense() {
        for (int par = 0; par < 2; ++par) {
            int m = count(par);
            M[par] = m;
            std::vector<double>& A = LU[par];
            A.assign((size_t)m * m, 0.0);
            int row = 0;
            for (int n = par; n <= P - 2; n += 2, ++row) {
                for (int j = 0; j < m; ++j) {
                    int mm = par + 2 * j;
                    double v = 0;
                    if (mm >= n + 2) v = th0 * (double)mm * ((double)mm * mm - (double)n * n) / cm(n);
                    if (mm == n) v -= th1;
                    A[(size_t)row * m + j] = v;
                }
            }
            // wall row
            for (int j = 0; j < m; ++j) {
                int mm = par + 2 * j;
                A[(size_t)row * m + j] = neumann ? (double)mm * mm : 1.0;
            }
            // LU with partial pivoting
            std::vector<int>& pv = piv[par];
            pv.resize(m);
            for (int c = 0; c < m; ++c) {
                int p = c;
                double best = std::fabs(A[(size_t)c * m + c]);
                for (int r = c + 1; r < m; ++r) {
                    double v = std::fabs(A[(size_t)r * m + c]);
                    if (v > best) { best = v; p = r; }
                }
                pv[c] = p;
                if (p != c)
                    for (int j = 0; j < m; ++j) std::swap(A[(size_t)c * m + j], A[(size_t)p * m + j]);
                double d = A[(size_t)c * m + c];
                for (int r = c + 1; r < m; ++r) {
                    double f = A[(size_t)r * m + c] / d;
                    A[(size_t)r * m + c] = f;
                    if (f != 0.0)
                        for (int j = c + 1; j < m; ++j) A[(size_t)r * m + j] -= f * A[(size_t)c * m + j];
                }
            }
        }
    }

    // coefficients of equation n (n >= 2): s a_{n-2} + d a_n + u a_{n+2} = g
    double eq_s(int n) const { return -cm(n - 2) * th1 / (4.0 * n * (n - 1)); }
    double eq_d(int n) const { return th0 + (n <= P - 2 ? th1 / (2.0 * ((double)n * n - 1.0)) : 0.0); }
    double eq_u(int n) const { return (n + 2 <= P - 2) ? -th1 / (4.0 * n * (n + 1)) : 0.0; }
    double wall_w(int n) const { return neumann ? (double)n * n : 1.0; }

    void init_qt() {
        alpha.assign(Ny + 2, 0.0);
        invden.assign(Ny + 2, 0.0);
        for (int par = 0; par < 2; ++par) {
            int top = par + 2 * (count(par) - 1);
            double anext = 0;
            for (int n = top; n >= par + 2; n -= 2) {
                double den = eq_d(n) + eq_u(n) * anext;
                invden[n] = 1.0 / den;
                alpha[n] = -eq_s(n) / den;
                anext = alpha[n];
            }
            double A = 1.0, sa = wall_w(par);
            for (int n = par + 2; n <= top; n += 2) {
                A *= alpha[n];
                sa += wall_w(n) * A;
            }
            SA[par] = sa;
        }
    }

    // solve for real coefficients a (length Ny) from f (length Ny)
    void solve(const double* f, double bp, double bm, double* a) const {
        double bc[2];
        if (!neumann) { bc[0] = 0.5 * (bp + bm); bc[1] = 0.5 * (bp - bm); }
        else { bc[0] = 0.5 * (bp - bm); bc[1] = 0.5 * (bp + bm); }
        if (dense) {
            std::vector<double> x;
            for (int par = 0; par < 2; ++par) {
                int m = M[par];
                if (m == 0) continue;
                x.assign(m, 0.0);
                int row = 0;
                for (int n = par; n <= P - 2; n += 2, ++row) x[row] = f[n];
                x[row] = bc[par];
                const std::vector<double>& A = LU[par];
                const std::vector<int>& pv = piv[par];
                // rows were interchanged whole during factorisation, so apply
                // every interchange before the forward substitution
                for (int c = 0; c < m; ++c)
                    if (pv[c] != c) std::swap(x[c], x[pv[c]]);
                for (int c = 0; c < m; ++c)
                    for (int r = c + 1; r < m; ++r) x[r] -= A[(size_t)r * m + c] * x[c];
                for (int c = m - 1; c >= 0; --c) {
                    double s = x[c];
                    for (int j = c + 1; j < m; ++j) s -= A[(size_t)c * m + j] * x[j];
                    x[c] = s / A[(size_t)c * m + c];
                }
                for (int j = 0; j < m; ++j) a[par + 2 * j] = x[j];
            }
            return;
        }
        // quasi-tridiagonal elimination
        std::vector<double> beta(Ny + 2, 0.0);
        for (int par = 0; par < 2; ++par) {
            int cnt = count(par);
            if (cnt == 0) continue;
            int top = par + 2 * (cnt - 1);
            double bnext = 0;
            for (int n = top; n >= par + 2; n -= 2) {
                double g = cm(n - 2) * f[n - 2] / (4.0 * n * (n - 1));
                if (n <= P - 2) g -= f[n] / (2.0 * ((double)n * n - 1.0));
                if (n + 2 <= P - 2) g += f[n + 2] / (4.0 * n * (n + 1));
                beta[n] = (g - eq_u(n) * bnext) * invden[n];
                bnext = beta[n];
            }
            double C = 0, sc = 0;
            for (int n = par + 2; n <= top; n += 2) {
                C = alpha[n] * C + beta[n];
                sc += wall_w(n) * C;
            }
            double a0 = (bc[par] - sc) / SA[par];
            a[par] = a0;
            double prev = a0;
            for (int n = par + 2; n <= top; n += 2) {
                prev = alpha[n] * prev + beta[n];
                a[n] = prev;
            }
        }
    }
    void solve_c(const cd* f, cd bp, cd bm, cd* a) const {
        std::vector<double> fr(Ny), fi(Ny), ar(Ny), ai(Ny);
        for (int n = 0; n < Ny; ++n) { fr[n] = f[n].real(); fi[n] = f[n].imag(); }
        solve(fr.data(), bp.real(), bm.real(), ar.data());
        solve(fi.data(), bp.imag(), bm.imag(), ai.data());
        for (int n = 0; n < Ny; ++n) a[n] = cd(ar[n], ai[n]);
    }
};

// ---------------------------------------------------------------------------
// Per-column influence/tau solver (influence.jl and the batched bank).  The
// batched bank (batchedinfluence.jl:45-98) computes exactly the same responses
// column by column, with the zero-wavenumber pressure placeholder kappa^2 -> 1.
// ---------------------------------------------------------------------------
struct ModeSolver {
    int Ny = 0;
    double k = 0, l = 0, nu = 0, shift = 0;
    Helm ph, vh;
    std::vector<double> pp, pm, vp, vm, p0, v0;
    double inf[4] = {0, 0, 0, 0};  // inverse influence matrix, row major
    double sigma[2] = {0, 0};

    // returns false when the influence matrix is singular
    bool init(int Ny_, double k_, double l_, double nu_, double lambda, bool placeholder) {
        Ny = Ny_; k = k_; l = l_; nu = nu_;
        const int P = Ny - 1;
        double kap2 = k * k + l * l;
        shift = lambda + nu * kap2;
        ph.init(Ny, 1.0, (placeholder && kap2 == 0.0) ? 1.0 : kap2, false);
        vh.init(Ny, nu, shift, false);
        std::vector<double> zero(Ny, 0.0), work(Ny);
        pp.resize(Ny); pm.resize(Ny); vp.resize(Ny); vm.resize(Ny); p0.resize(Ny); v0.resize(Ny);
        ph.solve(zero.data(), 1.0, 0.0, pp.data());
        cheb_diff(pp.data(), 1, work.data(), 1, Ny);
        vh.solve(work.data(), 0.0, 0.0, vp.data());
        ph.solve(zero.data(), 0.0, 1.0, pm.data());
        cheb_diff(pm.data(), 1, work.data(), 1, Ny);
        vh.solve(work.data(), 0.0, 0.0, vm.data());
        double a = wall_deriv(vp.data(), 1, Ny, true), b = wall_deriv(vm.data(), 1, Ny, true);
        double c = wall_deriv(vp.data(), 1, Ny, false), d = wall_deriv(vm.data(), 1, Ny, false);
        double scale = std::max(std::max(std::fabs(a), std::fabs(b)), std::max(std::fabs(c), std::fabs(d)));
        if (!(std::isfinite(scale) && scale > 0)) return false;
        a /= scale; b /= scale; c /= scale; d /= scale;
        double det = a * d - b * c;
        if (!(std::isfinite(det) && std::fabs(det) > 2.220446049250313e-16 * std::max(std::fabs(a * d), std::fabs(b * c))))
            return false;
        inf[0] = d / (det * scale); inf[1] = -b / (det * scale);
        inf[2] = -c / (det * scale); inf[3] = a / (det * scale);
        // auxiliary tau problem: source (T_{P-1} + T_P)'
        std::vector<double> src(Ny, 0.0), forcing(Ny);
        src[P - 1] = 1.0; src[P] = 1.0;
        cheb_diff(src.data(), 1, forcing.data(), 1, Ny);
        ph.solve(forcing.data(), 0.0, 0.0, p0.data());
        cheb_diff(p0.data(), 1, forcing.data(), 1, Ny);
        vh.solve(forcing.data(), 0.0, 0.0, v0.data());
        influence(p0.data(), v0.data());
        cheb_diff(p0.data(), 1, forcing.data(), 1, Ny);
        sigma[0] = shift * v0[P - 1] + forcing[P - 1];
        sigma[1] = shift * v0[P];
        return true;
    }
    template <class T>
    void influence(T* p, T* v) const {
        T upper = T(0), lower = T(0);
        for (int n = 1; n < Ny; ++n) {
            T term = (double)n * n * v[n];
            upper -= term;
            lower -= (n % 2 == 1 ? 1.0 : -1.0) * term;
        }
        T dp = inf[0] * upper + inf[1] * lower;
        T dm = inf[2] * upper + inf[3] * lower;
        for (int n = 0; n < Ny; ++n) {
            p[n] += dp * pp[n] + dm * pm[n];
            v[n] += dp * vp[n] + dm * vm[n];
        }
    }
    // Batched solve for one column (batchedinfluence.jl:129-160); sources
    // strided by s, outputs strided by s.
    void solve(cd* u, cd* v, cd* w, cd* p, const cd* Rx, const cd* Ry, const cd* Rz, long s) const {
        const int P = Ny - 1;
        std::vector<cd> rx(Ny), ry(Ny), rz(Ny), r(Ny), q(Ny), pc(Ny), vc(Ny), uc(Ny), wc(Ny), dp(Ny);
        for (int n = 0; n < Ny; ++n) { rx[n] = Rx[n * s]; ry[n] = Ry[n * s]; rz[n] = Rz[n * s]; }
        const cd I(0, 1);
        cheb_diff(ry.data(), 1, r.data(), 1, Ny);
        for (int n = 0; n < Ny; ++n) r[n] += I * k * rx[n] + I * l * rz[n];
        ph.solve_c(r.data(), 0.0, 0.0, pc.data());
        cheb_diff(pc.data(), 1, q.data(), 1, Ny);
        for (int n = 0; n < Ny; ++n) q[n] -= ry[n];
        vh.solve_c(q.data(), 0.0, 0.0, vc.data());
        influence(pc.data(), vc.data());
        cheb_diff(pc.data(), 1, dp.data(), 1, Ny);
        cd s1 = (shift * vc[P - 1] + dp[P - 1] - ry[P - 1]) / (1.0 - sigma[0]);
        cd s2 = (shift * vc[P] + dp[P] - ry[P]) / (1.0 - sigma[1]);
        for (int n = 0; n < Ny; ++n) {
            pc[n] += (n % 2 == 0 ? s1 : s2) * p0[n];
            vc[n] += (n % 2 == 0 ? s2 : s1) * v0[n];
        }
        for (int n = 0; n < Ny; ++n) r[n] = I * k * pc[n] - rx[n];
        vh.solve_c(r.data(), 0.0, 0.0, uc.data());
        for (int n = 0; n < Ny; ++n) r[n] = I * l * pc[n] - rz[n];
        vh.solve_c(r.data(), 0.0, 0.0, wc.data());
        for (int n = 0; n < Ny; ++n) {
            u[n * s] = uc[n]; v[n * s] = vc[n]; w[n * s] = wc[n]; p[n * s] = pc[n];
        }
    }
    // Scalar InfluenceModeSolver solve (influence.jl:205-316): real and
    // imaginary pressure/normal-velocity pairs solved separately.
    void solve_scalar(cd* u, cd* v, cd* w, cd* p, const cd* Rx, const cd* Ry, const cd* Rz) const {
        const int P = Ny - 1;
        std::vector<double> ryc(Ny), r(Ny), pc(Ny), vc(Ny), work(Ny), a(Ny), b(Ny);
        for (int imag = 0; imag < 2; ++imag) {
            for (int n = 0; n < Ny; ++n) ryc[n] = imag ? Ry[n].imag() : Ry[n].real();
            cheb_diff(ryc.data(), 1, r.data(), 1, Ny);
            for (int n = 0; n < Ny; ++n)
                r[n] += imag ? k * Rx[n].real() + l * Rz[n].real() : -k * Rx[n].imag() - l * Rz[n].imag();
            ph.solve(r.data(), 0.0, 0.0, pc.data());
            cheb_diff(pc.data(), 1, work.data(), 1, Ny);
            for (int n = 0; n < Ny; ++n) work[n] -= ryc[n];
            vh.solve(work.data(), 0.0, 0.0, vc.data());
            influence(pc.data(), vc.data());
            cheb_diff(pc.data(), 1, work.data(), 1, Ny);
            double sNm1 = (shift * vc[P - 1] + work[P - 1] - ryc[P - 1]) / (1.0 - sigma[0]);
            double sN = (shift * vc[P] + work[P] - ryc[P]) / (1.0 - sigma[1]);
            for (int n = 0; n < Ny; ++n) {
                pc[n] += (n % 2 == 0 ? sNm1 : sN) * p0[n];
                vc[n] += (n % 2 == 0 ? sN : sNm1) * v0[n];
            }
            for (int n = 0; n < Ny; ++n) {
                if (imag) { p[n] += cd(0, pc[n]); v[n] += cd(0, vc[n]); }
                else { p[n] = pc[n]; v[n] = vc[n]; }
            }
        }
        for (int c = 0; c < 2; ++c) {
            cd* out = c == 0 ? u : w;
            const cd* src = c == 0 ? Rx : Rz;
            double kk = c == 0 ? k : l;
            for (int n = 0; n < Ny; ++n) {
                pc[n] = -kk * p[n].imag() - src[n].real();
                vc[n] = kk * p[n].real() - src[n].imag();
            }
            vh.solve(pc.data(), 0.0, 0.0, a.data());
            vh.solve(vc.data(), 0.0, 0.0, b.data());
            for (int n = 0; n < Ny; ++n) out[n] = cd(a[n], b[n]);
        }
    }
};

// Mean mode (meanmode.jl:38-150)
struct MeanSolver {
    int Ny = 0;
    double nu = 0, lambda = 0;
    Helm vh;
    std::vector<double> response;
    double response_mean = 0;
    bool init(int Ny_, double nu_, double lambda_) {
        Ny = Ny_; nu = nu_; lambda = lambda_;
        if (Ny < 4 || !(std::isfinite(nu) && nu > 0) || !(std::isfinite(lambda) && lambda >= 0)) return false;
        vh.init(Ny, nu, lambda, false);
        std::vector<double> work(Ny, 0.0);
        work[0] = 1.0;
        response.resize(Ny);
        vh.solve(work.data(), 0.0, 0.0, response.data());
        response_mean = bulkmean(response.data(), 1, Ny);
        return std::isfinite(response_mean) && response_mean != 0.0;
    }
    // mode: 0 pressure gradient (gx, gz), 1 bulk velocity (perturbation targets)
    void solve(cd* u, cd* v, cd* w, cd* p, const cd* Rx, const cd* Ry, const cd* Rz, long s,
               int mode, double c1, double c2, double* grads) const {
        const int P = Ny - 1;
        std::vector<cd> pc(Ny, 0.0);
        for (int n = 1; n <= P; ++n) {
            cd lower = n == 1 ? Ry[0] : Ry[(n - 1) * s] / 2.0;
            cd upper = n + 1 < P ? Ry[(n + 1) * s] / 2.0 : cd(0);
            pc[n] = (lower - upper) / (double)n;
        }
        pc[0] = 0;
        pc[0] = -bulkmean(pc.data(), 1, Ny);
        for (int n = 0; n < Ny; ++n) { p[n * s] = pc[n]; v[n * s] = 0.0; }
        std::vector<double> fr(Ny), fi(Ny), ar(Ny), ai(Ny);
        for (int i = 0; i < 2; ++i) {
            cd* out = i == 0 ? u : w;
            const cd* src = i == 0 ? Rx : Rz;
            for (int n = 0; n < Ny; ++n) { fr[n] = -src[n * s].real(); fi[n] = -src[n * s].imag(); }
            vh.solve(fr.data(), 0.0, 0.0, ar.data());
            vh.solve(fi.data(), 0.0, 0.0, ai.data());
            double g;
            if (mode == 1) {
                double target = i == 0 ? c1 : c2;
                g = (target - bulkmean(ar.data(), 1, Ny)) / response_mean;
            } else {
                g = i == 0 ? c1 : c2;
            }
            for (int n = 0; n < Ny; ++n) out[n * s] = cd(ar[n] + g * response[n], ai[n]);
            grads[i] = g;
        }
    }
};

// ---------------------------------------------------------------------------
// Grid, fields and transforms
// ---------------------------------------------------------------------------
struct OGrid {
    int Nx, Ny, Nz;
    double Lx, Lz;
    int Nxh, Nxp, Nzp, Nxhp;
    long nr() const { return (long)Nxh * Nz * Ny; }
    long nphys() const { return (long)Nxp * Nzp * Ny; }
    double kx(int ix) const { return 2 * M_PI / Lx * ix; }
    double lz(int iz) const { return 2 * M_PI / Lz * (iz <= (Nz >> 1) ? iz : iz - Nz); }
    bool nyquist(int ix, int iz) const {
        return ((Nx % 2 == 0) && ix == Nx / 2) || ((Nz % 2 == 0) && iz == Nz / 2);
    }
    int zpad(int iz) const { return iz <= (Nz >> 1) ? iz : Nzp - (Nz - iz); }
};

static OGrid make_grid(int Nx, int Ny, int Nz, double Lx, double Lz) {
    OGrid g;
    g.Nx = Nx; g.Ny = Ny; g.Nz = Nz; g.Lx = Lx; g.Lz = Lz;
    g.Nxh = Nx / 2 + 1;
    g.Nxp = (3 * Nx + 1) / 2;
    g.Nzp = (3 * Nz + 1) / 2;
    g.Nxhp = g.Nxp / 2 + 1;
    return g;
}

static int nthreads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Inverse transform (ffts.jl:151-166): spectral (Ny,Nz,Nxh) -> padded physical (Ny,Nzp,Nxp)
// Work array of the padded spectrum, shared by the transforms (the oracle is
// single-caller) and allocated once, so a timed stage pays no allocation.
static std::vector<cd>& pad_buffer(size_t n) {
    static std::vector<cd> buf;
    if (buf.size() < n) buf.resize(n);
    return buf;
}

static void inverse_transform(const OGrid& g, const cd* U, double* u) {
    const int Ny = g.Ny, P = Ny - 1, Nz = g.Nz, Nxh = g.Nxh, Nzp = g.Nzp, Nxp = g.Nxp, Nxhp = g.Nxhp;
    const size_t npad = (size_t)Ny * Nzp * Nxhp;
    std::vector<cd>& pad = pad_buffer(npad);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < sampled((long)npad); ++i) pad[i] = cd(0);
#pragma omp parallel
    {
        std::vector<cd> col(Ny), buf(2 * P + 2), work(2 * P + 2);
#pragma omp for schedule(static)
        for (long c = 0; c < sampled((long)Nz * Nxh); ++c) {
            int iz = c / Nxh, ix = c % Nxh;
            for (int n = 0; n < Ny; ++n) col[n] = U[((long)n * Nz + iz) * Nxh + ix];
            col[0] *= 2.0;
            col[P] *= 2.0;
            redft00(col.data(), 1, P, buf.data(), work.data());
            if (g.nyquist(ix, iz)) continue;  // zero_nyquist! on the padded spectrum
            int izp = g.zpad(iz);
            for (int n = 0; n < Ny; ++n) pad[((size_t)n * Nzp + izp) * Nxhp + ix] = 0.5 * col[n];
        }
    }
#pragma omp parallel
    {
        std::vector<cd> line(std::max(Nzp, Nxp)), work(std::max(Nzp, Nxp));
#pragma omp for schedule(static)
        for (long c = 0; c < sampled((long)Ny * Nxh); ++c) {  // z backward c2c
            int n = c / Nxh, ix = c % Nxh;
            for (int z = 0; z < Nzp; ++z) line[z] = pad[((size_t)n * Nzp + z) * Nxhp + ix];
            fft_inplace(line.data(), work.data(), Nzp, +1);
            for (int z = 0; z < Nzp; ++z) pad[((size_t)n * Nzp + z) * Nxhp + ix] = line[z];
        }
#pragma omp for schedule(static)
        for (long c = 0; c < sampled((long)Ny * Nzp); ++c) {  // x c2r
            const cd* X = &pad[(size_t)c * Nxhp];
            line[0] = X[0].real();
            for (int k = 1; k < Nxhp; ++k) {
                if (2 * k == Nxp) { line[k] = X[k].real(); continue; }
                line[k] = X[k];
                line[Nxp - k] = std::conj(X[k]);
            }
            fft_inplace(line.data(), work.data(), Nxp, +1);
            for (int j = 0; j < Nxp; ++j) u[(size_t)c * Nxp + j] = line[j].real();
        }
    }
}

// Forward transform (ffts.jl:65-82, normalize_forward! :254-269)
static void forward_transform(const OGrid& g, const double* u, cd* U) {
    const int Ny = g.Ny, P = Ny - 1, Nz = g.Nz, Nxh = g.Nxh, Nzp = g.Nzp, Nxp = g.Nxp, Nxhp = g.Nxhp;
    std::vector<cd>& pad = pad_buffer((size_t)Ny * Nzp * Nxhp);
#pragma omp parallel
    {
        std::vector<cd> line(std::max(Nzp, Nxp)), work(std::max(Nzp, Nxp));
#pragma omp for schedule(static)
        for (long c = 0; c < sampled((long)Ny * Nzp); ++c) {  // x r2c
            for (int j = 0; j < Nxp; ++j) line[j] = u[(size_t)c * Nxp + j];
            fft_inplace(line.data(), work.data(), Nxp, -1);
            for (int k = 0; k < Nxhp; ++k) pad[(size_t)c * Nxhp + k] = line[k];
        }
#pragma omp for schedule(static)
        for (long c = 0; c < sampled((long)Ny * Nxh); ++c) {  // z forward c2c
            int n = c / Nxh, ix = c % Nxh;
            for (int z = 0; z < Nzp; ++z) line[z] = pad[((size_t)n * Nzp + z) * Nxhp + ix];
            fft_inplace(line.data(), work.data(), Nzp, -1);
            for (int z = 0; z < Nzp; ++z) pad[((size_t)n * Nzp + z) * Nxhp + ix] = line[z];
        }
    }
    const double norm = 1.0 / ((double)Nxp * Nzp * (Ny - 1));
#pragma omp parallel
    {
        std::vector<cd> col(Ny), buf(2 * P + 2), work(2 * P + 2);
#pragma omp for schedule(static)
        for (long c = 0; c < sampled((long)Nz * Nxh); ++c) {
            int iz = c / Nxh, ix = c % Nxh;
            int izp = g.zpad(iz);
            for (int n = 0; n < Ny; ++n) col[n] = pad[((size_t)n * Nzp + izp) * Nxhp + ix];
            redft00(col.data(), 1, P, buf.data(), work.data());
            bool nyq = g.nyquist(ix, iz);
            for (int n = 0; n < Ny; ++n) {
                double e = (n == 0 || n == P) ? 0.5 : 1.0;
                U[((long)n * Nz + iz) * Nxh + ix] = nyq ? cd(0) : col[n] * (norm * e);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Operators (src/fields/operators.jl)
// ---------------------------------------------------------------------------
static void op_ddx1(const OGrid& g, const cd* U, cd* O, bool add) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < sampled(g.nr()); ++i) {
        const int ix = (int)(i % g.Nxh);
        cd v = cd(0, g.kx(ix)) * U[i];
        O[i] = add ? O[i] + v : v;
    }
}
static void op_ddx3(const OGrid& g, const cd* U, cd* O, bool add) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < sampled(g.nr()); ++i) {
        const int iz = (int)((i / g.Nxh) % g.Nz);
        cd v = cd(0, g.lz(iz)) * U[i];
        O[i] = add ? O[i] + v : v;
    }
}
static void op_ddx2(const OGrid& g, const cd* U, cd* O, bool add) {
    const long S = (long)g.Nz * g.Nxh;
#pragma omp parallel
    {
        std::vector<cd> tmp(g.Ny);
#pragma omp for
        for (long c = 0; c < sampled(S); ++c) {
            cheb_diff(U + c, S, tmp.data(), 1, g.Ny);
            for (int n = 0; n < g.Ny; ++n) O[c + n * S] = add ? O[c + n * S] + tmp[n] : tmp[n];
        }
    }
}
// laplacian! non-aliased path (operators.jl:104-124)
static void op_laplacian(const OGrid& g, const cd* a, cd* b) {
    const int Ny = g.Ny, Nz = g.Nz, Nxh = g.Nxh;
    const double al2 = std::pow(2 * M_PI / g.Lx, 2), be2 = std::pow(2 * M_PI / g.Lz, 2);
    auto A = [&](int j, int iz, int ix) { return a[((long)(j - 1) * Nz + iz) * Nxh + ix]; };
    auto Bv = [&](int j, int iz, int ix) -> cd& { return b[((long)(j - 1) * Nz + iz) * Nxh + ix]; };
    // columns are independent; the recurrence runs down each column
#pragma omp parallel for schedule(static)
    for (long c = 0; c < sampled((long)Nz * Nxh); ++c) {
        const int iz = (int)(c / Nxh), ix = (int)(c % Nxh);
        const int l = iz <= (Nz >> 1) ? iz : iz - Nz;
        const double k2 = al2 * (double)ix * ix + be2 * (double)l * l;
        for (int j = Ny; j >= 1; --j) {
            cd d2 = 0;
            if (j + 2 <= Ny)
                d2 = (4.0 * j * (j + 1)) * A(j + 2, iz, ix) +
                     (2.0 * (j + 1) / (j + 2)) * (Bv(j + 2, iz, ix) + k2 * A(j + 2, iz, ix));
            if (j + 4 <= Ny) d2 -= ((double)j / (j + 2)) * (Bv(j + 4, iz, ix) + k2 * A(j + 4, iz, ix));
            Bv(j, iz, ix) = (j == 1 ? d2 / 2.0 : d2) - k2 * A(j, iz, ix);
        }
    }
}
// curl! (operators.jl:172-190)
static void op_curl(const OGrid& g, const cd* const U[3], cd* const O[3]) {
    op_ddx2(g, U[2], O[0], false);
    op_ddx2(g, U[0], O[2], false);
    const cd I(0, 1);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < sampled(g.nr()); ++i) {
        const int ix = (int)(i % g.Nxh), iz = (int)((i / g.Nxh) % g.Nz);
        double k = g.kx(ix), l = g.lz(iz);
        O[0][i] -= I * l * U[1][i];
        O[1][i] = I * (l * U[0][i] - k * U[2][i]);
        O[2][i] = I * k * U[1][i] - O[2][i];
    }
}
static void zero_nyquist(const OGrid& g, cd* U) {
    for (int iz = 0; iz < g.Nz; ++iz)
        for (int ix = 0; ix < g.Nxh; ++ix)
            if (g.nyquist(ix, iz))
                for (int n = 0; n < g.Ny; ++n) U[((long)n * g.Nz + iz) * g.Nxh + ix] = 0;
}

// ---------------------------------------------------------------------------
// Problem: CNRK2 scheme with Stokes banks and the rotational nonlinear term
// ---------------------------------------------------------------------------
static const double CA[3] = {0.0, -5.0 / 9.0, -153.0 / 128.0};
static const double CB[3] = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};
static const double CC[3] = {1.0 / 6.0, 5.0 / 24.0, 1.0 / 8.0};

struct Stokes {
    std::vector<ModeSolver> modes;
    MeanSolver mean;
    bool init(const OGrid& g, double nu, double lambda) {
        const long B = (long)g.Nxh * g.Nz;
        modes.resize(B);
        if (!mean.init(g.Ny, nu, lambda)) return false;
        bool ok = true;
#pragma omp parallel for schedule(dynamic, 16) reduction(&& : ok)
        for (long c = 0; c < B; ++c) {
            int iz = c / g.Nxh, ix = c % g.Nxh;
            if (!modes[c].init(g.Ny, g.kx(ix), g.lz(iz), nu, lambda, true)) ok = false;
        }
        return ok;
    }
    // solve! (stokes.jl:81-108); mode 0 pressure gradient, 1 bulk (total targets)
    void solve(const OGrid& g, cd* const U[3], cd* Pf, const cd* const R[3], int mode, double c1, double c2,
               double basemean, double* grads) const {
        const long S = (long)g.Nxh * g.Nz;
#pragma omp parallel for schedule(dynamic, 16)
        for (long c = 0; c < sampled(S); ++c) {
            if (c == 0) continue;
            modes[c].solve(U[0] + c, U[1] + c, U[2] + c, Pf + c, R[0] + c, R[1] + c, R[2] + c, S);
        }
        double t1 = mode == 1 ? c1 - basemean : c1;
        mean.solve(U[0], U[1], U[2], Pf, R[0], R[1], R[2], S, mode, t1, c2, grads);
        for (int i = 0; i < 3; ++i) zero_nyquist(g, U[i]);
        zero_nyquist(g, Pf);
    }
};

struct Problem {
    OGrid g;
    double nu, dt;
    int cmode;  // 0 pressure gradient, 1 bulk velocity
    double c1, c2;
    std::vector<double> base, basecurv;
    double basemean;
    Stokes stokes[3];
    bool stokes_ready = false;
    std::vector<cd> Q[3], N[3], R[3];
    std::vector<cd> TMP[3], OM[3];
    std::vector<double> uphys[3], wphys[3], nphys[3];
    // nonlinear form (nonlinear.jl:10-17): 0 rotational, 1 convective, 2 divergence
    int form = 0;
    std::vector<cd> GR[9];          // convective: spectral gradient (i, j) at 3 i + j
    std::vector<double> gphys[9];   // convective: its padded physical values
    std::vector<cd> UU[6];          // divergence: spectral products 00 01 02 11 12 22
    std::vector<double> uuphys[6];  // divergence: physical products

    long nr() const { return g.nr(); }
    void alloc_nl() {
        for (int i = 0; i < 3; ++i) {
            TMP[i].assign(nr(), 0); OM[i].assign(nr(), 0);
            uphys[i].assign(g.nphys(), 0); wphys[i].assign(g.nphys(), 0); nphys[i].assign(g.nphys(), 0);
        }
    }
};

// total velocity: TMP = U with the base profile added to mode (0,0) of u
// (nonlinear.jl:123-124, 153-154, 179-180)
static void total_velocity(Problem& pb, const cd* const U[3]) {
    const OGrid& g = pb.g;
    const long nr = g.nr(), S = (long)g.Nxh * g.Nz;
    for (int i = 0; i < 3; ++i) {
        cd* dst = pb.TMP[i].data();
        const cd* src = U[i];
#pragma omp parallel for schedule(static)
        for (long x = 0; x < sampled(nr); ++x) dst[x] = src[x];
    }
    for (int n = 0; n < g.Ny; ++n) pb.TMP[0][n * S] += pb.base[n];
}

// _store_rhs! with sign -1 (nonlinear.jl:200-208)
static void negate(const OGrid& g, cd* const N[3]) {
    for (int i = 0; i < 3; ++i) {
        cd* x = N[i];
#pragma omp parallel for schedule(static)
        for (long j = 0; j < g.nr(); ++j) x[j] = -x[j];
    }
}

// NonLinearTerm{ConvectiveForm} (nonlinear.jl:113-140): grad! of the total
// velocity (operators.jl:206-214), 12 inverse transforms, dot! (operators.jl:
// 247-254), 3 forward transforms, sign -1.
static void nonlinear_convective(Problem& pb, const cd* const U[3], cd* const Nout[3]) {
    const OGrid& g = pb.g;
    total_velocity(pb, U);
    for (int i = 0; i < 3; ++i) {
        const cd* T = pb.TMP[i].data();
        op_ddx1(g, T, pb.GR[3 * i + 0].data(), false);
        op_ddx2(g, T, pb.GR[3 * i + 1].data(), false);
        op_ddx3(g, T, pb.GR[3 * i + 2].data(), false);
    }
    for (int i = 0; i < 3; ++i) inverse_transform(g, pb.TMP[i].data(), pb.uphys[i].data());
    for (int m = 0; m < 9; ++m) inverse_transform(g, pb.GR[m].data(), pb.gphys[m].data());
    const long np = g.nphys();
    const double *u1 = pb.uphys[0].data(), *u2 = pb.uphys[1].data(), *u3 = pb.uphys[2].data();
    for (int i = 0; i < 3; ++i) {
        const double *g1 = pb.gphys[3 * i].data(), *g2 = pb.gphys[3 * i + 1].data(), *g3 = pb.gphys[3 * i + 2].data();
        double* n = pb.nphys[i].data();
#pragma omp parallel for schedule(static)
        for (long x = 0; x < sampled(np); ++x) n[x] = u1[x] * g1[x] + u2[x] * g2[x] + u3[x] * g3[x];
    }
    for (int i = 0; i < 3; ++i) forward_transform(g, pb.nphys[i].data(), Nout[i]);
    negate(g, Nout);
}

// index of the product u_i u_j among the six distinct ones (00 01 02 11 12 22)
static int sym6(int i, int j) {
    if (i > j) std::swap(i, j);
    return i == 0 ? j : (i == 1 ? 2 + j : 5);
}

// NonLinearTerm{DivergenceForm} (nonlinear.jl:146-167): 3 inverse transforms,
// outer! (operators.jl:227-234; u_i u_j = u_j u_i exactly, so the six distinct
// products are transformed), forward transforms, div! of the rows
// (operators.jl:270-294), sign -1.
static void nonlinear_divergence(Problem& pb, const cd* const U[3], cd* const Nout[3]) {
    const OGrid& g = pb.g;
    total_velocity(pb, U);
    for (int i = 0; i < 3; ++i) inverse_transform(g, pb.TMP[i].data(), pb.uphys[i].data());
    const long np = g.nphys();
    for (int i = 0; i < 3; ++i)
        for (int j = i; j < 3; ++j) {
            const double *a = pb.uphys[i].data(), *b = pb.uphys[j].data();
            double* o = pb.uuphys[sym6(i, j)].data();
#pragma omp parallel for schedule(static)
            for (long x = 0; x < sampled(np); ++x) o[x] = a[x] * b[x];
        }
    for (int m = 0; m < 6; ++m) forward_transform(g, pb.uuphys[m].data(), pb.UU[m].data());
    for (int i = 0; i < 3; ++i) {
        op_ddx1(g, pb.UU[sym6(i, 0)].data(), Nout[i], false);
        op_ddx2(g, pb.UU[sym6(i, 1)].data(), Nout[i], true);
        op_ddx3(g, pb.UU[sym6(i, 2)].data(), Nout[i], true);
    }
    negate(g, Nout);
}

static void nonlinear_rotational(Problem& pb, const cd* const U[3], cd* const Nout[3]);
// NonLinearTerm call of the problem's form; overwrites Nout.
static void nonlinear(Problem& pb, const cd* const U[3], cd* const Nout[3]) {
    if (pb.form == 1) nonlinear_convective(pb, U, Nout);
    else if (pb.form == 2) nonlinear_divergence(pb, U, Nout);
    else nonlinear_rotational(pb, U, Nout);
}

// NonLinearTerm{RotatingForm} (nonlinear.jl:173-193); overwrites Nout.
static void nonlinear_rotational(Problem& pb, const cd* const U[3], cd* const Nout[3]) {
    const OGrid& g = pb.g;
    total_velocity(pb, U);
    const cd* T[3] = {pb.TMP[0].data(), pb.TMP[1].data(), pb.TMP[2].data()};
    cd* O[3] = {pb.OM[0].data(), pb.OM[1].data(), pb.OM[2].data()};
    op_curl(g, T, O);
    for (int i = 0; i < 3; ++i) {
        inverse_transform(g, T[i], pb.uphys[i].data());
        inverse_transform(g, O[i], pb.wphys[i].data());
    }
    const long np = g.nphys();
    const double *u1 = pb.uphys[0].data(), *u2 = pb.uphys[1].data(), *u3 = pb.uphys[2].data();
    const double *w1 = pb.wphys[0].data(), *w2 = pb.wphys[1].data(), *w3 = pb.wphys[2].data();
    double *n1 = pb.nphys[0].data(), *n2 = pb.nphys[1].data(), *n3 = pb.nphys[2].data();
#pragma omp parallel for schedule(static)
    for (long i = 0; i < sampled(np); ++i) {
        n1[i] = u2[i] * w3[i] - u3[i] * w2[i];
        n2[i] = u3[i] * w1[i] - u1[i] * w3[i];
        n3[i] = u1[i] * w2[i] - u2[i] * w1[i];
    }
    for (int i = 0; i < 3; ++i) forward_transform(g, pb.nphys[i].data(), Nout[i]);
}

static bool problem_stokes(Problem& pb) {
    if (pb.stokes_ready) return true;
    for (int j = 0; j < 3; ++j)
        if (!pb.stokes[j].init(pb.g, pb.nu, 1.0 / (CC[j] * pb.dt))) return false;
    pb.stokes_ready = true;
    return true;
}

// One CNRK2 stage j (cnrk2.jl:170-205) of a step of duration dt with the
// Stokes solvers st (the problem's own for its nominal dt); gradients carries
// the previous stage's uniform gradients in and this stage's out.
static void cnrk2_stage(Problem& pb, cd* const U[3], cd* Pf, int j, double* gradients, double dt, const Stokes* st) {
    const OGrid& g = pb.g;
    const long nr = g.nr(), S = (long)g.Nxh * g.Nz;
    cd* Nf[3] = {pb.N[0].data(), pb.N[1].data(), pb.N[2].data()};
    cd* Rf[3] = {pb.R[0].data(), pb.R[1].data(), pb.R[2].data()};
    const cd* Uc[3] = {U[0], U[1], U[2]};
    nonlinear(pb, Uc, Nf);
    double old[2] = {gradients[0], gradients[1]};
    if (pb.cmode == 1) {
        for (int i = 0; i < 2; ++i) {
            int comp = i == 0 ? 0 : 2;
            cd sh = wall_deriv(U[comp], S, g.Ny, true) - wall_deriv(U[comp], S, g.Ny, false);
            double base = i == 0 ? pb.nu * bulkmean(pb.basecurv.data(), 1, g.Ny) : 0.0;
            old[i] = pb.nu * sh.real() / 2 + base + bulkmean(Nf[comp], S, g.Ny).real();
        }
    }
    for (int i = 0; i < 3; ++i) {
        cd* Qi = pb.Q[i].data();
        const cd* Ni = Nf[i];
        const double a = CA[j];
#pragma omp parallel for schedule(static)
        for (long x = 0; x < sampled(nr); ++x) Qi[x] = (j == 0) ? Ni[x] : a * Qi[x] + Ni[x];
    }
    const double lambda = 1.0 / (CC[j] * dt), weight = CB[j] / CC[j];
    for (int i = 0; i < 3; ++i) {
        op_laplacian(g, U[i], Rf[i]);
        if (i == 0) op_ddx1(g, Pf, Nf[i], false);
        else if (i == 1) op_ddx2(g, Pf, Nf[i], false);
        else op_ddx3(g, Pf, Nf[i], false);
        const cd* Qi = pb.Q[i].data();
        cd* Ri = Rf[i];
        const cd *Ui = U[i], *Ni = Nf[i];
        const double nu = pb.nu;
#pragma omp parallel for schedule(static)
        for (long x = 0; x < sampled(nr); ++x) Ri[x] = lambda * Ui[x] + nu * Ri[x] - Ni[x] + weight * Qi[x];
    }
    for (int n = 0; n < g.Ny; ++n) Rf[0][n * S] += 2 * pb.nu * pb.basecurv[n];
    Rf[0][0] -= old[0];
    Rf[2][0] -= old[1];
    const cd* Rc[3] = {Rf[0], Rf[1], Rf[2]};
    st[j].solve(g, U, Pf, Rc, pb.cmode, pb.c1, pb.c2, pb.basemean, gradients);
}

// step! (cnrk2.jl:149-207).  Returns the last stage's gradients in grads.
static void cnrk2_step(Problem& pb, cd* const U[3], cd* Pf, double* grads, double dt, const Stokes* st) {
    double gradients[2] = {pb.cmode == 0 ? pb.c1 : 0.0, pb.cmode == 0 ? pb.c2 : 0.0};
    for (int j = 0; j < 3; ++j) cnrk2_stage(pb, U, Pf, j, gradients, dt, st);
    grads[0] = gradients[0];
    grads[1] = gradients[1];
}

// project! (pressure.jl:36-54)
static bool project(Problem& pb, cd* const U[3]) {
    const OGrid& g = pb.g;
    Stokes st;
    if (!st.init(g, 1.0, 0.0)) return false;
    std::vector<cd> R[3], phi(g.nr());
    cd* Rp[3];
    for (int i = 0; i < 3; ++i) {
        R[i].assign(g.nr(), 0);
        op_laplacian(g, U[i], R[i].data());
        for (auto& x : R[i]) x = -x;
        Rp[i] = R[i].data();
    }
    const cd* Rc[3] = {Rp[0], Rp[1], Rp[2]};
    double grads[2];
    if (pb.cmode == 1) st.solve(g, U, phi.data(), Rc, 1, pb.c1, pb.c2, pb.basemean, grads);
    else st.solve(g, U, phi.data(), Rc, 0, 0.0, 0.0, pb.basemean, grads);
    return true;
}

// pressure (pressure.jl:95-204)
static bool pressure(Problem& pb, const cd* const U[3], cd* Pout) {
    const OGrid& g = pb.g;
    const long nr = g.nr(), S = (long)g.Nxh * g.Nz;
    const int Ny = g.Ny;
    std::vector<cd> A[3];
    cd* Ap[3];
    for (int i = 0; i < 3; ++i) { A[i].assign(nr, 0); Ap[i] = A[i].data(); }
    nonlinear(pb, U, Ap);
    // P = div(A)
    op_ddx1(g, Ap[0], Pout, false);
    op_ddx2(g, Ap[1], Pout, true);
    op_ddx3(g, Ap[2], Pout, true);
    const cd* V = U[1];
    bool ok = true;
#pragma omp parallel
    {
        Helm h;
        std::vector<cd> rhs(Ny), sol(Ny);
#pragma omp for schedule(dynamic, 16)
        for (long c = 0; c < S; ++c) {
            int iz = c / g.Nxh, ix = c % g.Nxh;
            if (c == 0 || g.nyquist(ix, iz)) continue;
            double k = g.kx(ix), l = g.lz(iz);
            h.init(Ny, 1.0, k * k + l * l, true);
            cd upper = 0, lower = 0;
            for (int n = 0; n < Ny; ++n) {
                cd a = Ap[1][c + n * S];
                upper += a;
                lower += (n % 2 == 0 ? 1.0 : -1.0) * a;
            }
            for (int n = 2; n <= Ny - 1; ++n) {
                cd wall = pb.nu * ((double)n * n * ((double)n * n - 1) / 3.0) * V[c + n * S];
                upper += wall;
                lower += (n % 2 == 0) ? wall : -wall;
            }
            for (int n = 0; n < Ny; ++n) rhs[n] = Pout[c + n * S];
            h.solve_c(rhs.data(), upper, lower, sol.data());
            for (int n = 0; n < Ny; ++n) Pout[c + n * S] = sol[n];
        }
    }
    // zero mode
    std::vector<cd> mean(Ny, 0.0);
    const cd* normal = Ap[1];
    for (int n = 1; n <= Ny - 1; ++n) {
        cd lo = n == 1 ? normal[0] : normal[(n - 1) * S] / 2.0;
        cd up = n + 1 < Ny - 1 ? normal[(n + 1) * S] / 2.0 : cd(0);
        mean[n] = (lo - up) / (double)n;
    }
    mean[0] = 0;
    mean[0] = -bulkmean(mean.data(), 1, Ny);
    for (int n = 0; n < Ny; ++n) Pout[n * S] = mean[n];
    zero_nyquist(g, Pout);
    return ok;
}

// Spectral inner product (postprocessing.jl:31-62)
static double spectral_dot(const OGrid& g, const cd* U, const cd* V) {
    const int Ny = g.Ny;
    const long S = (long)g.Nxh * g.Nz;
    auto moment = [](int n) { return (n % 2 == 0) ? 1.0 / (1.0 - (double)n * n) : 0.0; };
    std::vector<double> M((size_t)Ny * Ny);
    for (int m = 0; m < Ny; ++m)
        for (int n = 0; n < Ny; ++n) M[(size_t)m * Ny + n] = (moment(m + n) + moment(std::abs(m - n))) / 2;
    double result = 0;
    std::vector<cd> w(Ny);
    for (long c = 0; c < S; ++c) {
        int iz = c / g.Nxh, ix = c % g.Nxh;
        if (g.nyquist(ix, iz)) continue;
        for (int m = 0; m < Ny; ++m) {
            cd s = 0;
            for (int n = 0; n < Ny; ++n) s += M[(size_t)m * Ny + n] * V[c + n * S];
            w[m] = s;
        }
        cd d = 0;
        for (int m = 0; m < Ny; ++m) d += std::conj(U[c + m * S]) * w[m];
        result += (ix == 0 ? 1.0 : 2.0) * d.real();
    }
    return result;
}

// Deterministic synthetic initial coefficients (spectral Gaussian with a
// prescribed spectrum).  splitmix64 hash of (seed, component, ix, iz, n) ->
// two uniforms -> Box-Muller.  The same formula is used by the engine.
static inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}
static inline double u01(uint64_t h) { return ((h >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
static cd gauss_c(uint64_t seed, int comp, int ix, int iz, int n) {
    uint64_t key = splitmix64(seed ^ splitmix64(((uint64_t)comp << 56) ^ ((uint64_t)ix << 36) ^ ((uint64_t)iz << 16) ^ (uint64_t)n));
    double a = u01(splitmix64(key)), b = u01(splitmix64(key ^ 0xD1B54A32D192ED03ULL));
    double r = std::sqrt(-2.0 * std::log(a));
    return cd(r * std::cos(2 * M_PI * b), r * std::sin(2 * M_PI * b));
}
// shape: 0 exp(-(|k|+|l|)/4) exp(-n/4); 1 (1+k^2+l^2)^-1 rho^n with rho = param
static void synth_coeffs(const OGrid& g, uint64_t seed, double amp, int shape, double rho, cd* const U[3]) {
    const long S = (long)g.Nxh * g.Nz;
    for (int c = 0; c < 3; ++c)
        for (int n = 0; n < g.Ny; ++n)
            for (int iz = 0; iz < g.Nz; ++iz) {
                int l = iz <= (g.Nz >> 1) ? iz : iz - g.Nz;
                for (int ix = 0; ix < g.Nxh; ++ix) {
                    double s, r;
                    if (shape == 0) { s = std::exp(-(std::abs(ix) + std::abs(l)) / 4.0); r = std::exp(-n / 4.0); }
                    else { s = 1.0 / (1.0 + (double)ix * ix + (double)l * l); r = std::pow(rho, n); }
                    cd v = g.nyquist(ix, iz) ? cd(0) : amp * s * r * gauss_c(seed, c, ix, iz, n);
                    U[c][n * S + (long)iz * g.Nxh + ix] = v;
                }
            }
    // conjugate symmetry on the k = 0 plane; (0,0) real
    for (int c = 0; c < 3; ++c)
        for (int n = 0; n < g.Ny; ++n) {
            cd* col = U[c] + n * S;
            col[0] = col[0].real();
            for (int iz = (g.Nz >> 1) + 1; iz < g.Nz; ++iz) {
                int mirror = g.Nz - iz;
                col[(long)iz * g.Nxh] = std::conj(col[(long)mirror * g.Nxh]);
            }
        }
}

// ===========================================================================
// C API
// ===========================================================================
extern "C" {

const char* or_last_error() { return g_error.c_str(); }
void or_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#endif
}
int or_get_threads() { return nthreads(); }
void or_set_sample_div(long d) { g_sample_div = d > 1 ? d : 1; }
void or_set_helmholtz_method(int method, int dense_max_ny) {
    g_helm_method = method;
    if (dense_max_ny > 0) g_dense_max_ny = dense_max_ny;
}

// complex FFT of length n, sign -1/+1
void or_fft(double* x, int n, int sign) {
    std::vector<cd> work(n);
    fft_inplace(reinterpret_cast<cd*>(x), work.data(), n, sign);
}
// DCT-I (REDFT00) of complex column length P+1
void or_redft00(double* x, int Ny) {
    int P = Ny - 1;
    std::vector<cd> buf(2 * P), work(2 * P);
    redft00(reinterpret_cast<cd*>(x), 1, P, buf.data(), work.data());
}
void or_chebcoeffs(const double* vals, double* coef, int Ny) { cheb_coeffs(vals, coef, Ny); }
void or_diff(const double* a, double* b, int Ny) { cheb_diff(a, 1, b, 1, Ny); }

// Scalar Helmholtz solve
int or_helmholtz(int Ny, double th0, double th1, int neumann, const double* f, double bp, double bm, double* out) {
    Helm h;
    h.init(Ny, th0, th1, neumann != 0);
    h.solve(f, bp, bm, out);
    return 0;
}

// Scalar InfluenceModeSolver (influence.jl): batched=0 uses the scalar
// real/imaginary split, batched=1 the batched-bank arithmetic.
int or_influence_solve(int Ny, double k, double l, double nu, double lambda, int batched, const double* Rx,
                       const double* Ry, const double* Rz, double* u, double* v, double* w, double* p) {
    if (!(Ny >= 5 && Ny % 2 == 1)) { set_error("tau correction requires odd Ny >= 5"); return -1; }
    if (k * k + l * l <= 0 && !batched) { set_error("InfluenceModeSolver requires kappa2 > 0"); return -1; }
    ModeSolver m;
    if (!m.init(Ny, k, l, nu, lambda, batched != 0)) { set_error("singular influence matrix"); return -2; }
    auto C = [](const double* x) { return reinterpret_cast<const cd*>(x); };
    auto Cm = [](double* x) { return reinterpret_cast<cd*>(x); };
    if (batched) m.solve(Cm(u), Cm(v), Cm(w), Cm(p), C(Rx), C(Ry), C(Rz), 1);
    else m.solve_scalar(Cm(u), Cm(v), Cm(w), Cm(p), C(Rx), C(Ry), C(Rz));
    return 0;
}
// responses: out[6*Ny] = pp, pm, vp, vm, p0, v0 ; extra[6] = inf(4), sigma(2)
int or_influence_responses(int Ny, double k, double l, double nu, double lambda, double* out, double* extra) {
    ModeSolver m;
    if (!m.init(Ny, k, l, nu, lambda, true)) { set_error("singular influence matrix"); return -2; }
    const std::vector<double>* v[6] = {&m.pp, &m.pm, &m.vp, &m.vm, &m.p0, &m.v0};
    for (int i = 0; i < 6; ++i) std::memcpy(out + i * Ny, v[i]->data(), sizeof(double) * Ny);
    for (int i = 0; i < 4; ++i) extra[i] = m.inf[i];
    extra[4] = m.sigma[0]; extra[5] = m.sigma[1];
    return 0;
}

// MeanModeSolver solve; mode 0 gradient (c1,c2), 1 bulk (c1,c2) perturbation targets
int or_mean_solve(int Ny, double nu, double lambda, int mode, double c1, double c2, const double* Rx,
                  const double* Ry, const double* Rz, double* u, double* v, double* w, double* p, double* grads) {
    MeanSolver m;
    if (!m.init(Ny, nu, lambda)) { set_error("invalid mean-mode parameters"); return -1; }
    m.solve(reinterpret_cast<cd*>(u), reinterpret_cast<cd*>(v), reinterpret_cast<cd*>(w), reinterpret_cast<cd*>(p),
            reinterpret_cast<const cd*>(Rx), reinterpret_cast<const cd*>(Ry), reinterpret_cast<const cd*>(Rz), 1, mode,
            c1, c2, grads);
    return 0;
}

void* or_create(int Nx, int Ny, int Nz, double Lx, double Lz, double nu, double dt, const double* base_values,
                int cmode, double c1, double c2) {
    if (!(Ny >= 5 && Ny % 2 == 1)) { set_error("Gibson's tau correction requires odd Ny >= 5"); return nullptr; }
    if (!(Nx > 0 && Nz > 0)) { set_error("Nx and Nz must be positive"); return nullptr; }
    if (!(std::isfinite(dt) && dt > 0)) { set_error("dt must be finite and positive"); return nullptr; }
    auto* pb = new Problem();
    pb->g = make_grid(Nx, Ny, Nz, Lx, Lz);
    pb->nu = nu; pb->dt = dt; pb->cmode = cmode; pb->c1 = c1; pb->c2 = c2;
    pb->base.resize(Ny); pb->basecurv.resize(Ny);
    cheb_coeffs(base_values, pb->base.data(), Ny);
    std::vector<double> d1(Ny);
    cheb_diff(pb->base.data(), 1, d1.data(), 1, Ny);
    cheb_diff(d1.data(), 1, pb->basecurv.data(), 1, Ny);
    pb->basemean = bulkmean(pb->base.data(), 1, Ny);
    for (int i = 0; i < 3; ++i) {
        pb->Q[i].assign(pb->g.nr(), 0); pb->N[i].assign(pb->g.nr(), 0); pb->R[i].assign(pb->g.nr(), 0);
    }
    pb->alloc_nl();
    return pb;
}
// nonlinear form of the problem (NonLinearTerm(...; form), nonlinear.jl:55-70):
// 0 RotatingForm, 1 ConvectiveForm, 2 DivergenceForm
int or_set_form(void* h, int form) {
    auto* pb = static_cast<Problem*>(h);
    if (form < 0 || form > 2) { set_error("unknown nonlinear form"); return -1; }
    pb->form = form;
    const long nr = pb->g.nr(), np = pb->g.nphys();
    if (form == 1 && pb->GR[0].empty())
        for (int m = 0; m < 9; ++m) { pb->GR[m].assign(nr, 0); pb->gphys[m].assign(np, 0); }
    if (form == 2 && pb->UU[0].empty())
        for (int m = 0; m < 6; ++m) { pb->UU[m].assign(nr, 0); pb->uuphys[m].assign(np, 0); }
    return 0;
}
void or_destroy(void* h) { delete static_cast<Problem*>(h); }
void or_get_base(void* h, double* base, double* curv) {
    auto* pb = static_cast<Problem*>(h);
    std::memcpy(base, pb->base.data(), sizeof(double) * pb->g.Ny);
    std::memcpy(curv, pb->basecurv.data(), sizeof(double) * pb->g.Ny);
}
int or_prepare(void* h) {
    auto* pb = static_cast<Problem*>(h);
    if (!problem_stokes(*pb)) { set_error("singular influence matrix"); return -2; }
    return 0;
}
// U: 3 consecutive complex fields; P one field.  nsteps steps from t.
int or_step(void* h, double* U, double* P, int nsteps, double* grads) {
    auto* pb = static_cast<Problem*>(h);
    if (!problem_stokes(*pb)) { set_error("singular influence matrix"); return -2; }
    const long nr = pb->g.nr();
    cd* Uc = reinterpret_cast<cd*>(U);
    cd* Uf[3] = {Uc, Uc + nr, Uc + 2 * nr};
    for (int s = 0; s < nsteps; ++s) cnrk2_step(*pb, Uf, reinterpret_cast<cd*>(P), grads, pb->dt, pb->stokes);
    return 0;
}
// One step of duration dt with Stokes solvers built for it (the Flows
// adapter's temporary CNRK2 for a shortened final step,
// ext/ChannelFlowFlowsExt.jl:45-50); the problem's own solvers are untouched.
int or_step_dt(void* h, double* U, double* P, double dt, double* grads) {
    auto* pb = static_cast<Problem*>(h);
    if (!(std::isfinite(dt) && dt > 0)) { set_error("dt must be finite and positive"); return -1; }
    Stokes st[3];
    for (int j = 0; j < 3; ++j)
        if (!st[j].init(pb->g, pb->nu, 1.0 / (CC[j] * dt))) { set_error("singular influence matrix"); return -2; }
    const long nr = pb->g.nr();
    cd* Uc = reinterpret_cast<cd*>(U);
    cd* Uf[3] = {Uc, Uc + nr, Uc + 2 * nr};
    cnrk2_step(*pb, Uf, reinterpret_cast<cd*>(P), grads, dt, st);
    return 0;
}
// one stage j of a step (a bounded sample of the step's work)
int or_stage(void* h, double* U, double* P, int j) {
    auto* pb = static_cast<Problem*>(h);
    if (!problem_stokes(*pb)) { set_error("singular influence matrix"); return -2; }
    const long nr = pb->g.nr();
    cd* Uc = reinterpret_cast<cd*>(U);
    cd* Uf[3] = {Uc, Uc + nr, Uc + 2 * nr};
    double gr[2] = {pb->cmode == 0 ? pb->c1 : 0.0, pb->cmode == 0 ? pb->c2 : 0.0};
    cnrk2_stage(*pb, Uf, reinterpret_cast<cd*>(P), j, gr, pb->dt, pb->stokes);
    return 0;
}
void or_nonlinear(void* h, const double* U, double* N) {
    auto* pb = static_cast<Problem*>(h);
    const long nr = pb->g.nr();
    const cd* Uc = reinterpret_cast<const cd*>(U);
    cd* Nc = reinterpret_cast<cd*>(N);
    const cd* Uf[3] = {Uc, Uc + nr, Uc + 2 * nr};
    cd* Nf[3] = {Nc, Nc + nr, Nc + 2 * nr};
    nonlinear(*pb, Uf, Nf);
}
void or_inverse(void* h, const double* U, double* u) {
    auto* pb = static_cast<Problem*>(h);
    inverse_transform(pb->g, reinterpret_cast<const cd*>(U), u);
}
void or_forward(void* h, const double* u, double* U) {
    auto* pb = static_cast<Problem*>(h);
    forward_transform(pb->g, u, reinterpret_cast<cd*>(U));
}
// op: 1 ddx1, 2 ddx2, 3 ddx3, 4 laplacian
void or_operator(void* h, int op, const double* U, double* O, int add) {
    auto* pb = static_cast<Problem*>(h);
    const cd* a = reinterpret_cast<const cd*>(U);
    cd* b = reinterpret_cast<cd*>(O);
    if (op == 1) op_ddx1(pb->g, a, b, add);
    else if (op == 2) op_ddx2(pb->g, a, b, add);
    else if (op == 3) op_ddx3(pb->g, a, b, add);
    else op_laplacian(pb->g, a, b);
}
void or_curl(void* h, const double* U, double* O) {
    auto* pb = static_cast<Problem*>(h);
    const long nr = pb->g.nr();
    const cd* Uc = reinterpret_cast<const cd*>(U);
    cd* Oc = reinterpret_cast<cd*>(O);
    const cd* Uf[3] = {Uc, Uc + nr, Uc + 2 * nr};
    cd* Of[3] = {Oc, Oc + nr, Oc + 2 * nr};
    op_curl(pb->g, Uf, Of);
}
// Stokes solve with the stage-j bank (j = 0,1,2) or a fresh (nu, lambda) bank (j < 0)
int or_stokes(void* h, int j, double nu, double lambda, double* U, double* P, const double* R, int mode,
              double c1, double c2, double* grads) {
    auto* pb = static_cast<Problem*>(h);
    const long nr = pb->g.nr();
    cd* Uc = reinterpret_cast<cd*>(U);
    const cd* Rc = reinterpret_cast<const cd*>(R);
    cd* Uf[3] = {Uc, Uc + nr, Uc + 2 * nr};
    const cd* Rf[3] = {Rc, Rc + nr, Rc + 2 * nr};
    if (j >= 0) {
        if (!problem_stokes(*pb)) { set_error("singular influence matrix"); return -2; }
        pb->stokes[j].solve(pb->g, Uf, reinterpret_cast<cd*>(P), Rf, mode, c1, c2, pb->basemean, grads);
    } else {
        Stokes st;
        if (!st.init(pb->g, nu, lambda)) { set_error("singular influence matrix"); return -2; }
        st.solve(pb->g, Uf, reinterpret_cast<cd*>(P), Rf, mode, c1, c2, pb->basemean, grads);
    }
    return 0;
}
int or_project(void* h, double* U) {
    auto* pb = static_cast<Problem*>(h);
    const long nr = pb->g.nr();
    cd* Uc = reinterpret_cast<cd*>(U);
    cd* Uf[3] = {Uc, Uc + nr, Uc + 2 * nr};
    if (!project(*pb, Uf)) { set_error("singular influence matrix"); return -2; }
    return 0;
}
int or_pressure(void* h, const double* U, double* P) {
    auto* pb = static_cast<Problem*>(h);
    const long nr = pb->g.nr();
    const cd* Uc = reinterpret_cast<const cd*>(U);
    const cd* Uf[3] = {Uc, Uc + nr, Uc + 2 * nr};
    pressure(*pb, Uf, reinterpret_cast<cd*>(P));
    return 0;
}
double or_dot(void* h, const double* U, const double* V) {
    auto* pb = static_cast<Problem*>(h);
    return spectral_dot(pb->g, reinterpret_cast<const cd*>(U), reinterpret_cast<const cd*>(V));
}
// diagnostics of the perturbation velocity U (3 fields):
// out = [kinetic energy, dissipation nu<|curl U|^2>, max |div U| coefficient,
//        nu*u'(+1) (0,0), nu*u'(-1) (0,0)]
void or_diagnostics(void* h, const double* U, double* out) {
    auto* pb = static_cast<Problem*>(h);
    const OGrid& g = pb->g;
    const long nr = g.nr(), S = (long)g.Nxh * g.Nz;
    const cd* Uc = reinterpret_cast<const cd*>(U);
    const cd* Uf[3] = {Uc, Uc + nr, Uc + 2 * nr};
    double e = 0;
    for (int i = 0; i < 3; ++i) e += spectral_dot(g, Uf[i], Uf[i]);
    std::vector<cd> O[3];
    cd* Op[3];
    for (int i = 0; i < 3; ++i) { O[i].assign(nr, 0); Op[i] = O[i].data(); }
    op_curl(g, Uf, Op);
    double d = 0;
    for (int i = 0; i < 3; ++i) d += spectral_dot(g, Op[i], Op[i]);
    std::vector<cd> dv(nr);
    op_ddx1(g, Uf[0], dv.data(), false);
    op_ddx2(g, Uf[1], dv.data(), true);
    op_ddx3(g, Uf[2], dv.data(), true);
    double mx = 0;
    for (auto& x : dv) mx = std::max(mx, std::abs(x));
    out[0] = e / 2;
    out[1] = pb->nu * d;
    out[2] = mx;
    out[3] = pb->nu * wall_deriv(Uf[0], S, g.Ny, true).real();
    out[4] = pb->nu * wall_deriv(Uf[0], S, g.Ny, false).real();
}
void or_synth(void* h, unsigned long long seed, double amp, int shape, double rho, double* U) {
    auto* pb = static_cast<Problem*>(h);
    const long nr = pb->g.nr();
    cd* Uc = reinterpret_cast<cd*>(U);
    cd* Uf[3] = {Uc, Uc + nr, Uc + 2 * nr};
    synth_coeffs(pb->g, seed, amp, shape, rho, Uf);
}

}  // extern "C"
