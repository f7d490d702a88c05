// Oracle -- test infrastructure only.  A CPU FP64 restatement of the
// reference's SGT frequency loop, used by tests/, __graft_entry__.smoke()
// and bench.py (CPU baseline leg) as the checker of the CUDA library.  It
// is never linked into the product.
//
// Parity status: UNPINNED.  The reference (Fortran + MPI) cannot be built
// in this environment (no Fortran compiler) and ships no test vectors, so
// this restatement is checked against closed-form properties and its own
// committed fixtures, not against reference outputs.
//
// Arithmetic follows gfortran's rules: complex products (ac-bd, ad+bc),
// complex division by Smith's method (GCC's default for Fortran), no
// fused multiply-add (built with -ffp-contract=off), libm sin/cos/log.
#pragma once

#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstddef>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace oracle {

constexpr double kPi = 3.1415926535897932;

struct cplx {
    double re = 0.0, im = 0.0;
    cplx() = default;
    constexpr cplx(double r) : re(r), im(0.0) {}
    constexpr cplx(double r, double i) : re(r), im(i) {}
};

inline cplx operator+(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
inline cplx operator-(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
inline cplx operator-(cplx a) { return {-a.re, -a.im}; }
inline cplx operator*(cplx a, cplx b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
// real * complex: the Fortran front end promotes the real operand; GCC
// lowers the product with a zero imaginary part to two scalings.
inline cplx operator*(double a, cplx b) { return {a * b.re, a * b.im}; }
inline cplx operator*(cplx a, double b) { return {a.re * b, a.im * b}; }
inline cplx operator/(cplx a, double b) { return {a.re / b, a.im / b}; }
// Smith's division (GCC expand_complex_div_wide)
inline cplx operator/(cplx a, cplx b) {
    double c = b.re, d = b.im;
    if (std::fabs(c) < std::fabs(d)) {
        double ratio = c / d;
        double div = (c * ratio) + d;
        double tr = (a.re * ratio) + a.im;
        double ti = (a.im * ratio) - a.re;
        return {tr / div, ti / div};
    }
    double ratio = d / c;
    double div = (d * ratio) + c;
    double tr = (a.im * ratio) + a.re;
    double ti = a.im - (a.re * ratio);
    return {tr / div, ti / div};
}
inline cplx conj(cplx a) { return {a.re, -a.im}; }
inline double cabs(cplx a) { return std::hypot(a.re, a.im); }
inline cplx& operator+=(cplx& a, cplx b) { a = a + b; return a; }

// glu / glusub: Gaussian elimination with partial pivoting,
// src/SGTsh/glu2.f90:140-281 (identical in src/SGTpsv/glu2.f90).
// a is column-major (n1, n), 0-based storage a[i + n1*j].
// Returns ier (0 ok).  eps < 0 is replaced by 3.52e-15 as in the reference.
inline int glu(cplx* a, int n, int n1, cplx* b, double eps, int* ip) {
    if (eps < 0.0) eps = 3.52e-15;
    auto A = [&](int i, int j) -> cplx& { return a[(i - 1) + n1 * (j - 1)]; };
    if (n1 < n || n <= 0) return 3;
    std::vector<cplx> wk(n + 1);
    for (int i = 1; i <= n; ++i) wk[i] = cplx(cabs(A(i, 1)), 0.0);
    for (int j = 2; j <= n; ++j)
        for (int i = 1; i <= n; ++i)
            wk[i] = cplx(std::fmax(cabs(wk[i]), cabs(A(i, j))), 0.0);
    for (int i = 1; i <= n; ++i)
        if (cabs(wk[i]) < eps) return 2;
    for (int k = 1; k <= n; ++k) {
        double amax = cabs(A(k, k));
        int ipk = k;
        for (int i = k + 1; i <= n; ++i) {
            double aik = cabs(A(i, k));
            if (aik > amax) { ipk = i; amax = aik; }
        }
        ip[k - 1] = ipk;
        if (amax > eps) {
            if (ipk != k) { cplx w = A(ipk, k); A(ipk, k) = A(k, k); A(k, k) = w; }
            for (int i = k + 1; i <= n; ++i) {
                A(i, k) = -A(i, k) / A(k, k);
                wk[i] = A(i, k);
            }
            for (int j = k + 1; j <= n; ++j) {
                if (ipk != k) { cplx w = A(ipk, j); A(ipk, j) = A(k, j); A(k, j) = w; }
                cplx t = A(k, j);
                for (int i = k + 1; i <= n; ++i) A(i, j) = A(i, j) + wk[i] * t;
            }
        } else {
            ip[k - 1] = k;
            for (int i = k + 1; i <= n; ++i) A(i, k) = cplx(0.0);
            return 1;
        }
    }
    // glusub
    for (int k = 1; k <= n; ++k) {
        if (ip[k - 1] != k) { cplx w = b[ip[k - 1] - 1]; b[ip[k - 1] - 1] = b[k - 1]; b[k - 1] = w; }
        cplx t = b[k - 1];
        for (int i = k + 1; i <= n; ++i) b[i - 1] = b[i - 1] + A(i, k) * t;
    }
    b[n - 1] = b[n - 1] / A(n, n);
    for (int k = n - 1; k >= 1; --k) {
        cplx t = b[k];
        for (int i = 1; i <= k; ++i) b[i - 1] = b[i - 1] - A(i, k + 1) * t;
        b[k - 1] = b[k - 1] / A(k, k);
    }
    return 0;
}

// interpolate, src/SGTsh/others.f90:843-891 / src/SGTpsv/others.f90:1170-1212.
// g holds 3*ncomp values (node-major, component fastest); u gets ncomp.
inline void interpolate(int ncomp, int nderiv, double rsta, const double* rrsta, const cplx* g,
                        cplx* u) {
    for (int c = 0; c < ncomp; ++c) u[c] = cplx(0.0);
    double dh[3];
    for (int i = 0; i < 3; ++i) dh[i] = rrsta[i] - rsta;
    if (dh[1] == 0.0 && nderiv == 0) {
        for (int c = 0; c < ncomp; ++c) u[c] = g[ncomp + c];
        return;
    }
    cplx a[9];
    for (int i = 0; i < 3; ++i) {
        a[0 + 3 * i] = cplx(1.0);
        a[1 + 3 * i] = cplx(dh[i]);
        a[2 + 3 * i] = cplx(dh[i] * dh[i] / 2.0);
    }
    cplx b[3] = {cplx(0.0), cplx(0.0), cplx(0.0)};
    b[nderiv] = cplx(1.0);
    int ip[3];
    glu(a, 3, 3, b, -1.0, ip);
    for (int c = 0; c < ncomp; ++c)
        for (int i = 0; i < 3; ++i) u[c] = u[c] + b[i] * g[ncomp * i + c];
}

// calplm, src/SGTsh/trial.f90:85-118 (same in src/SGTpsv/trial.f90:294-323)
inline void calplm(int l, int m, double x, double* plm) {
    if (l == m) {
        double pmm = 1.0;
        if (m > 0) {
            double somx2 = std::sqrt((1.0 - x) * (1.0 + x));
            double fact = 1.0;
            for (int i = 1; i <= m; ++i) {
                pmm = -pmm * fact * somx2;
                fact = fact + 2.0;
            }
        }
        plm[2] = 0.0;
        plm[1] = 0.0;
        plm[0] = pmm;
    } else {
        plm[2] = plm[1];
        plm[1] = plm[0];
        if (l == m + 1) plm[0] = x * (double)(2 * m + 1) * plm[1];
        else plm[0] = (x * (double)(2 * l - 1) * plm[1] - (double)(l + m - 1) * plm[2]) / (double)(l - m);
    }
}

// uder(3,3) as a 0-based array U[i][j] = Fortran uder(i+1, j+1)
struct Uder {
    cplx u[3][3];
    void zero() {
        for (auto& r : u)
            for (auto& c : r) c = cplx(0.0);
    }
};


// Host thread pool of the oracle's parallel frequency loop: run(n, f) calls
// f(i, t) for i in [0, n) on the pool's threads (the caller is t = 0, the
// others 1 .. size()-1), indices handed out one at a time, and returns when
// all have finished.
class Pool {
  public:
    explicit Pool(int nthreads) : n_(nthreads < 1 ? 1 : nthreads) {
        for (int t = 1; t < n_; ++t) th_.emplace_back([this, t] { loop(t); });
    }
    ~Pool() {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_ = true;
            ++gen_;
        }
        cv_.notify_all();
        for (auto& t : th_) t.join();
    }
    int size() const { return n_; }
    void run(int n, const std::function<void(int, int)>& f) {
        if (n <= 0) return;
        if (n_ == 1) {
            for (int i = 0; i < n; ++i) f(i, 0);
            return;
        }
        {
            std::lock_guard<std::mutex> g(m_);
            job_ = &f;
            njob_ = n;
            next_.store(0);
            busy_ = n_ - 1;
            ++gen_;
        }
        cv_.notify_all();
        work(0);
        std::unique_lock<std::mutex> g(m_);
        done_.wait(g, [this] { return busy_ == 0; });
        job_ = nullptr;
    }

  private:
    void work(int t) {
        for (int i = next_.fetch_add(1); i < njob_; i = next_.fetch_add(1)) (*job_)(i, t);
    }
    void loop(int t) {
        unsigned long seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> g(m_);
                cv_.wait(g, [&] { return gen_ != seen; });
                seen = gen_;
                if (stop_) return;
            }
            work(t);
            {
                std::lock_guard<std::mutex> g(m_);
                --busy_;
            }
            done_.notify_one();
        }
    }
    int n_;
    std::vector<std::thread> th_;
    std::mutex m_;
    std::condition_variable cv_, done_;
    unsigned long gen_ = 0;
    bool stop_ = false;
    const std::function<void(int, int)>* job_ = nullptr;
    int njob_ = 0, busy_ = 0;
    std::atomic<int> next_{0};
};

}  // namespace oracle
