// Element integrals of the P-SV set-up on the device: the ω- and
// l-independent matrices the reference's driver builds once per run
// (src/SGTpsv/SGTpsv-MPI.f90:383-477 with calmatc, pinteg, pmulti, polint,
// caltl, calhl, calt, calh5, submat, mtrnp, calhm1, calhm2, mtrnp2 of
// src/SGTpsv/calmat.f90:1-404, and the structure values of calstg /
// caltstg, src/SGTpsv/others.f90:590-682, 767-831).  Used when many models
// are set up per request; the host restatement (host/setup.cpp) takes the
// same steps.
//
// One thread per layer computes every integral of its layer; one thread per
// node column computes the modified first-derivative operators.  The grid
// and the offsets come from the host builder.  This file is compiled
// without fused multiply-add and every value keeps the Fortran operation
// order, so the arrays equal the host builder's bit for bit.
#include <cstdio>
#include <string>
#include <vector>

#include "common.cuh"

namespace dsm {
namespace {

// one zone of the model and of the grid
struct ZoneDev {
    int phase;       // 1 solid, 2 fluid
    int nl;          // layers
    int node0;       // 0-based index of the zone's first node in ra
    int layer0;      // index of the zone's first layer among all layers
    int off;         // 0-based element offset (solid or fluid arrays)
    int col;         // 0-based first column of the hm arrays (solid), -1 fluid
    double c[6][4];  // rho, vpv, vph, vsv, vsh, eta coefficients in r / rmax
};

constexpr int NSOLID = DSM_PSV_NSOLID;

// sum of c(j) (r/rmax)^(j-1), accumulated as calstg does
__device__ double poly_at(const double* c, double r, double rmax) {
    const double x = r / rmax;
    double coef = 1.0;
    double s = 0.0 + c[0] * coef;
    for (int j = 1; j < 4; ++j) {
        coef = coef * x;
        s = s + c[j] * coef;
    }
    return s;
}

struct Cons {
    double rho, kappa, ecKx, ecKy, ecKz, ecL, ecN, rhoinv, kappainv;
};

// calstg (and caltstg, which evaluates the same values) + calinv at radius r
__device__ Cons cons_at(const ZoneDev& z, double r, double rmax) {
    const double trho = poly_at(z.c[0], r, rmax), tvpv = poly_at(z.c[1], r, rmax), tvph = poly_at(z.c[2], r, rmax);
    const double tvsv = poly_at(z.c[3], r, rmax), tvsh = poly_at(z.c[4], r, rmax), teta = poly_at(z.c[5], r, rmax);
    Cons k;
    k.rho = trho;
    k.ecL = k.rho * tvsv * tvsv;
    k.ecN = k.rho * tvsh * tvsh;
    const double ecA = trho * tvph * tvph;
    const double ecC = trho * tvpv * tvpv;
    const double ecF = teta * (ecA - 2.0 * k.ecL);
    k.kappa = (4.0 * ecA + ecC + 4.0 * ecF - 4.0 * k.ecN) / 9.0;
    k.ecKx = ecA - 4.0 / 3.0 * k.ecN;
    k.ecKy = ecF + 2.0 / 3.0 * k.ecN;
    k.ecKz = (ecC + 2.0 * ecF) / 3.0;
    k.rhoinv = 1.0 / k.rho;
    k.kappainv = 1.0 / k.kappa;
    return k;
}

// pinteg (calmat.f90:86-124) over the one structure segment [v0, v1] a
// layer lies in, con linear from c0 to c1; p has n coefficients (n <= 5):
// pmulti by q1 + q2 x, then polint (:128-161) from x1 to x2
__device__ double pinteg_seg(const double* p, int n, double x1, double x2, double c0, double c1, double v0,
                             double v1) {
    const double q2 = (c1 - c0) / (v1 - v0);
    const double q1 = -(q2 * v0) + c0;
    double pq[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (int i = 0; i < n; ++i) {
        pq[i] = pq[i] + p[i] * q1;
        pq[i + 1] = pq[i + 1] + p[i] * q2;
    }
    double a[6], b[6];
    a[0] = 1.0;
    b[0] = 1.0;
    for (int i = 1; i <= n; ++i) {
        a[i] = a[i - 1] * x1;
        b[i] = b[i - 1] * x2;
    }
    const double dx = x2 - x1;
    double pint = 0.0;
    for (int i = 1; i <= n + 1; ++i) {
        double xx = 0.0;
        for (int j = 1; j <= i; ++j) xx = xx + a[j - 1] * b[i - j] / (double)i;
        pint = pint + pq[i - 1] * dx * xx;
    }
    return pint;
}

// calmatc (calmat.f90:1-62) of one layer [lo, hi]: entries (1,1), (1,2),
// (2,1), (2,2) of the integral of r^rpow con W^(w1dn) W^(w2dn)
__device__ void calmatc_layer(double lo, double hi, double c0, double c1, int rpow, int w1dn, int w2dn,
                              double out[4]) {
    const double rh = hi - lo;
    double A[2][2], B[2][2];  // [j][0] constant, [j][1] linear coefficient
    if (w1dn == 0) {
        A[0][0] = hi / rh;    A[0][1] = -1.0 / rh;
        A[1][0] = -(lo / rh); A[1][1] = 1.0 / rh;
    } else {
        A[0][0] = -1.0 / rh;  A[0][1] = 0.0;
        A[1][0] = 1.0 / rh;   A[1][1] = 0.0;
    }
    if (w2dn == 0) {
        B[0][0] = hi / rh;    B[0][1] = -1.0 / rh;
        B[1][0] = -(lo / rh); B[1][1] = 1.0 / rh;
    } else {
        B[0][0] = -1.0 / rh;  B[0][1] = 0.0;
        B[1][0] = 1.0 / rh;   B[1][1] = 0.0;
    }
    for (int j = 0; j < 2; ++j)
        for (int k = 0; k < 2; ++k) {
            // pmulti(2, a, 2, b, 3, c), then the shift by rpow
            const double cc[3] = {0.0 + A[j][0] * B[k][0], (0.0 + A[j][0] * B[k][1]) + A[j][1] * B[k][0],
                                  0.0 + A[j][1] * B[k][1]};
            double c[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
            for (int l = 0; l < 3; ++l) c[l + rpow] = cc[l];
            out[2 * j + k] = pinteg_seg(c, 5, lo, hi, c0, c1, lo, hi);
        }
}

// caltl (mass, :165-195) / calhl (rigidity, :200-224) of one layer
__device__ void lumped_layer(double lo, double hi, double c0, double c1, bool mass, double out[4]) {
    const double mid = (lo + hi) / 2.0;
    const double pm[3] = {0.0, 0.0, 1.0}, pr[1] = {1.0};
    out[0] = mass ? pinteg_seg(pm, 3, lo, mid, c0, c1, lo, hi) : pinteg_seg(pr, 1, lo, mid, c0, c1, lo, hi);
    out[1] = 0.0;
    out[2] = 0.0;
    out[3] = mass ? pinteg_seg(pm, 3, mid, hi, c0, c1, lo, hi) : pinteg_seg(pr, 1, mid, hi, c0, c1, lo, hi);
}

// calh5 (:246-277) of one layer
__device__ void calh5_layer(double r0, double r1, double c0, double c1, double out[4]) {
    out[0] = -(3.0 / 8.0 * c0 * r0) - 1.0 / 8.0 * c1 * r1;
    out[1] = -out[0];
    out[2] = -(1.0 / 8.0 * c0 * r0) - 3.0 / 8.0 * c1 * r1;
    out[3] = -out[2];
}

__device__ void put4(double* a, size_t o, const double v[4]) {
    for (int e = 0; e < 4; ++e) a[o + e] = v[e];
}
__device__ void put4t(double* a, size_t o, const double v[4]) {  // mtrnp (:363-386)
    a[o] = v[0];
    a[o + 1] = v[2];
    a[o + 2] = v[1];
    a[o + 3] = v[3];
}

__global__ void k_psv_integrals(const ZoneDev* __restrict__ zones, int nz, int nlayers, const double* __restrict__ ra,
                                double rmax, double* __restrict__ solid, int n_sel, double* __restrict__ fluid,
                                int n_fel) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= nlayers) return;
    int z = 0;
    while (z + 1 < nz && zones[z + 1].layer0 <= g) ++z;
    const ZoneDev& Z = zones[z];
    const int i = g - Z.layer0;
    const double lo = ra[Z.node0 + i], hi = ra[Z.node0 + i + 1];
    const Cons a = cons_at(Z, lo, rmax), b = cons_at(Z, hi, rmax);
    const size_t o = (size_t)Z.off + 4 * (size_t)i;
    double m[4], w[4], t[4];
    auto calt4 = [&](const double* x, const double* y) {
        for (int e = 0; e < 4; ++e) t[e] = (x[e] + y[e]) / 2.0;
    };
    if (Z.phase == 1) {
        auto S = [&](int k) { return solid + (size_t)k * n_sel; };
        calmatc_layer(lo, hi, a.rho, b.rho, 2, 0, 0, m);
        lumped_layer(lo, hi, a.rho, b.rho, true, w);
        calt4(m, w);
        put4(S(DSM_PSV_T), o, t);
        calmatc_layer(lo, hi, a.ecKx, b.ecKx, 0, 0, 0, m);
        lumped_layer(lo, hi, a.ecKx, b.ecKx, false, w);
        calt4(m, w);
        put4(S(DSM_PSV_H1X), o, t);
        calmatc_layer(lo, hi, a.ecL, b.ecL, 0, 0, 0, m);
        lumped_layer(lo, hi, a.ecL, b.ecL, false, w);
        calt4(m, w);
        put4(S(DSM_PSV_H2L), o, t);
        calmatc_layer(lo, hi, a.ecN, b.ecN, 0, 0, 0, m);
        lumped_layer(lo, hi, a.ecN, b.ecN, false, w);
        calt4(m, w);
        put4(S(DSM_PSV_H2N), o, t);
        // h5a / h6a (rpow 1, W' W) and their transposes h3a / h4a; then
        // the modified operators h5 = h5a - calh5 (submat) and h3 = h5^T
        const double ca[3] = {a.ecKy, a.ecL, a.ecN}, cb[3] = {b.ecKy, b.ecL, b.ecN};
        const int ka[3] = {DSM_PSV_H5AY, DSM_PSV_H6AL, DSM_PSV_H6AN};
        const int kt[3] = {DSM_PSV_H3AY, DSM_PSV_H4AL, DSM_PSV_H4AN};
        const int km[3] = {DSM_PSV_H5Y, DSM_PSV_H6L, DSM_PSV_H6N};
        const int kmt[3] = {DSM_PSV_H3Y, DSM_PSV_H4L, DSM_PSV_H4N};
        for (int q = 0; q < 3; ++q) {
            calmatc_layer(lo, hi, ca[q], cb[q], 1, 0, 1, m);
            put4(S(ka[q]), o, m);
            put4t(S(kt[q]), o, m);
            calh5_layer(lo, hi, ca[q], cb[q], w);
            for (int e = 0; e < 4; ++e) t[e] = m[e] - w[e];
            put4(S(km[q]), o, t);
            put4t(S(kmt[q]), o, t);
        }
        calmatc_layer(lo, hi, a.ecKy, b.ecKy, 2, 1, 1, m);
        put4(S(DSM_PSV_H7Y), o, m);
        calmatc_layer(lo, hi, a.ecKz, b.ecKz, 2, 1, 1, m);
        put4(S(DSM_PSV_H7Z), o, m);
        calmatc_layer(lo, hi, a.ecL, b.ecL, 2, 1, 1, m);
        put4(S(DSM_PSV_H8L), o, m);
        calmatc_layer(lo, hi, a.ecN, b.ecN, 2, 1, 1, m);
        put4(S(DSM_PSV_H8N), o, m);
    } else {
        calmatc_layer(lo, hi, a.rhoinv, b.rhoinv, 2, 1, 1, m);
        put4(fluid, o, m);
        calmatc_layer(lo, hi, a.rhoinv, b.rhoinv, 0, 0, 0, m);
        lumped_layer(lo, hi, a.rhoinv, b.rhoinv, false, w);
        calt4(m, w);
        put4(fluid + n_fel, o, t);
        calmatc_layer(lo, hi, a.kappainv, b.kappainv, 2, 0, 0, m);
        lumped_layer(lo, hi, a.kappainv, b.kappainv, true, w);
        calt4(m, w);
        put4(fluid + 2 * (size_t)n_fel, o, t);
    }
}

// entry of calhm1 (:282-318): row r (-1..2) of column j (0..nl) for the
// zone's nodes x and constant values con at those nodes
__device__ double hm1_entry(int j, int r, int nl, double c, double x) {
    const double t7 = 7.0 / 12.0 * c * x, t8 = 8.0 / 12.0 * c * x, t1 = 1.0 / 12.0 * c * x;
    const double t5 = 5.0 / 12.0 * c * x, t3 = 3.0 / 12.0 * c * x, t9 = 9.0 / 12.0 * c * x;
    if (j == 0) return r == 0 ? 0.0 - t7 : (r == 1 ? 0.0 + t8 : (r == 2 ? 0.0 - t1 : 0.0));
    if (j <= nl - 2) return r == -1 ? 0.0 - t5 : (r == 0 ? 0.0 - t3 : (r == 1 ? 0.0 + t9 : 0.0 - t1));
    if (j == nl - 1) return r == -1 ? 0.0 - t5 : (r == 0 ? 0.0 - t3 : (r == 1 ? 0.0 + t8 : 0.0));
    return r == -1 ? 0.0 - t5 : (r == 0 ? 0.0 + t5 : 0.0);
}
// entry of calhm2 (:322-358): row r (-2..1) of column j (0..nl)
__device__ double hm2_entry(int j, int r, int nl, double c, double x) {
    const double t5 = 5.0 / 12.0 * c * x, t8 = 8.0 / 12.0 * c * x, t3 = 3.0 / 12.0 * c * x;
    const double t1 = 1.0 / 12.0 * c * x, t9 = 9.0 / 12.0 * c * x, t7 = 7.0 / 12.0 * c * x;
    if (j == 0) return r == 0 ? 0.0 - t5 : (r == 1 ? 0.0 + t5 : 0.0);
    if (j == 1) return r == -1 ? 0.0 - t8 : (r == 0 ? 0.0 + t3 : (r == 1 ? 0.0 + t5 : 0.0));
    if (j <= nl - 1) return r == -2 ? 0.0 + t1 : (r == -1 ? 0.0 - t9 : (r == 0 ? 0.0 + t3 : 0.0 + t5));
    return r == -2 ? 0.0 + t1 : (r == -1 ? 0.0 - t8 : (r == 0 ? 0.0 + t7 : 0.0));
}

enum { HM3Y = 0, HM5Y, HM41L, HM42N, HM61N, HM62L };  // packing order of hm_el

// one thread per (solid zone, node column): the columns of h5my, h6m1N
// (calhm1), h6m2L (calhm2) and, by mtrnp2 (:390-404), h3my, h4m2N (from
// hm1, rows -2..1) and h4m1L (from hm2, rows -1..2)
__global__ void k_psv_hm(const ZoneDev* __restrict__ zones, int nz, int ncols, const int* __restrict__ colzone,
                         const double* __restrict__ ra, double rmax, double* __restrict__ hm, int n_hm) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ncols) return;
    const int z = colzone[2 * g], j = colzone[2 * g + 1];
    const ZoneDev& Z = zones[z];
    const int nl = Z.nl;
    auto node = [&](int jj) { return ra[Z.node0 + jj]; };
    auto con = [&](int jj, int which) {
        const Cons k = cons_at(Z, node(jj), rmax);
        return which == 0 ? k.ecKy : (which == 1 ? k.ecL : k.ecN);
    };
    auto H = [&](int a, int row4) -> double& { return hm[((size_t)a * n_hm + Z.col + j) * 4 + row4]; };
    const double x = node(j);
    const double cy = con(j, 0), cl = con(j, 1), cn = con(j, 2);
    for (int r = -1; r <= 2; ++r) {
        H(HM5Y, r + 1) = hm1_entry(j, r, nl, cy, x);
        H(HM61N, r + 1) = hm1_entry(j, r, nl, cn, x);
    }
    for (int r = -2; r <= 1; ++r) H(HM62L, r + 2) = hm2_entry(j, r, nl, cl, x);
    // mtrnp2(p, q): hm2(i, j) = hm1(-i, i + j), i = -q..p, when column i + j exists
    for (int i = -2; i <= 1; ++i) {  // p = 1, q = 2: rows -2..1 from hm1 rows -1..2
        const int n = i + j;
        const bool in = n >= 0 && n <= nl;
        H(HM3Y, i + 2) = in ? hm1_entry(n, -i, nl, con(n, 0), node(n)) : 0.0;
        H(HM42N, i + 2) = in ? hm1_entry(n, -i, nl, con(n, 2), node(n)) : 0.0;
    }
    for (int i = -1; i <= 2; ++i) {  // p = 2, q = 1: rows -1..2 from hm2 rows -2..1
        const int n = i + j;
        const bool in = n >= 0 && n <= nl;
        H(HM41L, i + 1) = in ? hm2_entry(n, -i, nl, con(n, 1), node(n)) : 0.0;
    }
}

}  // namespace
}  // namespace dsm

// Called by the host set-up builder (host/setup.cpp) in place of its own
// element-integral loop: fills solid_el [NSOLID][n_sel], fluid_el
// [3][n_fel] and hm_el [NHM][n_hm][4] (zeros outside the zones) for the
// zones' offsets elem (1-based element offset) and hmoff (1-based column,
// 0 for fluid zones).  ra holds the nnode node radii; the coefficient
// arrays are (4, nzone) column-major.  Returns DSM_OK or a DSM_ERR_* code
// with the text in err.
extern "C" int dsm_psv_integrals_device(int device, int nzone, const int* iphase, const int* nlayer, const int* isp,
                                        const int* elem, const int* hmoff, const double* ra, int nnode, double rmax,
                                        const double* rho, const double* vpv, const double* vph, const double* vsv,
                                        const double* vsh, const double* eta, int n_sel, int n_fel, int n_hm,
                                        double* solid_el, double* fluid_el, double* hm_el, char* err, int errlen) {
    using namespace dsm;
    auto fail = [&](int code, const std::string& m) {
        if (err && errlen > 0) {
            std::snprintf(err, (size_t)errlen, "%s", m.c_str());
        }
        return code;
    };
    try {
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
            return fail(DSM_ERR_NODEVICE, "no CUDA device for the element integrals");
        DSM_CUDA(cudaSetDevice(device));
        std::vector<ZoneDev> zs(nzone);
        std::vector<int> colzone;
        int layers = 0;
        const double* cf[6] = {rho, vpv, vph, vsv, vsh, eta};
        for (int z = 0; z < nzone; ++z) {
            ZoneDev& Z = zs[z];
            Z.phase = iphase[z];
            Z.nl = nlayer[z];
            Z.node0 = isp[z] - 1;
            Z.layer0 = layers;
            Z.off = elem[z] - 1;
            Z.col = Z.phase == 1 ? hmoff[z] - 1 : -1;
            for (int k = 0; k < 6; ++k)
                for (int j = 0; j < 4; ++j) Z.c[k][j] = cf[k][4 * z + j];
            if (Z.node0 < 0 || Z.node0 + Z.nl >= nnode || Z.nl < 2)
                return fail(DSM_ERR_INVALID, "zone nodes outside the grid");
            const int cap = Z.phase == 1 ? n_sel : n_fel;
            if (Z.off < 0 || Z.off + 4 * Z.nl > cap) return fail(DSM_ERR_INVALID, "element offsets outside the arrays");
            if (Z.phase == 1) {
                if (Z.col < 0 || Z.col + Z.nl + 1 > n_hm) return fail(DSM_ERR_INVALID, "hm columns outside the arrays");
                for (int j = 0; j <= Z.nl; ++j) {
                    colzone.push_back(z);
                    colzone.push_back(j);
                }
            }
            layers += Z.nl;
        }
        cudaStream_t st;
        DSM_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        DBuf<ZoneDev> dz;
        DBuf<int> dcz;
        DBuf<double> dra, ds, df, dh;
        dz.upload(zs, st);
        if (!colzone.empty()) dcz.upload(colzone, st);
        dra.upload(ra, nnode, st);
        ds.reserve((size_t)NSOLID * n_sel);
        df.reserve((size_t)3 * n_fel);
        dh.reserve((size_t)DSM_PSV_NHM * 4 * n_hm);
        DSM_CUDA(cudaMemsetAsync(ds.p, 0, sizeof(double) * NSOLID * (size_t)n_sel, st));
        DSM_CUDA(cudaMemsetAsync(df.p, 0, sizeof(double) * 3 * (size_t)n_fel, st));
        DSM_CUDA(cudaMemsetAsync(dh.p, 0, sizeof(double) * DSM_PSV_NHM * 4 * (size_t)n_hm, st));
        if (layers > 0)
            k_psv_integrals<<<(layers + 127) / 128, 128, 0, st>>>(dz.p, nzone, layers, dra.p, rmax, ds.p, n_sel, df.p,
                                                                   n_fel);
        DSM_CUDA(cudaGetLastError());
        const int ncols = (int)colzone.size() / 2;
        if (ncols > 0)
            k_psv_hm<<<(ncols + 127) / 128, 128, 0, st>>>(dz.p, nzone, ncols, dcz.p, dra.p, rmax, dh.p, n_hm);
        DSM_CUDA(cudaGetLastError());
        DSM_CUDA(cudaMemcpyAsync(solid_el, ds.p, sizeof(double) * NSOLID * (size_t)n_sel, cudaMemcpyDeviceToHost, st));
        DSM_CUDA(cudaMemcpyAsync(fluid_el, df.p, sizeof(double) * 3 * (size_t)n_fel, cudaMemcpyDeviceToHost, st));
        DSM_CUDA(cudaMemcpyAsync(hm_el, dh.p, sizeof(double) * DSM_PSV_NHM * 4 * (size_t)n_hm, cudaMemcpyDeviceToHost,
                                 st));
        DSM_CUDA(cudaStreamSynchronize(st));
        DSM_CUDA(cudaStreamDestroy(st));
        return DSM_OK;
    } catch (const Error& e) {
        return fail(e.code, e.what());
    }
}
