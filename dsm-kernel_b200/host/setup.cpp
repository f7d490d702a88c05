// Driver-side set-up of the SGT engine: input parsing, radial grid and
// element integrals.  This is the part of SGTsh/SGTpsv that runs once per
// job before the frequency loop; each function restates the Fortran
// routine named in its comment (paths relative to the DSM Kernel Suite).
// Arithmetic is FP64 in the same operation order as the Fortran; the file
// is compiled with -ffp-contract=off so that no multiply-add is fused.
#include "dsmsgt_host.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

constexpr double kPi = 3.1415926535897932;

// ---------------------------------------------------------------- arrays
// 1-based vector, matching the Fortran declarations.
struct V1 {
    std::vector<double> v;
    explicit V1(size_t n = 0) : v(n + 1, 0.0) {}
    double &operator()(long i) { return v.at(i); }
    double operator()(long i) const { return v.at(i); }
    double *p(long i) { return &v.at(i); }
    void resize(size_t n) { v.assign(n + 1, 0.0); }
};
struct I1 {
    std::vector<int> v;
    explicit I1(size_t n = 0) : v(n + 1, 0) {}
    int &operator()(long i) { return v.at(i); }
    int operator()(long i) const { return v.at(i); }
    void resize(size_t n) { v.assign(n + 1, 0); }
};

// ------------------------------------------------------- list-directed I/O
// Lines of a file with '#' comment lines removed and everything from the
// first line starting with "end" dropped (pinput, readDSMconf,
// readpsvmodel: src/SGTpsv/others.f90:27-34, 90-97, 117-126).
std::vector<std::string> filtered_lines(const char *text) {
    std::vector<std::string> out;
    std::istringstream is(text ? text : "");
    std::string line;
    while (std::getline(is, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (line.size() > 120) line.resize(120);  // format a120
        if (!line.empty() && line[0] == '#') continue;
        if (line.compare(0, 3, "end") == 0) break;
        out.push_back(line);
    }
    return out;
}

// Fortran list-directed READ over a sequence of records: one READ takes as
// many records as it needs, the rest of its last record is skipped.
struct ListReader {
    const std::vector<std::string> &lines;
    size_t rec = 0;
    explicit ListReader(const std::vector<std::string> &l) : lines(l) {}
    static std::vector<std::string> tokens(const std::string &s) {
        std::vector<std::string> t;
        std::string cur;
        for (char c : s) {
            if (c == ' ' || c == '\t' || c == ',') {
                if (!cur.empty()) { t.push_back(cur); cur.clear(); }
            } else {
                cur.push_back(c);
            }
        }
        if (!cur.empty()) t.push_back(cur);
        return t;
    }
    static double to_double(std::string s) {
        for (char &c : s)
            if (c == 'd' || c == 'D') c = 'e';
        char *end = nullptr;
        double v = std::strtod(s.c_str(), &end);
        if (end == s.c_str()) throw std::runtime_error("not a number: " + s);
        return v;
    }
    // Reads n values; missing trailing values keep their defaults when
    // allow_short is set (the reference reads 4 switches where its example
    // files give 3).
    std::vector<double> read(size_t n, bool allow_short = false) {
        std::vector<double> v;
        while (v.size() < n) {
            if (rec >= lines.size()) {
                if (allow_short) break;
                throw std::runtime_error("unexpected end of input");
            }
            auto t = tokens(lines[rec++]);
            for (auto &s : t) {
                if (v.size() == n) break;
                v.push_back(to_double(s));
            }
        }
        return v;
    }
    std::string read_line() {
        if (rec >= lines.size()) throw std::runtime_error("unexpected end of input");
        std::string s = lines[rec++];
        size_t b = s.find_first_not_of(" \t");
        size_t e = s.find_last_not_of(" \t");
        return b == std::string::npos ? std::string() : s.substr(b, e - b + 1);
    }
};

void copy_str(char *dst, size_t n, const std::string &s) {
    std::snprintf(dst, n, "%s", s.c_str());
}

struct Conf {
    double re, ratc, ratl, omegai;
    int maxlmax;
};

// readDSMconf, src/SGTpsv/others.f90:74-111
Conf parse_conf(const char *text) {
    auto lines = filtered_lines(text);
    ListReader r(lines);
    Conf c;
    c.re = r.read(1)[0];
    c.ratc = r.read(1)[0];
    c.ratl = r.read(1)[0];
    c.omegai = r.read(1)[0];
    c.maxlmax = (int)r.read(1)[0];
    return c;
}

struct Model {
    int nzone = 0;
    V1 vrmin, vrmax, qmu, qkappa;
    std::vector<V1> rho, vpv, vph, vsv, vsh, eta;  // [4] each (1..nzone)
};

// Model file read, src/SGTpsv/SGTpsv-MPI.f90:100-105 after readpsvmodel.
Model parse_model(const char *text) {
    auto lines = filtered_lines(text);
    ListReader r(lines);
    Model m;
    m.nzone = (int)r.read(1)[0];
    if (m.nzone <= 0) throw std::runtime_error("model: nzone <= 0");
    int nz = m.nzone;
    m.vrmin.resize(nz); m.vrmax.resize(nz); m.qmu.resize(nz); m.qkappa.resize(nz);
    for (auto *a : {&m.rho, &m.vpv, &m.vph, &m.vsv, &m.vsh, &m.eta}) a->assign(5, V1(nz));
    for (int i = 1; i <= nz; ++i) {
        auto v = r.read(28);
        m.vrmin(i) = v[0]; m.vrmax(i) = v[1];
        for (int j = 1; j <= 4; ++j) {
            m.rho[j](i) = v[1 + j];
            m.vpv[j](i) = v[5 + j];
            m.vph[j](i) = v[9 + j];
            m.vsv[j](i) = v[13 + j];
            m.vsh[j](i) = v[17 + j];
            m.eta[j](i) = v[21 + j];
        }
        m.qmu(i) = v[26]; m.qkappa(i) = v[27];
    }
    return m;
}

// ------------------------------------------------ polynomial integration
// pmulti, src/SGTpsv/calmat.f90:67-82 (src/SGTsh/calmat.f90:164-182)
void pmulti(int n, const double *a, int m, const double *b, int l, double *c) {
    for (int i = 0; i < l; ++i) c[i] = 0.0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < m; ++j) c[i + j] = c[i + j] + a[i] * b[j];
}

// polint, src/SGTpsv/calmat.f90:128-161
double polint(int n, const double *p, double x1, double x2) {
    double a[6], b[6];
    a[0] = 1.0; b[0] = 1.0;
    for (int i = 1; i < n; ++i) { a[i] = a[i - 1] * x1; b[i] = b[i - 1] * x2; }
    double dx = x2 - x1, pint = 0.0;
    for (int i = 1; i <= n; ++i) {
        double xx = 0.0;
        for (int j = 1; j <= i; ++j) xx = xx + a[j - 1] * b[i - j] / (double)i;
        pint = pint + p[i - 1] * dx * xx;
    }
    return pint;
}

// pinteg, src/SGTpsv/calmat.f90:86-124.  vra/con are 1-based views of
// length vnp; snp is the caller's search hint (kept across calls).
double pinteg(int &snp, int n, const double *p, double from, double to, int vnp,
              const double *vra, const double *con) {
    if (snp >= vnp) snp = 1;
    double pint = 0.0, x1 = from, x2;
    int guard = 0;
    for (;;) {
        while (!((vra[snp] <= x1) && (vra[snp + 1] > x1))) {
            snp = snp + 1;
            if (snp == vnp) snp = 1;
            if (++guard > 4 * vnp + 8) throw std::runtime_error("pinteg: radius outside grid");
        }
        x2 = std::fmin(to, vra[snp + 1]);
        double q[2], pq[6];
        q[1] = (con[snp + 1] - con[snp]) / (vra[snp + 1] - vra[snp]);
        q[0] = -q[1] * vra[snp] + con[snp];
        pmulti(n, p, 2, q, n + 1, pq);
        pint = pint + polint(n + 1, pq, x1, x2);
        if (x2 == to) break;
        x1 = x2;
    }
    return pint;
}

// calmatc: src/SGTpsv/calmat.f90:1-62 (PSV) and src/SGTsh/calmat.f90:2-83
// (SH, which symmetrises when w1dn /= w2dn).  ra and m are 1-based views.
void calmatc(int nlayer, int vnp, const double *vra, const double *con, int rpow,
             int w1dn, int w2dn, const double *ra, double *m, bool sh_symmetrise) {
    if (rpow > 2 || w1dn < 0 || w1dn > 1 || w2dn < 0 || w2dn > 1)
        throw std::runtime_error("calmatc: invalid arguments");
    std::vector<double> work(4 * nlayer + 1, 0.0);
    int snp = 1;
    for (int i = 1; i <= nlayer; ++i) {
        double rh = ra[i + 1] - ra[i];
        double a[2][2], b[2][2];  // a[col][row] = Fortran a(row+1,col+1)
        if (w1dn == 0) {
            a[0][1] = -1.0 / rh; a[0][0] = ra[i + 1] / rh;
            a[1][1] = 1.0 / rh;  a[1][0] = -ra[i] / rh;
        } else {
            a[0][1] = 0.0; a[0][0] = -1.0 / rh; a[1][1] = 0.0; a[1][0] = 1.0 / rh;
        }
        if (w2dn == 0) {
            b[0][1] = -1.0 / rh; b[0][0] = ra[i + 1] / rh;
            b[1][1] = 1.0 / rh;  b[1][0] = -ra[i] / rh;
        } else {
            b[0][1] = 0.0; b[0][0] = -1.0 / rh; b[1][1] = 0.0; b[1][0] = 1.0 / rh;
        }
        for (int j = 1; j <= 2; ++j) {
            for (int k = 1; k <= 2; ++k) {
                double c[5] = {0, 0, 0, 0, 0};
                pmulti(2, a[j - 1], 2, b[k - 1], 3, c);
                for (int l = 3; l >= 1; --l) {
                    c[l + rpow - 1] = c[l - 1];
                    if (rpow > 0) c[l - 1] = 0.0;
                }
                int nn = 4 * (i - 1) + 2 * (j - 1) + k;
                work[nn] = pinteg(snp, 5, c, ra[i], ra[i + 1], vnp, vra, con);
            }
        }
    }
    if (sh_symmetrise && w1dn != w2dn) {
        for (int i = 1; i <= 4 * nlayer; ++i) {
            if ((i % 4 == 0) || (i % 4 == 1)) m[i] = 2.0 * work[i];
            else if (i % 4 == 2) m[i] = work[i] + work[i + 1];
            else m[i] = work[i - 1] + work[i];
        }
    } else {
        for (int i = 1; i <= 4 * nlayer; ++i) m[i] = work[i];
    }
}

// caltl: lumped mass, src/SGTpsv/calmat.f90:165-195
void caltl(int nlayer, int vnp, const double *vra, const double *rho, const double *ra,
           double *tl) {
    int snp = 1;
    for (int i = 1; i <= nlayer; ++i) {
        double c[3] = {0.0, 0.0, 1.0};
        double from = ra[i], to = (ra[i] + ra[i + 1]) / 2.0;
        int nn = 4 * (i - 1);
        tl[nn + 1] = pinteg(snp, 3, c, from, to, vnp, vra, rho);
        tl[nn + 2] = 0.0;
        tl[nn + 3] = 0.0;
        from = to; to = ra[i + 1];
        tl[nn + 4] = pinteg(snp, 3, c, from, to, vnp, vra, rho);
    }
}

// calhl: lumped rigidity, src/SGTpsv/calmat.f90:200-224
void calhl(int nlayer, int vnp, const double *vra, const double *mu, const double *ra,
           double *hl) {
    int snp = 1;
    for (int i = 1; i <= nlayer; ++i) {
        double c[1] = {1.0};
        double from = ra[i], to = (ra[i] + ra[i + 1]) / 2.0;
        int nn = 4 * (i - 1);
        hl[nn + 1] = pinteg(snp, 1, c, from, to, vnp, vra, mu);
        hl[nn + 2] = 0.0;
        hl[nn + 3] = 0.0;
        from = to; to = ra[i + 1];
        hl[nn + 4] = pinteg(snp, 1, c, from, to, vnp, vra, mu);
    }
}

// calt, src/SGTpsv/calmat.f90:231-241
void calt(int nlayer, const double *tl, const double *tc, double *t) {
    for (int i = 1; i <= 4 * nlayer; ++i) t[i] = (tl[i] + tc[i]) / 2.0;
}

// calgrid: src/SGTsh/others.f90:383-459 (SH uses vs only) and
// src/SGTpsv/others.f90:374-450 (PSV uses vp in fluid zones).
void calgrid(int nzone, const V1 &vrmin, const V1 &vrmax, const std::vector<V1> &vp,
             const std::vector<V1> &vs, bool psv, double rmin, double rmax, int imax, int lmin,
             double tlen, V1 &vmin, V1 &gridpar, V1 &dzpar) {
    for (int iz = 1; iz <= nzone; ++iz) {
        double v[5];
        bool usevp = psv && vs[1](iz) == 0.0;
        for (int i = 1; i <= 4; ++i) v[i] = usevp ? vp[i](iz) : vs[i](iz);
        double vs1 = 0.0, vs2 = 0.0, c1 = 1.0, c2 = 1.0;
        for (int j = 1; j <= 4; ++j) {
            if (j == 1) { c1 = 1.0; c2 = 1.0; }
            else { c1 = c1 * (vrmin(iz) / rmax); c2 = c2 * (vrmax(iz) / rmax); }
            vs1 = vs1 + v[j] * c1;
            vs2 = vs2 + v[j] * c2;
        }
        double rh = vrmax(iz) - vrmin(iz);
        double omega = 2.0 * kPi * (double)imax / tlen;
        vmin(iz) = (vs1 >= vs2) ? vs2 : vs1;
        double amax = vrmax(iz);
        double gtmp = (omega * omega) / (vmin(iz) * vmin(iz)) -
                      (((double)lmin + 0.5) * ((double)lmin + 0.5)) / (amax * amax);
        if (gtmp > 0.0) {
            dzpar(iz) = std::sqrt(1.0 / gtmp);
            gridpar(iz) = rh / dzpar(iz);
        } else {
            dzpar(iz) = 0.0;
            gridpar(iz) = 0.0;
        }
    }
    double gtmp = 0.0;
    for (int iz = 1; iz <= nzone; ++iz) gtmp = gtmp + gridpar(iz);
    for (int iz = 1; iz <= nzone; ++iz) {
        if (gridpar(iz) > 0.0) gridpar(iz) = gridpar(iz) / gtmp;
        else gridpar(iz) = (vrmax(iz) - vrmin(iz)) / (rmax - rmin) * 0.1;
    }
    gtmp = 0.0;
    for (int iz = 1; iz <= nzone; ++iz) gtmp = gtmp + gridpar(iz);
    for (int iz = 1; iz <= nzone; ++iz) gridpar(iz) = gridpar(iz) / gtmp;
}

// layers per zone: calra (src/SGTsh/others.f90:463-495) and calra_psv
// (src/SGTpsv/others.f90:1292-1340), see Geller & Takeuchi 1995 eq. 6.2.
int layers_per_zone(int nzone, const V1 &vrmin, const V1 &vrmax, const V1 &dzpar, double re,
                    I1 &nnl) {
    int total = 0;
    for (int iz = 1; iz <= nzone; ++iz) {
        double rh = vrmax(iz) - vrmin(iz);
        int ntmp;
        if (dzpar(iz) == 0.0) ntmp = 1;
        else ntmp = (int)(std::sqrt(3.3 / re) * rh / dzpar(iz) / 2.0 / kPi / 7.0e-1 + 1);
        nnl(iz) = ntmp < 5 ? 5 : ntmp;
        total += nnl(iz);
    }
    return total;
}

// node radii: first loop of calra2 / calra2_psv
void node_radii(int nzone, const V1 &vrmin, const V1 &vrmax, const I1 &nnl, double rmin, V1 &ra) {
    ra(1) = rmin;
    int itmp = 1;
    for (int iz = 1; iz <= nzone; ++iz) {
        double rh = vrmax(iz) - vrmin(iz);
        for (int i = 1; i <= nnl(iz); ++i) {
            itmp = itmp + 1;
            ra(itmp) = vrmin(iz) + rh * (double)i / (double)nnl(iz);
        }
    }
}

double poly4(const std::vector<V1> &c, int iz, double r, double rmax) {
    double s = 0.0, coef = 1.0;
    for (int j = 1; j <= 4; ++j) {
        if (j == 1) coef = 1.0;
        else coef = coef * (r / rmax);
        s = s + c[j](iz) * coef;
    }
    return s;
}

}  // namespace

// ============================================================== bundles
struct dsm_bundle {
    bool psv = false;
    int n_nodes = 0, n_unknowns = 0;
    // SH storage
    dsm_sh_setup_t sh{};
    // PSV storage
    dsm_psv_setup_t psvs{};
    std::vector<std::vector<double>> dvec;
    std::vector<std::vector<int>> ivec;
    const double *keep(std::vector<double> v) {
        dvec.push_back(std::move(v));
        return dvec.back().data();
    }
    const int *keepi(std::vector<int> v) {
        ivec.push_back(std::move(v));
        return ivec.back().data();
    }
    // converts a 1-based V1 to a 0-based stored array of n entries
    const double *keep1(const V1 &a, size_t n) {
        return keep(std::vector<double>(a.v.begin() + 1, a.v.begin() + 1 + n));
    }
    const int *keep1i(const I1 &a, size_t n) {
        return keepi(std::vector<int>(a.v.begin() + 1, a.v.begin() + 1 + n));
    }
};

extern "C" const char *dsm_host_last_error(void) { return g_err.c_str(); }

extern "C" int dsm_parse_params(const char *text, dsm_params_t *out) {
    try {
        if (!text || !out) throw std::runtime_error("null argument");
        auto lines = filtered_lines(text);
        ListReader r(lines);
        std::memset(out, 0, sizeof(*out));
        copy_str(out->dsmconf, sizeof out->dsmconf, r.read_line());
        copy_str(out->outdir, sizeof out->outdir, r.read_line());
        copy_str(out->model, sizeof out->model, r.read_line());
        copy_str(out->modelname, sizeof out->modelname, r.read_line());
        out->tlen = r.read(1)[0];
        auto rr = r.read(3);
        out->rmin_ = rr[0]; out->rmax_ = rr[1]; out->rdelta_ = rr[2];
        out->r0min = r.read(1)[0];
        auto th = r.read(3);
        out->thetamin = th[0]; out->thetamax = th[1]; out->thetadelta = th[2];
        auto ii = r.read(2);
        out->imin = (int)ii[0]; out->imax = (int)ii[1];
        auto sw = r.read(4, true);
        int *dst[4] = {&out->rsgt_switch, &out->tsgt_switch, &out->synn_switch, &out->psgt_switch};
        for (size_t k = 0; k < sw.size(); ++k) *dst[k] = (int)sw[k];
        return DSM_OK;
    } catch (const std::exception &e) {
        g_err = std::string("dsm_parse_params: ") + e.what();
        return DSM_ERR_INVALID;
    }
}

extern "C" void dsm_bundle_free(dsm_bundle_t *b) { delete b; }

extern "C" int dsm_bundle_info(const dsm_bundle_t *b, int *n_nodes, int *n_unknowns) {
    if (!b) return DSM_ERR_INVALID;
    if (n_nodes) *n_nodes = b->n_nodes;
    if (n_unknowns) *n_unknowns = b->n_unknowns;
    return DSM_OK;
}

// ============================================================== SH set-up
// src/SGTsh/SGTsh-MPI.f90:66-347
extern "C" int dsm_sh_setup_build(const dsm_params_t *par, const char *conf_text,
                                  const char *model_text, dsm_bundle_t **bundle_out,
                                  const dsm_sh_setup_t **setup_out) {
    try {
        if (!par || !bundle_out || !setup_out) throw std::runtime_error("null argument");
        Conf conf = parse_conf(conf_text);
        Model full = parse_model(model_text);
        // outer-core cut: ioutercore is the last fluid zone, 0 when there is
        // none (:83-102)
        int ioutercore = 0;
        for (int i = 1; i <= full.nzone; ++i) {
            bool fluid = full.vsv[1](i) == 0.0 && full.vsv[2](i) == 0.0 &&
                         full.vsv[3](i) == 0.0 && full.vsv[4](i) == 0.0;
            if (fluid) ioutercore = i;
        }
        int nzone = full.nzone - ioutercore;
        if (nzone <= 0) throw std::runtime_error("SH: no solid zone above the outer core");
        V1 vrmin(nzone), vrmax(nzone), qmu(nzone);
        std::vector<V1> rrho(5, V1(nzone)), vsv(5, V1(nzone)), vsh(5, V1(nzone));
        for (int i = 1; i <= nzone; ++i) {
            int s = i + ioutercore;
            vrmin(i) = full.vrmin(s); vrmax(i) = full.vrmax(s); qmu(i) = full.qmu(s);
            for (int j = 1; j <= 4; ++j) {
                rrho[j](i) = full.rho[j](s); vsv[j](i) = full.vsv[j](s); vsh[j](i) = full.vsh[j](s);
            }
        }
        double rmin = vrmin(1), rmax = vrmax(nzone);
        double tlen = par->tlen;
        double omegai = -std::log(conf.omegai) / tlen;
        // receiver radii above rmin (:152-179)
        double rmin_ = par->rmin_, rdelta_ = par->rdelta_;
        int r_n = (int)((par->rmax_ - rmin_) / rdelta_) + 1;
        int ir_ = 0;
        for (int i = 1; i <= r_n; ++i)
            if (rmin_ + (double)(i - 1) * rdelta_ <= rmin) ir_ = i;
        r_n = r_n - ir_;
        rmin_ = rmin_ + (double)ir_ * rdelta_;
        if (r_n <= 0) throw std::runtime_error("SH: no receiver above rmin");
        V1 r_(r_n);
        for (int i = 1; i <= r_n; ++i) r_(i) = rmin_ + (double)(i - 1) * rdelta_;
        int theta_n = (int)((par->thetamax - par->thetamin) / par->thetadelta) + 1;
        std::vector<double> theta(theta_n);
        for (int i = 1; i <= theta_n; ++i)
            theta[i - 1] = par->thetamin + (double)(i - 1) * par->thetadelta;
        double r0 = par->r0min;
        // grid (:276-287)
        V1 vmin(nzone), gridpar(nzone), dzpar(nzone);
        calgrid(nzone, vrmin, vrmax, vsv, vsv, false, rmin, rmax, par->imax, 1, tlen, vmin,
                gridpar, dzpar);
        I1 nlayer(nzone);
        int nnlayer = layers_per_zone(nzone, vrmin, vrmax, dzpar, conf.re, nlayer);
        V1 ra(nnlayer + nzone + 1);
        node_radii(nzone, vrmin, vrmax, nlayer, rmin, ra);
        // receiver bracketing, second loop of calra2 (src/SGTsh/others.f90:527-559)
        V1 rrsta(3 * r_n);
        I1 iista(3 * r_n);
        {
            int itmp = 1;
            for (int iz = 1; iz <= nzone; ++iz) {
                for (int i = 1; i <= nlayer(iz); ++i) {
                    for (int ista = 1; ista <= r_n; ++ista) {
                        if (ra(itmp) < r_(ista) && r_(ista) <= ra(itmp + 1)) {
                            int b = (i != nlayer(iz)) ? itmp : itmp - 1;
                            for (int k = 0; k < 3; ++k) {
                                rrsta(3 * (ista - 1) + 1 + k) = ra(b + k);
                                iista(3 * (ista - 1) + 1 + k) = b + k;
                            }
                        }
                    }
                    itmp = itmp + 1;
                }
            }
        }
        for (int ista = 1; ista <= r_n; ++ista)
            if (iista(3 * (ista - 1) + 1) <= 0)
                throw std::runtime_error("SH: receiver outside the grid");
        // stack points calsp (src/SGTsh/others.f90:569-584)
        I1 isp(nzone), jsp(nzone);
        isp(1) = 1; jsp(1) = 1;
        for (int i = 1; i <= nzone - 1; ++i) {
            isp(i + 1) = isp(i) + nlayer(i);
            jsp(i + 1) = jsp(i) + 4 * nlayer(i);
        }
        // source: calspo (src/SGTsh/others.f90:588-631), calgra (:637-647)
        int ndc = nzone - 1;
        if (r0 < rmin || r0 > rmax) throw std::runtime_error("The source location is improper.(calspo)");
        double spo;
        int spn;
        if (r0 == rmax) {
            spo = (double)nnlayer - 0.01;
            r0 = ra(nnlayer) + (spo - (double)(nnlayer - 1)) * (ra(nnlayer + 1) - ra(nnlayer));
        } else {
            int itmp;
            for (itmp = 2; itmp <= ndc + nnlayer + 2; ++itmp)
                if (r0 < ra(itmp)) break;
            spo = (double)(itmp - 2) + (r0 - ra(itmp - 1)) / (ra(itmp) - ra(itmp - 1));
            if ((spo - (double)(itmp - 2)) < 0.01) {
                spo = (double)(itmp - 2) + 0.01;
                r0 = ra(itmp - 1) + (spo - (double)(itmp - 2)) * (ra(itmp) - ra(itmp - 1));
            }
            if ((spo - (double)(itmp - 2)) > 0.99) {
                spo = (double)(itmp - 2) + 0.99;
                r0 = ra(itmp - 1) + (spo - (double)(itmp - 2)) * (ra(itmp) - ra(itmp - 1));
            }
        }
        spn = 0;
        for (int itmp = 1; itmp <= ndc + 1; ++itmp) {
            spn = spn + 1;
            if (r0 <= vrmax(itmp)) break;
        }
        spo = spo - (double)(isp(spn) - 1);
        int igr = isp(spn) + (int)std::trunc(spo);
        double gra[4] = {0.0, ra(igr), r0, ra(igr + 1)};
        // structure at grid points: calstg (src/SGTsh/others.f90:651-694)
        int nvra = nnlayer + 2 * nzone + 1;
        V1 vra(nvra), rho(nvra), ecL(nvra), ecN(nvra);
        int vnp;
        {
            int itmp = 0, jtmp = 0;
            for (int iz = 1; iz <= nzone; ++iz) {
                for (int i = 1; i <= nlayer(iz) + 1; ++i) {
                    itmp++; jtmp++;
                    vra(itmp) = ra(jtmp);
                    double trho = 0, tvsv = 0, tvsh = 0, coef = 1.0;
                    for (int j = 1; j <= 4; ++j) {
                        if (j == 1) coef = 1.0;
                        else coef = coef * (vra(itmp) / rmax);
                        trho = trho + rrho[j](iz) * coef;
                        tvsv = tvsv + vsv[j](iz) * coef;
                        tvsh = tvsh + vsh[j](iz) * coef;
                    }
                    rho(itmp) = trho;
                    ecL(itmp) = rho(itmp) * tvsv * tvsv;
                    ecN(itmp) = rho(itmp) * tvsh * tvsh;
                }
                jtmp = jtmp - 1;
            }
            vnp = itmp;
        }
        // calgstg (src/SGTsh/others.f90:699-742)
        double gvra[4], grho[4], gecL[4], gecN[4];
        for (int i = 1; i <= 3; ++i) {
            gvra[i] = gra[i];
            double trho = 0, tvsv = 0, tvsh = 0, coef = 1.0;
            for (int j = 1; j <= 4; ++j) {
                if (j == 1) coef = 1.0;
                else coef = coef * (gvra[i] / rmax);
                trho = trho + rrho[j](spn) * coef;
                tvsv = tvsv + vsv[j](spn) * coef;
                tvsh = tvsh + vsh[j](spn) * coef;
            }
            grho[i] = trho;
            gecL[i] = grho[i] * tvsv * tvsv;
            gecN[i] = grho[i] * tvsh * tvsh;
        }
        double mu0 = gecL[2];
        // element integrals (:314-339)
        V1 t(4 * nnlayer), h1(4 * nnlayer), h2(4 * nnlayer), h3(4 * nnlayer), h4(4 * nnlayer),
            work(4 * nnlayer);
        const double *pv = vra.v.data();
        for (int i = 1; i <= nzone; ++i) {
            const double *rz = ra.p(isp(i)) - 1;
            int o = jsp(i) - 1;
            calmatc(nlayer(i), vnp, pv, rho.v.data(), 2, 0, 0, rz, t.v.data() + o, true);
            calmatc(nlayer(i), vnp, pv, ecL.v.data(), 2, 1, 1, rz, h1.v.data() + o, true);
            calmatc(nlayer(i), vnp, pv, ecL.v.data(), 1, 1, 0, rz, h2.v.data() + o, true);
            calmatc(nlayer(i), vnp, pv, ecL.v.data(), 0, 0, 0, rz, h3.v.data() + o, true);
            calmatc(nlayer(i), vnp, pv, ecN.v.data(), 0, 0, 0, rz, h4.v.data() + o, true);
            caltl(nlayer(i), vnp, pv, rho.v.data(), rz, work.v.data() + o);
            calt(nlayer(i), t.v.data() + o, work.v.data() + o, t.v.data() + o);
            calhl(nlayer(i), vnp, pv, ecL.v.data(), rz, work.v.data() + o);
            calt(nlayer(i), h3.v.data() + o, work.v.data() + o, h3.v.data() + o);
            calhl(nlayer(i), vnp, pv, ecN.v.data(), rz, work.v.data() + o);
            calt(nlayer(i), h4.v.data() + o, work.v.data() + o, h4.v.data() + o);
        }
        double gt[9] = {0}, gh1[9] = {0}, gh2[9] = {0}, gh3[9] = {0}, gh4[9] = {0}, gw[9] = {0};
        calmatc(2, 3, gvra, grho, 2, 0, 0, gra, gt, true);
        calmatc(2, 3, gvra, gecL, 2, 1, 1, gra, gh1, true);
        calmatc(2, 3, gvra, gecL, 1, 1, 0, gra, gh2, true);
        calmatc(2, 3, gvra, gecL, 0, 0, 0, gra, gh3, true);
        calmatc(2, 3, gvra, gecN, 0, 0, 0, gra, gh4, true);
        caltl(2, 3, gvra, grho, gra, gw);
        calt(2, gt, gw, gt);
        calhl(2, 3, gvra, gecL, gra, gw);
        calt(2, gh3, gw, gh3);
        calhl(2, 3, gvra, gecN, gra, gw);
        calt(2, gh4, gw, gh4);
        int ns = isp(spn) + (int)std::trunc(spo);
        int ins = 4 * ns - 3;

        auto *b = new dsm_bundle;
        b->psv = false;
        b->n_nodes = nnlayer + 1;
        b->n_unknowns = nnlayer + 1;
        dsm_sh_setup_t &s = b->sh;
        s.nzone = nzone;
        s.vrmin = b->keep1(vrmin, nzone);
        s.vrmax = b->keep1(vrmax, nzone);
        {
            std::vector<double> v(4 * nzone);
            for (int i = 1; i <= nzone; ++i)
                for (int j = 1; j <= 4; ++j) v[4 * (i - 1) + (j - 1)] = vsv[j](i);
            s.vsv = b->keep(v);
        }
        s.qmu = b->keep1(qmu, nzone);
        s.nlayer = b->keep1i(nlayer, nzone);
        s.isp = b->keep1i(isp, nzone);
        s.jsp = b->keep1i(jsp, nzone);
        s.nnlayer = nnlayer;
        s.t = b->keep1(t, 4 * nnlayer);
        s.h1 = b->keep1(h1, 4 * nnlayer);
        s.h2 = b->keep1(h2, 4 * nnlayer);
        s.h3 = b->keep1(h3, 4 * nnlayer);
        s.h4 = b->keep1(h4, 4 * nnlayer);
        s.spn = spn; s.spo = spo; s.r0 = r0; s.mu0 = mu0; s.ins = ins;
        s.gt = b->keep(std::vector<double>(gt + 1, gt + 9));
        s.gh1 = b->keep(std::vector<double>(gh1 + 1, gh1 + 9));
        s.gh2 = b->keep(std::vector<double>(gh2 + 1, gh2 + 9));
        s.gh3 = b->keep(std::vector<double>(gh3 + 1, gh3 + 9));
        s.gh4 = b->keep(std::vector<double>(gh4 + 1, gh4 + 9));
        s.r_n = r_n;
        s.r = b->keep1(r_, r_n);
        s.rrsta = b->keep1(rrsta, 3 * r_n);
        s.iista = b->keep1i(iista, 3 * r_n);
        s.theta_n = theta_n;
        s.theta = b->keep(theta);
        s.tlen = tlen; s.omegai = omegai; s.ratl = conf.ratl; s.maxlmax = conf.maxlmax;
        s.imin = par->imin; s.imax = par->imax;
        s.rsgt_switch = par->rsgt_switch; s.tsgt_switch = par->tsgt_switch;
        s.synn_switch = par->synn_switch;
        *bundle_out = b;
        *setup_out = &b->sh;
        return DSM_OK;
    } catch (const std::exception &e) {
        g_err = std::string("dsm_sh_setup_build: ") + e.what();
        return DSM_ERR_INVALID;
    }
}

// ============================================================= PSV set-up
namespace {

// calh5, src/SGTpsv/calmat.f90:246-277.  vra, con, ra are 1-based views
// starting at the zone's first grid point.
void calh5(int nlayer, const double *vra, const double *con, const double *ra, double *h5) {
    for (int i = 1; i <= 4 * nlayer; ++i) h5[i] = 0.0;
    int itmp = 0;
    for (;;) {
        itmp++;
        if (vra[itmp] == ra[1]) {
            if (vra[itmp + 1] == vra[itmp]) itmp++;
            break;
        }
    }
    itmp = itmp - 1;
    for (int i = 1; i <= nlayer; ++i) {
        itmp++;
        h5[4 * i - 3] = -3.0 / 8.0 * con[itmp] * ra[i] - 1.0 / 8.0 * con[itmp + 1] * ra[i + 1];
        h5[4 * i - 2] = -h5[4 * i - 3];
        h5[4 * i - 1] = -1.0 / 8.0 * con[itmp] * ra[i] - 3.0 / 8.0 * con[itmp + 1] * ra[i + 1];
        h5[4 * i] = -h5[4 * i - 1];
    }
}

// hm views: column j (1-based) of a (lo:lo+3, *) array
struct HM {
    double *base;  // points at element (lo, 1)
    int lo;
    double &operator()(int i, int j) { return base[4 * (j - 1) + (i - lo)]; }
};

// calhm1, src/SGTpsv/calmat.f90:282-318 (accumulates)
void calhm1(int nlayer, const double *vra, const double *con, const double *ra, HM hm1) {
    int itmp = 0;
    for (;;) {
        itmp++;
        if (vra[itmp] == ra[1]) {
            if (vra[itmp + 1] == vra[itmp]) itmp++;
            break;
        }
    }
    hm1(0, 1) = hm1(0, 1) - 7.0 / 12.0 * con[itmp] * ra[1];
    hm1(1, 1) = hm1(1, 1) + 8.0 / 12.0 * con[itmp] * ra[1];
    hm1(2, 1) = hm1(2, 1) - 1.0 / 12.0 * con[itmp] * ra[1];
    for (int i = 2; i <= nlayer - 1; ++i) {
        itmp++;
        hm1(-1, i) = hm1(-1, i) - 5.0 / 12.0 * con[itmp] * ra[i];
        hm1(0, i) = hm1(0, i) - 3.0 / 12.0 * con[itmp] * ra[i];
        hm1(1, i) = hm1(1, i) + 9.0 / 12.0 * con[itmp] * ra[i];
        hm1(2, i) = hm1(2, i) - 1.0 / 12.0 * con[itmp] * ra[i];
    }
    itmp++;
    hm1(-1, nlayer) = hm1(-1, nlayer) - 5.0 / 12.0 * con[itmp] * ra[nlayer];
    hm1(0, nlayer) = hm1(0, nlayer) - 3.0 / 12.0 * con[itmp] * ra[nlayer];
    hm1(1, nlayer) = hm1(1, nlayer) + 8.0 / 12.0 * con[itmp] * ra[nlayer];
    itmp++;
    hm1(-1, nlayer + 1) = hm1(-1, nlayer + 1) - 5.0 / 12.0 * con[itmp] * ra[nlayer + 1];
    hm1(0, nlayer + 1) = hm1(0, nlayer + 1) + 5.0 / 12.0 * con[itmp] * ra[nlayer + 1];
}

// calhm2, src/SGTpsv/calmat.f90:322-358 (accumulates)
void calhm2(int nlayer, const double *vra, const double *con, const double *ra, HM hm2) {
    int itmp = 0;
    for (;;) {
        itmp++;
        if (vra[itmp] == ra[1]) {
            if (vra[itmp + 1] == vra[itmp]) itmp++;
            break;
        }
    }
    hm2(0, 1) = hm2(0, 1) - 5.0 / 12.0 * con[itmp] * ra[1];
    hm2(1, 1) = hm2(1, 1) + 5.0 / 12.0 * con[itmp] * ra[1];
    itmp++;
    hm2(-1, 2) = hm2(-1, 2) - 8.0 / 12.0 * con[itmp] * ra[2];
    hm2(0, 2) = hm2(0, 2) + 3.0 / 12.0 * con[itmp] * ra[2];
    hm2(1, 2) = hm2(1, 2) + 5.0 / 12.0 * con[itmp] * ra[2];
    for (int i = 3; i <= nlayer; ++i) {
        itmp++;
        hm2(-2, i) = hm2(-2, i) + 1.0 / 12.0 * con[itmp] * ra[i];
        hm2(-1, i) = hm2(-1, i) - 9.0 / 12.0 * con[itmp] * ra[i];
        hm2(0, i) = hm2(0, i) + 3.0 / 12.0 * con[itmp] * ra[i];
        hm2(1, i) = hm2(1, i) + 5.0 / 12.0 * con[itmp] * ra[i];
    }
    itmp++;
    hm2(-2, nlayer + 1) = hm2(-2, nlayer + 1) + 1.0 / 12.0 * con[itmp] * ra[nlayer + 1];
    hm2(-1, nlayer + 1) = hm2(-1, nlayer + 1) - 8.0 / 12.0 * con[itmp] * ra[nlayer + 1];
    hm2(0, nlayer + 1) = hm2(0, nlayer + 1) + 7.0 / 12.0 * con[itmp] * ra[nlayer + 1];
}

// mtrnp, src/SGTpsv/calmat.f90:363-386
void mtrnp(int nlayer, const double *a1, double *a2) {
    int nn = 4 * nlayer;
    for (int i = 1; i <= nn - 3; i += 4) a2[i] = a1[i];
    for (int i = 2; i <= nn - 2; i += 4) a2[i] = a1[i + 1];
    for (int i = 3; i <= nn - 1; i += 4) a2[i] = a1[i - 1];
    for (int i = 4; i <= nn; i += 4) a2[i] = a1[i];
}

// mtrnp2, src/SGTpsv/calmat.f90:390-404: hm2(-q:p) from hm1(-p:q)
void mtrnp2(int nlayer, int p, int q, HM hm1, HM hm2) {
    for (int i = -q; i <= p; ++i)
        for (int j = 1; j <= nlayer + 1; ++j) {
            int m = -i, n = i + j;
            if (n >= 1 && n <= nlayer + 1) hm2(i, j) = hm1(m, n);
        }
}

}  // namespace

// src/SGTpsv/SGTpsv-MPI.f90:98-477 and the l-independent parts of the
// omega/l loops (calspdr, ksta, nn: :621-629; source indices :557-558,
// :636-641).
// element integrals on the device (csrc/setup_dev.cu)
extern "C" int dsm_psv_integrals_device(int device, int nzone, const int *iphase, const int *nlayer, const int *isp,
                                        const int *elem, const int *hmoff, const double *ra, int nnode, double rmax,
                                        const double *rho, const double *vpv, const double *vph, const double *vsv,
                                        const double *vsh, const double *eta, int n_sel, int n_fel, int n_hm,
                                        double *solid_el, double *fluid_el, double *hm_el, char *err, int errlen);

namespace {
// device < 0: element integrals on the host; otherwise on that CUDA device
int psv_setup_build(const dsm_params_t *par, const char *conf_text, const char *model_text, int device,
                    dsm_bundle_t **bundle_out, const dsm_psv_setup_t **setup_out) {
    try {
        if (!par || !bundle_out || !setup_out) throw std::runtime_error("null argument");
        Conf conf = parse_conf(conf_text);
        Model md = parse_model(model_text);
        int nzone = md.nzone;
        double rmin = md.vrmin(1), rmax = md.vrmax(nzone);
        double tlen = par->tlen;
        double omegai = -std::log(conf.omegai) / tlen;
        int r_n = (int)((par->rmax_ - par->rmin_) / par->rdelta_) + 1;
        if (r_n <= 0) throw std::runtime_error("PSV: no receiver");
        V1 r_(r_n);
        for (int i = 1; i <= r_n; ++i) r_(i) = par->rmin_ + (double)(i - 1) * par->rdelta_;
        // calstg_for_stackpoints (src/SGTpsv/others.f90:687-762)
        V1 lambda(r_n), qkp(r_n);
        for (int ir = 1; ir <= r_n; ++ir) {
            double r = r_(ir);
            for (int iz = 1; iz <= nzone; ++iz) {
                if (r > md.vrmin(iz) && r <= md.vrmax(iz)) {
                    double trho = poly4(md.rho, iz, r, rmax);
                    double tvph = poly4(md.vph, iz, r, rmax);
                    lambda(ir) = trho * tvph * tvph;
                    qkp(ir) = md.qkappa(iz);
                }
            }
        }
        int theta_n = (int)((par->thetamax - par->thetamin) / par->thetadelta) + 1;
        std::vector<double> theta(theta_n);
        for (int i = 1; i <= theta_n; ++i)
            theta[i - 1] = par->thetamin + (double)(i - 1) * par->thetadelta;
        double r0 = par->r0min;
        // calnl (src/SGTpsv/others.f90:348-368)
        I1 iphase(nzone);
        int nsl = 0, nll = 0;
        for (int i = 1; i <= nzone; ++i) {
            bool fl = md.vsv[1](i) == 0.0 && md.vsv[2](i) == 0.0 && md.vsv[3](i) == 0.0 &&
                      md.vsv[4](i) == 0.0;
            if (fl) { nll++; iphase(i) = 2; }
            else { nsl++; iphase(i) = 1; }
        }
        if (nsl == 0) throw std::runtime_error("PSV: model has no solid zone");
        int ndc = nzone - 1;
        if (r0 < rmin || r0 > rmax) throw std::runtime_error("Location of the source is improper.");
        V1 vmin(nzone), gridpar(nzone), dzpar(nzone);
        calgrid(nzone, md.vrmin, md.vrmax, md.vpv, md.vsv, true, rmin, rmax, par->imax, 1, tlen,
                vmin, gridpar, dzpar);
        I1 nlayer(nzone);
        int nnlayer = layers_per_zone(nzone, md.vrmin, md.vrmax, dzpar, conf.re, nlayer);
        int nslay = 0, nllay = 0;
        for (int iz = 1; iz <= nzone; ++iz) {
            if (iphase(iz) == 1) nslay += nlayer(iz);
            else nllay += nlayer(iz);
        }
        int inlayer = nnlayer;
        V1 ra(nnlayer + nzone + 1);
        node_radii(nzone, md.vrmin, md.vrmax, nlayer, rmin, ra);
        // receiver bracketing, calra2_psv (src/SGTpsv/others.f90:1376-1416)
        V1 rrsta(3 * r_n);
        I1 iista(3 * r_n), istazone(r_n);
        {
            int itmp = 1;
            for (int iz = 1; iz <= nzone; ++iz) {
                for (int i = 1; i <= nlayer(iz); ++i) {
                    for (int ista = 1; ista <= r_n; ++ista) {
                        if (ra(itmp) < r_(ista) && r_(ista) <= ra(itmp + 1)) {
                            istazone(ista) = iz;
                            int gb = (i != nlayer(iz)) ? itmp : itmp - 1;
                            int lb = (i != nlayer(iz)) ? i : i - 1;
                            for (int k = 0; k < 3; ++k) {
                                rrsta(3 * (ista - 1) + 1 + k) = ra(gb + k);
                                iista(3 * (ista - 1) + 1 + k) = lb + k;
                            }
                        }
                    }
                    itmp = itmp + 1;
                }
            }
        }
        for (int ista = 1; ista <= r_n; ++ista)
            if (istazone(ista) == 0) throw std::runtime_error("PSV: receiver outside the grid");
        // calsp (src/SGTpsv/others.f90:455-522)
        I1 isp(nzone), jsp(nzone), ksp(nzone), issp(nzone), ilsp(nzone), lsp(nzone), jssp(nzone);
        isp(1) = jsp(1) = ksp(1) = issp(1) = ilsp(1) = lsp(1) = jssp(1) = 1;
        {
            int isl = 0, ill = 0;
            for (int i = 1; i <= ndc; ++i) {
                isp(i + 1) = isp(i) + nlayer(i);
                if (iphase(i) == 1) {
                    jsp(i + 1) = jsp(i) + 16 * nlayer(i);
                    ksp(i + 1) = ksp(i) + 2 * (nlayer(i) + 1);
                    lsp(i + 1) = lsp(i) + 4 * nlayer(i);
                    isl++;
                    if (isl != nsl) {
                        issp(isl + 1) = issp(isl) + 4 * nlayer(i);
                        jssp(isl + 1) = jssp(isl) + nlayer(i) + 1;
                    }
                } else {
                    jsp(i + 1) = jsp(i) + 4 * nlayer(i);
                    ksp(i + 1) = ksp(i) + (nlayer(i) + 1);
                    lsp(i + 1) = lsp(i) + 2 * nlayer(i);
                    ill++;
                    if (ill != nll) ilsp(ill + 1) = ilsp(ill) + 4 * nlayer(i);
                }
            }
        }
        int isdr = issp(nsl) - 1 + 4 * nlayer(ndc + 1);
        int jsdr = jssp(nsl) - 1 + nlayer(ndc + 1) + 1;
        int ildr = 4 * nllay;
        // calspo (src/SGTpsv/others.f90:527-584)
        double spo;
        int spn;
        if (r0 == rmax) {
            spo = (double)inlayer - 0.01;
            r0 = ra(inlayer) + (spo - (double)(inlayer - 1)) * (ra(inlayer + 1) - ra(inlayer));
        } else {
            int itmp = 2;
            while (!(r0 < ra(itmp))) {
                itmp++;
                if (itmp > nnlayer + 1) throw std::runtime_error("calspo: source above grid");
            }
            spo = (double)(itmp - 2) + (r0 - ra(itmp - 1)) / (ra(itmp) - ra(itmp - 1));
            if ((spo - (double)(itmp - 2)) < 0.01) {
                spo = (double)(itmp - 2) + 0.01;
                r0 = ra(itmp - 1) + (spo - (double)(itmp - 2)) * (ra(itmp) - ra(itmp - 1));
            }
            if ((spo - (double)(itmp - 2)) > 0.99) {
                spo = (double)(itmp - 2) + 0.99;
                r0 = ra(itmp - 1) + (spo - (double)(itmp - 2)) * (ra(itmp) - ra(itmp - 1));
            }
        }
        spn = 0;
        {
            int itmp = 1;
            for (;;) {
                if (itmp > nzone) throw std::runtime_error("calspo: zone search failed");
                if (iphase(itmp) == 1) {
                    spn++;
                    if (r0 <= md.vrmax(itmp)) break;
                    itmp++;
                } else {
                    spn++;
                    if (r0 <= md.vrmax(itmp))
                        throw std::runtime_error("The source is in the liquid layer.(calspo)");
                    itmp++;
                }
            }
        }
        spo = spo - (double)(isp(spn) - 1);
        // calstg (src/SGTpsv/others.f90:590-682); caltstg recomputes the same
        // point values (:767-831), so one evaluation serves both.
        int nvra = nnlayer + 2 * nzone + 1;
        V1 vra(nvra), rho(nvra), kappa(nvra), ecKx(nvra), ecKy(nvra), ecKz(nvra), ecL(nvra),
            ecN(nvra);
        int vnp;
        {
            int itmp = 0, jtmp = 0;
            for (int iz = 1; iz <= nzone; ++iz) {
                for (int i = 1; i <= nlayer(iz) + 1; ++i) {
                    itmp++; jtmp++;
                    vra(itmp) = ra(jtmp);
                    double trho = 0, tvpv = 0, tvph = 0, tvsv = 0, tvsh = 0, teta = 0, coef = 1.0;
                    for (int j = 1; j <= 4; ++j) {
                        if (j == 1) coef = 1.0;
                        else coef = coef * (vra(itmp) / rmax);
                        trho = trho + md.rho[j](iz) * coef;
                        tvpv = tvpv + md.vpv[j](iz) * coef;
                        tvph = tvph + md.vph[j](iz) * coef;
                        tvsv = tvsv + md.vsv[j](iz) * coef;
                        tvsh = tvsh + md.vsh[j](iz) * coef;
                        teta = teta + md.eta[j](iz) * coef;
                    }
                    rho(itmp) = trho;
                    ecL(itmp) = rho(itmp) * tvsv * tvsv;
                    ecN(itmp) = rho(itmp) * tvsh * tvsh;
                    double ecA = trho * tvph * tvph;
                    double ecC = trho * tvpv * tvpv;
                    double ecF = teta * (ecA - 2.0 * ecL(itmp));
                    kappa(itmp) = (4.0 * ecA + ecC + 4.0 * ecF - 4.0 * ecN(itmp)) / 9.0;
                    ecKx(itmp) = ecA - 4.0 / 3.0 * ecN(itmp);
                    ecKy(itmp) = ecF + 2.0 / 3.0 * ecN(itmp);
                    ecKz(itmp) = (ecC + 2.0 * ecF) / 3.0;
                }
                jtmp = jtmp - 1;
            }
            vnp = itmp;
        }
        double ecC0, ecF0, ecL0;
        {
            double trho = 0, tvpv = 0, tvph = 0, tvsv = 0, tvsh = 0, teta = 0, coef = 1.0;
            for (int j = 1; j <= 4; ++j) {
                if (j == 1) coef = 1.0;
                else coef = coef * (r0 / rmax);
                trho = trho + md.rho[j](spn) * coef;
                tvpv = tvpv + md.vpv[j](spn) * coef;
                tvph = tvph + md.vph[j](spn) * coef;
                tvsv = tvsv + md.vsv[j](spn) * coef;
                tvsh = tvsh + md.vsh[j](spn) * coef;
                teta = teta + md.eta[j](spn) * coef;
            }
            ecL0 = trho * tvsv * tvsv;
            double ecA0 = trho * tvph * tvph;
            ecC0 = trho * tvpv * tvpv;
            ecF0 = teta * (ecA0 - 2.0 * ecL0);
        }
        // calinv (src/SGTpsv/others.f90:835-847)
        V1 rhoinv(nvra), kappainv(nvra);
        for (int i = 1; i <= vnp; ++i) {
            rhoinv(i) = 1.0 / rho(i);
            kappainv(i) = 1.0 / kappa(i);
        }
        // element integrals (src/SGTpsv/SGTpsv-MPI.f90:385-477)
        int n_sel = 8 * nslay, n_fel = 8 * (nllay > 0 ? nllay : 1), n_hm = 2 * (nslay + nzone);
        const bool on_host = device < 0;
        std::vector<V1> S(on_host ? 31 : 0, V1(n_sel));  // every solid array of the reference
        enum { T, H1X, H1Y, H1Z, H2L, H2N, H3AX, H3AY, H3AZ, H4AL, H4AN, H5AX, H5AY, H5AZ, H6AL,
               H6AN, H3X, H3Y, H3Z, H4L, H4N, H5X, H5Y, H5Z, H6L, H6N, H7X, H7Y, H7Z, H8L, H8N };
        V1 p1(on_host ? n_fel : 0), p2(on_host ? n_fel : 0), p3(on_host ? n_fel : 0);
        V1 work(on_host ? (n_sel > n_fel ? n_sel : n_fel) : 0);
        std::vector<std::vector<double>> hmst(on_host ? 14 : 0, std::vector<double>(4 * n_hm, 0.0));
        enum { M3X, M3Y, M3Z, M5X, M5Y, M5Z, M41L, M41N, M42L, M42N, M61L, M61N, M62L, M62N };
        const int hmlo[14] = {-2, -2, -2, -1, -1, -1, -1, -1, -2, -2, -1, -1, -2, -2};
        auto hmv = [&](int a, int col) {
            return HM{hmst[a].data() + 4 * (col - 1), hmlo[a]};
        };
        const double *pv = vra.v.data();
        auto rz_of = [&](int iz) { return ra.p(isp(iz)) - 1; };
        if (on_host) {
            int isl = 0, ill = 0;
            for (int i = 1; i <= ndc + 1; ++i) {
                const double *rz = rz_of(i);
                int nl = nlayer(i);
                if (iphase(i) == 1) {
                    isl++;
                    int o = isdr + issp(isl) - 1;
                    auto P = [&](int a) { return S[a].v.data() + o; };
                    double *w = work.v.data() + o;
                    calmatc(nl, vnp, pv, rho.v.data(), 2, 0, 0, rz, P(T), false);
                    caltl(nl, vnp, pv, rho.v.data(), rz, w);
                    calt(nl, P(T), w, P(T));
                    const double *cons[5] = {ecKx.v.data(), ecKy.v.data(), ecKz.v.data(),
                                             ecL.v.data(), ecN.v.data()};
                    int h1s[5] = {H1X, H1Y, H1Z, H2L, H2N};
                    for (int k = 0; k < 5; ++k) {
                        calmatc(nl, vnp, pv, cons[k], 0, 0, 0, rz, P(h1s[k]), false);
                        calhl(nl, vnp, pv, cons[k], rz, w);
                        calt(nl, P(h1s[k]), w, P(h1s[k]));
                    }
                    int h5s[5] = {H5AX, H5AY, H5AZ, H6AL, H6AN};
                    int h3s[5] = {H3AX, H3AY, H3AZ, H4AL, H4AN};
                    for (int k = 0; k < 5; ++k) calmatc(nl, vnp, pv, cons[k], 1, 0, 1, rz, P(h5s[k]), false);
                    for (int k = 0; k < 5; ++k) mtrnp(nl, P(h5s[k]), P(h3s[k]));
                    int h7s[5] = {H7X, H7Y, H7Z, H8L, H8N};
                    for (int k = 0; k < 5; ++k) calmatc(nl, vnp, pv, cons[k], 2, 1, 1, rz, P(h7s[k]), false);
                } else {
                    ill++;
                    int o = ildr + ilsp(ill) - 1;
                    double *w = work.v.data() + o;
                    calmatc(nl, vnp, pv, rhoinv.v.data(), 2, 1, 1, rz, p1.v.data() + o, false);
                    calmatc(nl, vnp, pv, rhoinv.v.data(), 0, 0, 0, rz, p2.v.data() + o, false);
                    calhl(nl, vnp, pv, rhoinv.v.data(), rz, w);
                    calt(nl, p2.v.data() + o, w, p2.v.data() + o);
                    calmatc(nl, vnp, pv, kappainv.v.data(), 2, 0, 0, rz, p3.v.data() + o, false);
                    caltl(nl, vnp, pv, kappainv.v.data(), rz, w);
                    calt(nl, p3.v.data() + o, w, p3.v.data() + o);
                }
            }
            // modified first-derivative operator (:439-477); caltstg's values
            // equal calstg's for vra, ecKx, ecKy, ecKz, ecL, ecN.
            isl = 0;
            for (int i = 1; i <= ndc + 1; ++i) {
                if (iphase(i) != 1) continue;
                isl++;
                const double *rz = rz_of(i);
                int nl = nlayer(i);
                int o = isdr + issp(isl) - 1;
                auto P = [&](int a) { return S[a].v.data() + o; };
                double *w = work.v.data() + o;
                int jt = isp(i) + i - 1;
                const double *vz = vra.p(jt) - 1;
                const double *cons[5] = {ecKx.p(jt) - 1, ecKy.p(jt) - 1, ecKz.p(jt) - 1,
                                         ecL.p(jt) - 1, ecN.p(jt) - 1};
                int ha[5] = {H5AX, H5AY, H5AZ, H6AL, H6AN};
                int hb[5] = {H5X, H5Y, H5Z, H6L, H6N};
                int hc[5] = {H3X, H3Y, H3Z, H4L, H4N};
                for (int k = 0; k < 5; ++k) {
                    calh5(nl, vz, cons[k], rz, w);
                    for (int e = 1; e <= 4 * nl; ++e) P(hb[k])[e] = P(ha[k])[e] - w[e];
                }
                for (int k = 0; k < 5; ++k) mtrnp(nl, P(hb[k]), P(hc[k]));
                int col = jsdr + jssp(isl);
                calhm1(nl, vz, cons[0], rz, hmv(M5X, col));
                calhm1(nl, vz, cons[1], rz, hmv(M5Y, col));
                calhm1(nl, vz, cons[2], rz, hmv(M5Z, col));
                calhm1(nl, vz, cons[3], rz, hmv(M61L, col));
                calhm1(nl, vz, cons[4], rz, hmv(M61N, col));
                calhm2(nl, vz, cons[3], rz, hmv(M62L, col));
                calhm2(nl, vz, cons[4], rz, hmv(M62N, col));
                mtrnp2(nl, 1, 2, hmv(M5X, col), hmv(M3X, col));
                mtrnp2(nl, 1, 2, hmv(M5Y, col), hmv(M3Y, col));
                mtrnp2(nl, 1, 2, hmv(M5Z, col), hmv(M3Z, col));
                mtrnp2(nl, 1, 2, hmv(M61L, col), hmv(M42L, col));
                mtrnp2(nl, 1, 2, hmv(M61N, col), hmv(M42N, col));
                mtrnp2(nl, 2, 1, hmv(M62L, col), hmv(M41L, col));
                mtrnp2(nl, 2, 1, hmv(M62N, col), hmv(M41N, col));
            }
        }
        // calspdr (src/SGTpsv/others.f90:870-898) and the stack points of the
        // receivers (SGTpsv-MPI.f90:623-628)
        I1 kkdr(nzone);
        kkdr(1) = 1;
        for (int iz = 1; iz <= nzone - 1; ++iz) {
            if (iphase(iz) == 1) {
                kkdr(iz + 1) = kkdr(iz) + (iphase(iz + 1) == 1 ? 2 * nlayer(iz) : 2 * (nlayer(iz) + 1));
            } else {
                kkdr(iz + 1) = kkdr(iz) + (iphase(iz + 1) == 1 ? (nlayer(iz) + 1) : nlayer(iz));
            }
        }
        int nn = kkdr(nzone) + 2 * nlayer(nzone) + 1;
        // source indices (:557-558, :636-641)
        int ispo = (int)spo;  // Fortran int(): truncation
        int mtmp = isp(spn) + ispo;
        int jtmp = kkdr(spn) + 2 * ispo;
        if (spo == (double)ispo) { mtmp--; jtmp -= 2; }

        auto *b = new dsm_bundle;
        b->psv = true;
        b->n_nodes = nnlayer + 1;
        b->n_unknowns = nn;
        dsm_psv_setup_t &s = b->psvs;
        s.nzone = nzone;
        s.iphase = b->keep1i(iphase, nzone);
        s.nlayer = b->keep1i(nlayer, nzone);
        s.isp = b->keep1i(isp, nzone);
        s.kkdr = b->keep1i(kkdr, nzone);
        {
            std::vector<int> elem(nzone), hmoff(nzone);
            int isl = 0, ill = 0;
            for (int i = 1; i <= nzone; ++i) {
                if (iphase(i) == 1) {
                    isl++;
                    elem[i - 1] = isdr + issp(isl);
                    hmoff[i - 1] = jsdr + jssp(isl);
                } else {
                    ill++;
                    elem[i - 1] = ildr + ilsp(ill);
                    hmoff[i - 1] = 0;
                }
            }
            s.elem = b->keepi(elem);
            s.hmoff = b->keepi(hmoff);
        }
        s.vrmin = b->keep1(md.vrmin, nzone);
        s.vrmax = b->keep1(md.vrmax, nzone);
        s.qmu = b->keep1(md.qmu, nzone);
        s.qkappa = b->keep1(md.qkappa, nzone);
        {
            std::vector<double> v(4 * nzone);
            for (int i = 1; i <= nzone; ++i)
                for (int j = 1; j <= 4; ++j) v[4 * (i - 1) + (j - 1)] = md.vsv[j](i);
            s.vsv = b->keep(v);
        }
        s.nn = nn;
        s.rmin = rmin; s.rmax = rmax;
        s.n_sel = n_sel; s.n_fel = n_fel; s.n_hm = n_hm;
        {
          if (on_host) {
            const int order[DSM_PSV_NSOLID] = {T,    H1X,  H2L,  H2N, H3AY, H4AL, H4AN,
                                               H5AY, H6AL, H6AN, H7Y, H7Z,  H8L,  H8N,
                                               H3Y,  H4L,  H4N,  H5Y, H6L,  H6N};
            std::vector<double> el((size_t)DSM_PSV_NSOLID * n_sel);
            for (int k = 0; k < DSM_PSV_NSOLID; ++k)
                for (int e = 0; e < n_sel; ++e) el[(size_t)k * n_sel + e] = S[order[k]].v[e + 1];
            s.solid_el = b->keep(el);
            std::vector<double> fl((size_t)3 * n_fel);
            for (int e = 0; e < n_fel; ++e) {
                fl[e] = p1.v[e + 1];
                fl[(size_t)n_fel + e] = p2.v[e + 1];
                fl[(size_t)2 * n_fel + e] = p3.v[e + 1];
            }
            s.fluid_el = b->keep(fl);
            const int horder[DSM_PSV_NHM] = {M3Y, M5Y, M41L, M42N, M61N, M62L};
            std::vector<double> hm((size_t)DSM_PSV_NHM * 4 * n_hm);
            for (int k = 0; k < DSM_PSV_NHM; ++k)
                for (int e = 0; e < 4 * n_hm; ++e) hm[(size_t)k * 4 * n_hm + e] = hmst[horder[k]][e];
            s.hm_el = b->keep(hm);
          } else {
            std::vector<double> el((size_t)DSM_PSV_NSOLID * n_sel), fl((size_t)3 * n_fel),
                hm((size_t)DSM_PSV_NHM * 4 * n_hm);
            std::vector<double> cf[6];
            const std::vector<V1> *src[6] = {&md.rho, &md.vpv, &md.vph, &md.vsv, &md.vsh, &md.eta};
            for (int k = 0; k < 6; ++k) {
                cf[k].resize(4 * (size_t)nzone);
                for (int i = 1; i <= nzone; ++i)
                    for (int j = 1; j <= 4; ++j) cf[k][4 * (i - 1) + (j - 1)] = (*src[k])[j](i);
            }
            char err[256] = {0};
            const int rc = dsm_psv_integrals_device(
                device, nzone, s.iphase, s.nlayer, s.isp, s.elem, s.hmoff, ra.v.data() + 1, nnlayer + 1, rmax,
                cf[0].data(), cf[1].data(), cf[2].data(), cf[3].data(), cf[4].data(), cf[5].data(), n_sel, n_fel,
                n_hm, el.data(), fl.data(), hm.data(), err, (int)sizeof(err));
            if (rc != DSM_OK) {
                delete b;
                throw std::runtime_error(std::string("element integrals on the device: ") + err);
            }
            s.solid_el = b->keep(el);
            s.fluid_el = b->keep(fl);
            s.hm_el = b->keep(hm);
          }
        }
        s.spn = spn; s.spo = spo; s.r0 = r0;
        s.ecC0 = ecC0; s.ecF0 = ecF0; s.ecL0 = ecL0;
        s.ra_src[0] = ra(mtmp); s.ra_src[1] = ra(mtmp + 1);
        for (int j = 1; j <= 4; ++j) {
            s.src_poly[0 + j - 1] = md.rho[j](spn);
            s.src_poly[4 + j - 1] = md.vpv[j](spn);
            s.src_poly[8 + j - 1] = md.vph[j](spn);
            s.src_poly[12 + j - 1] = md.vsv[j](spn);
            s.src_poly[16 + j - 1] = md.vsh[j](spn);
            s.src_poly[20 + j - 1] = md.eta[j](spn);
        }
        s.jsrc = jtmp;
        s.r_n = r_n;
        s.r = b->keep1(r_, r_n);
        s.rrsta = b->keep1(rrsta, 3 * r_n);
        s.iista = b->keep1i(iista, 3 * r_n);
        s.istazone = b->keep1i(istazone, r_n);
        s.lambda = b->keep1(lambda, r_n);
        s.qkp = b->keep1(qkp, r_n);
        s.theta_n = theta_n;
        s.theta = b->keep(theta);
        s.tlen = tlen; s.omegai = omegai; s.ratl = conf.ratl; s.maxlmax = conf.maxlmax;
        s.imin = par->imin; s.imax = par->imax;
        s.rsgt_switch = par->rsgt_switch; s.tsgt_switch = par->tsgt_switch;
        s.synn_switch = par->synn_switch;
        *bundle_out = b;
        *setup_out = &b->psvs;
        return DSM_OK;
    } catch (const std::exception &e) {
        g_err = std::string("dsm_psv_setup_build: ") + e.what();
        return DSM_ERR_INVALID;
    }
}
}  // namespace

extern "C" int dsm_psv_setup_build(const dsm_params_t *par, const char *conf_text, const char *model_text,
                                   dsm_bundle_t **bundle_out, const dsm_psv_setup_t **setup_out) {
    return psv_setup_build(par, conf_text, model_text, -1, bundle_out, setup_out);
}

extern "C" int dsm_psv_setup_build_device(const dsm_params_t *par, const char *conf_text, const char *model_text,
                                          int device, dsm_bundle_t **bundle_out,
                                          const dsm_psv_setup_t **setup_out) {
    if (device < 0) {
        g_err = "dsm_psv_setup_build_device: negative device ordinal";
        return DSM_ERR_INVALID;
    }
    return psv_setup_build(par, conf_text, model_text, device, bundle_out, setup_out);
}
