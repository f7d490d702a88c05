// sgtpsv / sgtsh: drop-in drivers of the SGT engine.
//
// Same inputs and outputs as the reference programs SGTpsv and SGTsh
// (src/SGTpsv/SGTpsv-MPI.f90, src/SGTsh/SGTsh-MPI.f90):
//   * the parameter file on stdin (pinput), DSM.config and the polynomial
//     model named in it;
//   * catalogue records, one file per (source, receiver, frequency):
//       <outdir>/TSGT/<model>.<r0>.<r>.<i>.TSGT_PSV|SH   (num_tsgt x theta complex64)
//       <outdir>/RSGT/<model>.<r>.<i>.RSGT_PSV|SH        (num_rsgt x theta)
//       <outdir>/RSGT/<model>.<r0>.<i>.SYNN_PSV|SH       (num_synn x theta)
//     integers written as I7 with leading blanks turned into '0' and radii
//     in metres truncated (SGTpsv-MPI.f90:1103-1150); a record is the raw
//     array, component fastest (direct access, no record markers);
//   * logs <outdir>/log/calLog[SH].<model>.<imin>.<imax> (start / finish
//     times) and <outdir>/log/list[SH].<model>.<imin>.<imax>.<rank> (one
//     line "i  i/tlen  llog-1" per frequency, :1097-1099).
// Frequencies i in [imin, imax], i != 0, owned by this process under the
// reference's zig-zag rule (:550) for --rank/--nproc (default 0/1): run one
// process per GPU to share a frequency range.
//
// Usage: sgtpsv|sgtsh [--precision fp64|mixed|mixed_bf16] [--device N]
//                     [--rank p --nproc n] [--batch F] < parameter_file
#include <sys/stat.h>

#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "dsmsgt.h"
#include "dsmsgt_host.h"

namespace {

std::string slurp(std::istream& in) {
    std::ostringstream ss;
    ss << in.rdbuf();
    return ss.str();
}

std::string read_file(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open " + path);
    return slurp(f);
}

std::string trim(const char* s) {
    std::string t(s);
    size_t a = t.find_first_not_of(" \t\r\n"), b = t.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? std::string() : t.substr(a, b - a + 1);
}

// Fortran I7: right-justified in 7 characters, '*******' when it does not fit
std::string i7(long long v) {
    char b[32];
    std::snprintf(b, sizeof b, "%7lld", v);
    std::string s(b);
    return s.size() > 7 ? std::string(7, '*') : s;
}

// blanks of the first n characters become '0' (the reference's name loop)
std::string zero_fill(std::string s, size_t n) {
    for (size_t j = 0; j < n && j < s.size(); ++j)
        if (s[j] == ' ') s[j] = '0';
    return s;
}

long long fint(double x) { return (long long)x; }  // Fortran int(): toward zero

void mkdirs(const std::string& p) {
    if (p.empty()) return;
    std::string cur;
    std::stringstream ss(p);
    std::string part;
    if (p[0] == '/') cur = "/";
    while (std::getline(ss, part, '/')) {
        if (part.empty()) continue;
        cur += part + "/";
        if (mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST)
            throw std::runtime_error("cannot create directory " + cur);
    }
}

void write_record(const std::string& path, const float* data, size_t count) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write " + path);
    size_t w = std::fwrite(data, sizeof(float), count, f);
    std::fclose(f);
    if (w != count) throw std::runtime_error("short write to " + path);
}

std::string stamp(const char* what) {
    std::time_t t = std::time(nullptr);
    std::tm tm{};
    localtime_r(&t, &tm);
    char b[160];
    std::snprintf(b, sizeof b, "\n%s%04d-%02d-%02d.  %02d:%02d:%02d.%03d\n", what, tm.tm_year + 1900,
                  tm.tm_mon + 1, tm.tm_mday, tm.tm_hour, tm.tm_min, tm.tm_sec, 0);
    return b;
}

void append(const std::string& path, const std::string& text, bool truncate = false) {
    FILE* f = std::fopen(path.c_str(), truncate ? "w" : "a");
    if (!f) throw std::runtime_error("cannot write " + path);
    std::fputs(text.c_str(), f);
    std::fclose(f);
}

bool owns(int i, int imax, int rank, int nproc) {
    if (i == 0) return false;
    const int m = 2 * nproc;
    return ((imax - rank - i) % m == 0) || ((imax + rank + 1 - i) % m == 0);
}

int die(const std::string& msg) {
    std::fprintf(stderr, "%s\n", msg.c_str());
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    std::string prog = argv[0];
    prog = prog.substr(prog.find_last_of('/') + 1);
    bool psv = prog.find("sh") == std::string::npos || prog.find("psv") != std::string::npos;
    dsm_options_t opt{};
    opt.precision = DSM_PREC_FP64;
    int rank = 0, nproc = 1;
    for (int a = 1; a < argc; ++a) {
        std::string k = argv[a];
        auto val = [&]() -> std::string {
            if (a + 1 >= argc) throw std::runtime_error("missing value after " + k);
            return argv[++a];
        };
        try {
            if (k == "--precision") {
                std::string v = val();
                opt.precision = v == "fp64" ? DSM_PREC_FP64
                                : v == "mixed" ? DSM_PREC_MIXED
                                : v == "mixed_bf16" ? DSM_PREC_MIXED_BF16 : -1;
                if (opt.precision < 0) return die("unknown precision " + v);
            } else if (k == "--device") opt.device = std::atoi(val().c_str());
            else if (k == "--rank") rank = std::atoi(val().c_str());
            else if (k == "--nproc") nproc = std::atoi(val().c_str());
            else if (k == "--batch") opt.freq_batch = std::atoi(val().c_str());
            else if (k == "--psv") psv = true;
            else if (k == "--sh") psv = false;
            else return die("usage: " + prog + " [--precision fp64|mixed|mixed_bf16] [--device N] "
                                                "[--rank p --nproc n] [--batch F] < parameter_file");
        } catch (const std::exception& e) {
            return die(e.what());
        }
    }
    if (nproc < 1 || rank < 0 || rank >= nproc) return die("bad --rank/--nproc");

    try {
        const std::string ptext = slurp(std::cin);
        dsm_params_t par{};
        if (dsm_parse_params(ptext.c_str(), &par)) throw std::runtime_error(dsm_host_last_error());
        const std::string conf = read_file(trim(par.dsmconf));
        const std::string model = read_file(trim(par.model));
        const std::string outdir = trim(par.outdir), mname = trim(par.modelname);

        dsm_bundle_t* bundle = nullptr;
        dsm_ctx_t* ctx = nullptr;
        int r_n = 0, theta_n = 0, nt, nr, ns;
        const double* rr = nullptr;
        double tlen = par.tlen;
        int rc;
        if (psv) {
            const dsm_psv_setup_t* s = nullptr;
            if (dsm_psv_setup_build(&par, conf.c_str(), model.c_str(), &bundle, &s))
                throw std::runtime_error(dsm_host_last_error());
            r_n = s->r_n; theta_n = s->theta_n; rr = s->r;
            nt = DSM_PSV_NUM_TSGT; nr = DSM_PSV_NUM_RSGT; ns = DSM_PSV_NUM_SYNN;
            rc = dsm_psv_create(s, &opt, &ctx);
        } else {
            const dsm_sh_setup_t* s = nullptr;
            if (dsm_sh_setup_build(&par, conf.c_str(), model.c_str(), &bundle, &s))
                throw std::runtime_error(dsm_host_last_error());
            r_n = s->r_n; theta_n = s->theta_n; rr = s->r;
            nt = DSM_SH_NUM_TSGT; nr = DSM_SH_NUM_RSGT; ns = DSM_SH_NUM_SYNN;
            rc = dsm_sh_create(s, &opt, &ctx);
        }
        if (rc) throw std::runtime_error(std::string("context: ") + dsm_last_error(nullptr));

        const std::string tag = psv ? "PSV" : "SH", lsuffix = psv ? "" : "SH";
        mkdirs(outdir + "/log");
        mkdirs(outdir + "/TSGT");
        mkdirs(outdir + "/RSGT");
        const std::string range = zero_fill(i7(par.imin) + "." + i7(par.imax), 15);
        const std::string callog = outdir + "/log/calLog" + lsuffix + "." + mname + "." + range;
        const std::string list = outdir + "/log/list" + lsuffix + "." + mname + "." +
                                 zero_fill(i7(par.imin) + "." + i7(par.imax) + "." + i7(rank), 22);
        if (rank == 0) append(callog, stamp("    Starting date and time:                     "), true);
        append(list, "\n", true);
        if (rank == 0) append(callog, stamp("    here we go!:                     "));

        std::vector<int> mine;
        for (int i = par.imin; i <= par.imax; ++i)
            if (owns(i, par.imax, rank, nproc)) mine.push_back(i);
        const long long ir0 = fint(par.r0min * 1e3);
        const size_t pt = (size_t)nt * theta_n, pr = (size_t)nr * theta_n, ps = (size_t)ns * theta_n;
        const int B = 16;  // frequencies per library call
        std::vector<float> t32, r32, s32;
        std::vector<int> llog;
        for (size_t b0 = 0; b0 < mine.size(); b0 += B) {
            const int n = (int)std::min<size_t>(B, mine.size() - b0);
            t32.assign(2 * pt * r_n * n, 0.0f);
            r32.assign(2 * pr * r_n * n, 0.0f);
            s32.assign(2 * ps * n, 0.0f);
            llog.assign(n, 0);
            dsm_out_t out{};
            out.tsgt32 = t32.data();
            out.rsgt32 = par.rsgt_switch ? r32.data() : nullptr;
            out.synn32 = par.synn_switch ? s32.data() : nullptr;
            out.llog = llog.data();
            if (dsm_run_freqs(ctx, mine.data() + b0, n, &out))
                throw std::runtime_error(std::string("frequencies: ") + dsm_last_error(ctx));
            for (int k = 0; k < n; ++k) {
                const int i = mine[b0 + k];
                char line[128];
                std::snprintf(line, sizeof line, "%12d %24.16E %12d\n", i, (double)i / tlen, llog[k] - 1);
                append(list, line);
                for (int ir = 0; ir < r_n; ++ir) {
                    const long long irr = fint(rr[ir] * 1e3);
                    std::string f = zero_fill(i7(ir0) + "." + i7(irr) + "." + i7(i) + ".TSGT_" + tag, 29);
                    write_record(outdir + "/TSGT/" + mname + "." + f,
                                 t32.data() + 2 * pt * ((size_t)k * r_n + ir), 2 * pt);
                    if (par.rsgt_switch) {
                        std::string g = zero_fill(i7(irr) + "." + i7(i) + ".RSGT_" + tag, 21);
                        write_record(outdir + "/RSGT/" + mname + "." + g,
                                     r32.data() + 2 * pr * ((size_t)k * r_n + ir), 2 * pr);
                    }
                }
                if (par.synn_switch) {
                    std::string g = zero_fill(i7(ir0) + "." + i7(i) + ".SYNN_" + tag, 21);
                    write_record(outdir + "/RSGT/" + mname + "." + g, s32.data() + 2 * ps * k, 2 * ps);
                }
            }
        }
        dsm_ctx_destroy(ctx);
        dsm_bundle_free(bundle);
        if (rank == 0) append(callog, stamp("    Finishing date and time:                     "));
    } catch (const std::exception& e) {
        return die(prog + ": " + e.what());
    }
    return 0;
}
