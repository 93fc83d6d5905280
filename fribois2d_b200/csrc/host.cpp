// Host-side set-up: deck parsing, grid metrics, coefficients, Poisson eigen
// data, DGTTRF factors, marker initialisation.  Compiled without FP
// contraction so that every coefficient is bit-identical to the reference's
// left-to-right evaluation.
#include "host.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace fb {

// ---------------------------------------------------------------- parsing

namespace {

// Sequential records with Fortran list-directed semantics: values are
// separated by blanks and/or commas, a record is consumed per read
// statement, a read that needs more values continues on the next record,
// and '/' ends the input list.
class Records {
  public:
    explicit Records(const std::string &path) {
        std::ifstream f(path, std::ios::binary);
        ok_ = static_cast<bool>(f);
        if (!ok_) return;
        std::stringstream ss;
        ss << f.rdbuf();
        std::string all = ss.str();
        size_t s = 0;
        for (;;) {
            size_t e = all.find('\n', s);
            if (e == std::string::npos) {
                lines_.push_back(all.substr(s));
                break;
            }
            lines_.push_back(all.substr(s, e - s));
            s = e + 1;
        }
        newlines_ = std::count(all.begin(), all.end(), '\n');
    }
    bool ok() const { return ok_; }
    long newlines() const { return newlines_; }
    void skip() { ++pos_; }
    bool read(size_t n, std::vector<std::string> &out) {
        out.clear();
        while (out.size() < n) {
            if (pos_ >= lines_.size()) return false;
            const std::string &line = lines_[pos_++];
            std::string tok;
            bool stop = false;
            auto flush = [&]() {
                if (!tok.empty() && out.size() < n) out.push_back(tok);
                tok.clear();
            };
            for (char c : line) {
                if (c == ',' || c == ' ' || c == '\t' || c == '\r') {
                    flush();
                } else if (c == '/' && tok.empty()) {
                    stop = true;
                    break;
                } else {
                    tok.push_back(c);
                }
                if (out.size() == n) break;
            }
            flush();
            if (stop && out.size() < n) return false;
        }
        return true;
    }

  private:
    std::vector<std::string> lines_;
    size_t pos_ = 0;
    bool ok_ = false;
    long newlines_ = 0;
};

bool to_real(const std::string &t, double &v) {
    std::string s = t;
    for (auto &c : s)
        if (c == 'd' || c == 'D') c = 'e';
    char *end = nullptr;
    v = std::strtod(s.c_str(), &end);
    return end && *end == '\0' && !s.empty();
}
bool to_int(const std::string &t, int &v) {
    char *end = nullptr;
    long x = std::strtol(t.c_str(), &end, 10);
    v = static_cast<int>(x);
    return end && *end == '\0' && !t.empty();
}
bool to_logical(const std::string &t, bool &v) {
    size_t i = 0;
    if (i < t.size() && t[i] == '.') ++i;
    if (i >= t.size()) return false;
    char c = static_cast<char>(std::toupper(static_cast<unsigned char>(t[i])));
    if (c == 'T') return v = true, true;
    if (c == 'F') return v = false, true;
    return false;
}

struct Reader {
    Records r;
    std::string err;
    std::vector<std::string> tok;
    explicit Reader(const std::string &p) : r(p) {
        if (!r.ok()) err = "cannot open " + p;
    }
    void skip(int n = 1) {
        for (int i = 0; i < n; ++i) r.skip();
    }
    void reals(double *v, int n, const char *what) {
        if (!err.empty()) return;
        if (!r.read(static_cast<size_t>(n), tok)) {
            err = std::string("end of input reading ") + what;
            return;
        }
        for (int i = 0; i < n; ++i)
            if (!to_real(tok[i], v[i])) err = std::string("bad real for ") + what + ": " + tok[i];
    }
    void ints(int *v, int n, const char *what) {
        if (!err.empty()) return;
        if (!r.read(static_cast<size_t>(n), tok)) {
            err = std::string("end of input reading ") + what;
            return;
        }
        for (int i = 0; i < n; ++i)
            if (!to_int(tok[i], v[i])) err = std::string("bad integer for ") + what + ": " + tok[i];
    }
    void logical(bool &v, const char *what) {
        if (!err.empty()) return;
        if (!r.read(1, tok) || !to_logical(tok[0], v)) err = std::string("bad logical for ") + what;
    }
    void word(std::string &v, const char *what) {
        if (!err.empty()) return;
        if (!r.read(1, tok)) err = std::string("end of input reading ") + what;
        else v = tok[0];
    }
};

}  // namespace

std::string read_deck(const std::string &dir, Deck &d) {
    double dummy[5];
    {   // utils_proc.F90:59-83
        Reader g(dir + "/global_par.in");
        g.skip();
        g.reals(&d.dt, 1, "dt");
        g.logical(d.idtv, "idtv");
        g.reals(&d.dtmax, 1, "dtmax");
        g.reals(&d.cflmax, 1, "cflmax");
        g.reals(&d.cfllim, 1, "cfllim");
        g.word(d.outfol, "outfol");
        g.logical(d.irest, "irest");
        g.reals(&d.trestart, 1, "trestart");
        g.skip(3);
        g.logical(d.ibact, "ibact");
        g.skip(3);
        g.reals(&d.kprobe, 1, "kprobe");
        g.logical(d.prlgr, "prlgr");
        g.reals(&d.tprtag, 1, "tprtag");
        g.ints(&d.forst, 1, "forst");
        g.reals(&d.radiusSD, 1, "radiusSD");
        g.ints(&d.wfun, 1, "wfun");
        if (!g.err.empty()) return "global_par.in: " + g.err;
    }
    {   // utils_proc.F90:142-170
        Reader f(dir + "/fluid_par.in");
        int nn[2];
        f.skip();
        f.reals(&d.alx3, 1, "alx3");
        f.reals(&d.rext2, 1, "rext2");
        f.ints(nn, 2, "n3, n2");
        d.n3 = nn[0];
        d.n2 = nn[1];
        f.ints(&d.istr3, 1, "istr3");
        f.reals(dummy, 5, "str3u..n3strp");
        f.reals(dummy, 2, "int3");
        f.ints(&d.istr2, 1, "istr2");
        f.reals(dummy, 5, "str2u..n2strp");
        f.reals(dummy, 2, "int2");
        f.skip(3);
        f.ints(&d.nsst, 1, "nsst");
        f.logical(d.nwrit, "nwrit");
        f.reals(&d.tframef, 1, "tframef");
        f.reals(&d.resid, 1, "resid");
        f.reals(&d.cou, 1, "cou");
        f.skip(3);
        f.reals(&d.visc, 1, "visc");
        f.logical(d.inslws, "inslws");
        f.logical(d.inslwn, "inslwn");
        f.reals(&d.q3uw, 1, "q3uw");
        f.reals(&d.q3lw, 1, "q3lw");
        if (!f.err.empty()) return "fluid_par.in: " + f.err;
        // utils_proc.F90:174-190
        if (d.nsst != 1 && d.nsst != 3) return "fluid_par.in: nsst must be 1 or 3";
        if (d.istr2 != 100 || d.istr3 != 100)
            return "fluid_par.in: only grids read from ycoord.dat/zcoord.dat (istr = 100) are supported";
        if (d.n2 < 4 || d.n3 < 4) return "fluid_par.in: grid too small";
    }
    {   // utils_proc.F90:18-36; ipert is read into a scalar dummy (line 12)
        Reader r(dir + "/rigid_par.in");
        int ib;
        r.skip();
        r.logical(d.cbody, "cbody");
        r.reals(d.cmposi, 2, "cmposi");
        r.reals(&d.cmroti, 1, "cmroti");
        r.reals(d.ipert, 1, "ipert");
        d.ipert[1] = d.ipert[2] = 0.0;
        r.reals(d.rbgravF, 2, "rbgravF");
        r.reals(&d.rbden, 1, "rbden");
        r.reals(d.rba, 2, "rba");
        r.ints(d.rbmcon, 3, "rbmcon");
        r.reals(d.kk, 3, "kk");
        r.reals(d.kk3, 3, "kk3");
        r.reals(d.cc, 3, "cc");
        r.logical(d.rtcoup, "rtcoup");
        r.reals(&d.rrr, 1, "rrr");
        (void)ib;
        if (!r.err.empty()) {
            if (d.ibact) return "rigid_par.in: " + r.err;
        }
    }
    {   // cordin.F90:243-278
        Reader y(dir + "/ycoord.dat"), z(dir + "/zcoord.dat");
        d.ycoord.assign(static_cast<size_t>(d.n2), 0.0);
        d.zcoord.assign(static_cast<size_t>(d.n3), 0.0);
        for (int i = 0; i < d.n2; ++i) y.reals(&d.ycoord[i], 1, "ycoord");
        for (int i = 0; i < d.n3; ++i) z.reals(&d.zcoord[i], 1, "zcoord");
        if (!y.err.empty()) return "ycoord.dat: " + y.err;
        if (!z.err.empty()) return "zcoord.dat: " + z.err;
        for (int i = 1; i < d.n2; ++i)
            if (!(d.ycoord[i] > d.ycoord[i - 1])) return "ycoord.dat: coordinates not increasing";
        for (int i = 1; i < d.n3; ++i)
            if (!(d.zcoord[i] > d.zcoord[i - 1])) return "zcoord.dat: coordinates not increasing";
    }
    d.nlm = 0;
    d.vert.clear();
    if (d.ibact) {   // utils_proc.F90:529-548: markers = newline count - 1
        Reader m(dir + "/lmdata.in");
        if (!m.err.empty()) return "lmdata.in: " + m.err;
        d.nlm = static_cast<int>(m.r.newlines()) - 1;
        if (d.nlm < 3) return "lmdata.in: fewer than 3 markers";
        d.vert.assign(static_cast<size_t>(d.nlm + 1) * 2, 0.0);
        for (int i = 0; i <= d.nlm; ++i) m.reals(&d.vert[2 * i], 2, "vertex");
        if (!m.err.empty()) return "lmdata.in: " + m.err;
    }
    return "";
}

// ---------------------------------------------------------------- DGTTRF

int dgttrf(int n, double *dl, double *d, double *du, double *du2, int *ipiv) {
    if (n <= 0) return 0;
    for (int i = 0; i < n; ++i) ipiv[i] = i + 1;
    for (int i = 0; i < n - 2; ++i) du2[i] = 0.0;
    auto step = [&](int i, bool last) {
        if (std::fabs(d[i]) >= std::fabs(dl[i])) {
            if (d[i] != 0.0) {
                double fact = dl[i] / d[i];
                dl[i] = fact;
                d[i + 1] = d[i + 1] - fact * du[i];
            }
        } else {
            double fact = d[i] / dl[i];
            d[i] = dl[i];
            dl[i] = fact;
            double temp = du[i];
            du[i] = d[i + 1];
            d[i + 1] = temp - fact * d[i + 1];
            if (!last) {
                du2[i] = du[i + 1];
                du[i + 1] = -fact * du[i + 1];
            }
            ipiv[i] = i + 2;
        }
    };
    for (int i = 0; i < n - 2; ++i) step(i, false);
    if (n > 1) step(n - 2, true);
    for (int i = 0; i < n; ++i)
        if (d[i] == 0.0) return i + 1;
    return 0;
}

TriLU factor(const std::vector<double> &lower, const std::vector<double> &diag,
             const std::vector<double> &upper) {
    TriLU f;
    f.n = static_cast<int>(diag.size());
    f.dl = lower;
    f.d = diag;
    f.du = upper;
    f.du2.assign(static_cast<size_t>(std::max(f.n - 2, 1)), 0.0);
    f.ipiv.assign(static_cast<size_t>(f.n), 0);
    f.dl.resize(static_cast<size_t>(std::max(f.n - 1, 1)));
    f.du.resize(static_cast<size_t>(std::max(f.n - 1, 1)));
    f.info = dgttrf(f.n, f.dl.data(), f.d.data(), f.du.data(), f.du2.data(), f.ipiv.data());
    for (int i = 0; i < f.n; ++i)
        if (f.ipiv[i] != i + 1) f.pivoted = true;
    return f;
}

// ---------------------------------------------------------------- grid

void build_grid(const Deck &d, Grid &g) {
    const int n2 = d.n2, n3 = d.n3, n2m = n2 - 1, n3m = n3 - 1;
    g.n2 = n2;
    g.n3 = n3;
    g.n2m = n2m;
    g.n3m = n3m;
    // fluid_pre.F90:145-152
    g.dx2 = 1.0 / (d.rext2 / static_cast<double>(n2m));
    g.dx3 = 1.0 / (d.alx3 / static_cast<double>(n3m));
    g.dx2q = g.dx2 * g.dx2;
    g.dx3q = g.dx3 * g.dx3;
    g.ren = 1.0 / d.visc;
    auto R = [](std::vector<double> &v, int n) { v.assign(static_cast<size_t>(n) + 2, 0.0); };
    auto I = [](std::vector<int> &v, int n) { v.assign(static_cast<size_t>(n) + 2, 0); };
    R(g.rc, n2); R(g.rm, n2); R(g.zz, n3); R(g.zm, n3);
    R(g.g2rc, n2); R(g.g2rm, n2); R(g.g3rc, n3); R(g.g3rm, n3);
    R(g.udx2c, n2); R(g.udx2m, n2); R(g.udx3c, n3); R(g.udx3m, n3);
    I(g.jmv, n2); I(g.jpv, n2); I(g.jmc, n2); I(g.jpc, n2);
    I(g.kmv, n3); I(g.kpv, n3); I(g.kmc, n3); I(g.kpc, n3);
    R(g.am2j, n2); R(g.ac2j, n2); R(g.ap2j, n2); R(g.am3j, n2); R(g.ac3j, n2); R(g.ap3j, n2);
    R(g.am3ck, n3); R(g.ac3ck, n3); R(g.ap3ck, n3); R(g.am3sk, n3); R(g.ac3sk, n3); R(g.ap3sk, n3);
    R(g.amphj, n2); R(g.acphj, n2); R(g.apphj, n2); R(g.amphk, n3); R(g.acphk, n3); R(g.apphk, n3);

    // indic.F90:276-303
    for (int kc = 1; kc <= n3m; ++kc) {
        g.kmv[kc] = kc - 1;
        g.kpv[kc] = kc + 1;
        if (kc == 1) g.kmv[kc] = kc;
        if (kc == n3m) g.kpv[kc] = kc;
    }
    for (int kc = 1; kc <= n3m; ++kc) {
        g.kpc[kc] = g.kpv[kc] - kc;
        g.kmc[kc] = kc - g.kmv[kc];
    }
    for (int jc = 1; jc <= n2; ++jc) {
        g.jmv[jc] = jc - 1;
        g.jpv[jc] = jc + 1;
        if (jc == 1) g.jmv[jc] = jc;
        if (jc == n2m) g.jpv[jc] = jc;
        if (jc == n2) g.jpv[jc] = jc;
    }
    for (int jc = 1; jc <= n2m; ++jc) {
        g.jpc[jc] = g.jpv[jc] - jc;
        g.jmc[jc] = jc - g.jmv[jc];
    }

    // cordin.F90:105-233 (istr = 100)
    for (int j = 1; j <= n2; ++j) g.rc[j] = d.ycoord[j - 1];
    for (int k = 1; k <= n3; ++k) g.zz[k] = d.zcoord[k - 1];
    for (int j = 1; j <= n2m; ++j) {
        g.rm[j] = (g.rc[j] + g.rc[j + 1]) * 0.5;
        g.g2rm[j] = (g.rc[j + 1] - g.rc[j]) * g.dx2;
    }
    for (int j = 2; j <= n2m; ++j) g.g2rc[j] = (g.rc[j + 1] - g.rc[j - 1]) * g.dx2 * 0.5;
    g.g2rc[1] = (g.rc[2] - g.rc[1]) * g.dx2;
    g.g2rc[n2] = (g.rc[n2] - g.rc[n2m]) * g.dx2;
    g.rm[n2] = g.rc[n2];
    for (int j = 1; j <= n2m; ++j) {
        g.udx2m[j] = g.dx2 / g.g2rm[j];
        g.udx2c[j] = g.dx2 / g.g2rc[j];
    }
    g.udx2c[n2] = g.dx2 / g.g2rc[n2];
    for (int k = 1; k <= n3m; ++k) {
        g.zm[k] = (g.zz[k] + g.zz[k + 1]) * 0.5;
        g.g3rm[k] = (g.zz[k + 1] - g.zz[k]) * g.dx3;
    }
    for (int k = 2; k <= n3m; ++k) g.g3rc[k] = (g.zz[k + 1] - g.zz[k - 1]) * g.dx3 * 0.5;
    g.g3rc[1] = (g.zz[2] - g.zz[1]) * g.dx3;
    g.g3rc[n3] = (g.zz[n3] - g.zz[n3m]) * g.dx3;
    g.zm[n3] = g.zz[n3];
    for (int k = 1; k <= n3m; ++k) {
        g.udx3m[k] = g.dx3 / g.g3rm[k];
        g.udx3c[k] = g.dx3 / g.g3rc[k];
    }
    g.udx3c[n3] = g.dx3 / g.g3rc[n3];
    double dymin = 1.0e+6, dzmin = 1.0e+6;
    for (int i = 2; i <= n2; ++i) dymin = std::min(dymin, g.rc[i] - g.rc[i - 1]);
    for (int i = 2; i <= n3; ++i) dzmin = std::min(dzmin, g.zz[i] - g.zz[i - 1]);
    g.ddmin = std::min(dzmin, dymin) * d.kprobe;

    // coetar.F90:297-420
    const double inwn = d.inslwn ? 1.0 : 0.0, inws = d.inslws ? 1.0 : 0.0;
    const double dx2q = g.dx2q, dx3q = g.dx3q;
    g.am2j[1] = 0.0; g.ap2j[1] = 0.0; g.ac2j[1] = 1.0;
    g.am2j[n2] = 0.0; g.ap2j[n2] = 0.0; g.ac2j[n2] = 1.0;
    for (int jc = 2; jc <= n2m; ++jc) {
        double a22 = dx2q / g.g2rc[jc], a22p = 1.0 / g.g2rm[jc], a22m = 1.0 / g.g2rm[jc - 1];
        g.ap2j[jc] = a22 * a22p;
        g.am2j[jc] = a22 * a22m;
        g.ac2j[jc] = -(a22 * a22p + a22 * a22m);
    }
    for (int jc = 2; jc <= n2m - 1; ++jc) {
        int jp = g.jpv[jc];
        double a22 = dx2q / g.g2rm[jc], a22p = a22 / g.g2rc[jp], a22m = a22 / g.g2rc[jc];
        g.ap3j[jc] = a22p;
        g.am3j[jc] = a22m;
        g.ac3j[jc] = -(a22p + a22m);
    }
    {
        int jc = n2m, jp = jc + 1;
        double a22 = dx2q / g.g2rm[jc], a22p = +a22 / g.g2rc[jp], a22m = +a22 / g.g2rc[jc];
        g.am3j[jc] = a22m;
        g.ap3j[jc] = 2.0 * inwn * a22p;
        g.ac3j[jc] = -(a22m + inwn * a22p * 2.0);
    }
    {
        int jc = 1, jp = jc + 1;
        double a22 = dx2q / g.g2rm[jc], a22p = +a22 / g.g2rc[jp], a22m = +a22 / g.g2rc[jc];
        g.ap3j[jc] = a22p;
        g.am3j[jc] = 2.0 * a22m * inws;
        g.ac3j[jc] = -(a22p + 2.0 * inws * a22m);
    }
    g.am3ck[1] = 0.0; g.ap3ck[1] = 0.0; g.ac3ck[1] = 1.0;
    g.am3ck[n3] = 0.0; g.ap3ck[n3] = 0.0; g.ac3ck[n3] = 1.0;
    for (int kc = 2; kc <= n3m; ++kc) {
        double a33 = dx3q / g.g3rc[kc], a33p = 1.0 / g.g3rm[kc], a33m = 1.0 / g.g3rm[kc - 1];
        g.ap3ck[kc] = a33 * a33p;
        g.am3ck[kc] = a33 * a33m;
        g.ac3ck[kc] = -(g.ap3ck[kc] + g.am3ck[kc]);
    }
    for (int kc = 2; kc <= n3m - 1; ++kc) {
        double a33 = dx3q / g.g3rm[kc], a33p = +a33 / g.g3rc[kc + 1], a33m = +a33 / g.g3rc[kc];
        g.ap3sk[kc] = a33p;
        g.am3sk[kc] = a33m;
        g.ac3sk[kc] = -(g.ap3sk[kc] + g.am3sk[kc]);
    }
    {
        int kc = 1;
        double a33 = dx3q / g.g3rm[kc], a33p = +a33 / g.g3rc[kc + 1], a33m = +a33 / g.g3rc[kc];
        g.ap3sk[kc] = a33p;
        g.am3sk[kc] = 0.0;
        g.ac3sk[kc] = -(a33p + a33m * 2.0);
    }
    {
        int kc = n3m;
        double a33 = dx3q / g.g3rm[kc], a33p = +a33 / g.g3rc[kc + 1], a33m = +a33 / g.g3rc[kc];
        g.am3sk[kc] = a33m;
        g.ap3sk[kc] = 0.0;
        g.ac3sk[kc] = -(a33m + a33p * 2.0);
    }

    // phini.F90:121-142 (tridiag_matrices)
    for (int jc = 1; jc <= n2m; ++jc) {
        int jp = g.jpv[jc];
        double a22icc = static_cast<double>(g.jmc[jc]) * dx2q / g.g2rc[jc];
        double a22icp = static_cast<double>(g.jpc[jc]) * dx2q / g.g2rc[jp];
        double ugmmm = 1.0 / g.g2rm[jc];
        g.amphj[jc] = a22icc * ugmmm;
        g.apphj[jc] = a22icp * ugmmm;
        g.acphj[jc] = -(g.amphj[jc] + g.apphj[jc]);
    }
    for (int kc = 1; kc <= n3m; ++kc) {
        int kp = g.kpv[kc];
        double a33icc = static_cast<double>(g.kmc[kc]) * dx3q / g.g3rc[kc];
        double a33icp = static_cast<double>(g.kpc[kc]) * dx3q / g.g3rc[kp];
        double ugmmm = 1.0 / g.g3rm[kc];
        g.amphk[kc] = a33icc * ugmmm;
        g.apphk[kc] = a33icp * ugmmm;
        g.acphk[kc] = -(g.amphk[kc] + g.apphk[kc]);
    }
}

// ---------------------------------------------------------------- eigen

// The z operator B of phini.F90:59-65 is tridiagonal with positive
// off-diagonal products, so B = S T S^-1 with T symmetric tridiagonal,
// T(i,i+1) = sqrt(B(i,i+1) B(i+1,i)) and S = diag(s), s(i+1)/s(i) =
// sqrt(B(i+1,i)/B(i,i+1)).  With T = U L U^T (implicit QL, Wilkinson shift)
// the eigenvectors of B are Z = S U and their inverse is U^T S^-1, exactly
// what phini obtains from DGEEV followed by DGESV.
int eigen_tridiag(int n, const double *am, const double *ac, const double *ap, double *wr,
                  double *zmm, double *zmmt, double *zs) {
    std::vector<double> d(ac, ac + n), e(static_cast<size_t>(n), 0.0), s(static_cast<size_t>(n), 1.0);
    for (int i = 0; i + 1 < n; ++i) {
        double up = ap[i], lo = am[i + 1];
        if (!(up > 0.0 && lo > 0.0)) return 1;
        e[i] = std::sqrt(up * lo);
        s[i + 1] = s[i] * std::sqrt(lo / up);
    }
    // U accumulated row-major: U[r*n + c]
    std::vector<double> U(static_cast<size_t>(n) * n, 0.0);
    for (int i = 0; i < n; ++i) U[static_cast<size_t>(i) * n + i] = 1.0;
    std::vector<double> rc_(static_cast<size_t>(n)), rs_(static_cast<size_t>(n));
    const double eps = std::numeric_limits<double>::epsilon();
    for (int l = 0; l < n; ++l) {
        int iter = 0;
        for (;;) {
            int m = l;
            for (; m < n - 1; ++m) {
                double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
                if (std::fabs(e[m]) <= eps * dd) break;
            }
            if (m == l) break;
            if (++iter > 60) return 2;
            // Wilkinson-type shift from the leading 2x2 block
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = std::hypot(g, 1.0);
            g = d[m] - d[l] + e[l] / (g + (g >= 0.0 ? std::fabs(r) : -std::fabs(r)));
            double sn = 1.0, cs = 1.0, p = 0.0;
            int i = m - 1, nrot = 0;
            bool deflated = false;
            for (; i >= l; --i) {
                double f = sn * e[i], b = cs * e[i];
                r = std::hypot(f, g);
                e[i + 1] = r;
                if (r == 0.0) {
                    d[i + 1] -= p;
                    e[m] = 0.0;
                    deflated = true;
                    break;
                }
                sn = f / r;
                cs = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * sn + 2.0 * cs * b;
                p = sn * r;
                d[i + 1] = g + p;
                g = cs * r - b;
                rc_[static_cast<size_t>(nrot)] = cs;
                rs_[static_cast<size_t>(nrot)] = sn;
                ++nrot;
            }
            // apply the plane rotations (columns i+1, i for i = m-1 down) to U
            const int i_first = m - 1;
#pragma omp parallel for schedule(static) if (n >= 256)
            for (int row = 0; row < n; ++row) {
                double *u = &U[static_cast<size_t>(row) * n];
                for (int q = 0; q < nrot; ++q) {
                    int ii = i_first - q;
                    double c = rc_[static_cast<size_t>(q)], sq = rs_[static_cast<size_t>(q)];
                    double f = u[ii + 1];
                    u[ii + 1] = sq * u[ii] + c * f;
                    u[ii] = c * u[ii] - sq * f;
                }
            }
            if (deflated && i >= l) continue;
            d[l] -= p;
            e[l] = g;
            e[m] = 0.0;
        }
    }
    // order eigenvalues descending (0 first, as the Neumann operator is <= 0)
    std::vector<int> idx(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) idx[static_cast<size_t>(i)] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return d[a] > d[b]; });
    for (int c = 0; c < n; ++c) {
        int src = idx[static_cast<size_t>(c)];
        wr[c] = d[static_cast<size_t>(src)];
        for (int r = 0; r < n; ++r) {
            double u = U[static_cast<size_t>(r) * n + src];
            zmm[static_cast<size_t>(c) * n + r] = s[static_cast<size_t>(r)] * u;    // Z(r,c)
            zmmt[static_cast<size_t>(r) * n + c] = u / s[static_cast<size_t>(r)];   // Zinv(c,r)
        }
    }
    if (zs)
        for (int r = 0; r < n; ++r) zs[r] = s[static_cast<size_t>(r)];
    for (int i = 0; i < n; ++i)
        if (!std::isfinite(wr[i])) return 3;
    return 0;
}

// ---------------------------------------------------------------- markers

// rigid.F90:468-495
void createnorm(int nlm, const double *vert, double orient, double *norm) {
    for (int i = 0; i < nlm; ++i) {
        const double *a = vert + 2 * i, *b = vert + 2 * (i + 1);
        double v1[3] = {0.0 - 0.0, b[0] - a[0], b[1] - a[1]};
        double v2[3] = {orient - 0.0, (a[0] + b[0]) * 0.5 - a[0], (a[1] + b[1]) * 0.5 - a[1]};
        double c[3] = {v1[1] * v2[2] - v1[2] * v2[1], v1[2] * v2[0] - v1[0] * v2[2],
                       v1[0] * v2[1] - v1[1] * v2[0]};
        double den = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
        norm[2 * i] = c[1] / den;
        norm[2 * i + 1] = c[2] / den;
    }
}

std::string setup_case(const std::string &dir, HostCase &hc) {
    std::string err = read_deck(dir, hc.deck);
    if (!err.empty()) return err;
    const Deck &d = hc.deck;
    if (d.dt < 1.0e-8) return "global_par.in: too small time step size";
    build_grid(d, hc.grid);
    const Grid &g = hc.grid;
    // fluid_pre.F90:164-182
    if (d.nsst > 1) {
        hc.gam[0] = 8.0 / 15.0; hc.gam[1] = 5.0 / 12.0; hc.gam[2] = 3.0 / 4.0;
        hc.rom[0] = 0.0; hc.rom[1] = -17.0 / 60.0; hc.rom[2] = -5.0 / 12.0;
    } else {
        hc.gam[0] = 1.5; hc.rom[0] = -0.50;
    }
    for (int n = 0; n < d.nsst; ++n) hc.alm[n] = hc.gam[n] + hc.rom[n];

    // phini.F90:59-92
    const int n3m = g.n3m;
    std::vector<double> am(static_cast<size_t>(n3m)), ac(static_cast<size_t>(n3m)), ap(static_cast<size_t>(n3m));
    for (int k = 0; k < n3m; ++k) {
        am[static_cast<size_t>(k)] = g.amphk[k + 1];
        ac[static_cast<size_t>(k)] = g.acphk[k + 1];
        ap[static_cast<size_t>(k)] = g.apphk[k + 1];
    }
    hc.wr.assign(static_cast<size_t>(n3m), 0.0);
    hc.zmm.assign(static_cast<size_t>(n3m) * n3m, 0.0);
    hc.zmmt.assign(static_cast<size_t>(n3m) * n3m, 0.0);
    hc.zs.assign(static_cast<size_t>(n3m), 1.0);
    if (eigen_tridiag(n3m, am.data(), ac.data(), ap.data(), hc.wr.data(), hc.zmm.data(), hc.zmmt.data(),
                      hc.zs.data()))
        return "eigen-decomposition of the z Poisson operator failed";

    // markers: utils_proc.F90:540-548 then rigid_pre.F90:42-118
    const int nlm = d.nlm;
    hc.vert = d.vert;
    hc.lmcc.assign(static_cast<size_t>(nlm) * 2, 0.0);
    hc.lmvel.assign(static_cast<size_t>(nlm) * 2, 0.0);
    hc.lmacc.assign(static_cast<size_t>(nlm) * 2, 0.0);
    hc.lmnor.assign(static_cast<size_t>(nlm) * 2, 0.0);
    hc.lmA.assign(static_cast<size_t>(nlm), 0.0);
    if (nlm > 0) {
        double *v = hc.vert.data();
        for (int i = 0; i < nlm; ++i) {
            hc.lmcc[2 * i] = (v[2 * i] + v[2 * i + 2]) * 0.5;
            hc.lmcc[2 * i + 1] = (v[2 * i + 1] + v[2 * i + 3]) * 0.5;
            double dy = v[2 * i + 2] - v[2 * i], dz = v[2 * i + 3] - v[2 * i + 1];
            hc.lmA[i] = std::sqrt(dy * dy + dz * dz);
        }
        createnorm(nlm, v, -1.0, hc.lmnor.data());
        double *cmp_n = hc.rigid, *cmv_n = hc.rigid + 3, *cma_n = hc.rigid + 6;
        double *cmp_np1 = hc.rigid + 9, *cmv_np1 = hc.rigid + 12, *cma_np1 = hc.rigid + 15;
        cmp_n[0] = d.cmposi[0];
        cmp_n[1] = d.cmposi[1];
        cmp_n[2] = d.cmroti;
        hc.kinori[0] = d.cmposi[0];
        hc.kinori[1] = d.cmposi[1];
        hc.kinori[2] = d.cmroti;
        cmv_n[0] = d.ipert[0];
        if (d.rtcoup) cmv_n[2] = cmv_n[0] / d.rrr;
        for (int i = 0; i < 3; ++i) {
            cmp_np1[i] = cmp_n[i];
            cmv_np1[i] = cmv_n[i];
            cma_np1[i] = cma_n[i];
        }
        double c = std::cos(cmp_n[2]), sn = std::sin(cmp_n[2]);
        double r00 = c, r01 = -sn, r10 = sn, r11 = c;
        for (int i = 0; i < nlm; ++i) {
            double rho0 = hc.lmcc[2 * i] - cmp_n[0], rho1 = hc.lmcc[2 * i + 1] - cmp_n[1];
            double c10 = -cmv_np1[2] * rho1, c11 = cmv_np1[2] * rho0;
            double c20 = -cma_np1[2] * rho1, c21 = cma_np1[2] * rho0;
            double c30 = -cmv_np1[2] * c11, c31 = cmv_np1[2] * c10;
            hc.lmcc[2 * i] = cmp_np1[0] + (r00 * rho0 + r01 * rho1);
            hc.lmcc[2 * i + 1] = cmp_np1[1] + (r10 * rho0 + r11 * rho1);
            hc.lmvel[2 * i] = cmv_np1[0] + c10;
            hc.lmvel[2 * i + 1] = cmv_np1[1] + c11;
            hc.lmacc[2 * i] = cma_np1[0] + c20 + c30;
            hc.lmacc[2 * i + 1] = cma_np1[1] + c21 + c31;
        }
        for (int i = 0; i <= nlm; ++i) {
            double a0 = v[2 * i] - d.cmposi[0], a1 = v[2 * i + 1] - d.cmposi[1];
            v[2 * i] = cmp_np1[0] + (r00 * a0 + r01 * a1);
            v[2 * i + 1] = cmp_np1[1] + (r10 * a0 + r11 * a1);
        }
        createnorm(nlm, v, -1.0, hc.lmnor.data());
    }
    return "";
}

}  // namespace fb
