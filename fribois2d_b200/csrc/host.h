// Host-side set-up of one FRiBoIS2D case: input deck, grid metrics,
// operator coefficients, Poisson eigen data, line-solve factors, markers.
// Everything here runs on the CPU once per case; the device path consumes it.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace fb {

// Values of global_par.in / fluid_par.in / rigid_par.in plus the grid and
// marker files (utils_proc.F90:2-222,519-578; cordin.F90:243-278).
struct Deck {
    double dt = 0, dtmax = 0, cflmax = 0, cfllim = 0, trestart = 0;
    bool idtv = true, irest = false, ibact = true, prlgr = false;
    std::string outfol;
    double kprobe = 1, tprtag = 0, radiusSD = 1.6;
    int forst = 1, wfun = 1;
    double alx3 = 0, rext2 = 0;
    int n3 = 0, n2 = 0, istr3 = 100, istr2 = 100, nsst = 3;
    bool nwrit = false;
    double tframef = 0, resid = 0, cou = 0, visc = 0, q3uw = 0, q3lw = 0;
    bool inslws = false, inslwn = false;
    bool cbody = true, rtcoup = false;
    double cmposi[2] = {0, 0}, cmroti = 0, ipert[3] = {0, 0, 0}, rbgravF[2] = {0, 0};
    double rbden = 1, rba[2] = {0, 0}, kk[3] = {0, 0, 0}, kk3[3] = {0, 0, 0}, cc[3] = {0, 0, 0};
    double rrr = 1;
    int rbmcon[3] = {0, 0, 0};
    std::vector<double> ycoord, zcoord;  // n2, n3
    int nlm = 0;
    std::vector<double> vert;            // (nlm+1) x 2, row-major (y, z)
};

// Returns an empty string on success, else a message.
std::string read_deck(const std::string &dir, Deck &d);

// LU factors of one tridiagonal system as DGTTRF leaves them (0-based):
// dl (n-1), d (n), du (n-1), du2 (n-2), ipiv (n, 1-based rows as LAPACK).
struct TriLU {
    int n = 0;
    std::vector<double> dl, d, du, du2;
    std::vector<int> ipiv;
    bool pivoted = false;
    int info = 0;
};
// DGTTRF restated (LAPACK 3.8): in-place factorization with partial pivoting.
int dgttrf(int n, double *dl, double *d, double *du, double *du2, int *ipiv);
TriLU factor(const std::vector<double> &lower, const std::vector<double> &diag,
             const std::vector<double> &upper);

// Grid metrics and coefficients, 1-based arrays (index 0 unused) exactly as
// the reference names them.
struct Grid {
    int n2 = 0, n3 = 0, n2m = 0, n3m = 0;
    double dx2 = 0, dx3 = 0, dx2q = 0, dx3q = 0, ren = 0, ddmin = 0;
    std::vector<double> rc, rm, zz, zm, g2rc, g2rm, g3rc, g3rm, udx2c, udx2m, udx3c, udx3m;
    std::vector<int> jmv, jpv, jmc, jpc, kmv, kpv, kmc, kpc;
    std::vector<double> am2j, ac2j, ap2j, am3j, ac3j, ap3j;
    std::vector<double> am3ck, ac3ck, ap3ck, am3sk, ac3sk, ap3sk;
    std::vector<double> amphj, acphj, apphj, amphk, acphk, apphk;
};
void build_grid(const Deck &d, Grid &g);

// Symmetric-tridiagonal eigen-decomposition of the z Poisson operator.
// am/ac/ap: sub (row i, col i-1), diagonal, super (row i, col i+1), 0-based.
// zmm: eigenvectors (column-major), zmmt: their inverse; zs (may be null):
// the diagonal S with zmm = S U, zmmt = U^T S^-1, U orthogonal.  Returns 0 on
// success.
int eigen_tridiag(int n, const double *am, const double *ac, const double *ap, double *wr,
                  double *zmm, double *zmmt, double *zs = nullptr);

// Everything the device needs for one case.
struct HostCase {
    Deck deck;
    Grid grid;
    double gam[3] = {0, 0, 0}, rom[3] = {0, 0, 0}, alm[3] = {0, 0, 0};
    std::vector<double> wr, zmm, zmmt;    // n3m, n3m^2 (column-major)
    std::vector<double> zs;               // n3m: zmm = diag(zs) U with U orthogonal
    // initial state (inqpr, initial_sol.F90:251-299) and markers after rigid_pre
    std::vector<double> lmcc, lmvel, lmacc, lmnor, lmA, vert;
    double rigid[18] = {0};               // cmp_n, cmv_n, cma_n, cmp_np1, cmv_np1, cma_np1
    double kinori[9] = {0};
};
std::string setup_case(const std::string &dir, HostCase &hc);
void createnorm(int nlm, const double *vert, double orient, double *norm);

}  // namespace fb
