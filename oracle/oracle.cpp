// CPU oracle for the Canard per-step hot path — TEST INFRASTRUCTURE ONLY.
//
// A plain C++ FP64 restatement of the reference Fortran, statement by statement
// in the reference's operation order (compile with -ffp-contract=off; the
// reference's gfortran -O3 build on x86-64 emits no FMA). Only tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline leg load this library.
//
// Parity status: UNPINNED against the reference binary (no golden vectors are
// shipped and no Fortran compiler exists here); pinned against known answers of
// the scheme in tests/test_oracle_kat.py. Known deliberate difference: the
// reference computes the interface coefficients with libgfortran's blocked
// matmul (src/mo_numerics.f90:412); here the products sum in ascending index
// order, so pbci/pbco agree with the reference to rounding (~1e-16), not
// bit for bit.
//
// Citations are to the reference tree (src/...).
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <stdexcept>
#include <tuple>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---- constants: src/mo_parameters.f90:15-70 ---------------------------------
const double zero = 0.0, half = 0.5, one = 1.0, two = 2.0, three = 3.0;
const double pi = std::acos(-1.0);
const double sml = 1.0e-8;
const int BC_NON_REFLECTIVE = 10, BC_WALL_INVISCID = 20, BC_WALL_VISCOUS = 25,
          BC_INTER_CURV = 30, BC_INTER_STRAIGHT = 35, BC_INTER_SUBDOMAINS = 40,
          BC_PERIODIC = 45;
const double gam = 1.4;
const double gamm1 = gam - one;
const double ham = one / gam;
const double hamm1 = one / gamm1;
const double hamhamm1 = ham * hamm1;
const double prndtl = 0.71;
const double gamm1prndtli = one / (gamm1 * prndtl);
const double twothirds = two / three;
const double alpha = 4 / 9.0, beta = 1 / 36.0, aa = 20 / 27.0, ab = 25 / 216.0;
const double alpha10 = 0.09166666665902128, alpha12 = 1.3500000000438646,
             beta13 = 0.2666666666794667, a10 = -0.3506944444280639,
             a12 = 0.8249999999974599, a13 = 0.7444444444773477,
             a14 = 0.014583333334139971;
const double alpha01 = 8.000000000449464, beta02 = 6.000000000542,
             a01 = -6.666666667794732, a02 = 9.000000000052879,
             a03 = 1.333333333178555, a04 = -0.0833333333455545;
const int lmd = 11, lmf = 11;
const int nnf[3] = {2, 3, 1};  // src/mo_numerics.f90:22
const int nkrk = 4;

// ---- numerics coefficients (shared by all blocks of a case) ----------------
struct Coeffs {
  double alphf, betf, fa, fb, fc;
  double albef[5][3][2];      // (-2:2, 0:2, 0:1) -> [k+2][r][n]
  double fbc[5][3];           // (0:4, 0:2)
  double pbci[12][2][2];      // (0:lmp, 0:1, 0:1)
  double pbco[12][2][2];
  double pbcot[2][2];         // (0:1 jjk, 0:1 ntk)
};

// src/mo_utils.f90:15-50 — Gauss-Jordan inverse with partial pivoting.
// a, s are n x n column-major (1-based semantics mapped to 0-based).
void mtrxi(const std::vector<double>& ax, std::vector<double>& sx, int n) {
  auto R = [n](int i, int j) { return i + n * j; };
  std::vector<double> rx(ax), temp(n);
  std::vector<int> ipvt(n);
  for (int i = 0; i < n; ++i) ipvt[i] = i;
  for (int iik = 0; iik < n; ++iik) {
    int mk = iik;
    double best = std::fabs(rx[R(iik, iik)]);
    for (int r = iik + 1; r < n; ++r)
      if (std::fabs(rx[R(r, iik)]) > best) { best = std::fabs(rx[R(r, iik)]); mk = r; }
    if (mk != iik) {
      std::swap(ipvt[mk], ipvt[iik]);
      for (int c = 0; c < n; ++c) std::swap(rx[R(mk, c)], rx[R(iik, c)]);
    }
    double ra0k = one / rx[R(iik, iik)];
    for (int r = 0; r < n; ++r) temp[r] = rx[R(r, iik)];
    for (int jjk = 0; jjk < n; ++jjk) {
      double ra1k = ra0k * rx[R(iik, jjk)];
      for (int r = 0; r < n; ++r) rx[R(r, jjk)] = rx[R(r, jjk)] - ra1k * temp[r];
      rx[R(iik, jjk)] = ra1k;
    }
    for (int r = 0; r < n; ++r) rx[R(r, iik)] = -ra0k * temp[r];
    rx[R(iik, iik)] = ra0k;
  }
  sx.assign(n * n, 0.0);
  for (int c = 0; c < n; ++c)
    for (int r = 0; r < n; ++r) sx[R(r, ipvt[c])] = rx[R(r, c)];
}

// src/mo_numerics.f90:306-326
void fcint(double fltk, double fltr, double& alphz, double& betz, double& za,
           double& zb, double& zc) {
  double c1 = std::cos(fltk), c2 = std::cos(2 * fltk), c3 = std::cos(3 * fltk);
  double fctrk = 1 / (((30 + (5 * (7 - 16 * fltr)) * c1) + (2 * (1 + 8 * fltr)) * c2) - 3 * c3);
  alphz = fctrk * (((20 * (2 * fltr - 1) - 30 * c1) + (12 * (2 * fltr - 1)) * c2) - 2 * c3);
  betz = (half * fctrk) * (((2 * (13 - 8 * fltr) + (33 - 48 * fltr) * c1) + 6 * c2) - c3);
  double ch = std::cos(half * fltk);
  double ch2 = ch * ch;
  double ch4 = ch2 * ch2;
  za = ((60 * (1 - fltr)) * ch4) * fctrk;
  zb = (-2 * za) / 5;
  zc = za / 15;
}

// src/mo_numerics.f90:253-302
void fcbcm(Coeffs& C, double fltk, double fltrbc) {
  double alphz, betz, za, zb, zc;
  double aok = std::log(fltrbc);
  fcint(fltk, half, alphz, betz, za, zb, zc);
  double fctrk = one / ((one + alphz * fltrbc) + betz * (fltrbc * fltrbc));
  double r0[5] = {zero, zero, one, alphz * fctrk, betz * fctrk};
  for (int k = 0; k < 5; ++k) C.albef[k][0][0] = r0[k];
  double resk = ((fltrbc - 1) * ((za + zc) + (fltrbc + 1) * (zb + fltrbc * zc))) / aok;
  double f0[5] = {za - (5 * resk) / 3, zb + (10 * resk) / 21, zc - (5 * resk) / 42,
                  (5 * resk) / 252, (-resk) / 630};
  for (int k = 0; k < 5; ++k) C.fbc[k][0] = f0[k] * fctrk;
  double r1[5] = {zero, alphz + betz * fltrbc, one, alphz, betz};
  for (int k = 0; k < 5; ++k) C.albef[k][1][0] = r1[k];
  resk = ((fltrbc - 1) * (zb + zc * (fltrbc + 1))) / aok;
  double f1[5] = {((za + zb) + zc) + (1627 * resk) / 1260, za + (10 * resk) / 21,
                  zb - (5 * resk) / 42, zc + (5 * resk) / 252, (-resk) / 630};
  for (int k = 0; k < 5; ++k) C.fbc[k][1] = f1[k];
  double r2[5] = {betz, alphz, one, alphz, betz};
  for (int k = 0; k < 5; ++k) C.albef[k][2][0] = r2[k];
  resk = (zc * (fltrbc - 1)) / aok;
  double f2[5] = {(zb + zc) + (1627 * resk) / 1260, za - (5 * resk) / 3,
                  za - (5 * resk) / 42, zb + (5 * resk) / 252, zc - resk / 630};
  for (int k = 0; k < 5; ++k) C.fbc[k][2] = f2[k];
}

// sum of a (0:n) product in ascending order, as Fortran's SUM does
inline double seqdot(const double* a, const double* b, int n) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s = s + a[i] * b[i];
  return s;
}

// src/mo_numerics.f90:330-425
void sbcco(Coeffs& C) {
  for (int ntk = 0; ntk <= 1; ++ntk) {
    int llk = (ntk == 0) ? lmd : lmf;
    int n = 2 * (llk + 1);
    auto R = [n](int i, int j) { return (i - 1) + n * (j - 1); };  // 1-based
    std::vector<double> ax(n * n, 0.0), bx(n * n, 0.0), rx, sx;
    if (ntk == 0) {
      ax[R(1, 1)] = one; ax[R(1, 2)] = alpha01; ax[R(1, 3)] = beta02;
      double b1[5] = {-(((a01 + a02) + a03) + a04), a01, a02, a03, a04};
      for (int k = 0; k < 5; ++k) bx[R(1, 1 + k)] = b1[k];
      double a2[4] = {alpha10, one, alpha12, beta13};
      for (int k = 0; k < 4; ++k) ax[R(2, 1 + k)] = a2[k];
      double b2[5] = {a10, -(((a10 + a12) + a13) + a14), a12, a13, a14};
      for (int k = 0; k < 5; ++k) bx[R(2, 1 + k)] = b2[k];
      for (int i = 3; i <= n - 2; ++i) {
        double ar[5] = {beta, alpha, one, alpha, beta};
        double br[5] = {-ab, -aa, zero, aa, ab};
        for (int k = 0; k < 5; ++k) { ax[R(i, i - 2 + k)] = ar[k]; bx[R(i, i - 2 + k)] = br[k]; }
      }
      for (int k = 0; k < 4; ++k) ax[R(n - 1, n - k)] = ax[R(2, 1 + k)];
      for (int k = 0; k < 5; ++k) bx[R(n - 1, n - k)] = -bx[R(2, 1 + k)];
      for (int k = 0; k < 3; ++k) ax[R(n, n - k)] = ax[R(1, 1 + k)];
      for (int k = 0; k < 5; ++k) bx[R(n, n - k)] = -bx[R(1, 1 + k)];
    } else {
      for (int k = 0; k < 3; ++k) ax[R(1, 1 + k)] = C.albef[k + 2][0][0];
      for (int k = 0; k < 5; ++k) bx[R(1, 1 + 1 + k)] = C.fbc[k][0];
      bx[R(1, 1)] = -((((C.fbc[0][0] + C.fbc[1][0]) + C.fbc[2][0]) + C.fbc[3][0]) + C.fbc[4][0]);
      for (int k = 0; k < 4; ++k) ax[R(2, 1 + k)] = C.albef[k + 1][1][0];
      {
        int off[5] = {0, 2, 3, 4, 5};
        for (int k = 0; k < 5; ++k) bx[R(2, 1 + off[k])] = C.fbc[k][1];
        bx[R(2, 2)] = -((((C.fbc[0][1] + C.fbc[1][1]) + C.fbc[2][1]) + C.fbc[3][1]) + C.fbc[4][1]);
      }
      for (int k = 0; k < 5; ++k) ax[R(3, 1 + k)] = C.albef[k][2][0];
      {
        int off[5] = {0, 1, 3, 4, 5};
        for (int k = 0; k < 5; ++k) bx[R(3, 1 + off[k])] = C.fbc[k][2];
        bx[R(3, 3)] = -((((C.fbc[0][2] + C.fbc[1][2]) + C.fbc[2][2]) + C.fbc[3][2]) + C.fbc[4][2]);
      }
      for (int i = 4; i <= n - 3; ++i) {
        double ar[5] = {C.betf, C.alphf, one, C.alphf, C.betf};
        for (int k = 0; k < 5; ++k) ax[R(i, i - 2 + k)] = ar[k];
        double br[7] = {C.fc, C.fb, C.fa, -2 * ((C.fa + C.fb) + C.fc), C.fa, C.fb, C.fc};
        for (int k = 0; k < 7; ++k) bx[R(i, i - 3 + k)] = br[k];
      }
      for (int k = 0; k < 5; ++k) ax[R(n - 2, n - k)] = ax[R(3, 1 + k)];
      for (int k = 0; k < 6; ++k) bx[R(n - 2, n - k)] = bx[R(3, 1 + k)];
      for (int k = 0; k < 4; ++k) ax[R(n - 1, n - k)] = ax[R(2, 1 + k)];
      for (int k = 0; k < 6; ++k) bx[R(n - 1, n - k)] = bx[R(2, 1 + k)];
      for (int k = 0; k < 3; ++k) ax[R(n, n - k)] = ax[R(1, 1 + k)];
      for (int k = 0; k < 6; ++k) bx[R(n, n - k)] = bx[R(1, 1 + k)];
    }
    mtrxi(ax, sx, n);
    rx = ax;
    int iik = n / 2 - 1;
    rx[R(iik, iik + 2)] = 0; rx[R(iik + 1, iik + 2)] = 0; rx[R(iik + 1, iik + 3)] = 0;
    iik = n / 2 + 2;
    rx[R(iik, iik - 2)] = 0; rx[R(iik - 1, iik - 2)] = 0; rx[R(iik - 1, iik - 3)] = 0;
    // ax = matmul(rx, matmul(sx, bx)), ascending-index summation
    std::vector<double> t(n * n), p(n * n);
    for (int j = 1; j <= n; ++j)
      for (int i = 1; i <= n; ++i) {
        double s = 0;
        for (int k = 1; k <= n; ++k) s = s + sx[R(i, k)] * bx[R(k, j)];
        t[R(i, j)] = s;
      }
    for (int j = 1; j <= n; ++j)
      for (int i = 1; i <= n; ++i) {
        double s = 0;
        for (int k = 1; k <= n; ++k) s = s + rx[R(i, k)] * t[R(k, j)];
        p[R(i, j)] = s;
      }
    iik = n / 2 + 1;
    for (int c = 0; c <= llk; ++c) C.pbco[llk - c][0][ntk] = p[R(iik, 1 + c)];
    for (int c = 0; c <= llk; ++c) C.pbci[c][0][ntk] = p[R(iik, 1 + llk + 1 + c)];
    iik = n / 2 + 2;
    for (int c = 0; c <= llk; ++c) C.pbco[llk - c][1][ntk] = p[R(iik, 1 + c)];
    for (int c = 0; c <= llk; ++c) C.pbci[c][1][ntk] = p[R(iik, 1 + llk + 1 + c)];
  }
}

// src/mo_numerics.f90:114-134
void init_coeffs(Coeffs& C, double fltk_nml, double fltrbc) {
  double fltk = pi * fltk_nml;
  std::memset(&C, 0, sizeof(C));
  fcbcm(C, fltk, fltrbc);
  fcint(fltk, half, C.alphf, C.betf, C.fa, C.fb, C.fc);
  double r0[5] = {zero, zero, one, C.alphf, C.betf};
  double r1[5] = {zero, C.alphf, one, C.alphf, C.betf};
  double r2[5] = {C.betf, C.alphf, one, C.alphf, C.betf};
  for (int k = 0; k < 5; ++k) { C.albef[k][0][1] = r0[k]; C.albef[k][1][1] = r1[k]; C.albef[k][2][1] = r2[k]; }
  sbcco(C);
  for (int ntk = 0; ntk <= 1; ++ntk)
    for (int jjk = 0; jjk <= 1; ++jjk) {
      double s = 0;
      for (int i = 0; i <= lmd; ++i) s = s + C.pbco[i][jjk][ntk];
      C.pbcot[jjk][ntk] = s;
    }
}

// src/mo_numerics.f90:179-249; xu (0:lim,3), xl (0:lim,2) column-major.
void penta(const Coeffs& C, double* xu, double* xl, int lim1, int is, int ie, int ns,
           int ne, int nt) {
  double albe[5][3][2];
  double alpho, beto;
  if (nt == 0) {
    double t[3][2][5] = {{{zero, zero, one, alpha01, beta02}, {zero, zero, one, alpha, beta}},
                         {{zero, alpha10, one, alpha12, beta13}, {zero, alpha, one, alpha, beta}},
                         {{beta, alpha, one, alpha, beta}, {beta, alpha, one, alpha, beta}}};
    for (int r = 0; r < 3; ++r)
      for (int n = 0; n < 2; ++n)
        for (int k = 0; k < 5; ++k) albe[k][r][n] = t[r][n][k];
    alpho = alpha;
    beto = beta;
  } else {
    std::memcpy(albe, C.albef, sizeof(albe));
    alpho = C.alphf;
    beto = C.betf;
  }
  auto U = [&](int i, int c) -> double& { return xu[i + lim1 * (c - 1)]; };
  auto L = [&](int i, int c) -> double& { return xl[i + lim1 * (c - 1)]; };
  auto A = [&](int k, int r, int n) { return albe[k + 2][r][n]; };
  for (int i = is; i <= ie; ++i) {
    L(i, 1) = L(i, 2) = one;
    U(i, 1) = U(i, 2) = U(i, 3) = one;
  }
  int i = is;
  U(i, 1) = one; U(i, 2) = A(1, 0, ns); U(i, 3) = A(2, 0, ns);
  i = is + 1;
  L(i, 2) = A(-1, 1, ns) * U(i - 1, 1);
  U(i, 1) = one / (one - U(i - 1, 2) * L(i, 2));
  U(i, 2) = A(1, 1, ns) - U(i - 1, 3) * L(i, 2);
  U(i, 3) = A(2, 1, ns);
  i = is + 2;
  L(i, 1) = A(-2, 2, ns) * U(i - 2, 1);
  L(i, 2) = (A(-1, 2, ns) - U(i - 2, 2) * L(i, 1)) * U(i - 1, 1);
  U(i, 1) = one / ((one - U(i - 2, 3) * L(i, 1)) - U(i - 1, 2) * L(i, 2));
  U(i, 2) = A(1, 2, ns) - U(i - 1, 3) * L(i, 2);
  U(i, 3) = A(2, 2, ns);
  for (i = is + 3; i <= ie - 3; ++i) {
    L(i, 1) = beto * U(i - 2, 1);
    L(i, 2) = (alpho - U(i - 2, 2) * L(i, 1)) * U(i - 1, 1);
    U(i, 1) = one / ((one - U(i - 2, 3) * L(i, 1)) - U(i - 1, 2) * L(i, 2));
    U(i, 2) = alpho - U(i - 1, 3) * L(i, 2);
    U(i, 3) = beto;
  }
  i = ie - 2;
  L(i, 1) = A(2, 2, ne) * U(i - 2, 1);
  L(i, 2) = (A(1, 2, ne) - U(i - 2, 2) * L(i, 1)) * U(i - 1, 1);
  U(i, 1) = one / ((one - U(i - 2, 3) * L(i, 1)) - U(i - 1, 2) * L(i, 2));
  U(i, 2) = A(-1, 2, ne) - U(i - 1, 3) * L(i, 2);
  U(i, 3) = A(-2, 2, ne);
  i = ie - 1;
  L(i, 1) = A(2, 1, ne) * U(i - 2, 1);
  L(i, 2) = (A(1, 1, ne) - U(i - 2, 2) * L(i, 1)) * U(i - 1, 1);
  U(i, 1) = one / ((one - U(i - 2, 3) * L(i, 1)) - U(i - 1, 2) * L(i, 2));
  U(i, 2) = A(-1, 1, ne) - U(i - 1, 3) * L(i, 2);
  i = ie;
  L(i, 1) = A(2, 0, ne) * U(i - 2, 1);
  L(i, 2) = (A(1, 0, ne) - U(i - 2, 2) * L(i, 1)) * U(i - 1, 1);
  U(i, 1) = one / ((one - U(i - 2, 3) * L(i, 1)) - U(i - 1, 2) * L(i, 2));
  for (i = is; i <= ie; ++i) {
    U(i, 2) = U(i, 2) * U(i, 1);
    U(i, 3) = U(i, 3) * U(i, 1);
  }
}

// ---- simulated MPI point-to-point: non-overtaking FIFO per (src,dst,tag) ----
struct MpiSim {
  struct Snd { int src, dst, tag; std::vector<double> data; };
  struct Rcv { int dst, src, tag; double* buf; size_t n; };
  std::vector<Snd> snd;
  std::vector<Rcv> rcv;
  void isend(int src, int dst, int tag, const double* p, size_t n) {
    snd.push_back({src, dst, tag, std::vector<double>(p, p + n)});
  }
  void irecv(int me, int src, int tag, double* p, size_t n) { rcv.push_back({me, src, tag, p, n}); }
  void waitall() {
    std::map<std::tuple<int, int, int>, std::deque<size_t>> q;
    for (size_t i = 0; i < snd.size(); ++i) q[std::make_tuple(snd[i].src, snd[i].dst, snd[i].tag)].push_back(i);
    for (auto& r : rcv) {
      auto& d = q[std::make_tuple(r.src, r.dst, r.tag)];
      if (d.empty()) throw std::runtime_error("mpi sim: unmatched receive");
      const Snd& s = snd[d.front()];
      d.pop_front();
      if (s.data.size() > r.n) throw std::runtime_error("mpi sim: message truncated");
      std::copy(s.data.begin(), s.data.end(), r.buf);
    }
    snd.clear();
    rcv.clear();
  }
};

// ---- one block = one rank ---------------------------------------------------
struct Block {
  int lxi, let, lze, lmx, lim;
  int nbc[3][2], mcd[3][2];
  int ijk[3][3];      // ijk[a][nn], a=0..2 (Fortran ijk(a+1, nn+1))
  int nbs[3];
  int ndf[3][2][2];   // [nn][ip][nt]
  std::vector<double> xu, yu, xl, yl;
  std::vector<double> send0[3], send1[3], recv0[3], recv1[3], drva[3], drvb[3], cm[3];
  std::vector<double> qa, qo, de, p, ss, rr;   // ss (0:lmx,3), rr (0:lmx,3)
  std::vector<double> xim, etm, zem, yaco;
  std::vector<double> txx, tyy, tzz, txy, tyz, tzx, hxx, hyy, hzz;
  std::vector<double> xyz;
  std::vector<double> sbcc;
  std::vector<int> nrr, npex;
  std::vector<int> lcsz;
  std::vector<double> asz, bsz;
  // junctions: src/mo_domdcomp.f90:17-34
  int njp[8], njl[12];
  // sub-domain of parent block mb at position ijkp (src/mo_domdcomp.f90:110-119)
  int mb = 0, ijkp[3] = {0, 0, 0};
  std::vector<int> imjp, jptag, imjl, jltag;
  std::vector<std::vector<int>> jjp, jjl;
  int jpcd[8][101], jlcd[12][101];
  size_t L() const { return (size_t)lmx + 1; }
  int indx3(int i, int j, int k, int nn) const {  // src/mo_utils.f90:54-69
    switch (nn) {
      case 1: return (k * (let + 1) + j) * (lxi + 1) + i;
      case 2: return (j * (let + 1) + i) * (lxi + 1) + k;
      default: return (i * (let + 1) + k) * (lxi + 1) + j;
    }
  }
};

}  // namespace

// A block of the input (nbbc / mbcd / nbpc of nml_domdcomp) whose sub-domains
// are ranks mo .. mo + nbpc[0] nbpc[1] nbpc[2] - 1.
struct Parent {
  int nbpc[3] = {1, 1, 1};
  int mbcd[3][2];
  int mo = 0;
};

struct orc_solver {
  orc_hook_fn hook = nullptr;  // exchange hook (orc_set_hook)
  void* hook_user = nullptr;
  void call_hook(int kind, int a, int b, double* data = nullptr, int n = 0) {
    if (hook) hook(hook_user, kind, a, b, data, n);
  }
  orc_case_desc cs;
  std::vector<Block> B;       // ranks (sub-domains)
  std::vector<Parent> P;      // blocks; by default every rank is its own block
  Coeffs C;
  double srefoo, srefp1dre, reoo, amachoo, uoo[3];
  double umf[3] = {0, 0, 0}, dudtmf[3] = {0, 0, 0};
  // time loop state (src/mo_canard_driver.f90:204-216)
  int n = 0, ndt = 0;
  double dt = 0, dts = 0, dte = 0, timo = 0;
  int nblk() const { return (int)B.size(); }
};

namespace {

using S = orc_solver;

// ---- t_numerics%mpigo: src/mo_numerics.f90:429-705 -------------------------
// cols[b] points at rfield(0:lmx, ncols) of block b; column nzk per direction.
void mpigo(S& s, double* const* cols, int nt, int nrt, int n45, int itag, int m) {
  MpiSim mpi;
  const int mpk = (nt == 0) ? lmd : lmf;
  for (int b = 0; b < s.nblk(); ++b) {
    Block& k = s.B[b];
    for (int nnk = 1; nnk <= 3; ++nnk) {
      int nzk = (1 - nrt) * (nnk - 1) + 1;
      const double* rf = cols[b] + (size_t)(nzk - 1) * k.L();
      int nb = k.nbs[nnk - 1];
      int ncomp = nt == 0 ? 2 : 3;
      std::vector<double>& send = nt == 0 ? k.send0[nnk - 1] : k.send1[nnk - 1];
      std::vector<double>& recv = nt == 0 ? k.recv0[nnk - 1] : k.recv1[nnk - 1];
      for (int ipk = 0; ipk <= 1; ++ipk) {
        int iqk = 1 - ipk;
        int istart = ipk * k.ijk[0][nnk - 1];
        int iend = 1 - 2 * ipk;
        double ra0k = 0;
        int iik = 0;
        switch (k.nbc[nnk - 1][ipk]) {
          case BC_INTER_STRAIGHT: ra0k = zero; iik = 1; break;
          case BC_INTER_SUBDOMAINS: ra0k = zero; iik = 0; break;
          case BC_PERIODIC: ra0k = n45; iik = 1; break;
        }
        if (k.ndf[nnk - 1][ipk][nt] == 1) {
          for (int kk = 0; kk <= k.ijk[2][nnk - 1]; ++kk) {
            int kpp = kk * (k.ijk[1][nnk - 1] + 1);
            for (int jj = 0; jj <= k.ijk[1][nnk - 1]; ++jj) {
              int jkk = kpp + jj;
              double resk = ra0k * rf[k.indx3(istart, jj, kk, nnk)];
              double sap[12];
              for (int iii = 0; iii <= mpk; ++iii)
                sap[iii] = rf[k.indx3(istart + iend * (iii + iik), jj, kk, nnk)];
              double* sd = &send[jkk + (size_t)nb * (ncomp * ipk)];
              double s0 = 0, s1 = 0;
              for (int iii = 0; iii <= mpk; ++iii) s0 = s0 + s.C.pbco[iii][0][nt] * sap[iii];
              for (int iii = 0; iii <= mpk; ++iii) s1 = s1 + s.C.pbco[iii][1][nt] * sap[iii];
              sd[0] = s0 - resk * s.C.pbcot[0][nt];
              sd[(size_t)nb] = s1 - resk * s.C.pbcot[1][nt];
              double* snt = &send[jkk + (size_t)nb * ((nt + 1) + ncomp * ipk)];
              *snt = *snt + nt * ((sap[0] - resk) - *snt);
            }
          }
          mpi.isend(b, k.mcd[nnk - 1][ipk], itag + iqk, &send[(size_t)nb * ncomp * ipk], (size_t)ncomp * nb);
          mpi.irecv(b, k.mcd[nnk - 1][ipk], itag + ipk,
                    &recv[(size_t)nb * ncomp * (ipk + 2 * (m - 1))], (size_t)ncomp * nb);
        }
      }
    }
  }
  mpi.waitall();
  s.call_hook(0, nt, m);
  if (n45 == 1) {
    for (int b = 0; b < s.nblk(); ++b) {
      Block& k = s.B[b];
      for (int nnk = 1; nnk <= 3; ++nnk) {
        int nzk = (1 - nrt) * (nnk - 1) + 1;
        const double* rf = cols[b] + (size_t)(nzk - 1) * k.L();
        int nb = k.nbs[nnk - 1];
        int ncomp = nt == 0 ? 2 : 3;
        std::vector<double>& recv = nt == 0 ? k.recv0[nnk - 1] : k.recv1[nnk - 1];
        for (int ipk = 0; ipk <= 1; ++ipk) {
          int istart = ipk * k.ijk[0][nnk - 1];
          if (k.nbc[nnk - 1][ipk] == BC_PERIODIC) {
            for (int kk = 0; kk <= k.ijk[2][nnk - 1]; ++kk) {
              int kpp = kk * (k.ijk[1][nnk - 1] + 1);
              for (int jj = 0; jj <= k.ijk[1][nnk - 1]; ++jj) {
                int jkk = kpp + jj;
                double f = rf[k.indx3(istart, jj, kk, nnk)];
                double* rv = &recv[jkk + (size_t)nb * ncomp * (ipk + 2 * (m - 1))];
                rv[0] = rv[0] + f * s.C.pbcot[0][nt];
                rv[(size_t)nb] = rv[(size_t)nb] + f * s.C.pbcot[1][nt];
                rv[(size_t)nb * (nt + 1)] = rv[(size_t)nb * (nt + 1)] + nt * f;
              }
            }
          }
        }
      }
    }
  }
}

// ---- t_numerics%deriv: src/mo_numerics.f90:709-886 --------------------------
// in/out: one column each (0:lmx); may alias (lines are gathered first).
void deriv(S& s, Block& k, const double* in, double* out, int nn, int m) {
  const int nstart = k.ndf[nn - 1][0][0], nend = k.ndf[nn - 1][1][0];
  int istart = nn == 1 ? 0 : nn == 2 ? k.lxi + 1 : k.lxi + k.let + 2;
  int iend = istart + k.ijk[0][nn - 1];
  const int nb = k.nbs[nn - 1];
  const std::vector<double>& recv = k.recv0[nn - 1];
  std::vector<double>& drva = k.drva[nn - 1];
  const int lim1 = k.lim + 1;
  const double* xu = k.xu.data();
  const double* xl = k.xl.data();
  const int nk = k.ijk[2][nn - 1] + 1, nj = k.ijk[1][nn - 1] + 1;
#pragma omp parallel
  {
    std::vector<double> sa(lim1), sb(lim1);
    std::vector<int> li(lim1);
#pragma omp for schedule(static)
    for (int kj = 0; kj < nk * nj; ++kj) {
      int kkk = kj / nj, jjj = kj % nj;
      int jkk = kkk * nj + jjj;
      for (int iii = istart; iii <= iend; ++iii) {
        int lll = k.indx3(iii - istart, jjj, kkk, nn);
        li[iii] = lll;
        sa[iii] = in[lll];
      }
      auto rv = [&](int c, int ip) { return recv[jkk + (size_t)nb * (c + 2 * (ip + 2 * (m - 1)))]; };
      if (nstart == 0) {
        int i0 = istart;
        sb[i0] = (((a01 * (sa[i0 + 1] - sa[i0]) + a02 * (sa[i0 + 2] - sa[i0])) + a03 * (sa[i0 + 3] - sa[i0])) +
                  a04 * (sa[i0 + 4] - sa[i0]));
        int i1 = istart + 1;
        sb[i1] = (((a10 * (sa[i0] - sa[i1]) + a12 * (sa[i0 + 2] - sa[i1])) + a13 * (sa[i0 + 3] - sa[i1])) +
                  a14 * (sa[i0 + 4] - sa[i1]));
      } else {
        double s0 = 0, s1 = 0;
        for (int i = 0; i <= lmd; ++i) s0 = s0 + s.C.pbci[i][0][0] * sa[istart + i];
        for (int i = 0; i <= lmd; ++i) s1 = s1 + s.C.pbci[i][1][0] * sa[istart + i];
        sb[istart] = s0 + rv(0, 0);
        sb[istart + 1] = s1 + rv(1, 0);
      }
      for (int iii = istart + 2; iii <= iend - 2; ++iii)
        sb[iii] = aa * (sa[iii + 1] - sa[iii - 1]) + ab * (sa[iii + 2] - sa[iii - 2]);
      if (nend == 0) {
        int e = iend;
        sb[e] = (((a01 * (sa[e] - sa[e - 1]) + a02 * (sa[e] - sa[e - 2])) + a03 * (sa[e] - sa[e - 3])) +
                 a04 * (sa[e] - sa[e - 4]));
        int e1 = iend - 1;
        sb[e1] = (((a10 * (sa[e1] - sa[e]) + a12 * (sa[e1] - sa[e - 2])) + a13 * (sa[e1] - sa[e - 3])) +
                  a14 * (sa[e1] - sa[e - 4]));
      } else {
        double s0 = 0, s1 = 0;
        for (int i = 0; i <= lmd; ++i) s0 = s0 + s.C.pbci[i][0][0] * sa[iend - i];
        for (int i = 0; i <= lmd; ++i) s1 = s1 + s.C.pbci[i][1][0] * sa[iend - i];
        sb[iend] = -s0 - rv(0, 1);
        sb[iend - 1] = -s1 - rv(1, 1);
      }
      sa[istart] = sb[istart];
      sa[istart + 1] = sb[istart + 1] - xl[istart + 1 + lim1] * sa[istart];
      for (int iii = istart + 2; iii <= iend; ++iii)
        sa[iii] = (sb[iii] - xl[iii] * sa[iii - 2]) - xl[iii + lim1] * sa[iii - 1];
      sb[iend] = xu[iend] * sa[iend];
      sb[iend - 1] = xu[iend - 1] * sa[iend - 1] - xu[iend - 1 + lim1] * sb[iend];
      for (int iii = iend - 2; iii >= istart; --iii)
        sb[iii] = (xu[iii] * sa[iii] - xu[iii + lim1] * sb[iii + 1]) - xu[iii + 2 * lim1] * sb[iii + 2];
      for (int iii = istart; iii <= iend; ++iii) out[li[iii]] = sb[iii];
      drva[jkk + (size_t)nb * ((m - 1) + 5 * 0)] = sb[istart];
      drva[jkk + (size_t)nb * ((m - 1) + 5 * 1)] = sb[iend];
    }
  }
}

// ---- t_numerics%filte: src/mo_numerics.f90:890-987 --------------------------
void filte(S& s, Block& k, double* rf, int inn, int m) {
  const int nn = nnf[inn - 1];
  const int nstart = k.ndf[nn - 1][0][1], nend = k.ndf[nn - 1][1][1];
  int istart = nn == 1 ? 0 : nn == 2 ? k.lxi + 1 : k.lxi + k.let + 2;
  int iend = istart + k.ijk[0][nn - 1];
  const int nb = k.nbs[nn - 1];
  const std::vector<double>& recv = k.recv1[nn - 1];
  const int lim1 = k.lim + 1;
  const double* yu = k.yu.data();
  const double* yl = k.yl.data();
  const double fa = s.C.fa, fb = s.C.fb, fc = s.C.fc;
  const int nk = k.ijk[2][nn - 1] + 1, nj = k.ijk[1][nn - 1] + 1;
#pragma omp parallel
  {
    std::vector<double> sa(lim1), sb(lim1);
    std::vector<int> li(lim1);
#pragma omp for schedule(static)
    for (int kj = 0; kj < nk * nj; ++kj) {
      int kkk = kj / nj, jjj = kj % nj;
      int jkk = kkk * nj + jjj;
      for (int iii = istart; iii <= iend; ++iii) {
        int lll = k.indx3(iii - istart, jjj, kkk, nn);
        li[iii] = lll;
        sa[iii] = rf[lll];
      }
      auto rv = [&](int c, int ip) { return recv[jkk + (size_t)nb * (c + 3 * (ip + 2 * (m - 1)))]; };
      const double(*fbc)[3] = s.C.fbc;
      if (nstart == 0) {
        int i = istart;
        sb[i] = ((((fbc[0][0] * (sa[i + 1] - sa[i]) + fbc[1][0] * (sa[i + 2] - sa[i])) +
                   fbc[2][0] * (sa[i + 3] - sa[i])) + fbc[3][0] * (sa[i + 4] - sa[i])) +
                 fbc[4][0] * (sa[i + 5] - sa[i]));
        int j = istart + 1;
        sb[j] = ((((fbc[0][1] * (sa[i] - sa[j]) + fbc[1][1] * (sa[i + 2] - sa[j])) +
                   fbc[2][1] * (sa[i + 3] - sa[j])) + fbc[3][1] * (sa[i + 4] - sa[j])) +
                 fbc[4][1] * (sa[i + 5] - sa[j]));
        int q = istart + 2;
        sb[q] = ((((fbc[0][2] * (sa[i] - sa[q]) + fbc[1][2] * (sa[i + 1] - sa[q])) +
                   fbc[2][2] * (sa[i + 3] - sa[q])) + fbc[3][2] * (sa[i + 4] - sa[q])) +
                 fbc[4][2] * (sa[i + 5] - sa[q]));
      } else {
        int i = istart;
        double ra2k = sa[i + 2] + sa[i + 2];
        double s0 = 0, s1 = 0;
        for (int c = 0; c <= lmf; ++c) s0 = s0 + s.C.pbci[c][0][1] * sa[i + c];
        for (int c = 0; c <= lmf; ++c) s1 = s1 + s.C.pbci[c][1][1] * sa[i + c];
        sb[i] = s0 + rv(0, 0);
        sb[i + 1] = s1 + rv(1, 0);
        sb[i + 2] = (fa * ((sa[i + 1] + sa[i + 3]) - ra2k) + fb * ((sa[i] + sa[i + 4]) - ra2k)) +
                    fc * ((rv(2, 0) + sa[i + 5]) - ra2k);
      }
      for (int iii = istart + 3; iii <= iend - 3; ++iii) {
        double resk = sa[iii] + sa[iii];
        sb[iii] = (fa * ((sa[iii - 1] + sa[iii + 1]) - resk) + fb * ((sa[iii - 2] + sa[iii + 2]) - resk)) +
                  fc * ((sa[iii - 3] + sa[iii + 3]) - resk);
      }
      if (nend == 0) {
        int e = iend;
        sb[e] = ((((fbc[0][0] * (sa[e - 1] - sa[e]) + fbc[1][0] * (sa[e - 2] - sa[e])) +
                   fbc[2][0] * (sa[e - 3] - sa[e])) + fbc[3][0] * (sa[e - 4] - sa[e])) +
                 fbc[4][0] * (sa[e - 5] - sa[e]));
        int j = iend - 1;
        sb[j] = ((((fbc[0][1] * (sa[e] - sa[j]) + fbc[1][1] * (sa[e - 2] - sa[j])) +
                   fbc[2][1] * (sa[e - 3] - sa[j])) + fbc[3][1] * (sa[e - 4] - sa[j])) +
                 fbc[4][1] * (sa[e - 5] - sa[j]));
        int q = iend - 2;
        sb[q] = ((((fbc[0][2] * (sa[e] - sa[q]) + fbc[1][2] * (sa[e - 1] - sa[q])) +
                   fbc[2][2] * (sa[e - 3] - sa[q])) + fbc[3][2] * (sa[e - 4] - sa[q])) +
                 fbc[4][2] * (sa[e - 5] - sa[q]));
      } else {
        int e = iend;
        double ra2k = sa[e - 2] + sa[e - 2];
        double s0 = 0, s1 = 0;
        for (int c = 0; c <= lmf; ++c) s0 = s0 + s.C.pbci[c][0][1] * sa[e - c];
        for (int c = 0; c <= lmf; ++c) s1 = s1 + s.C.pbci[c][1][1] * sa[e - c];
        sb[e] = s0 + rv(0, 1);
        sb[e - 1] = s1 + rv(1, 1);
        sb[e - 2] = (fa * ((sa[e - 3] + sa[e - 1]) - ra2k) + fb * ((sa[e - 4] + sa[e]) - ra2k)) +
                    fc * ((sa[e - 5] + rv(2, 1)) - ra2k);
      }
      sa[istart] = sb[istart];
      sa[istart + 1] = sb[istart + 1] - yl[istart + 1 + lim1] * sa[istart];
      for (int iii = istart + 2; iii <= iend; ++iii)
        sa[iii] = (sb[iii] - yl[iii] * sa[iii - 2]) - yl[iii + lim1] * sa[iii - 1];
      sb[iend] = yu[iend] * sa[iend];
      sb[iend - 1] = yu[iend - 1] * sa[iend - 1] - yu[iend - 1 + lim1] * sb[iend];
      for (int iii = iend - 2; iii >= istart; --iii)
        sb[iii] = (yu[iii] * sa[iii] - yu[iii + lim1] * sb[iii + 1]) - yu[iii + 2 * lim1] * sb[iii + 2];
      for (int iii = istart; iii <= iend; ++iii) rf[li[iii]] = rf[li[iii]] + sb[iii];
    }
  }
}

// ---- numerics initialisation (src/mo_numerics.f90:77-95, 136-175) ----------
void init_block_numerics(S& s, Block& k) {
  k.lim = (k.lxi + 1) + (k.let + 1) + (k.lze + 1) - 1;
  int lim1 = k.lim + 1;
  k.xu.assign(3 * lim1, 0); k.yu.assign(3 * lim1, 0);
  k.xl.assign(2 * lim1, 0); k.yl.assign(2 * lim1, 0);
  int ls[3] = {k.lxi, k.let, k.lze};
  int is = 0;
  for (int nn = 1; nn <= 3; ++nn) {
    int ie = is + ls[nn - 1];
    for (int ip = 0; ip <= 1; ++ip) {
      int np = k.nbc[nn - 1][ip];
      if (np == BC_NON_REFLECTIVE || np == BC_WALL_INVISCID || np == BC_WALL_VISCOUS || np == BC_INTER_CURV) {
        k.ndf[nn - 1][ip][0] = k.ndf[nn - 1][ip][1] = 0;
      } else {
        k.ndf[nn - 1][ip][0] = k.ndf[nn - 1][ip][1] = 1;
      }
    }
    penta(s.C, k.xu.data(), k.xl.data(), lim1, is, ie, k.ndf[nn - 1][0][0], k.ndf[nn - 1][1][0], 0);
    penta(s.C, k.yu.data(), k.yl.data(), lim1, is, ie, k.ndf[nn - 1][0][1], k.ndf[nn - 1][1][1], 1);
    is = ie + 1;
  }
  for (int d = 0; d < 3; ++d) {
    int nb = k.nbs[d];
    k.send0[d].assign((size_t)nb * 2 * 2, 0); k.send1[d].assign((size_t)nb * 3 * 2, 0);
    k.recv0[d].assign((size_t)nb * 2 * 2 * 5, 0); k.recv1[d].assign((size_t)nb * 3 * 2 * 5, 0);
    k.drva[d].assign((size_t)nb * 5 * 2, 0); k.drvb[d].assign((size_t)nb * 5 * 2, 0);
    k.cm[d].assign((size_t)nb * 3 * 2, 0);
  }
}

// ---- t_grid%grid_metrics: src/mo_grid.f90:52-189 ---------------------------
void grid_metrics(S& s) {
  const int nb = s.nblk();
  std::vector<std::vector<double>> rrk(nb), qok(nb), qak(nb), dek(nb);
  for (int b = 0; b < nb; ++b) {
    size_t L = s.B[b].L();
    rrk[b].assign(3 * L, 0); qok[b].assign(3 * L, 0); qak[b].assign(3 * L, 0); dek[b].assign(3 * L, 0);
  }
  std::vector<double*> cols(nb);
  std::vector<std::vector<double>>* dst[3] = {&qok, &qak, &dek};
  for (int m = 1; m <= 3; ++m) {
    for (int b = 0; b < nb; ++b) {
      size_t L = s.B[b].L();
      std::copy(s.B[b].xyz.begin() + (m - 1) * L, s.B[b].xyz.begin() + m * L, rrk[b].begin());
      cols[b] = rrk[b].data();
    }
    mpigo(s, cols.data(), 0, 1, 1, m, m);
    for (int b = 0; b < nb; ++b) {
      Block& k = s.B[b];
      size_t L = k.L();
      double* r = rrk[b].data();
      deriv(s, k, r, r + 2 * L, 3, m);
      deriv(s, k, r, r + 1 * L, 2, m);
      deriv(s, k, r, r, 1, m);
      (*dst[m - 1])[b] = rrk[b];
    }
  }
  for (int b = 0; b < nb; ++b) {
    Block& k = s.B[b];
    size_t L = k.L();
    k.xim.assign(3 * L, 0); k.etm.assign(3 * L, 0); k.zem.assign(3 * L, 0); k.yaco.assign(L, 0);
    const double *qo = qok[b].data(), *qa = qak[b].data(), *de = dek[b].data();
    for (size_t l = 0; l < L; ++l) {
      double q1 = qo[l], q2 = qo[l + L], q3 = qo[l + 2 * L];
      double a1 = qa[l], a2 = qa[l + L], a3 = qa[l + 2 * L];
      double d1 = de[l], d2 = de[l + L], d3 = de[l + 2 * L];
      k.xim[l] = a2 * d3 - d2 * a3;
      k.xim[l + L] = d2 * q3 - q2 * d3;
      k.xim[l + 2 * L] = q2 * a3 - a2 * q3;
      k.etm[l] = a3 * d1 - d3 * a1;
      k.etm[l + L] = d3 * q1 - q3 * d1;
      k.etm[l + 2 * L] = q3 * a1 - a3 * q1;
      k.zem[l] = a1 * d2 - d1 * a2;
      k.zem[l + L] = d1 * q2 - q1 * d2;
      k.zem[l + 2 * L] = q1 * a2 - a1 * q2;
    }
  }
  std::vector<double>* mets[3];
  for (int m = 1; m <= 3; ++m) {
    for (int w = 0; w < 3; ++w) {
      for (int inn = 1; inn <= 3; ++inn) {
        for (int b = 0; b < nb; ++b) {
          Block& k = s.B[b];
          mets[0] = &k.xim; mets[1] = &k.etm; mets[2] = &k.zem;
          cols[b] = mets[w]->data() + (size_t)(m - 1) * k.L();
        }
        mpigo(s, cols.data(), 1, 1, 0, 9 * (m - 1) + 3 * w + inn, m);
        for (int b = 0; b < nb; ++b) filte(s, s.B[b], cols[b], inn, m);
      }
    }
  }
  for (int b = 0; b < nb; ++b) {
    Block& k = s.B[b];
    size_t L = k.L();
    const double *qo = qok[b].data(), *qa = qak[b].data(), *de = dek[b].data();
    for (size_t l = 0; l < L; ++l) {
      double sum = qo[l] * k.xim[l];
      sum = sum + qo[l + L] * k.etm[l];
      sum = sum + qo[l + 2 * L] * k.zem[l];
      sum = sum + qa[l] * k.xim[l + L];
      sum = sum + qa[l + L] * k.etm[l + L];
      sum = sum + qa[l + 2 * L] * k.zem[l + L];
      sum = sum + de[l] * k.xim[l + 2 * L];
      sum = sum + de[l + L] * k.etm[l + 2 * L];
      sum = sum + de[l + 2 * L] * k.zem[l + 2 * L];
      k.yaco[l] = three / sum;
    }
    for (int nn = 1; nn <= 3; ++nn) {
      const std::vector<double>& met = nn == 1 ? k.xim : nn == 2 ? k.etm : k.zem;
      int nbsz = k.nbs[nn - 1];
      for (int ip = 0; ip <= 1; ++ip) {
        int i = ip * k.ijk[0][nn - 1];
        for (int kk = 0; kk <= k.ijk[2][nn - 1]; ++kk) {
          int kp = kk * (k.ijk[1][nn - 1] + 1);
          for (int j = 0; j <= k.ijk[1][nn - 1]; ++j) {
            int jk = kp + j;
            int l = k.indx3(i, j, kk, nn);
            double rv[3] = {k.yaco[l] * met[l], k.yaco[l] * met[l + L], k.yaco[l] * met[l + 2 * L]};
            double fctr = one / std::sqrt((rv[0] * rv[0] + rv[1] * rv[1]) + rv[2] * rv[2]);
            for (int d = 0; d < 3; ++d) k.cm[nn - 1][jk + (size_t)nbsz * (d + 3 * ip)] = fctr * rv[d];
          }
        }
      }
    }
  }
}

// ---- GCBC: src/mo_gcbc.f90 ---------------------------------------------------
struct Elem { double ao, aoi, ve[3], hv2, vn, vs; };

// src/mo_gcbc.f90:595-611
Elem eleme(const double cm[3], double qa1, const double qa24[3], double pp, const double umf[3]) {
  Elem e;
  double rhoi = one / qa1;
  e.ao = std::sqrt((gam * rhoi) * pp);
  e.aoi = one / e.ao;
  for (int d = 0; d < 3; ++d) e.ve[d] = rhoi * qa24[d];
  e.hv2 = half * ((e.ve[0] * e.ve[0] + e.ve[1] * e.ve[1]) + e.ve[2] * e.ve[2]);
  e.vn = (cm[0] * e.ve[0] + cm[1] * e.ve[1]) + cm[2] * e.ve[2];
  e.vs = (cm[0] * umf[0] + cm[1] * umf[1]) + cm[2] * umf[2];
  return e;
}

// src/mo_gcbc.f90:506-548 (xt row-major here: xt[r][c] = Fortran xt(r+1,c+1))
void xtq2r(const Elem& e, const double cm[3], double xt[5][5]) {
  double ho = (gamm1 * e.aoi) * e.aoi;
  double bo = 1 - ho * e.hv2;
  double co = e.aoi * e.vn;
  double dm[3], rv[3];
  for (int d = 0; d < 3; ++d) { dm[d] = e.aoi * cm[d]; rv[d] = ho * e.ve[d]; }
  const double* ve = e.ve;
  xt[0][0] = (bo * cm[0] + dm[1] * ve[2]) - dm[2] * ve[1];
  xt[0][1] = cm[0] * rv[0];
  xt[0][2] = cm[0] * rv[1] + dm[2];
  xt[0][3] = cm[0] * rv[2] - dm[1];
  xt[0][4] = -ho * cm[0];
  xt[1][0] = (bo * cm[1] + dm[2] * ve[0]) - dm[0] * ve[2];
  xt[1][1] = cm[1] * rv[0] - dm[2];
  xt[1][2] = cm[1] * rv[1];
  xt[1][3] = cm[1] * rv[2] + dm[0];
  xt[1][4] = -ho * cm[1];
  xt[2][0] = (bo * cm[2] + dm[0] * ve[1]) - dm[1] * ve[0];
  xt[2][1] = cm[2] * rv[0] + dm[1];
  xt[2][2] = cm[2] * rv[1] - dm[0];
  xt[2][3] = cm[2] * rv[2];
  xt[2][4] = -ho * cm[2];
  xt[3][0] = (one - bo) - co;
  xt[3][1] = dm[0] - rv[0];
  xt[3][2] = dm[1] - rv[1];
  xt[3][3] = dm[2] - rv[2];
  xt[3][4] = ho;
  xt[4][0] = (one - bo) + co;
  xt[4][1] = -dm[0] - rv[0];
  xt[4][2] = -dm[1] - rv[1];
  xt[4][3] = -dm[2] - rv[2];
  xt[4][4] = ho;
}

// src/mo_gcbc.f90:552-591
void xtr2q(const Elem& e, const double cm[3], double xt[5][5]) {
  double bo = e.hv2 + (hamm1 * e.ao) * e.ao;
  double co = e.ao * e.vn;
  double dm[3];
  for (int d = 0; d < 3; ++d) dm[d] = e.ao * cm[d];
  const double* ve = e.ve;
  xt[0][0] = cm[0]; xt[0][1] = cm[1]; xt[0][2] = cm[2]; xt[0][3] = half; xt[0][4] = half;
  xt[1][0] = cm[0] * ve[0];
  xt[1][1] = cm[1] * ve[0] - dm[2];
  xt[1][2] = cm[2] * ve[0] + dm[1];
  xt[1][3] = half * (ve[0] + dm[0]);
  xt[1][4] = xt[1][3] - dm[0];
  xt[2][0] = cm[0] * ve[1] + dm[2];
  xt[2][1] = cm[1] * ve[1];
  xt[2][2] = cm[2] * ve[1] - dm[0];
  xt[2][3] = half * (ve[1] + dm[1]);
  xt[2][4] = xt[2][3] - dm[1];
  xt[3][0] = cm[0] * ve[2] - dm[1];
  xt[3][1] = cm[1] * ve[2] + dm[0];
  xt[3][2] = cm[2] * ve[2];
  xt[3][3] = half * (ve[2] + dm[2]);
  xt[3][4] = xt[3][3] - dm[2];
  xt[4][0] = (e.hv2 * cm[0] + dm[2] * ve[1]) - dm[1] * ve[2];
  xt[4][1] = (e.hv2 * cm[1] + dm[0] * ve[2]) - dm[2] * ve[0];
  xt[4][2] = (e.hv2 * cm[2] + dm[1] * ve[0]) - dm[0] * ve[1];
  xt[4][3] = half * (bo + co);
  xt[4][4] = xt[4][3] - co;
}

inline void matvec5(const double xt[5][5], const double v[5], double r[5]) {
  for (int i = 0; i < 5; ++i) {
    double s = 0;
    for (int c = 0; c < 5; ++c) s = s + xt[i][c] * v[c];
    r[i] = s;
  }
}

inline bool is_gcbc(int np) {
  return np == BC_NON_REFLECTIVE || np == BC_WALL_INVISCID || np == BC_WALL_VISCOUS || np == BC_INTER_CURV;
}
inline bool is_avg(int np) { return np == BC_INTER_CURV || np == BC_INTER_STRAIGHT || np == BC_PERIODIC; }

// src/mo_gcbc.f90:40-131
void gcbc_init(S& s, Block& k) {
  const int mbci = 4;
  std::vector<double> cbca(16, 0.0), cbcs;
  auto Cb = [](int i, int j) { return (i - 1) + 4 * (j - 1); };
  cbca[Cb(1, 1)] = alpha01; cbca[Cb(1, 2)] = beta02;
  cbca[Cb(2, 1)] = one; cbca[Cb(2, 2)] = alpha12; cbca[Cb(2, 3)] = beta13;
  cbca[Cb(3, 1)] = alpha; cbca[Cb(3, 2)] = one; cbca[Cb(3, 3)] = alpha; cbca[Cb(3, 4)] = beta;
  for (int i = 4; i <= mbci; ++i) {
    cbca[Cb(i, i - 3)] = beta; cbca[Cb(i, i - 2)] = alpha; cbca[Cb(i, i - 1)] = one; cbca[Cb(i, i)] = alpha;
    if (i < mbci) cbca[Cb(i, i + 1)] = beta;
  }
  double rbci[4] = {one, alpha10, beta, zero};
  mtrxi(cbca, cbcs, 4);
  double sbci[4];
  for (int i = 1; i <= 4; ++i) {
    double sum = 0;
    for (int c = 1; c <= 4; ++c) sum = sum + cbcs[Cb(i, c)] * rbci[c - 1];
    sbci[i - 1] = -sum;
  }
  double fctr = pi / (mbci + 1);
  double res = zero;
  for (int i = 1; i <= mbci; ++i) {
    res = res + one;
    sbci[i - 1] = (half * sbci[i - 1]) * (one + std::cos(res * fctr));
  }
  size_t L = k.L();
  k.nrr.assign(L, 0); k.npex.assign(L, 0);
  std::vector<double> cnt(L, 0.0);
  std::vector<double> val;
  std::vector<int> pt;
  for (int nn = 1; nn <= 3; ++nn)
    for (int ip = 0; ip <= 1; ++ip) {
      int np = k.nbc[nn - 1][ip];
      int i = ip * k.ijk[0][nn - 1];
      int iq = 1 - 2 * ip;
      if (is_gcbc(np)) {
        for (int kk = 0; kk <= k.ijk[2][nn - 1]; ++kk)
          for (int j = 0; j <= k.ijk[1][nn - 1]; ++j) {
            int l = k.indx3(i, j, kk, nn);
            double r = one / k.yaco[l];
            cnt[l] = cnt[l] + one;
            val.push_back(r);
            pt.push_back(l);
            for (int ii = 1; ii <= mbci; ++ii) {
              int l2 = k.indx3(i + iq * ii, j, kk, nn);
              cnt[l2] = cnt[l2] + one;
              val.push_back(r * sbci[ii - 1]);
              pt.push_back(l2);
            }
          }
      }
      if (is_avg(np)) {
        for (int kk = 0; kk <= k.ijk[2][nn - 1]; ++kk)
          for (int j = 0; j <= k.ijk[1][nn - 1]; ++j) k.nrr[k.indx3(i, j, kk, nn)] = 1;
      }
    }
  for (size_t l = 0; l < L; ++l) k.nrr[l] = std::min(k.nrr[l] + k.npex[l], 1);
  k.sbcc.resize(val.size());
  for (size_t ll = 0; ll < val.size(); ++ll) k.sbcc[ll] = val[ll] / cnt[pt[ll]];
}

// src/mo_gcbc.f90:133-340 (setup, comm, update)
// part 0: the whole of gcbc_setup, gcbc_comm and gcbc_update; 1: setup only;
// 2: comm and update only (a test places ranks on several processes in between)
void gcbc_all(S& s, int nk_unused, double dt, int part = 0) {
  (void)nk_unused;
  // setup
  for (int b = 0; b < s.nblk() && part != 2; ++b) {
    Block& k = s.B[b];
    size_t L = k.L();
    for (int nn = 1; nn <= 3; ++nn) {
      int nb = k.nbs[nn - 1];
      for (int ip = 0; ip <= 1; ++ip) {
        int np = k.nbc[nn - 1][ip];
        int i = ip * k.ijk[0][nn - 1];
        if (!is_gcbc(np)) continue;
        double ra0 = (double)(((BC_WALL_INVISCID - np) * (BC_WALL_VISCOUS - np) * (BC_INTER_CURV - np)) / 3000);
        double ra1 = one - ra0;
        for (int kk = 0; kk <= k.ijk[2][nn - 1]; ++kk) {
          int kp = kk * (k.ijk[1][nn - 1] + 1);
          for (int j = 0; j <= k.ijk[1][nn - 1]; ++j) {
            int jk = kp + j;
            int l = k.indx3(i, j, kk, nn);
            double cm[3], qa24[3] = {k.qa[l + L], k.qa[l + 2 * L], k.qa[l + 3 * L]};
            for (int d = 0; d < 3; ++d) cm[d] = k.cm[nn - 1][jk + (size_t)nb * (d + 3 * ip)];
            Elem e = eleme(cm, k.qa[l], qa24, k.p[l], s.umf);
            double xt[5][5];
            xtq2r(e, cm, xt);
            double v[5], r[5];
            for (int c = 0; c < 5; ++c) {
              double cha = ra0 * k.drva[nn - 1][jk + (size_t)nb * (c + 5 * ip)] + ra1 * k.de[l + c * L];
              v[c] = k.yaco[l] * cha;
            }
            matvec5(xt, v, r);
            for (int c = 0; c < 5; ++c) k.drva[nn - 1][jk + (size_t)nb * (c + 5 * ip)] = r[c];
          }
        }
      }
    }
  }
  if (part == 1) return;
  s.call_hook(1, 0, 0);
  // comm (BC_INTER_CURV faces)
  MpiSim mpi;
  for (int b = 0; b < s.nblk(); ++b) {
    Block& k = s.B[b];
    for (int nn = 1; nn <= 3; ++nn) {
      int nb = k.nbs[nn - 1];
      for (int ip = 0; ip <= 1; ++ip) {
        int iq = 1 - ip;
        if (k.nbc[nn - 1][ip] != BC_INTER_CURV) continue;
        mpi.isend(b, k.mcd[nn - 1][ip], 30 + iq, &k.drva[nn - 1][(size_t)nb * 5 * ip], (size_t)5 * nb);
        mpi.irecv(b, k.mcd[nn - 1][ip], 30 + ip, &k.drvb[nn - 1][(size_t)nb * 5 * ip], (size_t)5 * nb);
      }
    }
  }
  mpi.waitall();
  // update
  for (int b = 0; b < s.nblk(); ++b) {
    Block& k = s.B[b];
    size_t L = k.L();
    int ll = -1;
    for (int nn = 1; nn <= 3; ++nn) {
      int nb = k.nbs[nn - 1];
      for (int ip = 0; ip <= 1; ++ip) {
        int np = k.nbc[nn - 1][ip];
        int i = ip * k.ijk[0][nn - 1];
        int iq = 1 - 2 * ip;
        double ra0 = iq;
        if (!is_gcbc(np)) continue;
        double dtwi = one / (nkrk * dt + sml);
        for (int kk = 0; kk <= k.ijk[2][nn - 1]; ++kk) {
          int kp = kk * (k.ijk[1][nn - 1] + 1);
          for (int j = 0; j <= k.ijk[1][nn - 1]; ++j) {
            int jk = kp + j;
            int l = k.indx3(i, j, kk, nn);
            double cm[3], qa24[3] = {k.qa[l + L], k.qa[l + 2 * L], k.qa[l + 3 * L]};
            for (int d = 0; d < 3; ++d) cm[d] = k.cm[nn - 1][jk + (size_t)nb * (d + 3 * ip)];
            Elem e = eleme(cm, k.qa[l], qa24, k.p[l], s.umf);
            double cha[5], dha[5], drv[5];
            for (int c = 0; c < 5; ++c) {
              drv[c] = k.drva[nn - 1][jk + (size_t)nb * (c + 5 * ip)];
              cha[c] = drv[c];
              dha[c] = k.drvb[nn - 1][jk + (size_t)nb * (c + 5 * ip)];
            }
            if (np == BC_NON_REFLECTIVE) {
              if (ra0 * ((e.vn + e.vs) + e.ao) > zero) cha[3] = zero;
              if (ra0 * ((e.vn + e.vs) - e.ao) > zero) cha[4] = zero;
            } else if (np == BC_WALL_INVISCID || np == BC_WALL_VISCOUS) {
              if (k.npex[l] == 0) {
                double sd = 0;
                for (int d = 0; d < 3; ++d) sd = sd + cm[d] * s.dudtmf[d];
                cha[3 + ip] = cha[4 - ip] + (((two * ra0) * e.aoi) * k.qa[l]) * (sd + dtwi * (e.vn + e.vs));
              }
            } else {  // BC_INTER_CURV
              if (ra0 * (e.vn + e.vs) > zero) { cha[0] = dha[0]; cha[1] = dha[1]; cha[2] = dha[2]; }
              if (ra0 * ((e.vn + e.vs) + e.ao) > zero) cha[3] = dha[3];
              if (ra0 * ((e.vn + e.vs) - e.ao) > zero) cha[4] = dha[4];
            }
            double xt[5][5], v[5];
            xtr2q(e, cm, xt);
            for (int c = 0; c < 5; ++c) v[c] = cha[c] - drv[c];
            matvec5(xt, v, dha);
            for (int ii = 0; ii <= 4; ++ii) {
              int l2 = k.indx3(i + iq * ii, j, kk, nn);
              ++ll;
              for (int c = 0; c < 5; ++c) k.de[l2 + c * L] = k.de[l2 + c * L] + k.sbcc[ll] * dha[c];
            }
          }
        }
      }
    }
  }
}

// src/mo_gcbc.f90:342-422
void average_surface(S& s) {
  s.call_hook(2, 2, 0);
  MpiSim mpi;
  for (int b = 0; b < s.nblk(); ++b) {
    Block& k = s.B[b];
    size_t L = k.L();
    for (int nn = 1; nn <= 3; ++nn) {
      int nb = k.nbs[nn - 1];
      for (int ip = 0; ip <= 1; ++ip) {
        int iq = 1 - ip;
        int np = k.nbc[nn - 1][ip];
        int i = ip * k.ijk[0][nn - 1];
        if (!is_avg(np)) continue;
        for (int kk = 0; kk <= k.ijk[2][nn - 1]; ++kk) {
          int kp = kk * (k.ijk[1][nn - 1] + 1);
          for (int j = 0; j <= k.ijk[1][nn - 1]; ++j) {
            int l = k.indx3(i, j, kk, nn);
            int jk = kp + j;
            for (int c = 0; c < 5; ++c) k.drva[nn - 1][jk + (size_t)nb * (c + 5 * ip)] = k.qa[l + c * L];
            k.rr[l] = one;
          }
        }
        mpi.isend(b, k.mcd[nn - 1][ip], 30 + iq, &k.drva[nn - 1][(size_t)nb * 5 * ip], (size_t)5 * nb);
        mpi.irecv(b, k.mcd[nn - 1][ip], 30 + ip, &k.drvb[nn - 1][(size_t)nb * 5 * ip], (size_t)5 * nb);
      }
    }
  }
  mpi.waitall();
  for (int b = 0; b < s.nblk(); ++b) {
    Block& k = s.B[b];
    size_t L = k.L();
    for (int nn = 1; nn <= 3; ++nn) {
      int nb = k.nbs[nn - 1];
      for (int ip = 0; ip <= 1; ++ip) {
        int np = k.nbc[nn - 1][ip];
        int i = ip * k.ijk[0][nn - 1];
        if (!is_avg(np)) continue;
        for (int kk = 0; kk <= k.ijk[2][nn - 1]; ++kk) {
          int kp = kk * (k.ijk[1][nn - 1] + 1);
          for (int j = 0; j <= k.ijk[1][nn - 1]; ++j) {
            int l = k.indx3(i, j, kk, nn);
            int jk = kp + j;
            k.rr[l] = k.rr[l] + k.nrr[l];
            k.rr[l + L] = k.nrr[l] / k.rr[l];
            for (int c = 0; c < 5; ++c)
              k.qa[l + c * L] = k.rr[l + L] * ((k.rr[l] - one) * k.qa[l + c * L] +
                                               k.drvb[nn - 1][jk + (size_t)nb * (c + 5 * ip)]) +
                                (double)(1 - k.nrr[l]) * k.qa[l + c * L];
          }
        }
      }
    }
  }
}

// src/mo_gcbc.f90:424-459
void wall_condition_update(S& s) {
  for (int b = 0; b < s.nblk(); ++b) {
    Block& k = s.B[b];
    size_t L = k.L();
    for (int nn = 1; nn <= 3; ++nn)
      for (int ip = 0; ip <= 1; ++ip) {
        int np = k.nbc[nn - 1][ip];
        int i = ip * k.ijk[0][nn - 1];
        if (np != BC_WALL_INVISCID && np != BC_WALL_VISCOUS) continue;
        for (int kk = 0; kk <= k.ijk[2][nn - 1]; ++kk)
          for (int j = 0; j <= k.ijk[1][nn - 1]; ++j) {
            int l = k.indx3(i, j, kk, nn);
            double* q = k.qa.data();
            double npx = k.npex[l];
            if (np == BC_WALL_INVISCID) {
              double ke = (q[l + L] * q[l + L] + q[l + 2 * L] * q[l + 2 * L]) + q[l + 3 * L] * q[l + 3 * L];
              q[l + 4 * L] = npx * q[l + 4 * L] +
                             (one - npx) * (hamhamm1 * std::pow(q[l], gam) + (half * ke) / q[l]);
            } else {
              double fctr = (one - npx) * q[l];
              for (int d = 0; d < 3; ++d) q[l + (d + 1) * L] = npx * q[l + (d + 1) * L] - fctr * s.umf[d];
              double ke = (q[l + L] * q[l + L] + q[l + 2 * L] * q[l + 2 * L]) + q[l + 3 * L] * q[l + 3 * L];
              q[l + 4 * L] = npx * q[l + 4 * L] + (one - npx) * (hamhamm1 * q[l] + (half * ke) / q[l]);
            }
          }
      }
  }
}

// ---- junction search and averaging: src/mo_domdcomp.f90:269-585 ----------------
// trimm: src/mo_domdcomp.f90:563-585
void trimm(std::vector<int>& it, int& lene, int lens) {
  for (int k = 0; k <= lens - 1; ++k)
    for (int kk = k + 1; kk <= lens; ++kk)
      if (it[kk] - it[k] == 0) it[kk] = -1;
  lene = lens;
  for (int k = 0; k <= lens; ++k)
    if (it[k] == -1) {
      lene = lene - 1;
      it[k] = it[k + 1];
      it[k + 1] = -1;
    }
}

int idsd3_rank(const Parent& p, const int* pos) {
  return p.mo + (pos[2] * p.nbpc[1] + pos[1]) * p.nbpc[0] + pos[0];
}

// rank of block mm's sub-domain at position (i along nn, j along nn+1, k
// along nn+2, cyclically): src/mo_domdcomp.f90:588-605
int idsd3(const S& s, int i, int j, int k, int mm, int nn) {
  const Parent& p = s.P[mm];
  int pos[3];
  pos[nn - 1] = i;
  pos[nn % 3] = j;
  pos[(nn + 1) % 3] = k;
  return p.mo + (pos[2] * p.nbpc[1] + pos[1]) * p.nbpc[0] + pos[0];
}

// search_point / search_line (src/mo_domdcomp.f90:269-437): the junctions of
// block corners / edges over the blocks' neighbour graph, then per rank the
// corners / edge segments it owns and the ranks owning the partners
void search_junctions(S& s, bool points) {
  const int mbki = (int)s.P.size() - 1;
  const int per = points ? 8 : 12;
  const int lp = per * mbki + per - 1;
  std::vector<int> imj(lp + 1, 0);
  std::vector<std::vector<int>> jj(lp + 1, std::vector<int>(102, -1));
  int ij[4][3][2];
  if (points) {
    for (int ip = 0; ip <= 1; ++ip) {
      int a[4] = {0, 2, 4, 6}, b2[4] = {0, 4, 1, 5}, c[4] = {0, 1, 2, 3};
      for (int i = 0; i < 4; ++i) {
        ij[i][0][ip] = a[i] + ip; ij[i][1][ip] = b2[i] + 2 * ip; ij[i][2][ip] = c[i] + 4 * ip;
      }
    }
  } else {
    int njl0[4] = {2, 2, 1, 1};
    for (int ip = 0; ip <= 1; ++ip) {
      int a[4] = {0, 1, 8, 10}, b2[4] = {4, 5, 0, 2}, c[4] = {8, 9, 4, 6};
      for (int i = 0; i < 4; ++i) {
        ij[i][0][ip] = a[i] + ip * njl0[i]; ij[i][1][ip] = b2[i] + ip * njl0[i]; ij[i][2][ip] = c[i] + ip * njl0[i];
      }
    }
  }
  for (int i = 0; i <= lp; ++i) jj[i][0] = i;
  for (int mm = 0; mm <= mbki; ++mm)
    for (int nn = 1; nn <= 3; ++nn)
      for (int ip = 0; ip <= 1; ++ip) {
        int mp = s.P[mm].mbcd[nn - 1][ip];
        if (mp == -1) continue;
        for (int i = 0; i <= 3; ++i) {
          int is = per * mm + ij[i][nn - 1][ip];
          int ie = per * mp + ij[i][nn - 1][1 - ip];
          imj[is] = imj[is] + 1;
          jj[is][imj[is]] = jj[ie][0];
        }
      }
  for (int i = 0; i <= lp; ++i)
    for (int j = 0; j <= lp; ++j) {
      int ll = 0;
      if ((i - j) * imj[i] * imj[j] != 0) {
        for (int k = 0; k <= imj[i]; ++k)
          for (int kk = 0; kk <= imj[j]; ++kk)
            if (jj[j][kk] - jj[i][k] == 0) ll = ll + 1;
        if (ll != 0) {
          int ks = imj[i] + 1;
          int ke = ks + imj[j];
          if (ke + 1 > 100) throw std::runtime_error("junction list overflow");
          for (int c = 0; c <= ke - ks; ++c) jj[i][ks + c] = jj[j][c];
          trimm(jj[i], imj[i], ke);
        }
      }
    }
  std::vector<int> tag(lp + 1);
  for (int i = 0; i <= lp; ++i) {
    int mn = jj[i][0];
    for (int c = 1; c <= imj[i]; ++c) mn = std::min(mn, jj[i][c]);
    tag[i] = mn;
  }
  for (int r = 0; r < s.nblk(); ++r) {
    Block& k = s.B[r];
    const int mb = k.mb;
    const Parent& pb = s.P[mb];
    if (points) {
      k.imjp = imj; k.jptag = tag; k.jjp = jj;
      for (int i = 0; i < 8; ++i) {
        k.njp[i] = -1;
        for (int c = 0; c < 101; ++c) k.jpcd[i][c] = -1;
      }
      for (int i = 0; i <= 7; ++i) {
        const int ip = i % 2, jp = (i % 4) / 2, kp = i / 4;
        const int l = 8 * mb + i;
        if (k.ijkp[0] == ip * (pb.nbpc[0] - 1) && k.ijkp[1] == jp * (pb.nbpc[1] - 1) &&
            k.ijkp[2] == kp * (pb.nbpc[2] - 1) && imj[l] >= 3) {
          k.njp[i] = l;
          for (int c = 1; c <= imj[l]; ++c) {
            const int mm = jj[l][c] / 8, j = jj[l][c] - 8 * mm;
            const Parent& pm = s.P[mm];
            k.jpcd[i][c] = idsd3(s, (j % 2) * (pm.nbpc[0] - 1), ((j % 4) / 2) * (pm.nbpc[1] - 1),
                                 (j / 4) * (pm.nbpc[2] - 1), mm, 1);
          }
        }
      }
    } else {
      k.imjl = imj; k.jltag = tag; k.jjl = jj;
      for (int i = 0; i < 12; ++i) {
        k.njl[i] = -1;
        for (int c = 0; c < 101; ++c) k.jlcd[i][c] = -1;
      }
      for (int i = 0; i <= 11; ++i) {
        const int nn = i / 4 + 1, ns = nn % 3 + 1, ne = ns % 3 + 1;
        const int ip = (i % 4) / 2, jp = (i % 4) % 2;
        const int l = 12 * mb + i;
        if (k.ijkp[nn - 1] == ip * (pb.nbpc[nn - 1] - 1) && k.ijkp[ns - 1] == jp * (pb.nbpc[ns - 1] - 1) &&
            imj[l] >= 2) {
          k.njl[i] = l;
          for (int c = 1; c <= imj[l]; ++c) {
            const int mm = jj[l][c] / 12, j = jj[l][c] - 12 * mm;
            const int np = j / 4 + 1, nq = np % 3 + 1;
            const Parent& pm = s.P[mm];
            k.jlcd[i][c] = idsd3(s, ((j % 4) / 2) * (pm.nbpc[np - 1] - 1), ((j % 4) % 2) * (pm.nbpc[nq - 1] - 1),
                                 k.ijkp[ne - 1], mm, np);
          }
        }
      }
    }
  }
}

// src/mo_domdcomp.f90:439-490
void average_point(S& s) {
  s.call_hook(2, 0, 0);
  MpiSim mpi;
  std::vector<std::vector<double>> r1(s.nblk()), r2(s.nblk());
  for (int b = 0; b < s.nblk(); ++b) {
    Block& k = s.B[b];
    r1[b].assign(8 * 5 + 5, 0); r2[b].assign(8 * 5 * 102, 0);
    size_t L = k.L();
    int lp = -5, lq = -5;
    for (int i = 0; i <= 7; ++i) {
      int ii = k.njp[i];
      if (ii == -1) continue;
      int itag = k.jptag[ii];
      int ip = i % 2, jp = (i % 4) / 2, kp = i / 4;
      lp += 5;
      int l = k.indx3(ip * k.lxi, jp * k.let, kp * k.lze, 1);
      for (int c = 0; c < 5; ++c) r1[b][lp + c] = k.qa[l + c * L];
      for (int j = 1; j <= k.imjp[ii]; ++j) {
        lq += 5;
        mpi.isend(b, k.jpcd[i][j], itag, &r1[b][lp], 5);
        mpi.irecv(b, k.jpcd[i][j], itag, &r2[b][lq], 5);
      }
    }
  }
  mpi.waitall();
  for (int b = 0; b < s.nblk(); ++b) {
    Block& k = s.B[b];
    size_t L = k.L();
    int lp = -5, lq = -5;
    for (int i = 0; i <= 7; ++i) {
      int ii = k.njp[i];
      if (ii == -1) continue;
      int ip = i % 2, jp = (i % 4) / 2, kp = i / 4;
      lp += 5;
      for (int j = 1; j <= k.imjp[ii]; ++j) {
        lq += 5;
        for (int c = 0; c < 5; ++c) r1[b][lp + c] = r1[b][lp + c] + r2[b][lq + c];
      }
      double fctr = one / (k.imjp[ii] + 1);
      int l = k.indx3(ip * k.lxi, jp * k.let, kp * k.lze, 1);
      for (int c = 0; c < 5; ++c) k.qa[l + c * L] = fctr * r1[b][lp + c];
    }
  }
}

// src/mo_domdcomp.f90:493-559
void average_line(S& s) {
  s.call_hook(2, 1, 0);
  MpiSim mpi;
  std::vector<std::vector<double>> r1(s.nblk()), r2(s.nblk());
  for (int b = 0; b < s.nblk(); ++b) {
    Block& k = s.B[b];
    size_t L = k.L();
    size_t cap = 0;
    for (int i = 0; i <= 11; ++i) {
      int ii = k.njl[i];
      if (ii == -1) continue;
      int nn = i / 4 + 1;
      cap += (size_t)5 * (k.ijk[2][nn - 1] + 1) * (k.imjl[ii] + 1);
    }
    r1[b].assign(cap + 5, 0); r2[b].assign(cap + 5, 0);
    int lp = 0, lq = 0;
    for (int i = 0; i <= 11; ++i) {
      int ii = k.njl[i];
      if (ii == -1) continue;
      int itag = k.jltag[ii];
      int nn = i / 4 + 1, ip = (i % 4) / 2, jp = (i % 4) % 2;
      int ks = lp, ke = ks + 5 * (k.ijk[2][nn - 1] + 1) - 1;
      lp = lp + ke - ks + 1;
      for (int kk = 0; kk <= k.ijk[2][nn - 1]; ++kk) {
        int ll = ks + 5 * kk;
        int l = k.indx3(ip * k.ijk[0][nn - 1], jp * k.ijk[1][nn - 1], kk, nn);
        for (int c = 0; c < 5; ++c) r1[b][ll + c] = k.qa[l + c * L];
      }
      for (int j = 1; j <= k.imjl[ii]; ++j) {
        int js = lq, je = js + ke - ks;
        lq = lq + je - js + 1;
        mpi.isend(b, k.jlcd[i][j], itag, &r1[b][ks], (size_t)(ke - ks + 1));
        mpi.irecv(b, k.jlcd[i][j], itag, &r2[b][js], (size_t)(je - js + 1));
      }
    }
  }
  mpi.waitall();
  for (int b = 0; b < s.nblk(); ++b) {
    Block& k = s.B[b];
    size_t L = k.L();
    int lp = 0, lq = 0;
    for (int i = 0; i <= 11; ++i) {
      int ii = k.njl[i];
      if (ii == -1) continue;
      int nn = i / 4 + 1, ip = (i % 4) / 2, jp = (i % 4) % 2;
      int ks = lp, ke = ks + 5 * (k.ijk[2][nn - 1] + 1) - 1;
      lp = lp + ke - ks + 1;
      for (int j = 1; j <= k.imjl[ii]; ++j) {
        int js = lq, je = js + ke - ks;
        lq = lq + je - js + 1;
        for (int c = 0; c <= ke - ks; ++c) r1[b][ks + c] = r1[b][ks + c] + r2[b][js + c];
      }
      double fctr = one / (k.imjl[ii] + 1);
      for (int kk = 0; kk <= k.ijk[2][nn - 1]; ++kk) {
        int ll = ks + 5 * kk;
        int l = k.indx3(ip * k.ijk[0][nn - 1], jp * k.ijk[1][nn - 1], kk, nn);
        for (int c = 0; c < 5; ++c) k.qa[l + c * L] = fctr * r1[b][ll + c];
      }
    }
  }
}

// ---- sponge: src/mo_sponge.f90:34-88 ---------------------------------------
inline double fmaxn(double a, double b) { return std::fmax(a, b); }
inline double fminn(double a, double b) { return std::fmin(a, b); }

void spongeup(S& s, Block& k) {
  size_t L = k.L();
  k.lcsz.clear(); k.asz.clear(); k.bsz.clear();
  const double ra2 = zero;
  const double tmpa = pi / s.cs.szth0, tmpb = pi / s.cs.szth1;
  for (size_t l = 0; l < L; ++l) {
    double x = k.xyz[l], y = k.xyz[l + L];
    double ra3 = ra2 * y;
    double ra0 = tmpa * (x - ((ra3 - s.cs.doml0) + s.cs.szth0));
    double ra1 = tmpb * (((ra3 + s.cs.doml1) - s.cs.szth1) - x);
    double c0 = std::cos(fmaxn(fminn(ra0, pi), zero));
    double c1 = std::cos(fmaxn(fminn(ra1, pi), zero));
    double d1 = (s.cs.szco * half) * ((two + c0) + c1);
    double d2 = (s.cs.szco * half) * (one + c0);
    if (d1 > sml) {
      k.lcsz.push_back((int)l);
      k.asz.push_back(d1 / k.yaco[l]);
      k.bsz.push_back(d2 / k.yaco[l]);
    }
  }
}

void spongego(S& s) {
  for (auto& k : s.B) {
    size_t L = k.L();
    for (size_t ll = 0; ll < k.lcsz.size(); ++ll) {
      int l = k.lcsz[ll];
      k.de[l] = k.de[l] + k.asz[ll] * (k.qa[l] - one);
      for (int d = 1; d <= 3; ++d) k.de[l + d * L] = k.de[l + d * L] + k.bsz[ll] * (k.qa[l + d * L] - zero);
      k.de[l + 4 * L] = k.de[l + 4 * L] + k.asz[ll] * (k.qa[l + 4 * L] - hamhamm1);
    }
  }
}

// ---- physics: src/mo_physics.f90 ----------------------------------------------
void movef(S& s, double dtko, double dtk) {  // src/mo_physics.f90:144-169
  if (s.cs.nsmf == 0) {
    double ra0 = pi / s.cs.timf;
    double ra1 = ra0 * std::min(s.timo, s.cs.timf);
    double ra2 = ra0 * std::min(s.timo + dtko, s.cs.timf);
    double fctr = one - std::cos(ra1);
    double dfdt = ra0 * std::sin(ra2);
    double progmf = half * (fctr + dtk * dfdt);
    for (int d = 0; d < 3; ++d) s.umf[d] = progmf * s.uoo[d];
    fctr = std::sin(ra1);
    dfdt = ra0 * std::cos(ra2);
    progmf = (half * ra0) * (fctr + dtk * dfdt);
    for (int d = 0; d < 3; ++d) s.dudtmf[d] = progmf * s.uoo[d];
  } else {
    for (int d = 0; d < 3; ++d) { s.umf[d] = s.uoo[d]; s.dudtmf[d] = zero; }
  }
}

void primitives(S& s) {  // src/mo_canard_driver.f90:267-275
  for (auto& k : s.B) {
    size_t L = k.L();
    double *q = k.qa.data(), *de = k.de.data();
#pragma omp parallel for schedule(static)
    for (long l = 0; l < (long)L; ++l) {
      de[l] = one / q[l];
      de[l + L] = q[l + L] * de[l];
      de[l + 2 * L] = q[l + 2 * L] * de[l];
      de[l + 3 * L] = q[l + 3 * L] * de[l];
      k.p[l] = gamm1 * (q[l + 4 * L] - half * ((q[l + L] * de[l + L] + q[l + 2 * L] * de[l + 2 * L]) +
                                               q[l + 3 * L] * de[l + 3 * L]));
      de[l + 4 * L] = (gam * k.p[l]) * de[l];
      k.ss[l] = (s.srefp1dre * std::pow(de[l + 4 * L], 1.5)) / (de[l + 4 * L] + s.srefoo);
    }
  }
}

void calc_time_step(S& s) {  // src/mo_physics.f90:171-211
  const int nb = s.nblk();
  std::vector<double> res(2 * nb, -1e300);  // per rank: res1, then res2
  for (int b = 0; b < nb; ++b) {
    Block& k = s.B[b];
    double res1 = -1e300, res2 = -1e300;
    size_t L = k.L();
    const double *de = k.de.data(), *xi = k.xim.data(), *et = k.etm.data(), *ze = k.zem.data();
    for (size_t l = 0; l < L; ++l) {
      double r1 = xi[l] * xi[l];
      r1 = r1 + xi[l + L] * xi[l + L];
      r1 = r1 + xi[l + 2 * L] * xi[l + 2 * L];
      r1 = r1 + et[l] * et[l];
      r1 = r1 + et[l + L] * et[l + L];
      r1 = r1 + et[l + 2 * L] * et[l + 2 * L];
      r1 = r1 + ze[l] * ze[l];
      r1 = r1 + ze[l + L] * ze[l + L];
      r1 = r1 + ze[l + 2 * L] * ze[l + 2 * L];
      double u = de[l + L] + s.umf[0], v = de[l + 2 * L] + s.umf[1], w = de[l + 3 * L] + s.umf[2];
      double r2 = std::fabs((xi[l] * u + xi[l + L] * v) + xi[l + 2 * L] * w) +
                  std::fabs((et[l] * u + et[l + L] * v) + et[l + 2 * L] * w);
      r2 = r2 + std::fabs((ze[l] * u + ze[l + L] * v) + ze[l + 2 * L] * w);
      double ssi = std::fabs(k.yaco[l]);
      res1 = std::max(res1, (std::sqrt(de[l + 4 * L] * r1) + r2) * ssi);
      if (s.cs.viscous) res2 = std::max(res2, (((de[l] * k.ss[l]) * r1) * ssi) * ssi);
    }
    res[b] = res1;
    res[nb + b] = res2;
  }
  s.call_hook(3, 0, 0, res.data(), nb);
  // the maximum does not depend on the order of the ranks
  double res1 = -1e300, res2 = -1e300;
  for (int b = 0; b < nb; ++b) {
    res1 = std::max(res1, res[b]);
    res2 = std::max(res2, res[nb + b]);
  }
  double ra0 = s.cs.cfl / res1;
  double ra1 = ra0;
  if (s.cs.viscous) ra1 = half / res2;
  s.dte = std::min(ra0, ra1);
}

void calc_viscous(S& s) {  // src/mo_physics.f90:216-301
  const int nb = s.nblk();
  std::vector<std::vector<double>> rr(nb);
  std::vector<double*> cols(nb);
  for (int b = 0; b < nb; ++b) {
    Block& k = s.B[b];
    size_t L = k.L();
    std::copy(k.ss.begin(), k.ss.begin() + L, k.de.begin());  // de(:,1) = ssk
    rr[b].assign(3 * L * 4, 0.0);  // rr(:,3,2:5)
  }
  for (int m = 2; m <= 5; ++m) {
    for (int b = 0; b < nb; ++b) {
      Block& k = s.B[b];
      size_t L = k.L();
      double* r = rr[b].data() + 3 * L * (m - 2);
      std::copy(k.de.begin() + (m - 1) * L, k.de.begin() + m * L, r);
      cols[b] = r;
    }
    mpigo(s, cols.data(), 0, 1, 0, m, m);
  }
  for (int b = 0; b < nb; ++b) {
    Block& k = s.B[b];
    size_t L = k.L();
    for (int m = 2; m <= 5; ++m) {
      double* r = rr[b].data() + 3 * L * (m - 2);
      deriv(s, k, r, r + 2 * L, 3, m);
      deriv(s, k, r, r + L, 2, m);
      deriv(s, k, r, r, 1, m);
    }
    const double *xi = k.xim.data(), *et = k.etm.data(), *ze = k.zem.data();
    std::vector<double> ssv(3 * L);
    auto comb = [&](const double* r, size_t l, int c) {
      return (xi[l + c * L] * r[l] + et[l + c * L] * r[l + L]) + ze[l + c * L] * r[l + 2 * L];
    };
    const double *r2 = rr[b].data(), *r3 = r2 + 3 * L, *r4 = r3 + 3 * L, *r5 = r4 + 3 * L;
#pragma omp parallel for schedule(static)
    for (long l = 0; l < (long)L; ++l) {
      k.txx[l] = comb(r2, l, 0); k.hzz[l] = comb(r2, l, 1); k.tzx[l] = comb(r2, l, 2);
      k.txy[l] = comb(r3, l, 0); k.tyy[l] = comb(r3, l, 1); k.hxx[l] = comb(r3, l, 2);
      k.hyy[l] = comb(r4, l, 0); k.tyz[l] = comb(r4, l, 1); k.tzz[l] = comb(r4, l, 2);
      ssv[l] = comb(r5, l, 0); ssv[l + L] = comb(r5, l, 1); ssv[l + 2 * L] = comb(r5, l, 2);
      double* de = k.de.data();
      double rr1 = de[l] * k.yaco[l];
      double rr2 = gamm1prndtli * rr1;
      de[l + 4 * L] = twothirds * ((k.txx[l] + k.tyy[l]) + k.tzz[l]);
      k.txx[l] = rr1 * ((k.txx[l] + k.txx[l]) - de[l + 4 * L]);
      k.tyy[l] = rr1 * ((k.tyy[l] + k.tyy[l]) - de[l + 4 * L]);
      k.tzz[l] = rr1 * ((k.tzz[l] + k.tzz[l]) - de[l + 4 * L]);
      k.txy[l] = rr1 * (k.txy[l] + k.hzz[l]);
      k.tyz[l] = rr1 * (k.tyz[l] + k.hxx[l]);
      k.tzx[l] = rr1 * (k.tzx[l] + k.hyy[l]);
      double u = de[l + L], v = de[l + 2 * L], w = de[l + 3 * L];
      k.hxx[l] = ((rr2 * ssv[l] + u * k.txx[l]) + v * k.txy[l]) + w * k.tzx[l];
      k.hyy[l] = ((rr2 * ssv[l + L] + u * k.txy[l]) + v * k.tyy[l]) + w * k.tyz[l];
      k.hzz[l] = ((rr2 * ssv[l + 2 * L] + u * k.tzx[l]) + v * k.tyz[l]) + w * k.tzz[l];
    }
  }
}

void calc_fluxes(S& s) {  // src/mo_physics.f90:306-402
  const int nb = s.nblk();
  std::vector<std::vector<double>> rr(nb);
  const bool visc = s.cs.viscous != 0;
  const double* umf = s.umf;
  for (int b = 0; b < nb; ++b) {
    Block& k = s.B[b];
    size_t L = k.L();
    rr[b].assign(3 * L * 5, 0.0);  // rr(:,3,5)
    double* R = rr[b].data();
    const double *q = k.qa.data(), *p = k.p.data();
    double* de = k.de.data();
    const double *xi = k.xim.data(), *et = k.etm.data(), *ze = k.zem.data();
#pragma omp parallel for schedule(static)
    for (long l = 0; l < (long)L; ++l) {
      double u = de[l + L] + umf[0], v = de[l + 2 * L] + umf[1], w = de[l + 3 * L] + umf[2];
      const double* mt[3] = {xi, et, ze};
      double ssd[3];
      for (int d = 0; d < 3; ++d) ssd[d] = (mt[d][l] * u + mt[d][l + L] * v) + mt[d][l + 2 * L] * w;
      for (int d = 0; d < 3; ++d) R[l + d * L + 0 * 3 * L] = q[l] * ssd[d];
      double tau[3][3] = {{k.txx[l], k.txy[l], k.tzx[l]}, {k.txy[l], k.tyy[l], k.tyz[l]}, {k.tzx[l], k.tyz[l], k.tzz[l]}};
      for (int c = 0; c < 3; ++c)
        for (int d = 0; d < 3; ++d) {
          double v1 = q[l + (c + 1) * L] * ssd[d] + mt[d][l + c * L] * p[l];
          if (visc) {
            v1 = v1 - mt[d][l] * tau[c][0];
            v1 = v1 - mt[d][l + L] * tau[c][1];
            v1 = v1 - mt[d][l + 2 * L] * tau[c][2];
          }
          R[l + d * L + (c + 1) * 3 * L] = v1;
        }
      de[l + 4 * L] = q[l + 4 * L] + p[l];
      for (int d = 0; d < 3; ++d) {
        double v1 = de[l + 4 * L] * ssd[d] -
                    p[l] * ((umf[0] * mt[d][l] + umf[1] * mt[d][l + L]) + umf[2] * mt[d][l + 2 * L]);
        if (visc) {
          v1 = v1 - mt[d][l] * k.hxx[l];
          v1 = v1 - mt[d][l + L] * k.hyy[l];
          v1 = v1 - mt[d][l + 2 * L] * k.hzz[l];
        }
        R[l + d * L + 4 * 3 * L] = v1;
      }
    }
  }
  std::vector<double*> cols(nb);
  for (int m = 1; m <= 5; ++m) {
    for (int b = 0; b < nb; ++b) cols[b] = rr[b].data() + 3 * s.B[b].L() * (m - 1);
    mpigo(s, cols.data(), 0, 0, 0, m, m);
  }
  for (int b = 0; b < nb; ++b) {
    Block& k = s.B[b];
    size_t L = k.L();
    for (int m = 1; m <= 5; ++m) {
      double* r = rr[b].data() + 3 * L * (m - 1);
      deriv(s, k, r, r, 1, m);
      deriv(s, k, r + L, r + L, 2, m);
      deriv(s, k, r + 2 * L, r + 2 * L, 3, m);
      double* de = k.de.data() + (m - 1) * L;
#pragma omp parallel for schedule(static)
      for (long l = 0; l < (long)L; ++l) de[l] = (r[l] + r[l + L]) + r[l + 2 * L];
    }
  }
}

void filter_all(S& s) {  // src/mo_canard_driver.f90:234-250
  const int nb = s.nblk();
  std::vector<double*> cols(nb);
  for (int m = 1; m <= 5; ++m)
    for (int inn = 1; inn <= 3; ++inn) {
      for (int b = 0; b < nb; ++b) cols[b] = s.B[b].qa.data() + (size_t)(m - 1) * s.B[b].L();
      mpigo(s, cols.data(), 1, 1, 0, 3 * (m - 1) + inn, m);
      for (int b = 0; b < nb; ++b) filte(s, s.B[b], cols[b], inn, m);
    }
}

void rk_update(S& s, double dtk) {  // src/mo_canard_driver.f90:329-334
  for (auto& k : s.B) {
    size_t L = k.L();
#pragma omp parallel for schedule(static)
    for (long l = 0; l < (long)L; ++l) {
      double r1 = dtk * k.yaco[l];
      for (int c = 0; c < 5; ++c) k.qa[l + c * L] = k.qo[l + c * L] - r1 * k.de[l + c * L];
    }
  }
}

int run_phase(S& s, int phase, int nk) {
  switch (phase) {
    case ORC_PH_FILTER: filter_all(s); break;
    case ORC_PH_COPYQO: for (auto& k : s.B) k.qo = k.qa; break;
    case ORC_PH_MOVEF_A: {
      double dtko = (s.dt * std::min(std::max(nk - 2, 0), 1)) / (nkrk - nk + 3);
      double dtk = (s.dt * std::min(nk - 1, 1)) / (nkrk - nk + 2);
      movef(s, dtko, dtk);
      break;
    }
    case ORC_PH_PRIM: primitives(s); break;
    case ORC_PH_TIMESTEP:
      if (nk == 1) {
        if (s.n % 10 == 1) {
          s.ndt = s.n;
          s.dts = s.dte;
          calc_time_step(s);
        }
        double sn = std::sin((0.05 * pi) * (s.n - s.ndt));
        s.dt = s.dts + (s.dte - s.dts) * (sn * sn);
      }
      break;
    case ORC_PH_VISCOUS: if (s.cs.viscous) calc_viscous(s); break;
    case ORC_PH_FLUXES: calc_fluxes(s); break;
    case ORC_PH_GCBC: gcbc_all(s, nk, s.dt); break;
    case ORC_PH_GCBC_SETUP: gcbc_all(s, nk, s.dt, 1); break;
    case ORC_PH_GCBC_COMM_UPDATE: gcbc_all(s, nk, s.dt, 2); break;
    case ORC_PH_SPONGE: spongego(s); break;
    case ORC_PH_RKUPDATE: {
      double dtko = (s.dt * std::min(nk - 1, 1)) / (nkrk - nk + 2);
      double dtk = s.dt / (nkrk - nk + 1);
      movef(s, dtko, dtk);
      rk_update(s, dtk);
      break;
    }
    case ORC_PH_WALL: wall_condition_update(s); break;
    case ORC_PH_AVERAGE:
      average_point(s);
      average_line(s);
      average_surface(s);
      break;
    case ORC_PH_ADVANCE:
      s.n = s.n + 1;
      s.timo = s.timo + s.dt;
      break;
    default: return -1;
  }
  return 0;
}

int one_step(S& s) {
  run_phase(s, ORC_PH_FILTER, 0);
  run_phase(s, ORC_PH_COPYQO, 0);
  for (int nk = 1; nk <= nkrk; ++nk) {
    run_phase(s, ORC_PH_MOVEF_A, nk);
    run_phase(s, ORC_PH_PRIM, nk);
    run_phase(s, ORC_PH_TIMESTEP, nk);
    run_phase(s, ORC_PH_VISCOUS, nk);
    run_phase(s, ORC_PH_FLUXES, nk);
    run_phase(s, ORC_PH_GCBC, nk);
    run_phase(s, ORC_PH_SPONGE, nk);
    run_phase(s, ORC_PH_RKUPDATE, nk);
    run_phase(s, ORC_PH_WALL, nk);
    run_phase(s, ORC_PH_AVERAGE, nk);
  }
  run_phase(s, ORC_PH_ADVANCE, 0);
  return 0;
}

}  // namespace

extern "C" {

int orc_coeffs(double fltk_nml, double fltrbc, double* o) {
  Coeffs C;
  init_coeffs(C, fltk_nml, fltrbc);
  int p = 0;
  for (int nt = 0; nt < 2; ++nt)
    for (int j = 0; j < 2; ++j)
      for (int i = 0; i < 12; ++i) o[p++] = C.pbci[i][j][nt];
  for (int nt = 0; nt < 2; ++nt)
    for (int j = 0; j < 2; ++j)
      for (int i = 0; i < 12; ++i) o[p++] = C.pbco[i][j][nt];
  for (int nt = 0; nt < 2; ++nt)
    for (int j = 0; j < 2; ++j) o[p++] = C.pbcot[j][nt];
  o[p++] = C.alphf; o[p++] = C.betf; o[p++] = C.fa; o[p++] = C.fb; o[p++] = C.fc;
  for (int n = 0; n < 2; ++n)
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k < 5; ++k) o[p++] = C.albef[k][r][n];
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 5; ++k) o[p++] = C.fbc[k][r];
  return p;
}

int orc_penta(double fltk_nml, double fltrbc, int n, int ns, int ne, int nt, double* xu, double* xl) {
  if (n < 8) return -1;
  Coeffs C;
  init_coeffs(C, fltk_nml, fltrbc);
  penta(C, xu, xl, n, 0, n - 1, ns, ne, nt);
  return 0;
}

void orc_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : 1);
#else
  (void)n;
#endif
}

orc_solver* orc_create(const orc_case_desc* c, const orc_block_desc* bd) {
  try {
    auto* s = new orc_solver();
    s->cs = *c;
    init_coeffs(s->C, c->fltk, c->fltrbc);
    // src/mo_physics.f90:101-111
    s->amachoo = std::sqrt((c->amach1 * c->amach1 + c->amach2 * c->amach2) + c->amach3 * c->amach3);
    s->reoo = c->reoo;
    if (s->amachoo > sml) s->reoo = s->reoo / s->amachoo;
    s->srefoo = 111 / c->tempoo;
    s->srefp1dre = (s->srefoo + one) / s->reoo;
    s->uoo[0] = c->amach1; s->uoo[1] = c->amach2; s->uoo[2] = c->amach3;
    s->B.resize(c->nblocks);
    for (int b = 0; b < c->nblocks; ++b) {
      Block& k = s->B[b];
      k.lxi = bd[b].lxi; k.let = bd[b].let; k.lze = bd[b].lze;
      for (int d = 0; d < 3; ++d)
        for (int ip = 0; ip < 2; ++ip) { k.nbc[d][ip] = bd[b].nbc[d][ip]; k.mcd[d][ip] = bd[b].mbcd[d][ip]; }
      k.lmx = (k.lxi + 1) * (k.let + 1) * (k.lze + 1) - 1;
      int I[3][3] = {{k.lxi, k.let, k.lze}, {k.let, k.lze, k.lxi}, {k.lze, k.lxi, k.let}};
      for (int nn = 0; nn < 3; ++nn)
        for (int a = 0; a < 3; ++a) k.ijk[a][nn] = I[nn][a];
      for (int nn = 0; nn < 3; ++nn) k.nbs[nn] = (k.ijk[1][nn] + 1) * (k.ijk[2][nn] + 1);
      init_block_numerics(*s, k);
      size_t L = k.L();
      k.qa.assign(5 * L, 0); k.qo.assign(5 * L, 0); k.de.assign(5 * L, 0);
      k.p.assign(L, 0); k.ss.assign(3 * L, 0); k.rr.assign(3 * L, 0);
      for (auto* v : {&k.txx, &k.tyy, &k.tzz, &k.txy, &k.tyz, &k.tzx, &k.hxx, &k.hyy, &k.hzz}) v->assign(L, 0);
      k.xyz.assign(3 * L, 0);
      k.mb = b;
    }
    // without orc_set_subdomains every rank is a block of its own (nbpc = 1)
    s->P.resize(c->nblocks);
    for (int b = 0; b < c->nblocks; ++b) {
      s->P[b].mo = b;
      for (int d = 0; d < 3; ++d)
        for (int ip = 0; ip < 2; ++ip) s->P[b].mbcd[d][ip] = bd[b].mbcd[d][ip];
    }
    return s;
  } catch (...) {
    return nullptr;
  }
}

void orc_destroy(orc_solver* s) { delete s; }

int orc_set_subdomains(orc_solver* s, int nblocks, const int32_t* nbpc, const int32_t* mbcd, const int32_t* sub) {
  if (!s || nblocks < 1 || !nbpc || !mbcd || !sub) return -1;
  std::vector<Parent> P(nblocks);
  int mo = 0;
  for (int m = 0; m < nblocks; ++m) {
    P[m].mo = mo;
    for (int d = 0; d < 3; ++d) {
      P[m].nbpc[d] = nbpc[3 * m + d];
      if (P[m].nbpc[d] < 1) return -1;
      for (int ip = 0; ip < 2; ++ip) P[m].mbcd[d][ip] = mbcd[6 * m + 2 * d + ip];
    }
    mo += P[m].nbpc[0] * P[m].nbpc[1] * P[m].nbpc[2];
  }
  if (mo != s->nblk()) return -1;  // one rank per sub-domain
  for (int r = 0; r < s->nblk(); ++r) {
    Block& k = s->B[r];
    k.mb = sub[4 * r];
    if (k.mb < 0 || k.mb >= nblocks) return -1;
    for (int d = 0; d < 3; ++d) {
      k.ijkp[d] = sub[4 * r + 1 + d];
      if (k.ijkp[d] < 0 || k.ijkp[d] >= P[k.mb].nbpc[d]) return -1;
    }
    if (idsd3_rank(P[k.mb], k.ijkp) != r) return -1;  // ranks numbered as domdcomp_init numbers them
  }
  s->P = P;
  return 0;
}

int orc_lmx(orc_solver* s, int b) { return s->B[b].lmx; }

int orc_set_grid(orc_solver* s, int b, const double* xyz) {
  if (b < 0 || b >= s->nblk()) return -1;
  std::copy(xyz, xyz + 3 * s->B[b].L(), s->B[b].xyz.begin());
  return 0;
}

int orc_setup(orc_solver* s) {
  try {
    grid_metrics(*s);
    for (auto& k : s->B) gcbc_init(*s, k);
    search_junctions(*s, true);
    search_junctions(*s, false);
    for (auto& k : s->B) spongeup(*s, k);
    return 0;
  } catch (std::exception& e) {
    std::fprintf(stderr, "orc_setup: %s\n", e.what());
    return -2;
  }
}

int orc_set_state(orc_solver* s, int b, const double* qa) {
  if (b < 0 || b >= s->nblk()) return -1;
  std::copy(qa, qa + 5 * s->B[b].L(), s->B[b].qa.begin());
  return 0;
}

static std::vector<double>* arr(orc_solver* s, int b, int which) {
  Block& k = s->B[b];
  switch (which) {
    case ORC_A_QA: return &k.qa;
    case ORC_A_QO: return &k.qo;
    case ORC_A_DE: return &k.de;
    case ORC_A_P: return &k.p;
    case ORC_A_SS1: return &k.ss;
    case ORC_A_XIM: return &k.xim;
    case ORC_A_ETM: return &k.etm;
    case ORC_A_ZEM: return &k.zem;
    case ORC_A_YACO: return &k.yaco;
    case ORC_A_DRVA1: return &k.drva[0];
    case ORC_A_DRVA2: return &k.drva[1];
    case ORC_A_DRVA3: return &k.drva[2];
    case ORC_A_CM1: return &k.cm[0];
    case ORC_A_CM2: return &k.cm[1];
    case ORC_A_CM3: return &k.cm[2];
    case ORC_A_SBCC: return &k.sbcc;
  }
  return nullptr;
}

long orc_get_array(orc_solver* s, int b, int which, double* out) {
  if (b < 0 || b >= s->nblk()) return -1;
  Block& k = s->B[b];
  size_t L = k.L();
  if (which == ORC_A_SS1) {
    if (out) std::copy(k.ss.begin(), k.ss.begin() + L, out);
    return (long)L;
  }
  if (which == ORC_A_TAU) {
    const std::vector<double>* v[9] = {&k.txx, &k.tyy, &k.tzz, &k.txy, &k.tyz, &k.tzx, &k.hxx, &k.hyy, &k.hzz};
    if (out)
      for (int i = 0; i < 9; ++i) std::copy(v[i]->begin(), v[i]->end(), out + i * L);
    return (long)(9 * L);
  }
  if (which == ORC_A_RECV0 || which == ORC_A_RECV1 || which == ORC_A_SEND1) {
    long p = 0;
    for (int d = 0; d < 3; ++d) {
      const std::vector<double>& v = which == ORC_A_RECV0 ? k.recv0[d] : which == ORC_A_RECV1 ? k.recv1[d] : k.send1[d];
      if (out) std::copy(v.begin(), v.end(), out + p);
      p += (long)v.size();
    }
    return p;
  }
  if (which == ORC_A_SPONGE) {
    if (out)
      for (size_t i = 0; i < k.lcsz.size(); ++i) {
        out[3 * i] = k.lcsz[i]; out[3 * i + 1] = k.asz[i]; out[3 * i + 2] = k.bsz[i];
      }
    return (long)(3 * k.lcsz.size());
  }
  std::vector<double>* v = arr(s, b, which);
  if (!v) return -2;
  if (out) std::copy(v->begin(), v->end(), out);
  return (long)v->size();
}

int orc_set_array(orc_solver* s, int b, int which, const double* in) {
  if (b < 0 || b >= s->nblk()) return -1;
  Block& k = s->B[b];
  if (which == ORC_A_SS1) {
    std::copy(in, in + k.L(), k.ss.begin());
    return 0;
  }
  if (which == ORC_A_TAU) {
    std::vector<double>* v[9] = {&k.txx, &k.tyy, &k.tzz, &k.txy, &k.tyz, &k.tzx, &k.hxx, &k.hyy, &k.hzz};
    for (int i = 0; i < 9; ++i) std::copy(in + i * k.L(), in + (i + 1) * k.L(), v[i]->begin());
    return 0;
  }
  if (which == ORC_A_SEND1 || which == ORC_A_RECV0 || which == ORC_A_RECV1) {
    std::vector<double>* v = which == ORC_A_SEND1 ? k.send1 : which == ORC_A_RECV0 ? k.recv0 : k.recv1;
    long p = 0;
    for (int d = 0; d < 3; ++d) {
      std::copy(in + p, in + p + v[d].size(), v[d].begin());
      p += (long)v[d].size();
    }
    return 0;
  }
  std::vector<double>* v = arr(s, b, which);
  if (!v) return -2;
  std::copy(in, in + v->size(), v->begin());
  return 0;
}

int orc_step(orc_solver* s, int nsteps) {
  try {
    for (int i = 0; i < nsteps; ++i) one_step(*s);
    return 0;
  } catch (std::exception& e) {
    std::fprintf(stderr, "orc_step: %s\n", e.what());
    return -2;
  }
}

void orc_set_hook(orc_solver* s, orc_hook_fn fn, void* user) {
  s->hook = fn;
  s->hook_user = user;
}

int orc_phase(orc_solver* s, int phase, int nk) {
  try {
    return run_phase(*s, phase, nk);
  } catch (std::exception& e) {
    std::fprintf(stderr, "orc_phase: %s\n", e.what());
    return -2;
  }
}

int orc_get_time(orc_solver* s, double* o) {
  o[0] = s->n; o[1] = s->ndt; o[2] = s->dt; o[3] = s->dts; o[4] = s->dte; o[5] = s->timo;
  return 0;
}
int orc_set_time(orc_solver* s, const double* in) {
  s->n = (int)in[0]; s->ndt = (int)in[1]; s->dt = in[2]; s->dts = in[3]; s->dte = in[4]; s->timo = in[5];
  return 0;
}

int orc_mpigo(orc_solver* s, double* const* fields, int ncols, int nt, int nrt, int n45, int itag, int m) {
  (void)ncols;
  try {
    mpigo(*s, fields, nt, nrt, n45, itag, m);
    return 0;
  } catch (std::exception& e) {
    std::fprintf(stderr, "orc_mpigo: %s\n", e.what());
    return -2;
  }
}

int orc_deriv(orc_solver* s, int b, const double* in, double* out, int nn, int m) {
  if (b < 0 || b >= s->nblk() || nn < 1 || nn > 3 || m < 1 || m > 5) return -1;
  deriv(*s, s->B[b], in, out, nn, m);
  return 0;
}

int orc_filte(orc_solver* s, int b, double* f, int inn, int m) {
  if (b < 0 || b >= s->nblk() || inn < 1 || inn > 3 || m < 1 || m > 5) return -1;
  filte(*s, s->B[b], f, inn, m);
  return 0;
}

}  // extern "C"
