// Host-side set-up of the Canard hot path (see host.h). Compiled without FMA
// contraction so every coefficient rounds exactly like the reference's
// double-precision statements.
#include "host.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <stdexcept>
#include <tuple>

namespace canard {
namespace {

const double kPi = std::acos(-1.0);
// src/mo_parameters.f90:52-70
const double kAlpha = 4 / 9.0, kBeta = 1 / 36.0, kAa = 20 / 27.0, kAb = 25 / 216.0;
const double kAlpha10 = 0.09166666665902128, kAlpha12 = 1.3500000000438646, kBeta13 = 0.2666666666794667;
const double kA10 = -0.3506944444280639, kA12 = 0.8249999999974599, kA13 = 0.7444444444773477,
             kA14 = 0.014583333334139971;
const double kAlpha01 = 8.000000000449464, kBeta02 = 6.000000000542, kA01 = -6.666666667794732,
             kA02 = 9.000000000052879, kA03 = 1.333333333178555, kA04 = -0.0833333333455545;

// Dense n x n matrix, row-major, 0-based.
struct Mat {
  int n;
  std::vector<double> a;
  explicit Mat(int n_) : n(n_), a((size_t)n_ * n_, 0.0) {}
  double& operator()(int r, int c) { return a[(size_t)r * n + c]; }
  double operator()(int r, int c) const { return a[(size_t)r * n + c]; }
};

// Gauss-Jordan inversion with partial pivoting, column by column in place,
// followed by the column permutation of the pivots (src/mo_utils.f90:15-50).
Mat invert(const Mat& A) {
  const int n = A.n;
  Mat R = A;
  std::vector<int> perm(n);
  for (int i = 0; i < n; ++i) perm[i] = i;
  std::vector<double> col(n);
  for (int p = 0; p < n; ++p) {
    int piv = p;
    for (int r = p + 1; r < n; ++r)
      if (std::fabs(R(r, p)) > std::fabs(R(piv, p))) piv = r;
    if (piv != p) {
      std::swap(perm[piv], perm[p]);
      for (int c = 0; c < n; ++c) std::swap(R(piv, c), R(p, c));
    }
    const double inv = 1.0 / R(p, p);
    for (int r = 0; r < n; ++r) col[r] = R(r, p);
    for (int c = 0; c < n; ++c) {
      const double f = inv * R(p, c);
      for (int r = 0; r < n; ++r) R(r, c) = R(r, c) - f * col[r];
      R(p, c) = f;
    }
    for (int r = 0; r < n; ++r) R(r, p) = -inv * col[r];
    R(p, p) = inv;
  }
  Mat S(n);
  for (int c = 0; c < n; ++c)
    for (int r = 0; r < n; ++r) S(r, perm[c]) = R(r, c);
  return S;
}

Mat matmul(const Mat& A, const Mat& B) {
  const int n = A.n;
  Mat C(n);
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < n; ++c) {
      double s = 0.0;
      for (int k = 0; k < n; ++k) s = s + A(r, k) * B(k, c);
      C(r, c) = s;
    }
  return C;
}

// Interior filter coefficients for cut-off fltk (src/mo_numerics.f90:306-326).
void filter_interior(double fltk, double fltr, double& al, double& be, double& za, double& zb, double& zc) {
  const double c1 = std::cos(fltk), c2 = std::cos(2 * fltk), c3 = std::cos(3 * fltk);
  const double den = ((30 + (5 * (7 - 16 * fltr)) * c1) + (2 * (1 + 8 * fltr)) * c2) - 3 * c3;
  const double f = 1 / den;
  al = f * (((20 * (2 * fltr - 1) - 30 * c1) + (12 * (2 * fltr - 1)) * c2) - 2 * c3);
  be = (0.5 * f) * (((2 * (13 - 8 * fltr) + (33 - 48 * fltr) * c1) + 6 * c2) - c3);
  const double ch = std::cos(0.5 * fltk);
  const double ch2 = ch * ch;
  za = ((60 * (1 - fltr)) * (ch2 * ch2)) * f;
  zb = (-2 * za) / 5;
  zc = za / 15;
}

inline double sum5(const double* v) { return (((v[0] + v[1]) + v[2]) + v[3]) + v[4]; }

}  // namespace

void Scheme::build(double fltk_nml, double fltrbc) {
  const double fltk = kPi * fltk_nml;
  *this = Scheme();
  // boundary filter rows (src/mo_numerics.f90:253-302)
  double al, be, za, zb, zc;
  filter_interior(fltk, 0.5, al, be, za, zb, zc);
  const double lg = std::log(fltrbc);
  const double f0 = 1.0 / ((1.0 + al * fltrbc) + be * (fltrbc * fltrbc));
  const double row0[5] = {0.0, 0.0, 1.0, al * f0, be * f0};
  double r = ((fltrbc - 1) * ((za + zc) + (fltrbc + 1) * (zb + fltrbc * zc))) / lg;
  const double c0[5] = {za - (5 * r) / 3, zb + (10 * r) / 21, zc - (5 * r) / 42, (5 * r) / 252, (-r) / 630};
  const double row1[5] = {0.0, al + be * fltrbc, 1.0, al, be};
  r = ((fltrbc - 1) * (zb + zc * (fltrbc + 1))) / lg;
  const double c1[5] = {((za + zb) + zc) + (1627 * r) / 1260, za + (10 * r) / 21, zb - (5 * r) / 42,
                        zc + (5 * r) / 252, (-r) / 630};
  const double row2[5] = {be, al, 1.0, al, be};
  r = (zc * (fltrbc - 1)) / lg;
  const double c2[5] = {(zb + zc) + (1627 * r) / 1260, za - (5 * r) / 3, za - (5 * r) / 42,
                        zb + (5 * r) / 252, zc - r / 630};
  for (int k = 0; k < 5; ++k) {
    albef[0][0][k] = row0[k]; albef[0][1][k] = row1[k]; albef[0][2][k] = row2[k];
    fbc[0][k] = c0[k] * f0; fbc[1][k] = c1[k]; fbc[2][k] = c2[k];
  }
  filter_interior(fltk, 0.5, alphf, betf, fa, fb, fc);
  const double i0[5] = {0.0, 0.0, 1.0, alphf, betf}, i1[5] = {0.0, alphf, 1.0, alphf, betf},
               i2[5] = {betf, alphf, 1.0, alphf, betf};
  for (int k = 0; k < 5; ++k) { albef[1][0][k] = i0[k]; albef[1][1][k] = i1[k]; albef[1][2][k] = i2[k]; }

  // Interface (quasi-disjoint) closures, src/mo_numerics.f90:330-425: the
  // 24-point operator spanning an interface, inverted, re-multiplied by its
  // decoupled left-hand side; rows 13 and 14 give the coupling coefficients.
  for (int nt = 0; nt < 2; ++nt) {
    const int n = 24;
    Mat A(n), B(n);
    if (nt == 0) {
      A(0, 0) = 1.0; A(0, 1) = kAlpha01; A(0, 2) = kBeta02;
      const double b0[5] = {-(((kA01 + kA02) + kA03) + kA04), kA01, kA02, kA03, kA04};
      const double a1[4] = {kAlpha10, 1.0, kAlpha12, kBeta13};
      const double b1[5] = {kA10, -(((kA10 + kA12) + kA13) + kA14), kA12, kA13, kA14};
      for (int k = 0; k < 5; ++k) { B(0, k) = b0[k]; B(1, k) = b1[k]; }
      for (int k = 0; k < 4; ++k) A(1, k) = a1[k];
      for (int i = 2; i <= n - 3; ++i) {
        const double ar[5] = {kBeta, kAlpha, 1.0, kAlpha, kBeta}, br[5] = {-kAb, -kAa, 0.0, kAa, kAb};
        for (int k = 0; k < 5; ++k) { A(i, i - 2 + k) = ar[k]; B(i, i - 2 + k) = br[k]; }
      }
      for (int k = 0; k < 4; ++k) A(n - 2, n - 1 - k) = A(1, k);
      for (int k = 0; k < 5; ++k) B(n - 2, n - 1 - k) = -B(1, k);
      for (int k = 0; k < 3; ++k) A(n - 1, n - 1 - k) = A(0, k);
      for (int k = 0; k < 5; ++k) B(n - 1, n - 1 - k) = -B(0, k);
    } else {
      for (int k = 0; k < 3; ++k) A(0, k) = albef[0][0][k + 2];
      for (int k = 0; k < 5; ++k) B(0, 1 + k) = fbc[0][k];
      B(0, 0) = -sum5(fbc[0]);
      for (int k = 0; k < 4; ++k) A(1, k) = albef[0][1][k + 1];
      const int o1[5] = {0, 2, 3, 4, 5}, o2[5] = {0, 1, 3, 4, 5};
      for (int k = 0; k < 5; ++k) B(1, o1[k]) = fbc[1][k];
      B(1, 1) = -sum5(fbc[1]);
      for (int k = 0; k < 5; ++k) A(2, k) = albef[0][2][k];
      for (int k = 0; k < 5; ++k) B(2, o2[k]) = fbc[2][k];
      B(2, 2) = -sum5(fbc[2]);
      for (int i = 3; i <= n - 4; ++i) {
        const double ar[5] = {betf, alphf, 1.0, alphf, betf};
        const double br[7] = {fc, fb, fa, -2 * ((fa + fb) + fc), fa, fb, fc};
        for (int k = 0; k < 5; ++k) A(i, i - 2 + k) = ar[k];
        for (int k = 0; k < 7; ++k) B(i, i - 3 + k) = br[k];
      }
      for (int k = 0; k < 5; ++k) A(n - 3, n - 1 - k) = A(2, k);
      for (int k = 0; k < 6; ++k) B(n - 3, n - 1 - k) = B(2, k);
      for (int k = 0; k < 4; ++k) A(n - 2, n - 1 - k) = A(1, k);
      for (int k = 0; k < 6; ++k) B(n - 2, n - 1 - k) = B(1, k);
      for (int k = 0; k < 3; ++k) A(n - 1, n - 1 - k) = A(0, k);
      for (int k = 0; k < 6; ++k) B(n - 1, n - 1 - k) = B(0, k);
    }
    Mat Ainv = invert(A);
    Mat D = A;  // decoupled left-hand side
    int i = n / 2 - 2;  // 1-based n/2-1
    D(i, i + 2) = 0; D(i + 1, i + 2) = 0; D(i + 1, i + 3) = 0;
    i = n / 2 + 1;      // 1-based n/2+2
    D(i, i - 2) = 0; D(i - 1, i - 2) = 0; D(i - 1, i - 3) = 0;
    Mat P = matmul(D, matmul(Ainv, B));
    for (int side = 0; side < 2; ++side) {
      const int row = n / 2 + side;  // 1-based n/2+1, n/2+2
      for (int c = 0; c < 12; ++c) {
        pbco[nt][side][11 - c] = P(row, c);
        pbci[nt][side][c] = P(row, 12 + c);
      }
    }
    for (int side = 0; side < 2; ++side) {
      double s = 0;
      for (int c = 0; c < 12; ++c) s = s + pbco[nt][side][c];
      pbcot[nt][side] = s;
    }
  }
}

// Pentadiagonal LU with pre-inverted pivots (src/mo_numerics.f90:179-249).
void Scheme::lu(int n, int ns, int ne, int nt, double* o) const {
  double* l1 = o;
  double* l2 = o + n;
  double* u1 = o + 2 * n;
  double* u2 = o + 3 * n;
  double* u3 = o + 4 * n;
  double rows[2][3][5];  // [closure kind][row][k+2]
  double ai, bi;
  if (nt == 0) {
    const double t[2][3][5] = {{{0, 0, 1, kAlpha01, kBeta02}, {0, kAlpha10, 1, kAlpha12, kBeta13},
                                {kBeta, kAlpha, 1, kAlpha, kBeta}},
                               {{0, 0, 1, kAlpha, kBeta}, {0, kAlpha, 1, kAlpha, kBeta},
                                {kBeta, kAlpha, 1, kAlpha, kBeta}}};
    std::memcpy(rows, t, sizeof(rows));
    ai = kAlpha; bi = kBeta;
  } else {
    std::memcpy(rows, albef, sizeof(rows));
    ai = alphf; bi = betf;
  }
  auto R = [&](int kind, int row, int k) { return rows[kind][row][k + 2]; };
  for (int i = 0; i < n; ++i) { l1[i] = l2[i] = 1.0; u1[i] = u2[i] = u3[i] = 1.0; }
  const int e = n - 1;
  u1[0] = 1.0; u2[0] = R(ns, 0, 1); u3[0] = R(ns, 0, 2);
  l2[1] = R(ns, 1, -1) * u1[0];
  u1[1] = 1.0 / (1.0 - u2[0] * l2[1]);
  u2[1] = R(ns, 1, 1) - u3[0] * l2[1];
  u3[1] = R(ns, 1, 2);
  auto row = [&](int i, double sub2, double sub1, double sup1) {
    l1[i] = sub2 * u1[i - 2];
    l2[i] = (sub1 - u2[i - 2] * l1[i]) * u1[i - 1];
    u1[i] = 1.0 / ((1.0 - u3[i - 2] * l1[i]) - u2[i - 1] * l2[i]);
    u2[i] = sup1 - u3[i - 1] * l2[i];
  };
  row(2, R(ns, 2, -2), R(ns, 2, -1), R(ns, 2, 1));
  u3[2] = R(ns, 2, 2);
  for (int i = 3; i <= e - 3; ++i) {
    row(i, bi, ai, ai);
    u3[i] = bi;
  }
  row(e - 2, R(ne, 2, 2), R(ne, 2, 1), R(ne, 2, -1));
  u3[e - 2] = R(ne, 2, -2);
  row(e - 1, R(ne, 1, 2), R(ne, 1, 1), R(ne, 1, -1));
  {  // last row: no super-diagonals
    const int i = e;
    l1[i] = R(ne, 0, 2) * u1[i - 2];
    l2[i] = (R(ne, 0, 1) - u2[i - 2] * l1[i]) * u1[i - 1];
    u1[i] = 1.0 / ((1.0 - u3[i - 2] * l1[i]) - u2[i - 1] * l2[i]);
  }
  for (int i = 0; i < n; ++i) {
    u2[i] = u2[i] * u1[i];
    u3[i] = u3[i] * u1[i];
  }
}

void Scheme::pack150(double* o) const {
  int p = 0;
  for (int nt = 0; nt < 2; ++nt)
    for (int s = 0; s < 2; ++s)
      for (int i = 0; i < 12; ++i) o[p++] = pbci[nt][s][i];
  for (int nt = 0; nt < 2; ++nt)
    for (int s = 0; s < 2; ++s)
      for (int i = 0; i < 12; ++i) o[p++] = pbco[nt][s][i];
  for (int nt = 0; nt < 2; ++nt)
    for (int s = 0; s < 2; ++s) o[p++] = pbcot[nt][s];
  o[p++] = alphf; o[p++] = betf; o[p++] = fa; o[p++] = fb; o[p++] = fc;
  for (int n = 0; n < 2; ++n)
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k < 5; ++k) o[p++] = albef[n][r][k];
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 5; ++k) o[p++] = fbc[r][k];
}

void make_geom(const canard_block_desc& d, int case_id, int bic, BlockGeom& g) {
  g.lxi = d.lxi; g.let = d.let; g.lze = d.lze;
  g.X = d.lxi + 1; g.Y = d.let + 1; g.Z = d.lze + 1;
  g.Xp = (g.X + 3) / 4 * 4;
  g.npad = (int64_t)g.Xp * g.Y * g.Z;
  for (int a = 0; a < 3; ++a)
    for (int s = 0; s < 2; ++s) { g.nbc[a][s] = d.nbc[a][s]; g.nbr[a][s] = d.mbcd[a][s]; }
  const int I[3][3] = {{g.lxi, g.let, g.lze}, {g.let, g.lze, g.lxi}, {g.lze, g.lxi, g.let}};
  for (int nn = 0; nn < 3; ++nn)
    for (int a = 0; a < 3; ++a) g.ijk[a][nn] = I[nn][a];
  for (int nn = 0; nn < 3; ++nn) g.nbs[nn] = (g.ijk[1][nn] + 1) * (g.ijk[2][nn] + 1);
  g.case_id = case_id;
  g.block_in_case = bic;
}

namespace {
// Message matching with MPI's non-overtaking rule: the k-th receive posted at
// `dst` for (src, tag) takes the k-th message `src` sent to `dst` with that tag.
struct Matcher {
  struct Msg { int src, dst, tag; int64_t id; };
  std::vector<Msg> sends, recvs;
  void send(int src, int dst, int tag, int64_t id) { sends.push_back({src, dst, tag, id}); }
  void recv(int me, int src, int tag, int64_t id) { recvs.push_back({src, me, tag, id}); }
  // result[i] = id of the send matched by recvs[i]
  std::vector<int64_t> match(std::string& err) const {
    std::map<std::tuple<int, int, int>, std::deque<int64_t>> q;
    for (const auto& s : sends) q[std::make_tuple(s.src, s.dst, s.tag)].push_back(s.id);
    std::vector<int64_t> out;
    for (const auto& r : recvs) {
      auto& d = q[std::make_tuple(r.src, r.dst, r.tag)];
      if (d.empty()) { err = "exchange: a receive has no matching send"; return {}; }
      out.push_back(d.front());
      d.pop_front();
    }
    return out;
  }
};
}  // namespace

std::string face_links(const std::vector<BlockGeom>& B, std::vector<FaceLink>& out) {
  // Pattern of the mpigo / gcbc_comm / average_surface exchanges: a face sends
  // with tag base+(1-side) and receives with tag base+side.
  Matcher M;
  auto id = [](int b, int nn, int s) { return (int64_t)(b * 3 + nn) * 2 + s; };
  for (int b = 0; b < (int)B.size(); ++b)
    for (int nn = 0; nn < 3; ++nn)
      for (int s = 0; s < 2; ++s) {
        const int np = B[b].nbc[nn][s];
        if (!(bc_interface(np) || np == BC_CURV)) continue;
        const int nb = B[b].nbr[nn][s];
        if (nb < 0 || nb >= (int)B.size()) return "face with interface boundary code but no neighbour block";
        M.send(b, nb, 1 - s, id(b, nn, s));
        M.recv(b, nb, s, id(b, nn, s));
      }
  std::string err;
  auto m = M.match(err);
  if (!err.empty()) return err;
  out.clear();
  for (size_t i = 0; i < M.recvs.size(); ++i) {
    const int64_t r = M.recvs[i].id, s = m[i];
    FaceLink L;
    L.dst_b = (int)(r / 6); L.nn = (int)(r / 2 % 3); L.dst_side = (int)(r % 2);
    L.src_b = (int)(s / 6); int snn = (int)(s / 2 % 3); L.src_side = (int)(s % 2);
    if (snn != L.nn || L.src_side != 1 - L.dst_side)
      return "block interface joins faces of different directions or equal sides (unsupported)";
    if (B[L.src_b].nbs[L.nn] != B[L.dst_b].nbs[L.nn] || B[L.src_b].ijk[1][L.nn] != B[L.dst_b].ijk[1][L.nn])
      return "block interface joins faces of different sizes";
    out.push_back(L);
  }
  return "";
}

Decomp unsplit(const std::vector<BlockGeom>& B) {
  Decomp d;
  for (int b = 0; b < (int)B.size(); ++b) {
    Decomp::Parent p;
    for (int a = 0; a < 3; ++a) {
      p.nbpc[a] = 1;
      for (int s = 0; s < 2; ++s) p.nbr[a][s] = B[b].nbr[a][s];
    }
    p.mo = b;
    d.parents.push_back(p);
    d.mb.push_back(b);
    d.pos.push_back({0, 0, 0});
  }
  return d;
}

std::string check_decomp(const std::vector<BlockGeom>& B, const Decomp& d) {
  int mo = 0;
  for (const auto& p : d.parents) {
    if (p.mo != mo) return "sub-domains: ranks of a block must follow the previous block's";
    for (int a = 0; a < 3; ++a)
      if (p.nbpc[a] < 1) return "sub-domains: nbpc must be positive";
    mo += p.nbpc[0] * p.nbpc[1] * p.nbpc[2];
  }
  if (mo != (int)B.size() || d.mb.size() != B.size() || d.pos.size() != B.size())
    return "sub-domains: one rank per sub-domain of the blocks";
  for (int r = 0; r < (int)B.size(); ++r) {
    const int m = d.mb[r];
    if (m < 0 || m >= (int)d.parents.size()) return "sub-domains: rank in no block";
    for (int a = 0; a < 3; ++a)
      if (d.pos[r][a] < 0 || d.pos[r][a] >= d.parents[m].nbpc[a]) return "sub-domains: position outside the split";
    if (d.idsd3(d.pos[r][0], d.pos[r][1], d.pos[r][2], m, 1) != r)
      return "sub-domains: ranks must be numbered as the reference numbers them";
  }
  return "";
}

namespace {
// Junction search of src/mo_domdcomp.f90:269-437 over the blocks of a case
// (the parents when they are split into sub-domains).
struct Junction {
  std::vector<int> cnt;                 // imjp / imjl
  std::vector<std::vector<int>> list;   // jjp / jjl
  std::vector<int> tag;                 // jptag / jltag
};

void compact(std::vector<int>& it, int& lene, int lens) {  // trimm, src/mo_domdcomp.f90:563-585
  for (int k = 0; k < lens; ++k)
    for (int kk = k + 1; kk <= lens; ++kk)
      if (it[kk] == it[k]) it[kk] = -1;
  lene = lens;
  for (int k = 0; k <= lens; ++k)
    if (it[k] == -1) {
      --lene;
      it[k] = it[k + 1];
      it[k + 1] = -1;
    }
}

std::string search(const Decomp& D, bool points, Junction& J) {
  const int per = points ? 8 : 12;
  const int nbl = (int)D.parents.size();
  const int lp = per * nbl - 1;
  J.cnt.assign(lp + 1, 0);
  J.list.assign(lp + 1, std::vector<int>(102, -1));
  int on_face[3][2][4];
  for (int s = 0; s < 2; ++s)
    for (int i = 0; i < 4; ++i) {
      if (points) {
        const int a[4] = {0, 2, 4, 6}, b[4] = {0, 4, 1, 5}, c[4] = {0, 1, 2, 3};
        on_face[0][s][i] = a[i] + s; on_face[1][s][i] = b[i] + 2 * s; on_face[2][s][i] = c[i] + 4 * s;
      } else {
        const int step[4] = {2, 2, 1, 1};
        const int a[4] = {0, 1, 8, 10}, b[4] = {4, 5, 0, 2}, c[4] = {8, 9, 4, 6};
        on_face[0][s][i] = a[i] + s * step[i]; on_face[1][s][i] = b[i] + s * step[i];
        on_face[2][s][i] = c[i] + s * step[i];
      }
    }
  for (int i = 0; i <= lp; ++i) J.list[i][0] = i;
  for (int mm = 0; mm < nbl; ++mm)
    for (int nn = 0; nn < 3; ++nn)
      for (int s = 0; s < 2; ++s) {
        const int mp = D.parents[mm].nbr[nn][s];
        if (mp == -1) continue;
        for (int i = 0; i < 4; ++i) {
          const int is = per * mm + on_face[nn][s][i];
          const int ie = per * mp + on_face[nn][1 - s][i];
          J.cnt[is] += 1;
          J.list[is][J.cnt[is]] = J.list[ie][0];
        }
      }
  for (int i = 0; i <= lp; ++i)
    for (int j = 0; j <= lp; ++j) {
      if ((i - j) * J.cnt[i] * J.cnt[j] == 0) continue;
      int hits = 0;
      for (int k = 0; k <= J.cnt[i]; ++k)
        for (int kk = 0; kk <= J.cnt[j]; ++kk)
          if (J.list[j][kk] == J.list[i][k]) ++hits;
      if (hits == 0) continue;
      const int ks = J.cnt[i] + 1, ke = ks + J.cnt[j];
      if (ke + 1 > 100) return "junction list longer than the reference's 100 entries";
      for (int c = 0; c <= ke - ks; ++c) J.list[i][ks + c] = J.list[j][c];
      compact(J.list[i], J.cnt[i], ke);
    }
  J.tag.assign(lp + 1, 0);
  for (int i = 0; i <= lp; ++i) {
    int mn = J.list[i][0];
    for (int c = 1; c <= J.cnt[i]; ++c) mn = std::min(mn, J.list[i][c]);
    J.tag[i] = mn;
  }
  return "";
}
}  // namespace

std::string junction_plans(const std::vector<BlockGeom>& B, AvgPlan& P, AvgPlan& Lp) {
  return junction_plans(B, unsplit(B), P, Lp);
}

std::string junction_plans(const std::vector<BlockGeom>& B, const Decomp& D, AvgPlan& P, AvgPlan& Lp) {
  std::string e = check_decomp(B, D);
  if (!e.empty()) return e;
  Junction JP, JL;
  e = search(D, true, JP);
  if (!e.empty()) return e;
  e = search(D, false, JL);
  if (!e.empty()) return e;
  const int nbl = (int)B.size();  // ranks
  // search_point's owner test and partner ranks: rank b averages block corner i
  // of its block if it holds that corner and three or more corners meet there
  auto point_partner = [&](int b, int i, int j) -> int {
    const int g = 8 * D.mb[b] + i;
    if (j == 0) {
      const Decomp::Parent& p = D.parents[D.mb[b]];
      const int c[3] = {i % 2, (i % 4) / 2, i / 4};
      for (int a = 0; a < 3; ++a)
        if (D.pos[b][a] != c[a] * (p.nbpc[a] - 1)) return -1;
      return JP.cnt[g] >= 3 ? b : -1;
    }
    const int mm = JP.list[g][j] / 8, jc = JP.list[g][j] - 8 * mm;
    const Decomp::Parent& q = D.parents[mm];
    return D.idsd3((jc % 2) * (q.nbpc[0] - 1), ((jc % 4) / 2) * (q.nbpc[1] - 1), (jc / 4) * (q.nbpc[2] - 1), mm, 1);
  };
  // search_line's: rank b averages its segment of block edge i if it touches
  // the edge and two or more edges meet there; partners hold the same segment
  auto line_partner = [&](int b, int i, int j) -> int {
    const int g = 12 * D.mb[b] + i;
    const int nn = i / 4 + 1, ns = nn % 3 + 1, ne = ns % 3 + 1;
    if (j == 0) {
      const Decomp::Parent& p = D.parents[D.mb[b]];
      if (D.pos[b][nn - 1] != ((i % 4) / 2) * (p.nbpc[nn - 1] - 1)) return -1;
      if (D.pos[b][ns - 1] != ((i % 4) % 2) * (p.nbpc[ns - 1] - 1)) return -1;
      return JL.cnt[g] >= 2 ? b : -1;
    }
    const int mm = JL.list[g][j] / 12, jc = JL.list[g][j] - 12 * mm;
    const int np = jc / 4 + 1, nq = np % 3 + 1;
    const Decomp::Parent& q = D.parents[mm];
    return D.idsd3(((jc % 4) / 2) * (q.nbpc[np - 1] - 1), ((jc % 4) % 2) * (q.nbpc[nq - 1] - 1), D.pos[b][ne - 1],
                   mm, np);
  };
  // ---- points (average_point, src/mo_domdcomp.f90:439-490)
  {
    Matcher M;
    struct Slot { int b, corner; };
    std::vector<Slot> owners;  // message id -> (block, corner)
    std::vector<std::vector<int>> recv_ids(nbl * 8);
    for (int b = 0; b < nbl; ++b)
      for (int i = 0; i < 8; ++i) {
        if (point_partner(b, i, 0) < 0) continue;
        const int g = 8 * D.mb[b] + i;
        for (int j = 1; j <= JP.cnt[g]; ++j) {
          const int dst = point_partner(b, i, j);
          const int64_t mid = (int64_t)owners.size();
          owners.push_back({b, i});
          M.send(b, dst, JP.tag[g], mid);
          M.recv(b, dst, JP.tag[g], (int64_t)(b * 8 + i) * 1000 + j);
        }
      }
    std::string err;
    auto m = M.match(err);
    if (!err.empty()) return err;
    std::map<int64_t, int64_t> got;
    for (size_t r = 0; r < M.recvs.size(); ++r) got[M.recvs[r].id] = m[r];
    auto corner_l = [&](int b, int i) {
      const BlockGeom& g = B[b];
      return g.dev((i % 2) * g.lxi, ((i % 4) / 2) * g.let, (i / 4) * g.lze);
    };
    P = AvgPlan();
    for (int b = 0; b < nbl; ++b)
      for (int i = 0; i < 8; ++i) {
        if (point_partner(b, i, 0) < 0) continue;
        const int g = 8 * D.mb[b] + i;
        AvgTarget t{b, corner_l(b, i), (int)P.src_b.size(), JP.cnt[g] + 1};
        P.src_b.push_back(b);
        P.src_l.push_back(t.l);
        for (int j = 1; j <= JP.cnt[g]; ++j) {
          const Slot& o = owners[got[(int64_t)(b * 8 + i) * 1000 + j]];
          P.src_b.push_back(o.b);
          P.src_l.push_back(corner_l(o.b, o.corner));
        }
        P.targets.push_back(t);
      }
  }
  // ---- lines (average_line, src/mo_domdcomp.f90:493-559)
  {
    Matcher M;
    struct Slot { int b, edge; };
    std::vector<Slot> owners;
    for (int b = 0; b < nbl; ++b)
      for (int i = 0; i < 12; ++i) {
        if (line_partner(b, i, 0) < 0) continue;
        const int g = 12 * D.mb[b] + i;
        for (int j = 1; j <= JL.cnt[g]; ++j) {
          const int dst = line_partner(b, i, j);
          const int64_t mid = (int64_t)owners.size();
          owners.push_back({b, i});
          M.send(b, dst, JL.tag[g], mid);
          M.recv(b, dst, JL.tag[g], (int64_t)(b * 12 + i) * 1000 + j);
        }
      }
    std::string err;
    auto m = M.match(err);
    if (!err.empty()) return err;
    std::map<int64_t, int64_t> got;
    for (size_t r = 0; r < M.recvs.size(); ++r) got[M.recvs[r].id] = m[r];
    auto edge_len = [&](int b, int i) { return B[b].ijk[2][i / 4] + 1; };
    auto edge_l = [&](int b, int i, int k) {
      const BlockGeom& g = B[b];
      const int nn = i / 4 + 1, ip = (i % 4) / 2, jp = (i % 4) % 2;
      int x, y, z;
      g.line_xyz(nn, ip * g.ijk[0][nn - 1], jp * g.ijk[1][nn - 1], k, x, y, z);
      return g.dev(x, y, z);
    };
    Lp = AvgPlan();
    for (int b = 0; b < nbl; ++b)
      for (int i = 0; i < 12; ++i) {
        if (line_partner(b, i, 0) < 0) continue;
        const int g = 12 * D.mb[b] + i;
        const int len = edge_len(b, i);
        std::vector<Slot> src;
        for (int j = 1; j <= JL.cnt[g]; ++j) {
          const Slot& o = owners[got[(int64_t)(b * 12 + i) * 1000 + j]];
          if (edge_len(o.b, o.edge) != len) return "junction line of different lengths";
          src.push_back(o);
        }
        for (int k = 0; k < len; ++k) {
          AvgTarget t{b, edge_l(b, i, k), (int)Lp.src_b.size(), JL.cnt[g] + 1};
          Lp.src_b.push_back(b);
          Lp.src_l.push_back(t.l);
          for (const Slot& o : src) {
            Lp.src_b.push_back(o.b);
            Lp.src_l.push_back(edge_l(o.b, o.edge, k));
          }
          Lp.targets.push_back(t);
        }
      }
    // A block corner lies on three of its edges; the reference writes it once
    // per edge in edge order, so the last edge's average is the one that stays.
    // Keep only that target (the combine kernel then writes every point once).
    std::map<std::pair<int, int64_t>, size_t> last;
    for (size_t i = 0; i < Lp.targets.size(); ++i) last[{Lp.targets[i].b, Lp.targets[i].l}] = i;
    std::vector<AvgTarget> kept;
    for (size_t i = 0; i < Lp.targets.size(); ++i)
      if (last[{Lp.targets[i].b, Lp.targets[i].l}] == i) kept.push_back(Lp.targets[i]);
    Lp.targets.swap(kept);
  }
  return "";
}

std::string surface_plan(const std::vector<BlockGeom>& B, const std::vector<FaceLink>& links, AvgPlan& S) {
  // average_surface (src/mo_gcbc.f90:342-422): every point of a face with code
  // 30/35/45 takes a running average with the neighbour's snapshot, face by
  // face in (direction, side) order. Targets: unique points in the first face
  // they appear on; sources: ordered snapshots (own value is the running one).
  S = AvgPlan();
  std::map<std::tuple<int, int, int>, const FaceLink*> by_dst;
  for (const auto& L : links) by_dst[std::make_tuple(L.dst_b, L.nn, L.dst_side)] = &L;
  for (int b = 0; b < (int)B.size(); ++b) {
    const BlockGeom& g = B[b];
    std::map<int64_t, std::vector<std::pair<int, int64_t>>> per_point;  // l -> (src block, src l)
    std::vector<int64_t> order;
    for (int nn = 0; nn < 3; ++nn)
      for (int s = 0; s < 2; ++s) {
        if (!bc_averaged(g.nbc[nn][s])) continue;
        auto it = by_dst.find(std::make_tuple(b, nn, s));
        if (it == by_dst.end()) return "averaged face without exchange partner";
        const FaceLink& L = *it->second;
        const BlockGeom& h = B[L.src_b];
        const int pos = s * g.ijk[0][nn], spos = L.src_side * h.ijk[0][nn];
        for (int k = 0; k <= g.ijk[2][nn]; ++k)
          for (int j = 0; j <= g.ijk[1][nn]; ++j) {
            int x, y, z, sx, sy, sz;
            g.line_xyz(nn + 1, pos, j, k, x, y, z);
            h.line_xyz(nn + 1, spos, j, k, sx, sy, sz);
            const int64_t l = g.dev(x, y, z);
            auto& v = per_point[l];
            if (v.empty()) order.push_back(l);
            v.push_back({L.src_b, h.dev(sx, sy, sz)});
          }
      }
    for (int64_t l : order) {
      const auto& v = per_point[l];
      AvgTarget t{b, l, (int)S.src_b.size(), (int)v.size()};
      for (const auto& p : v) { S.src_b.push_back(p.first); S.src_l.push_back(p.second); }
      S.targets.push_back(t);
    }
  }
  return "";
}

void gcbc_tables(const BlockGeom& g, const double* yaco, std::vector<GcbcFace>& faces,
                 std::vector<int64_t>& pts, std::vector<double>& w) {
  // taper weights of the 4 inward points: sbci = -cbca^-1 rbci, times a cosine
  // ramp (src/mo_gcbc.f90:56-76)
  Mat C(4);
  C(0, 0) = kAlpha01; C(0, 1) = kBeta02;
  C(1, 0) = 1.0; C(1, 1) = kAlpha12; C(1, 2) = kBeta13;
  C(2, 0) = kAlpha; C(2, 1) = 1.0; C(2, 2) = kAlpha; C(2, 3) = kBeta;
  C(3, 0) = kBeta; C(3, 1) = kAlpha; C(3, 2) = 1.0; C(3, 3) = kAlpha;
  Mat Ci = invert(C);
  const double rb[4] = {1.0, kAlpha10, kBeta, 0.0};
  double sb[4];
  for (int i = 0; i < 4; ++i) {
    double s = 0;
    for (int c = 0; c < 4; ++c) s = s + Ci(i, c) * rb[c];
    sb[i] = -s;
  }
  const double f = kPi / 5;
  double r = 0.0;
  for (int i = 0; i < 4; ++i) {
    r = r + 1.0;
    sb[i] = (0.5 * sb[i]) * (1.0 + std::cos(r * f));
  }
  faces.clear(); pts.clear(); w.clear();
  std::vector<double> cnt((size_t)g.X * g.Y * g.Z, 0.0);
  std::vector<int64_t> refp;
  for (int nn = 0; nn < 3; ++nn)
    for (int s = 0; s < 2; ++s) {
      const int np = g.nbc[nn][s];
      if (!bc_gcbc(np)) continue;
      faces.push_back({nn + 1, s, np, (int64_t)pts.size()});
      const int pos = s * g.ijk[0][nn], dir = 1 - 2 * s;
      for (int k = 0; k <= g.ijk[2][nn]; ++k)
        for (int j = 0; j <= g.ijk[1][nn]; ++j)
          for (int ii = 0; ii <= 4; ++ii) {
            int x, y, z, fx, fy, fz;
            g.line_xyz(nn + 1, pos, j, k, fx, fy, fz);
            g.line_xyz(nn + 1, pos + dir * ii, j, k, x, y, z);
            const int64_t lr = g.ref_index(x, y, z);
            const double inv = 1.0 / yaco[g.ref_index(fx, fy, fz)];
            cnt[lr] = cnt[lr] + 1.0;
            pts.push_back(g.dev(x, y, z));
            refp.push_back(lr);
            w.push_back(ii == 0 ? inv : inv * sb[ii - 1]);
          }
    }
  for (size_t e = 0; e < w.size(); ++e) w[e] = w[e] / cnt[refp[e]];
}

void sponge_list(const BlockGeom& g, const canard_case_desc& c, const double* xyz, const double* yaco,
                 std::vector<int64_t>& pts, std::vector<double>& asz, std::vector<double>& bsz) {
  pts.clear(); asz.clear(); bsz.clear();
  const int64_t L = (int64_t)g.X * g.Y * g.Z;
  const double ta = kPi / c.szth0, tb = kPi / c.szth1;
  for (int64_t l = 0; l < L; ++l) {
    const double x = xyz[l], y = xyz[l + L];
    const double r3 = 0.0 * y;
    const double r0 = ta * (x - ((r3 - c.doml0) + c.szth0));
    const double r1 = tb * (((r3 + c.doml1) - c.szth1) - x);
    // MIN/MAX return the non-NaN argument, as gfortran's do
    const double c0 = std::cos(std::fmax(std::fmin(r0, kPi), 0.0));
    const double c1 = std::cos(std::fmax(std::fmin(r1, kPi), 0.0));
    const double d1 = (c.szco * 0.5) * ((2.0 + c0) + c1);
    const double d2 = (c.szco * 0.5) * (1.0 + c0);
    if (d1 > 1.0e-8) {
      const int x0 = (int)(l % g.X), y0 = (int)(l / g.X % g.Y), z0 = (int)(l / ((int64_t)g.X * g.Y));
      pts.push_back(g.dev(x0, y0, z0));
      asz.push_back(d1 / yaco[l]);
      bsz.push_back(d2 / yaco[l]);
    }
  }
}

}  // namespace canard

namespace {

// Ranks, decomposition and the face-link and averaging plans of one case, from
// the arguments canard_average_host and canard_plan_export share.
int case_plans(int32_t nranks, const canard_block_desc* ranks, int32_t nblocks, const int32_t* nbpc,
               const int32_t* mbcd, const int32_t* sub, std::vector<canard::BlockGeom>& B,
               std::vector<canard::FaceLink>& links, canard::AvgPlan& P, canard::AvgPlan& L,
               canard::AvgPlan& S) {
  using namespace canard;
  if (nranks < 1 || !ranks) return CANARD_ERR_ARG;
  B.assign(nranks, BlockGeom{});
  for (int r = 0; r < nranks; ++r) make_geom(ranks[r], 0, r, B[r]);
  Decomp D;
  if (nbpc) {
    if (nblocks < 1 || !mbcd || !sub) return CANARD_ERR_ARG;
    int mo = 0;
    for (int m = 0; m < nblocks; ++m) {
      Decomp::Parent p;
      for (int a = 0; a < 3; ++a) {
        p.nbpc[a] = nbpc[3 * m + a];
        for (int s2 = 0; s2 < 2; ++s2) p.nbr[a][s2] = mbcd[6 * m + 2 * a + s2];
      }
      p.mo = mo;
      mo += p.nbpc[0] * p.nbpc[1] * p.nbpc[2];
      D.parents.push_back(p);
    }
    for (int r = 0; r < nranks; ++r) {
      D.mb.push_back(sub[4 * r]);
      D.pos.push_back({sub[4 * r + 1], sub[4 * r + 2], sub[4 * r + 3]});
    }
  } else {
    D = unsplit(B);
  }
  if (!face_links(B, links).empty() || !junction_plans(B, D, P, L).empty() || !surface_plan(B, links, S).empty())
    return CANARD_ERR_UNSUPPORTED;
  return CANARD_OK;
}

}  // namespace

// Junction averaging of one case on the host, through the plans the device
// applies (k_avg_snapshot / k_avg_combine, same arithmetic in the same order):
// the check of the plan builder against the oracle without a GPU.
extern "C" int canard_average_host(int32_t nranks, const canard_block_desc* ranks, int32_t nblocks,
                                   const int32_t* nbpc, const int32_t* mbcd, const int32_t* sub,
                                   double* const* qa) {
  using namespace canard;
  if (nranks < 1 || !ranks || !qa) return CANARD_ERR_ARG;
  for (int r = 0; r < nranks; ++r)
    if (!qa[r]) return CANARD_ERR_ARG;
  std::vector<BlockGeom> B;
  std::vector<FaceLink> links;
  AvgPlan P, L, S;
  if (int rc = case_plans(nranks, ranks, nblocks, nbpc, mbcd, sub, B, links, P, L, S)) return rc;
  std::vector<std::vector<double>> q(nranks);
  for (int r = 0; r < nranks; ++r) {
    const BlockGeom& g = B[r];
    q[r].assign((size_t)5 * g.npad, 0.0);
    for (int c = 0; c < 5; ++c)
      for (int z = 0; z < g.Z; ++z)
        for (int y = 0; y < g.Y; ++y)
          for (int x = 0; x < g.X; ++x)
            q[r][(size_t)c * g.npad + g.dev(x, y, z)] = qa[r][(size_t)c * g.X * g.Y * g.Z + g.ref_index(x, y, z)];
  }
  auto apply = [&](const AvgPlan& p, int mode) {
    std::vector<double> snap((size_t)5 * p.src_b.size());
    for (size_t e = 0; e < p.src_b.size(); ++e)
      for (int c = 0; c < 5; ++c) snap[5 * e + c] = q[p.src_b[e]][(size_t)c * B[p.src_b[e]].npad + p.src_l[e]];
    for (const AvgTarget& t : p.targets) {
      std::vector<double>& v = q[t.b];
      const size_t np = (size_t)B[t.b].npad;
      for (int c = 0; c < 5; ++c) {
        if (mode == 0) {
          double acc = snap[(size_t)t.first * 5 + c];
          for (int j = 1; j < t.count; ++j) acc = acc + snap[(size_t)(t.first + j) * 5 + c];
          v[t.l + c * np] = (1.0 / (double)t.count) * acc;
        } else {
          double x = v[t.l + c * np];
          double r1 = 1.0;
          for (int j = 0; j < t.count; ++j) {
            r1 = r1 + 1.0;
            const double r2 = 1.0 / r1;
            x = r2 * ((r1 - 1.0) * x + snap[(size_t)(t.first + j) * 5 + c]) + 0.0 * x;
          }
          v[t.l + c * np] = x;
        }
      }
    }
  };
  apply(P, 0);
  apply(L, 0);
  apply(S, 1);
  for (int r = 0; r < nranks; ++r) {
    const BlockGeom& g = B[r];
    for (int c = 0; c < 5; ++c)
      for (int z = 0; z < g.Z; ++z)
        for (int y = 0; y < g.Y; ++y)
          for (int x = 0; x < g.X; ++x)
            qa[r][(size_t)c * g.X * g.Y * g.Z + g.ref_index(x, y, z)] = q[r][(size_t)c * g.npad + g.dev(x, y, z)];
  }
  return CANARD_OK;
}


// Face links and averaging plans of one case, exported for placing its ranks
// on several devices: the pieces of every exchange a rank takes part in.
extern "C" int canard_plan_export(int32_t nranks, const canard_block_desc* ranks, int32_t nblocks,
                                  const int32_t* nbpc, const int32_t* mbcd, const int32_t* sub, int32_t kind,
                                  int64_t* out, int64_t cap, int64_t* n) {
  using namespace canard;
  if (kind < 0 || kind > 6 || !n || cap < 0 || (cap > 0 && !out)) return CANARD_ERR_ARG;
  std::vector<BlockGeom> B;
  std::vector<FaceLink> links;
  AvgPlan plans[3];
  if (int rc = case_plans(nranks, ranks, nblocks, nbpc, mbcd, sub, B, links, plans[0], plans[1], plans[2]))
    return rc;
  // device index of rank b -> index in the reference's (0:lmx) layout
  auto ref = [&](int b, int64_t l) {
    const BlockGeom& g = B[b];
    const int64_t x = l % g.Xp, y = l / g.Xp % g.Y, z = l / ((int64_t)g.Xp * g.Y);
    return g.ref_index((int)x, (int)y, (int)z);
  };
  std::vector<int64_t> v;
  if (kind == 0) {
    for (const FaceLink& L : links) {
      const BlockGeom& g = B[L.src_b];
      const int64_t row[7] = {L.dst_b, L.nn + 1, L.dst_side, L.src_b, L.src_side, g.nbs[L.nn],
                              g.nbc[L.nn][L.src_side]};
      v.insert(v.end(), row, row + 7);
    }
  } else if (kind <= 3) {
    for (const AvgTarget& t : plans[kind - 1].targets) {
      const int64_t row[4] = {t.b, ref(t.b, t.l), t.first, t.count};
      v.insert(v.end(), row, row + 4);
    }
  } else {
    const AvgPlan& p = plans[kind - 4];
    for (size_t e = 0; e < p.src_b.size(); ++e) {
      v.push_back(p.src_b[e]);
      v.push_back(ref(p.src_b[e], p.src_l[e]));
    }
  }
  *n = (int64_t)v.size();
  if (cap == 0) return CANARD_OK;
  if (cap < *n) return CANARD_ERR_ARG;
  std::copy(v.begin(), v.end(), out);
  return CANARD_OK;
}
