// FP64 line solves along eta and zeta with the forward-elimination results held
// in tensor memory (TMEM) instead of shared memory.
//
// The one-lane kernel (k_line) keeps a whole 32-line tile in shared memory:
// 257 FP64 rows are 66 KB, so three tiles fit per SM and each SM runs three
// dependent-chain warps on its four schedulers. Here each warp keeps its 32
// lines' elimination results in its own 32 TMEM lanes (row r in columns 2r,
// 2r+1; 512 columns hold rows 0..255, row 256 stays in registers), so shared
// memory only streams the input: a 128-row ring of 32-row TMA boxes per warp
// plus one box with the top rows for the closures. One CTA of four warps per
// SM owns all 512 TMEM columns; every scheduler runs a chain, warps loop over
// tiles, and the next tile's boxes load during the current back substitution.
// Results leave by coalesced stores (32 consecutive x per row).
//
// Every row is evaluated with the same operations in the same order as
// sweep_deriv / sweep_filter (src/mo_numerics.f90:742-792, 922-977), so the
// results are bit-identical to k_line's.
#pragma once
#include "kernels.cuh"

namespace canard {

constexpr int kTmWarps = 4;      // tiles in flight per CTA (one per TMEM lane quarter)
constexpr int kTmChunk = 32;     // rows per TMA box
#ifndef CANARD_TM_RING
#define CANARD_TM_RING 128
#endif
constexpr int kTmRing = CANARD_TM_RING;  // rows of a warp's input ring (boxes of 32)
static_assert(kTmRing % 32 == 0 && kTmRing / 32 + 1 <= 8, "ring boxes and the top box need <= 8 barriers");
constexpr int kTmMaxL = 257;     // rows 0..255 in TMEM, row 256 in registers
constexpr int kTmMinL = 16;      // closures read 12 rows from each end
constexpr int kTmTopSlot = kTmRing / kTmChunk;  // barrier index of the top box
constexpr size_t kTmWarpDoubles = (size_t)(kTmRing + kTmChunk) * kLanes;
constexpr size_t kTmBarOff = 128;  // TMEM address at 0; 8 barrier slots per warp from here
constexpr size_t kTmHeader = 512;  // >= kTmBarOff + kTmWarps * 8 * 8
constexpr size_t kTmSmem = kTmHeader + kTmWarps * kTmWarpDoubles * sizeof(double);

#ifdef CANARD_TRACE
#define TM_TRACE(k) \
  if (lane == 0) g_trace[(long long)t * 8 + (k)] = clock64();
#else
#define TM_TRACE(k)
#endif

// TMEM is not memory the compiler tracks: no "memory" clobbers, so shared and
// global accesses can be scheduled across these; the tcgen05 statements stay
// in program order among themselves (volatile), and tcgen05.wait::st before
// the back substitution orders the stores before the loads.
__device__ __forceinline__ void tm_st(uint32_t taddr, double v) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(taddr), "r"(__double2loint(v)),
               "r"(__double2hiint(v)));
}

// rows i, i-1, ..., i-7 of this warp's lanes; the wait names the destination
// registers so that no use can be scheduled before the data has arrived
__device__ __forceinline__ void tm_ld8(uint32_t tw, int i, double (&v)[8]) {
  uint32_t lo[8], hi[8];
#pragma unroll
  for (int k = 0; k < 8; ++k)
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];"
                 : "=r"(lo[k]), "=r"(hi[k])
                 : "r"(tw + 2u * (uint32_t)(i - k)));
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(lo[0]), "+r"(hi[0]), "+r"(lo[1]), "+r"(hi[1]), "+r"(lo[2]), "+r"(hi[2]), "+r"(lo[3]),
                 "+r"(hi[3]), "+r"(lo[4]), "+r"(hi[4]), "+r"(lo[5]), "+r"(hi[5]), "+r"(lo[6]), "+r"(hi[6]),
                 "+r"(lo[7]), "+r"(hi[7]));
#pragma unroll
  for (int k = 0; k < 8; ++k) v[k] = __hiloint2double((int)hi[k], (int)lo[k]);
}
__device__ __forceinline__ double tm_ld1(uint32_t tw, int i) {
  uint32_t lo, hi;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(lo), "=r"(hi) : "r"(tw + 2u * (uint32_t)i));
  asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(lo), "+r"(hi));
  return __hiloint2double((int)hi, (int)lo);
}

// Geometry of one tile (32 consecutive x lines at one y (eta) or z (zeta)).
struct TmTile {
  int ti, L, N, nch, x0, fix, nval;
  long long base, pstride;
};

template <int DIR>
__device__ __forceinline__ TmTile tm_tile(const LineTask* __restrict__ tasks, const int* __restrict__ tile_task,
                                          int ntasks, int t) {
  TmTile g;
  g.ti = __ldg(tile_task + t);
  (void)ntasks;
  const LineTask& T = tasks[g.ti];
  const int lt = t - T.tile0;
  g.L = T.L;
  g.N = T.L - 1;
  g.nch = (T.L + kTmChunk - 1) / kTmChunk;
  g.fix = lt / T.ntx;
  g.x0 = (lt % T.ntx) * kLanes;
  g.nval = min(kLanes, T.X - g.x0);
  g.pstride = (DIR == 2) ? (long long)T.Xp : (long long)T.Xp * T.Y;
  g.base = (DIR == 2) ? (long long)g.fix * T.Y * T.Xp + g.x0 : (long long)g.fix * T.Xp + g.x0;
  return g;
}

// One warp's input boxes: ring slot q % (kTmRing / 32) holds box q (rows
// 32q..32q+31); the top box holds rows L-32..L-1 (zero-filled below row 0).
template <int DIR>
struct TmIn {
  double* ring;  // this warp's ring; row r at ring[(r % kTmRing) * 32 + lane]
  double* top;   // row r at top[(r - (L - 32)) * 32 + lane]
  uint64_t* bars;
  uint32_t phase = 0;  // parity per barrier
  uint32_t pend = 0;   // barriers with a load in flight
  int lane;

  __device__ __forceinline__ void issue_box(const CUtensorMap* map, const TmTile& g, int slot, int row0,
                                            double* dst) {
    fence_proxy_async();
    if (lane == 0) {
      mbar_expect_tx(bars + slot, (uint32_t)(kTmChunk * kLanes * sizeof(double)));
      if (DIR == 2) tma_load_3d(dst, map, g.x0, row0, g.fix, bars + slot);
      else tma_load_3d(dst, map, g.x0, g.fix, row0, bars + slot);
    }
    pend |= 1u << slot;
  }
  __device__ __forceinline__ void issue_chunk(const CUtensorMap* map, const TmTile& g, int q) {
    const int slot = q % (kTmRing / kTmChunk);
    issue_box(map, g, slot, q * kTmChunk, ring + (size_t)slot * kTmChunk * kLanes);
  }
  // the first boxes of a tile: its top rows and as many boxes as the ring holds
  __device__ __forceinline__ void issue_tile(const CUtensorMap* map, const TmTile& g) {
    issue_box(map, g, kTmTopSlot, g.L - kTmChunk, top);
    for (int q = 0; q < min(g.nch, kTmRing / kTmChunk); ++q) issue_chunk(map, g, q);
  }
  __device__ __forceinline__ bool wait(int slot) {
    const bool ok = mbar_wait(bars + slot, (phase >> slot) & 1u);
    phase ^= 1u << slot;
    pend &= ~(1u << slot);
    return ok;
  }
  // after a failed wait: let the copies in flight land (bounded) before exit
  __device__ __forceinline__ void drain() {
    for (int s = 0; s <= kTmTopSlot; ++s)
      if (pend & (1u << s)) wait(s);
  }
};

// Input rows of the forward sweep: waits for boxes as rows are first read and
// refills box q's slot with the box kTmRing / 32 further once rows of box q
// are no longer read.
template <int DIR>
struct TmStream {
  TmIn<DIR>& in;
  const CUtensorMap* map;
  const TmTile& g;
  int arrived = -1, freed = -1;
  bool ok = true;
#ifdef CANARD_TRACE
  long long waited = 0;  // cycles spent waiting for boxes
#endif
  __device__ __forceinline__ TmStream(TmIn<DIR>& i, const CUtensorMap* m, const TmTile& t) : in(i), map(m), g(t) {}
  __device__ __forceinline__ void ensure(int row) {
    const int q = min(row, g.N) / kTmChunk;
    while (ok && arrived < q) {
      ++arrived;
#ifdef CANARD_TRACE
      const long long c0 = clock64();
#endif
      if (!in.wait(arrived % (kTmRing / kTmChunk))) ok = false;
#ifdef CANARD_TRACE
      waited += clock64() - c0;
#endif
    }
  }
  // rows below `row` are not read again
  __device__ __forceinline__ void release_below(int row) {
    while (ok && (freed + 1) * kTmChunk + kTmChunk - 1 < row) {
      ++freed;
      const int q = freed + kTmRing / kTmChunk;
      if (q < g.nch) in.issue_chunk(map, g, q);
    }
  }
  // every box of the tile lands before the ring is reused (all rows have been
  // read: each wait first frees the boxes before it, which issues the rest)
  __device__ __forceinline__ void finish() {
    while (ok && arrived < g.nch - 1) {
      release_below((arrived + 1) * kTmChunk);
      ensure((arrived + 1) * kTmChunk);
    }
  }
  __device__ __forceinline__ double S(int r) const { return in.ring[(size_t)(r % kTmRing) * kLanes + in.lane]; }
  __device__ __forceinline__ double TOP(int r) const {
    return in.top[(size_t)(r - (g.L - kTmChunk)) * kLanes + in.lane];
  }
};

// Forward rows [i, last] in blocks of eight: BLOCK(i, f) eliminates rows
// i..i+7 (it reads input rows up to i + LA, none below i + LS). Boxes are
// waited for once per run of blocks, and each coefficient segment (table
// rows, the constant interior, table rows) runs as a straight-line loop, so
// the scheduler can overlap a block's loads and right-hand sides with the
// previous chain. Returns the first row not done (single rows follow).
template <int DIR, int LA, int LS, class Block>
__device__ __forceinline__ int tm_blocks(TmStream<DIR>& R, const LuRows<double>& F, int i, int last,
                                         Block&& block) {
  const CoefTable<double> CT{F.l1, F.l2, F.u1, F.u2, F.u3};
  while (i + 7 <= last) {
    R.release_below(i + LS);
    R.ensure(i + LA);
    if (!R.ok) return -1;
    const int avail = min(R.g.N, (R.arrived + 1) * kTmChunk - 1);  // rows present in the ring
    const int imax = min(last - 7, avail - LA);                     // last block start possible now
    for (; i <= imax && i < F.c0; i += 8) {
      F8<double> f;
      f.load(CT, i);
      block(i, f);
    }
    {
      F8<double> f;
#pragma unroll
      for (int k = 0; k < 8; ++k) { f.l1[k] = F.cl1; f.l2[k] = F.cl2; }
      for (; i <= imax && i + 7 <= F.c1; i += 8) block(i, f);
    }
    for (; i <= imax; i += 8) {
      F8<double> f;
      f.load(CT, i);
      block(i, f);
    }
  }
  return i;
}

// Back substitution from the TMEM rows. Row r's final value goes to
// op[r * ps] (if has); ADD (filter) adds the original og[r * ps], loaded one
// block of eight ahead. first / lastv: the final values of rows 0 and N.
template <int ADD>
__device__ __forceinline__ void tm_backward(const LuRows<double>& F, int N, uint32_t tw, double aN, double aN1,
                                            const double* og, double* op, long long ps, bool has, double& first,
                                            double& lastv) {
  auto put = [&](int r, double v) {
    if (has) op[(long long)r * ps] = v;
  };
  double cp1 = __ldg(F.u1 + N) * aN;
  double v = ADD ? og[(long long)N * ps] + cp1 : cp1;
  put(N, v);
  lastv = v;
  double c = __ldg(F.u1 + N - 1) * aN1 - __ldg(F.u2 + N - 1) * cp1;
  put(N - 1, ADD ? og[(long long)(N - 1) * ps] + c : c);
  double cp2 = cp1;
  cp1 = c;
  int i = N - 2;
  double on[8] = {};
  if (ADD)
#pragma unroll
    for (int k = 0; k < 8; ++k) on[k] = og[(long long)max(i - k, 0) * ps];
  // rows i..i-7; the next block's originals load under this block's chain
  // (rows clamped at 0 so that the body stays branch-free)
  auto block = [&](int i, const B8<double>& b) {
    double ou[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) ou[k] = on[k];
    if (ADD)
#pragma unroll
      for (int k = 0; k < 8; ++k) on[k] = og[(long long)max(i - 8 - k, 0) * ps];
    double a[8], p[8], cc[8];
    tm_ld8(tw, i, a);
#pragma unroll
    for (int k = 0; k < 8; ++k) p[k] = b.u1[k] * a[k];
    cc[0] = (p[0] - b.u2[0] * cp1) - b.u3[0] * cp2;
    cc[1] = (p[1] - b.u2[1] * cc[0]) - b.u3[1] * cp1;
#pragma unroll
    for (int k = 2; k < 8; ++k) cc[k] = (p[k] - b.u2[k] * cc[k - 1]) - b.u3[k] * cc[k - 2];
    double* o = op + (long long)i * ps;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const double r = ADD ? ou[k] + cc[k] : cc[k];
      if (has) o[-(long long)k * ps] = r;
      if (i - k == 0) first = r;
    }
    cp2 = cc[6];
    cp1 = cc[7];
  };
  const CoefTable<double> CT{F.l1, F.l2, F.u1, F.u2, F.u3};
  for (; i - 7 >= 0 && i > F.c1; i -= 8) {
    B8<double> b;
    b.load(CT, i);
    block(i, b);
  }
  {
    B8<double> b;
#pragma unroll
    for (int k = 0; k < 8; ++k) { b.u1[k] = F.cu1; b.u2[k] = F.cu2; b.u3[k] = F.cu3; }
    for (; i - 7 >= 0 && i - 7 >= F.c0; i -= 8) block(i, b);
  }
  for (; i - 7 >= 0; i -= 8) {
    B8<double> b;
    b.load(CT, i);
    block(i, b);
  }
  for (; i >= 0; --i) {
    c = (__ldg(F.u1 + i) * tm_ld1(tw, i) - __ldg(F.u2 + i) * cp1) - __ldg(F.u3 + i) * cp2;
    const double r = ADD ? og[(long long)i * ps] + c : c;
    put(i, r);
    if (i == 0) first = r;
    cp2 = cp1;
    cp1 = c;
  }
}

// Derivative forward sweep (sweep_deriv's rows); returns a(N), a(N-1).
template <int DIR>
__device__ __forceinline__ bool tm_forward_deriv(TmStream<DIR>& R, const LuRows<double>& F, int ndf0, int ndf1,
                                                 const DevScheme* __restrict__ sc, double r00, double r10,
                                                 double r01, double r11, uint32_t tw, double& aN, double& aN1) {
  const int N = R.g.N;
  R.ensure(11);
  if (!R.ok) return false;
  double b0, b1, bn1, bn;
  if (ndf0 == 0) {
    const double s0 = R.S(0), s1 = R.S(1), s2 = R.S(2), s3 = R.S(3), s4 = R.S(4);
    b0 = ((CA_A01 * (s1 - s0) + CA_A02 * (s2 - s0)) + CA_A03 * (s3 - s0)) + CA_A04 * (s4 - s0);
    b1 = ((CA_A10 * (s0 - s1) + CA_A12 * (s2 - s1)) + CA_A13 * (s3 - s1)) + CA_A14 * (s4 - s1);
  } else {
    double t0 = 0, t1 = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      const double v = R.S(i);
      t0 = t0 + sc->pbci[0][0][i] * v;
      t1 = t1 + sc->pbci[0][1][i] * v;
    }
    b0 = t0 + r00;
    b1 = t1 + r10;
  }
  if (ndf1 == 0) {
    const double e0 = R.TOP(N), e1 = R.TOP(N - 1), e2 = R.TOP(N - 2), e3 = R.TOP(N - 3), e4 = R.TOP(N - 4);
    bn = ((CA_A01 * (e0 - e1) + CA_A02 * (e0 - e2)) + CA_A03 * (e0 - e3)) + CA_A04 * (e0 - e4);
    bn1 = ((CA_A10 * (e1 - e0) + CA_A12 * (e1 - e2)) + CA_A13 * (e1 - e3)) + CA_A14 * (e1 - e4);
  } else {
    double t0 = 0, t1 = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      const double v = R.TOP(N - i);
      t0 = t0 + sc->pbci[0][0][i] * v;
      t1 = t1 + sc->pbci[0][1][i] * v;
    }
    bn = -t0 - r01;
    bn1 = -t1 - r11;
  }
  double w0 = R.S(0), w1 = R.S(1), w2 = R.S(2), w3 = R.S(3);
  double am2 = b0;
  double am1 = b1 - __ldg(F.l2 + 1) * am2;
  tm_st(tw, am2);
  tm_st(tw + 2, am1);
  const int last = N - 2;
  int i = tm_blocks<DIR, 9, 2>(R, F, 2, last, [&](int i, const F8<double>& f) {
    double win[12], r[8], a[8];
    win[0] = w0; win[1] = w1; win[2] = w2; win[3] = w3;
#pragma unroll
    for (int k = 0; k < 8; ++k) win[4 + k] = R.S(i + 2 + k);
#pragma unroll
    for (int k = 0; k < 8; ++k) r[k] = CA_AA * (win[k + 3] - win[k + 1]) + CA_AB * (win[k + 4] - win[k]);
    a[0] = (r[0] - f.l1[0] * am2) - f.l2[0] * am1;
    a[1] = (r[1] - f.l1[1] * am1) - f.l2[1] * a[0];
#pragma unroll
    for (int k = 2; k < 8; ++k) a[k] = (r[k] - f.l1[k] * a[k - 2]) - f.l2[k] * a[k - 1];
#pragma unroll
    for (int k = 0; k < 8; ++k) tm_st(tw + 2u * (uint32_t)(i + k), a[k]);
    w0 = win[8]; w1 = win[9]; w2 = win[10]; w3 = win[11];
    am2 = a[6]; am1 = a[7];
  });
  if (i < 0) return false;
  for (; i <= last; ++i) {
    R.release_below(i + 2);  // with a ring of two boxes the last box is issued from here
    R.ensure(i + 2);
    if (!R.ok) return false;
    const double w4 = R.S(i + 2);
    const double rhs = CA_AA * (w3 - w1) + CA_AB * (w4 - w0);
    const double a = (rhs - __ldg(F.l1 + i) * am2) - __ldg(F.l2 + i) * am1;
    tm_st(tw + 2u * (uint32_t)i, a);
    w0 = w1; w1 = w2; w2 = w3; w3 = w4;
    am2 = am1; am1 = a;
  }
  {
    const double a = (bn1 - __ldg(F.l1 + N - 1) * am2) - __ldg(F.l2 + N - 1) * am1;
    am2 = am1; am1 = a;
    aN1 = a;
    aN = (bn - __ldg(F.l1 + N) * am2) - __ldg(F.l2 + N) * am1;
  }
  R.finish();  // every box of the tile has landed (none left in flight)
  return R.ok;
}

// Filter forward sweep (sweep_filter's rows); returns a(N), a(N-1).
template <int DIR>
__device__ __forceinline__ bool tm_forward_filter(TmStream<DIR>& R, const LuRows<double>& F, int ndf0, int ndf1,
                                                  const DevScheme* __restrict__ sc, double r00, double r10,
                                                  double r20, double r01, double r11, double r21, uint32_t tw,
                                                  double& aN, double& aN1) {
  const int N = R.g.N;
  R.ensure(11);
  if (!R.ok) return false;
  const double fa = sc->fa, fb = sc->fb, fc = sc->fc;
  auto fbc = [&](int r, int k) { return sc->fbc[r][k]; };
  double b0, b1, b2, bn2, bn1, bn;
  if (ndf0 == 0) {
    const double s0 = R.S(0), s1 = R.S(1), s2 = R.S(2), s3 = R.S(3), s4 = R.S(4), s5 = R.S(5);
    b0 = (((fbc(0, 0) * (s1 - s0) + fbc(0, 1) * (s2 - s0)) + fbc(0, 2) * (s3 - s0)) + fbc(0, 3) * (s4 - s0)) +
         fbc(0, 4) * (s5 - s0);
    b1 = (((fbc(1, 0) * (s0 - s1) + fbc(1, 1) * (s2 - s1)) + fbc(1, 2) * (s3 - s1)) + fbc(1, 3) * (s4 - s1)) +
         fbc(1, 4) * (s5 - s1);
    b2 = (((fbc(2, 0) * (s0 - s2) + fbc(2, 1) * (s1 - s2)) + fbc(2, 2) * (s3 - s2)) + fbc(2, 3) * (s4 - s2)) +
         fbc(2, 4) * (s5 - s2);
  } else {
    double t0 = 0, t1 = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      const double v = R.S(i);
      t0 = t0 + sc->pbci[1][0][i] * v;
      t1 = t1 + sc->pbci[1][1][i] * v;
    }
    const double s0 = R.S(0), s1 = R.S(1), s2 = R.S(2), s3 = R.S(3), s4 = R.S(4), s5 = R.S(5);
    const double ra2 = s2 + s2;
    b0 = t0 + r00;
    b1 = t1 + r10;
    b2 = (fa * ((s1 + s3) - ra2) + fb * ((s0 + s4) - ra2)) + fc * ((r20 + s5) - ra2);
  }
  if (ndf1 == 0) {
    const double e0 = R.TOP(N), e1 = R.TOP(N - 1), e2 = R.TOP(N - 2), e3 = R.TOP(N - 3), e4 = R.TOP(N - 4),
                 e5 = R.TOP(N - 5);
    bn = (((fbc(0, 0) * (e1 - e0) + fbc(0, 1) * (e2 - e0)) + fbc(0, 2) * (e3 - e0)) + fbc(0, 3) * (e4 - e0)) +
         fbc(0, 4) * (e5 - e0);
    bn1 = (((fbc(1, 0) * (e0 - e1) + fbc(1, 1) * (e2 - e1)) + fbc(1, 2) * (e3 - e1)) + fbc(1, 3) * (e4 - e1)) +
          fbc(1, 4) * (e5 - e1);
    bn2 = (((fbc(2, 0) * (e0 - e2) + fbc(2, 1) * (e1 - e2)) + fbc(2, 2) * (e3 - e2)) + fbc(2, 3) * (e4 - e2)) +
          fbc(2, 4) * (e5 - e2);
  } else {
    double t0 = 0, t1 = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      const double v = R.TOP(N - i);
      t0 = t0 + sc->pbci[1][0][i] * v;
      t1 = t1 + sc->pbci[1][1][i] * v;
    }
    const double e0 = R.TOP(N), e1 = R.TOP(N - 1), e2 = R.TOP(N - 2), e3 = R.TOP(N - 3), e4 = R.TOP(N - 4),
                 e5 = R.TOP(N - 5);
    const double ra2 = e2 + e2;
    bn = t0 + r01;
    bn1 = t1 + r11;
    bn2 = (fa * ((e3 + e1) - ra2) + fb * ((e4 + e0) - ra2)) + fc * ((e5 + r21) - ra2);
  }
  double w0 = R.S(0), w1 = R.S(1), w2 = R.S(2), w3 = R.S(3), w4 = R.S(4), w5 = R.S(5);
  double am2 = b0;
  double am1 = b1 - __ldg(F.l2 + 1) * am2;
  const double a2 = (b2 - __ldg(F.l1 + 2) * am2) - __ldg(F.l2 + 2) * am1;
  tm_st(tw, am2);
  tm_st(tw + 2, am1);
  tm_st(tw + 4, a2);
  am2 = am1;
  am1 = a2;
  const int last = N - 3;
  int i = tm_blocks<DIR, 10, 3>(R, F, 3, last, [&](int i, const F8<double>& f) {
    double win[14], r[8], a[8];
    win[0] = w0; win[1] = w1; win[2] = w2; win[3] = w3; win[4] = w4; win[5] = w5;
#pragma unroll
    for (int k = 0; k < 8; ++k) win[6 + k] = R.S(i + 3 + k);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const double rk = win[k + 3] + win[k + 3];
      r[k] = (fa * ((win[k + 2] + win[k + 4]) - rk) + fb * ((win[k + 1] + win[k + 5]) - rk)) +
             fc * ((win[k] + win[k + 6]) - rk);
    }
    a[0] = (r[0] - f.l1[0] * am2) - f.l2[0] * am1;
    a[1] = (r[1] - f.l1[1] * am1) - f.l2[1] * a[0];
#pragma unroll
    for (int k = 2; k < 8; ++k) a[k] = (r[k] - f.l1[k] * a[k - 2]) - f.l2[k] * a[k - 1];
#pragma unroll
    for (int k = 0; k < 8; ++k) tm_st(tw + 2u * (uint32_t)(i + k), a[k]);
    w0 = win[8]; w1 = win[9]; w2 = win[10]; w3 = win[11]; w4 = win[12]; w5 = win[13];
    am2 = a[6]; am1 = a[7];
  });
  if (i < 0) return false;
  for (; i <= last; ++i) {
    R.release_below(i + 3);
    R.ensure(i + 3);
    if (!R.ok) return false;
    const double w6 = R.S(i + 3);
    const double rk = w3 + w3;
    const double rhs = (fa * ((w2 + w4) - rk) + fb * ((w1 + w5) - rk)) + fc * ((w0 + w6) - rk);
    const double a = (rhs - __ldg(F.l1 + i) * am2) - __ldg(F.l2 + i) * am1;
    tm_st(tw + 2u * (uint32_t)i, a);
    w0 = w1; w1 = w2; w2 = w3; w3 = w4; w4 = w5; w5 = w6;
    am2 = am1; am1 = a;
  }
  {
    double a = (bn2 - __ldg(F.l1 + N - 2) * am2) - __ldg(F.l2 + N - 2) * am1;
    tm_st(tw + 2u * (uint32_t)(N - 2), a);
    am2 = am1; am1 = a;
    a = (bn1 - __ldg(F.l1 + N - 1) * am2) - __ldg(F.l2 + N - 1) * am1;
    am2 = am1; am1 = a;
    aN1 = a;
    aN = (bn - __ldg(F.l1 + N) * am2) - __ldg(F.l2 + N) * am1;
  }
  R.finish();
  return R.ok;
}

// DIR: 2 eta, 3 zeta. OP: 0 derivative, 1 filter (out = original + increment).
// One CTA of kTmWarps warps per SM (its shared memory admits no second CTA),
// persistent over the tiles of all tasks. Tasks need kTmMinL <= L <= kTmMaxL
// and 32-row boxes in their tensor maps.
template <int DIR, int OP>
__global__ void __launch_bounds__(kTmWarps * 32) k_line_tm(const LineTask* __restrict__ tasks,
                                                          const int* __restrict__ tile_task, int ntasks, int ntiles,
                                                          const CUtensorMap* __restrict__ maps,
                                                          int* __restrict__ err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint32_t* tbase = reinterpret_cast<uint32_t*>(smem_raw);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  {
    // after an earlier bounded wait gave up: no work (uniform over the CTA,
    // before any barrier or TMEM allocation)
    __shared__ int stop;
    if (threadIdx.x == 0) stop = *reinterpret_cast<const volatile int*>(err);
    __syncthreads();
    if (stop) return;
  }
  TmIn<DIR> in;
  in.lane = lane;
  in.bars = reinterpret_cast<uint64_t*>(smem_raw + kTmBarOff) + w * 8;
  in.ring = reinterpret_cast<double*>(smem_raw + kTmHeader) + (size_t)w * kTmWarpDoubles;
  in.top = in.ring + (size_t)kTmRing * kLanes;
  if (lane == 0) {
    for (int s = 0; s <= kTmTopSlot; ++s) mbar_init(in.bars + s, 1);
    mbar_init_done();
  }
  if (w == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tbase)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tw = tbase[0] + ((uint32_t)(32 * w) << 16);

  const int stride = gridDim.x * kTmWarps;
  int t = blockIdx.x * kTmWarps + w;
  bool ok = true;
  TmTile g;
  if (t < ntiles) {
    g = tm_tile<DIR>(tasks, tile_task, ntasks, t);
    in.issue_tile(maps + 2 * g.ti, g);
  }
  for (; ok && t < ntiles; t += stride) {
    TM_TRACE(0)
    const LineTask& T = tasks[g.ti];
    const CUtensorMap* map = maps + 2 * g.ti;
    const bool has = lane < g.nval;
    int jk = 0;
    if (DIR == 2) jk = (g.x0 + lane) * T.Z + g.fix;
    else jk = g.fix * T.X + g.x0 + lane;
    const int nbs = T.nbs;
    const double* recv = static_cast<const double*>(T.recv);
    const LuRows<double> F(static_cast<const double*>(T.lu), g.L, T.cl1, T.cl2, T.cu1, T.cu2, T.cu3, T.c0);
    TmStream<DIR> R(in, map, g);
    if (!in.wait(kTmTopSlot)) { ok = false; break; }
    TM_TRACE(1)
    double aN = 0, aN1 = 0;
    bool fw;
    __syncwarp();
    if (OP == 0) {
      double r00 = 0, r10 = 0, r01 = 0, r11 = 0;
      if (T.selfp) {
        // periodic onto itself: the contraction the other end would send
        // (src/mo_numerics.f90:503-518 with n45 = 0), formed from the tile
        R.ensure(12);
        const DevScheme* sc = T.sc;
        const int N = g.N;
#pragma unroll
        for (int i = 0; i < 12; ++i) {
          const double v = R.TOP(N - 1 - i), u = R.S(1 + i);
          r00 = r00 + sc->pbco[0][0][i] * v;
          r10 = r10 + sc->pbco[0][1][i] * v;
          r01 = r01 + sc->pbco[0][0][i] * u;
          r11 = r11 + sc->pbco[0][1][i] * u;
        }
      } else {
        if (has && T.ndf0) { r00 = recv[jk]; r10 = recv[nbs + jk]; }
        if (has && T.ndf1) { r01 = recv[2 * nbs + jk]; r11 = recv[3 * nbs + jk]; }
      }
      fw = tm_forward_deriv<DIR>(R, F, T.ndf0, T.ndf1, T.sc, r00, r10, r01, r11, tw, aN, aN1);
    } else {
      double r00 = 0, r10 = 0, r20 = 0, r01 = 0, r11 = 0, r21 = 0;
      if (has && T.ndf0) { r00 = recv[jk]; r10 = recv[nbs + jk]; r20 = recv[2 * nbs + jk]; }
      if (has && T.ndf1) { r01 = recv[3 * nbs + jk]; r11 = recv[4 * nbs + jk]; r21 = recv[5 * nbs + jk]; }
      fw = tm_forward_filter<DIR>(R, F, T.ndf0, T.ndf1, T.sc, r00, r10, r20, r01, r11, r21, tw, aN, aN1);
    }
    if (!fw) { ok = false; break; }
    TM_TRACE(2)
#ifdef CANARD_TRACE
    if (lane == 0) g_trace[(long long)t * 8 + 5] = R.waited;
#endif
    __syncwarp();
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    // the input ring is free: start the next tile's boxes under the back substitution
    const TmTile cur = g;
    const int tn = t + stride;
    if (tn < ntiles) {
      g = tm_tile<DIR>(tasks, tile_task, ntasks, tn);
      in.issue_tile(maps + 2 * g.ti, g);
    }
    // lanes without a line read lane 0's column (valid memory) and store nothing;
    // the filter's originals use plain loads because this kernel writes that array
    const long long col = cur.base + (has ? lane : 0);
    double* out = static_cast<double*>(T.out) + col;
    const double* orig = static_cast<const double*>(T.in) + col;
    double first = 0, lastv = 0;
    TM_TRACE(3)
    __syncwarp();
    tm_backward<OP>(F, cur.N, tw, aN, aN1, orig, out, cur.pstride, has, first, lastv);
    if (OP == 0 && has && T.drva) {
      double* drva = static_cast<double*>(T.drva);
      drva[jk + (long long)nbs * (T.m - 1)] = first;
      drva[jk + (long long)nbs * ((T.m - 1) + 5)] = lastv;
    }
    TM_TRACE(4)
  }
  if (!ok) {
    if (lane == 0) atomicExch(err, kErrTimeout);
    in.drain();
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (w == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase[0]), "r"(512));
}

template <int DIR, int OP>
void launch_line_tm_t(int grid, cudaStream_t st, const LineTask* t, const int* f, int nt, int ntiles,
                      const CUtensorMap* maps, int* err) {
  k_line_tm<DIR, OP><<<grid, kTmWarps * 32, kTmSmem, st>>>(t, f, nt, ntiles, maps, err);
}
template <int DIR, int OP>
cudaError_t line_tm_smem_limit() {
  return cudaFuncSetAttribute(k_line_tm<DIR, OP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTmSmem);
}

}  // namespace canard
