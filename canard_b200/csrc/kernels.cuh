// Device kernels of the Canard hot path for sm_100a.
//
// Every kernel is a template over its arithmetic types and is instantiated
// twice:
//  * FP64 plain: all types double, compiled without FMA contraction
//    (-fmad=false) and evaluating every expression in the reference's order,
//    so on identical inputs it reproduces the CPU restatement bit for bit (the
//    Sutherland power is the only library function, see pow15);
//  * FP32 mixed: line solves, fluxes, viscous stresses and GCBC in float with
//    FMA contraction (a separate translation unit), while the conserved state,
//    the RK update, the metric and Jacobian masters, the primitive
//    computation and the LU factorisation stay FP64.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace canard {

constexpr int kLanes = 32;            // lines per tile (one warp, one line per lane)
constexpr int kErrTimeout = 4;
constexpr int kErrOverflow = 8;  // dt == 0 after step 2 ("Canard: Overflow.")
constexpr long long kSpinLimit = 1LL << 28;  // bounded mbarrier waits: polls at most
constexpr unsigned long long kWaitNs = 500000000ull;  // and 0.5 s of %globaltimer

struct DevScheme {
  double pbci[2][2][12];  // [nt][side][i]
  double pbco[2][2][12];
  double pbcot[2][2];
  double fa, fb, fc;
  double fbc[3][5];       // [row][k]
  double alphf, betf;     // the filter's interior left-hand side (beta, alpha, 1, alpha, beta)
  double albef[2][3][5];  // its first three rows [closure kind][row][k+2]: 0 boundary, 1 interface
};

// Per-case scalars of one RK stage (written by the host before each step).
struct StageParams {
  double umf[3], dudtmf[3];   // moving frame for fluxes / GCBC (movef before the update)
  double umfb[3];             // moving frame after the update (wall condition)
  double dtk, dt;
};

struct CaseConst {
  double srefoo, srefp1dre;
  int viscous;
  int nsmf;                // 1: constant moving frame; 0: frame ramped over timf
  double cfl, timf, uoo[3];
};

// Time-loop state of one case (src/mo_canard_driver.f90:226-370), kept on the
// device so that a whole step needs no host round trip.
struct TimeDev {
  long long n, ndt;
  double dt, dts, dte, timo;
};

// Work fields of one block in the arithmetic type R of the flux path.
template <class R>
struct Work {
  R *de, *p, *mu, *tau, *scr;
  const R *xim, *etm, *zem, *yaco;
};

struct BlockDev {
  int X, Y, Z, Xp;
  long long npad;
  int case_id;
  // FP64: state, metric and Jacobian masters, and the FP64 work fields
  double *qa, *qo, *de, *p, *mu, *xim, *etm, *zem, *yaco, *tau, *scr, *xyz;
  Work<float> f;  // FP32 work fields and metric copies (mixed precision only)
};

template <class R>
__device__ __forceinline__ Work<R> work(const BlockDev& B);
template <>
__device__ __forceinline__ Work<double> work<double>(const BlockDev& B) {
  return {B.de, B.p, B.mu, B.tau, B.scr, B.xim, B.etm, B.zem, B.yaco};
}
template <>
__device__ __forceinline__ Work<float> work<float>(const BlockDev& B) {
  return B.f;
}

// ---------------------------------------------------------------------------
// A family of lines of one block, direction and field, solved by one launch
// together with other families (tile prefix sums select the family). Field
// pointers have the tile type TT of the launch, factor tables the solve type.
struct LineTask {
  const void* in;
  void* out;
  const void* lu;       // xl1, xl2, xu1, xu2, xu3 (each L entries)
  double cl1, cl2, cu1, cu2, cu3;  // the factors of rows [c0, L-4], bitwise constant there
  int c0;
  const void* recv;     // [side][comp][jk], comp stride nbs, side stride ncomp*nbs
  void* drva;           // drva(jk, m, side) of this block and direction, or null
  const DevScheme* sc;
  int X, Y, Z, Xp;
  int L, nbs, m, ndf0, ndf1;
  int selfp;               // derivative of a line periodic onto itself: contraction formed in the kernel
  int h, kg, ke;           // split solves: first row of the second half; homogeneous table lengths
  int kf;                  // split solves: rows the forward homogeneous solutions from h span
  int q2, q3;              // quad split: first rows of the third and fourth segments (h: of the second)
  int tile0, ntiles, ntx;  // first global tile, tiles, x-tiles per row (dir 2/3)
  int nbox, by;            // chunks per tile and positions per chunk
};

// Interface contraction of one face (t_numerics%mpigo): the sender's face
// lines are contracted with pbco and written into the receiver's buffers.
struct FaceTask {
  const void* src;      // sender field column for this direction
  const void* dstf;     // receiver field column (coordinate-jump correction)
  void* recv;           // receiver buffer [comp][jk] for (direction, side, m)
  double* chain;        // sender's persistent send(:,nt+1,side) of the filter
                        // (null: the fields are filtered direction-major, no chain)
  const DevScheme* sc;
  int nn, sb, nt, exch, corr, iik;
  double ra0k;
  int X, Y, Z, Xp, N;       // sender geometry
  int XA, YA, ZA, XpA, NA;  // receiver geometry
  int nbs, nj, line0;
};

struct GcbcTask {  // one GCBC face of one block
  int b, nn, side, bc;
  const double* cm;       // cm(jk,3,side) base of this face side: [d][jk]
  void* drva;             // drva(jk,5,side): [c][jk], in the flux type
  const void* drvb;
  const long long* pts;   // 5 device indices per line
  const double* w;        // 5 weights per line
  int nbs, nj, line0;
  int X, Y, Z, Xp, N;
};

struct SpongeTask { int b; const long long* pts; const double* asz; const double* bsz; int count, first; };

// ---------------------------------------------------------------------------
// small PTX helpers: mbarrier + bulk and element asynchronous copies
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// one fence after a thread's initialisations (their visibility to the copies)
__device__ __forceinline__ void mbar_init_done() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// L1 prefetch of one cache line
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }
// Bounded wait for phase `parity`; returns false if the limit expired.
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// false after kWaitNs (a copy that never completes sets the error flag in the
// caller instead of holding the GPU)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (int it = 0; it < 16; ++it)
    if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (long long it = 0; it < kSpinLimit; ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 63) == 0 && global_ns() - t0 > kWaitNs) return false;
  }
  return false;
}
// the error flag's load issued at a kernel's start and decided later (the
// load's latency then overlaps the task decode and barrier set-up)
__device__ __forceinline__ int error_flag_early(const int* err) {
  return (threadIdx.x & 31) == 0 ? *reinterpret_cast<const volatile int*>(err) : 0;
}
// a kernel launched after a bounded wait gave up does no work (the host
// reports the error at its next synchronisation); uniform over the warp
__device__ __forceinline__ bool error_pending(const int* err) {
  int e = 0;
  if ((threadIdx.x & 31) == 0) e = *reinterpret_cast<const volatile int*>(err);
  return __shfl_sync(0xffffffffu, e, 0) != 0;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)),
               "r"(bytes)
               : "memory");
}
// dst[k] = dst[k] + src[k] over bytes / 8 doubles, one FP64 add with
// round-to-nearest per element done at the memory side: the filter's
// in-place f = f + increment without reading f back into the SM
__device__ __forceinline__ void bulk_s2g_add_f64(void* dst, const void* src, uint32_t bytes) {
  asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f64 [%0], [%1], %2;" ::"l"(dst),
               "r"(smem_u32(src)), "r"(bytes)
               : "memory");
}
// TMA tile copies of a 3-D box (coordinates x, y, z in elements)
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, int x, int y, int z, const void* src) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(map),
               "r"(x), "r"(y), "r"(z), "r"(smem_u32(src))
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read0() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Correctly rounded x^1.5 for x > 0 (up to rare ties): x*sqrt(x) carried in
// double-double arithmetic (Dekker's exact product, Newton remainder of sqrt).
__device__ __forceinline__ double pow15(double x) {
  const double s = sqrt(x);
  const double r = fma(-s, s, x);          // exact: x - s^2
  const double e = r / (2.0 * s);          // sqrt(x) = s + e + O(ulp^2)
  const double p = x * s;
  const double pe = fma(x, s, -p);         // exact: x*s - p
  return p + (pe + x * e);
}

// ---------------------------------------------------------------------------
// scheme constants (src/mo_parameters.f90:52-70)
#define CA_ALPHA (4 / 9.0)
#define CA_BETA (1 / 36.0)
#define CA_AA (20 / 27.0)
#define CA_AB (25 / 216.0)
#define CA_A10 (-0.3506944444280639)
#define CA_A12 (0.8249999999974599)
#define CA_A13 (0.7444444444773477)
#define CA_A14 (0.014583333334139971)
#define CA_A01 (-6.666666667794732)
#define CA_A02 (9.000000000052879)
#define CA_A03 (1.333333333178555)
#define CA_A04 (-0.0833333333455545)

// The LU factors of the Toeplitz interior converge to a fixed point: rows
// [c0, L-4] hold bitwise identical factors (found on the host), which the
// sweeps keep in registers. Only the closure rows near the ends read the
// factor tables, so the dependent chain carries no memory latency there.
template <class RS>
struct LuRows {
  const RS* __restrict__ l1;
  const RS* __restrict__ l2;
  const RS* __restrict__ u1;
  const RS* __restrict__ u2;
  const RS* __restrict__ u3;
  RS cl1, cl2, cu1, cu2, cu3;
  int c0, c1;
  __device__ __forceinline__ LuRows(const RS* lu, int L, RS a, RS b, RS c, RS d, RS e, int c0_)
      : l1(lu), l2(lu + L), u1(lu + 2 * L), u2(lu + 3 * L), u3(lu + 4 * L), cl1(a), cl2(b), cu1(c), cu2(d),
        cu3(e), c0(c0_), c1(L - 4) {}
};

constexpr int kMaxChunks = 8;

// While a tile's copies are in flight: the scheme's coefficients (1.2 KB)
// and the first 16 rows of the five factor tables into L1, which the closures
// and the first blocks of the sweeps read as soon as the tile has arrived.
template <class RS>
__device__ __forceinline__ void prefetch_sweep_start(const DevScheme* sc, const RS* lu, int L, int lane) {
  if (lane < 10) {
    prefetch_l1(reinterpret_cast<const char*>(sc) + 128 * lane);
  } else if (lane < 20) {
    const int k = (lane - 10) % 5, e = (lane - 10) / 5 ? 15 : 0;
    prefetch_l1(lu + (size_t)k * L + e);
  }
}

#ifdef CANARD_TRACE
__device__ long long* g_trace;  // per CTA: start, loads issued, data ready, forward done, end, SM id
#define TRACE(k) \
  if (threadIdx.x == 0) g_trace[(long long)blockIdx.x * 8 + (k)] = clock64();
#else
#define TRACE(k)
#endif

// A tile arrives in NC chunks of CR positions (rows), chunk 0 and the last
// chunk first (the closures read both ends), then 1, 2, ...; the forward
// sweep waits for a chunk only when its look-ahead reaches it.
struct ChunkIn {
  uint64_t* bars;
  int CR, NC, L;
  int next;   // next middle chunk to wait for
  int ready;  // rows [0, ready) and the last chunk have arrived
  __device__ __forceinline__ bool wait_next(int* err) {
    if (next >= NC - 1) { ready = L; return true; }
    if (!mbar_wait(bars + next, 0)) { atomicExch(err, kErrTimeout); return false; }
    ++next;
    ready = (next >= NC - 1) ? L : next * CR;
    return true;
  }
};

// Factor providers: the interior constants or the per-row tables.
template <class RS>
struct CoefConst {
  RS l1, l2, u1, u2, u3;
  __device__ __forceinline__ RS L1(int) const { return l1; }
  __device__ __forceinline__ RS L2(int) const { return l2; }
  __device__ __forceinline__ RS U1(int) const { return u1; }
  __device__ __forceinline__ RS U2(int) const { return u2; }
  __device__ __forceinline__ RS U3(int) const { return u3; }
};
template <class RS>
struct CoefTable {
  const RS* __restrict__ l1;
  const RS* __restrict__ l2;
  const RS* __restrict__ u1;
  const RS* __restrict__ u2;
  const RS* __restrict__ u3;
  __device__ __forceinline__ RS L1(int i) const { return __ldg(l1 + i); }
  __device__ __forceinline__ RS L2(int i) const { return __ldg(l2 + i); }
  __device__ __forceinline__ RS U1(int i) const { return __ldg(u1 + i); }
  __device__ __forceinline__ RS U2(int i) const { return __ldg(u2 + i); }
  __device__ __forceinline__ RS U3(int i) const { return __ldg(u3 + i); }
};

// per-row factors staged in shared memory (the two-ended solve's closure rows)
template <class RS>
struct CoefShared {
  const RS* l1;
  const RS* l2;
  const RS* u1;
  const RS* u2;
  const RS* u3;
  __device__ __forceinline__ RS L1(int i) const { return l1[i]; }
  __device__ __forceinline__ RS L2(int i) const { return l2[i]; }
  __device__ __forceinline__ RS U1(int i) const { return u1[i]; }
  __device__ __forceinline__ RS U2(int i) const { return u2[i]; }
  __device__ __forceinline__ RS U3(int i) const { return u3[i]; }
};

// Rows are processed in blocks of eight: the block's inputs, right-hand sides
// and factors are all formed before its dependent chain, so their latency
// overlaps the chain. Every row is still evaluated with the reference's
// operations in the reference's order (bit-identical to one row at a time).
// Right-hand sides are formed in the tile type TT, the elimination runs in the
// solve type RS.

// Factors of one block of eight rows, loaded ahead of the block that uses
// them (forward: l1, l2 of rows i..i+7; backward: u1, u2, u3 of rows i..i-7),
// and the filter's originals of a backward block.
template <class RS>
struct F8 {
  RS l1[8], l2[8];
  template <class CF>
  __device__ __forceinline__ void load(const CF& cf, int i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) { l1[k] = cf.L1(i + k); l2[k] = cf.L2(i + k); }
  }
};
template <class RS>
struct B8 {
  RS u1[8], u2[8], u3[8];
  template <class CF>
  __device__ __forceinline__ void load(const CF& cf, int i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) { u1[k] = cf.U1(i - k); u2[k] = cf.U2(i - k); u3[k] = cf.U3(i - k); }
  }
};
template <class TT>
struct O8 {
  TT o[8];
  __device__ __forceinline__ void load(const TT* __restrict__ og, int ogs, int i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) o[k] = __ldg(og + (long long)(i - k) * ogs);
  }
};

// Right-hand sides of the derivative's rows i..i+7 (reads rows up to i+9);
// window w0..w3 = s[i-2..i+1] on entry, s[i+6..i+9] on return
template <int ST, class TT>
__device__ __forceinline__ void rhs8_deriv(const TT* __restrict__ s, int i, TT& w0, TT& w1, TT& w2, TT& w3,
                                           TT (&r)[8]) {
  TT win[12];
  win[0] = w0; win[1] = w1; win[2] = w2; win[3] = w3;
#pragma unroll
  for (int k = 0; k < 8; ++k) win[4 + k] = s[(i + 2 + k) * ST];
#pragma unroll
  for (int k = 0; k < 8; ++k) r[k] = TT(CA_AA) * (win[k + 3] - win[k + 1]) + TT(CA_AB) * (win[k + 4] - win[k]);
  w0 = win[8]; w1 = win[9]; w2 = win[10]; w3 = win[11];
}

// forward elimination of rows i..i+7 from their right-hand sides
template <int ST, class TT, class RS>
__device__ __forceinline__ void chain8_fwd(TT* __restrict__ s, int i, const F8<RS>& f, const TT (&r)[8], RS& am2,
                                           RS& am1) {
  RS a[8];
  a[0] = (RS(r[0]) - f.l1[0] * am2) - f.l2[0] * am1;
  a[1] = (RS(r[1]) - f.l1[1] * am1) - f.l2[1] * a[0];
#pragma unroll
  for (int k = 2; k < 8; ++k) a[k] = (RS(r[k]) - f.l1[k] * a[k - 2]) - f.l2[k] * a[k - 1];
#pragma unroll
  for (int k = 0; k < 8; ++k) s[(i + k) * ST] = TT(a[k]);
  am2 = a[6]; am1 = a[7];
}

// forward rows i..i+7 of the derivative; window w0..w3 = s[i-2..i+1]
template <int ST, class TT, class RS>
__device__ __forceinline__ void fwd8_deriv_c(TT* __restrict__ s, int i, const F8<RS>& f, TT& w0, TT& w1, TT& w2,
                                             TT& w3, RS& am2, RS& am1) {
  TT r[8];
  rhs8_deriv<ST, TT>(s, i, w0, w1, w2, w3, r);
  chain8_fwd<ST, TT, RS>(s, i, f, r, am2, am1);
}
template <int ST, class TT, class RS, class CF>
__device__ __forceinline__ void fwd8_deriv(TT* __restrict__ s, int i, const CF& cf, TT& w0, TT& w1, TT& w2, TT& w3,
                                           RS& am2, RS& am1) {
  F8<RS> f;
  f.load(cf, i);
  fwd8_deriv_c<ST, TT, RS>(s, i, f, w0, w1, w2, w3, am2, am1);
}

// Right-hand sides of the filter's rows i..i+7 (reads rows up to i+10);
// window w0..w5 = s[i-3..i+2] on entry, s[i+5..i+10] on return
// DIRECT: the right-hand side of the filtered values themselves, (B x)_i =
// (A x)_i + ((B - A) x)_i with A's interior row (beta, alpha, 1, alpha, beta)
template <int ST, class TT, bool DIRECT = false>
__device__ __forceinline__ void rhs8_filter(const TT* __restrict__ s, int i, TT fa, TT fb, TT fc, TT& w0, TT& w1,
                                            TT& w2, TT& w3, TT& w4, TT& w5, TT (&r)[8], TT al = 0, TT be = 0) {
  TT win[14];
  win[0] = w0; win[1] = w1; win[2] = w2; win[3] = w3; win[4] = w4; win[5] = w5;
#pragma unroll
  for (int k = 0; k < 8; ++k) win[6 + k] = s[(i + 3 + k) * ST];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const TT rk = win[k + 3] + win[k + 3];
    r[k] = (fa * ((win[k + 2] + win[k + 4]) - rk) + fb * ((win[k + 1] + win[k + 5]) - rk)) +
           fc * ((win[k] + win[k + 6]) - rk);
    if (DIRECT) r[k] = r[k] + ((win[k + 3] + al * (win[k + 2] + win[k + 4])) + be * (win[k + 1] + win[k + 5]));
  }
  w0 = win[8]; w1 = win[9]; w2 = win[10]; w3 = win[11]; w4 = win[12]; w5 = win[13];
}

// forward rows i..i+7 of the filter; window w0..w5 = s[i-3..i+2]
template <int ST, class TT, class RS>
__device__ __forceinline__ void fwd8_filter_c(TT* __restrict__ s, int i, const F8<RS>& f, TT fa, TT fb, TT fc,
                                              TT& w0, TT& w1, TT& w2, TT& w3, TT& w4, TT& w5, RS& am2, RS& am1) {
  TT r[8];
  rhs8_filter<ST, TT>(s, i, fa, fb, fc, w0, w1, w2, w3, w4, w5, r);
  chain8_fwd<ST, TT, RS>(s, i, f, r, am2, am1);
}
template <int ST, class TT, class RS, class CF>
__device__ __forceinline__ void fwd8_filter(TT* __restrict__ s, int i, const CF& cf, TT fa, TT fb, TT fc, TT& w0,
                                            TT& w1, TT& w2, TT& w3, TT& w4, TT& w5, RS& am2, RS& am1) {
  F8<RS> f;
  f.load(cf, i);
  fwd8_filter_c<ST, TT, RS>(s, i, f, fa, fb, fc, w0, w1, w2, w3, w4, w5, am2, am1);
}

// back substitution rows i, i-1, ..., i-7. ADD (filter): each row is stored
// as original + increment, the originals in o.
template <int ST, class TT, class RS>
__device__ __forceinline__ void bwd_p8(const TT* __restrict__ s, int i, const B8<RS>& b, RS (&p)[8]) {
#pragma unroll
  for (int k = 0; k < 8; ++k) p[k] = b.u1[k] * RS(s[(i - k) * ST]);
}
template <int ST, class TT, class RS, int ADD>
__device__ __forceinline__ void bwd_chain8(TT* __restrict__ s, int i, const B8<RS>& b, const RS (&p)[8],
                                           const O8<TT>& o, RS& cp1, RS& cp2) {
  RS c[8];
  c[0] = (p[0] - b.u2[0] * cp1) - b.u3[0] * cp2;
  c[1] = (p[1] - b.u2[1] * c[0]) - b.u3[1] * cp1;
#pragma unroll
  for (int k = 2; k < 8; ++k) c[k] = (p[k] - b.u2[k] * c[k - 1]) - b.u3[k] * c[k - 2];
#pragma unroll
  for (int k = 0; k < 8; ++k) s[(i - k) * ST] = ADD ? o.o[k] + TT(c[k]) : TT(c[k]);
  cp2 = c[6];
  cp1 = c[7];
}
template <int ST, class TT, class RS, int ADD>
__device__ __forceinline__ void bwd8_c(TT* __restrict__ s, int i, const B8<RS>& b, const O8<TT>& o, RS& cp1,
                                       RS& cp2) {
  RS p[8];
  bwd_p8<ST, TT, RS>(s, i, b, p);
  bwd_chain8<ST, TT, RS, ADD>(s, i, b, p, o, cp1, cp2);
}
template <int ST, class TT, class RS, class CF>
__device__ __forceinline__ void bwd8(TT* __restrict__ s, int i, const CF& cf, RS& cp1, RS& cp2) {
  B8<RS> b;
  b.load(cf, i);
  O8<TT> o;
  bwd8_c<ST, TT, RS, 0>(s, i, b, o, cp1, cp2);
}

// A run of forward blocks of eight while COND(i) holds, software-pipelined:
// one straight-line body forms the next block's right-hand sides (RHS8) and
// loads its factors while the current block's dependent chain runs, so the
// scheduler can fill the chain's latency. RHS8(i + 8) reads rows i+8.. that
// the chain of rows i..i+7 does not write. CONST: register constants, no loads.
#define FWD_RUN(COND, CF, CONST, RHS8)                                        \
  if (COND(i)) {                                                              \
    F8<RS> nx;                                                                \
    nx.load(CF, i);                                                           \
    TT rr[8];                                                                 \
    RHS8(i, rr);                                                              \
    while (COND(i + 8)) {                                                     \
      const F8<RS> cu = nx;                                                   \
      TT rc[8];                                                               \
      _Pragma("unroll") for (int k = 0; k < 8; ++k) rc[k] = rr[k];            \
      if (!(CONST)) nx.load(CF, i + 8);                                       \
      RHS8(i + 8, rr);                                                        \
      chain8_fwd<ST, TT, RS>(s, i, cu, rc, am2, am1);                         \
      i += 8;                                                                 \
    }                                                                         \
    chain8_fwd<ST, TT, RS>(s, i, nx, rr, am2, am1);                           \
    i += 8;                                                                   \
  }

// The same for back substitution blocks: the next block's u1 * (forward
// result) products, factors and (ADD) originals are formed during the current
// block's chain; they read rows below the ones the chain writes.
#define BWD_RUN(COND, CF, CONST)                                              \
  if (COND(i)) {                                                              \
    B8<RS> bn;                                                                \
    O8<TT> on;                                                                \
    RS pn[8];                                                                 \
    bn.load(CF, i);                                                           \
    if (ADD) on.load(og, ogs, i);                                             \
    bwd_p8<ST, TT, RS>(s, i, bn, pn);                                         \
    while (COND(i - 8)) {                                                     \
      const B8<RS> bu = bn;                                                   \
      const O8<TT> ou = on;                                                   \
      RS pu[8];                                                               \
      _Pragma("unroll") for (int k = 0; k < 8; ++k) pu[k] = pn[k];            \
      if (!(CONST)) bn.load(CF, i - 8);                                       \
      if (ADD) on.load(og, ogs, i - 8);                                       \
      bwd_p8<ST, TT, RS>(s, i - 8, bn, pn);                                   \
      bwd_chain8<ST, TT, RS, ADD>(s, i, bu, pu, ou, cp1, cp2);                \
      i -= 8;                                                                 \
    }                                                                         \
    bwd_chain8<ST, TT, RS, ADD>(s, i, bn, pn, on, cp1, cp2);                  \
    i -= 8;                                                                   \
  }

// Drives the forward rows [FIRST, LAST] with look-ahead LA: blocks of eight
// where the look-ahead rows have arrived, single rows otherwise.
#define FORWARD_ROWS(FIRST, LAST, LA, RHS8, STEP)                             \
  {                                                                           \
    const CoefConst<RS> CC{F.cl1, F.cl2, F.cu1, F.cu2, F.cu3};                \
    const CoefTable<RS> CT{F.l1, F.l2, F.u1, F.u2, F.u3};                     \
    int i = (FIRST);                                                          \
    while (i <= (LAST)) {                                                     \
      const int e = min((LAST), CI.ready - 1 - (LA));                         \
      if (e < i) {                                                            \
        if (!CI.wait_next(err)) return false;                                 \
        __syncwarp();                                                         \
        continue;                                                             \
      }                                                                       \
      {                                                                       \
        const int h = min(F.c0, e + 1);                                       \
        FWD_RUN(FR_H, CT, false, RHS8)                                        \
        for (; i < h; ++i) STEP(CT.L1(i), CT.L2(i))                           \
        const int ce = min(F.c1, e);                                          \
        FWD_RUN(FR_CE, CC, true, RHS8)                                        \
        FWD_RUN(FR_E, CT, false, RHS8)                                        \
        for (; i <= e; ++i) STEP(CT.L1(i), CT.L2(i))                          \
      }                                                                       \
    }                                                                         \
  }

#define FR_H(x) ((x) + 7 < h)
#define FR_CE(x) ((x) + 7 <= ce)
#define FR_E(x) ((x) + 7 <= e)
#define BR_TOP(x) ((x) > F.c1 && (x) - 7 >= lo)
#define BR_CE(x) ((x) - 7 >= ce)
#define BR_LO(x) ((x) - 7 >= lo)

// Back substitution over rows N-2 .. 0; after the lowest row of chunk c the
// chunk is final and DONE(c) runs (stores it). With ADD (filter) every row is
// stored as original + increment (OUT).
#define OUT(i, v) (ADD ? __ldg(og + (long long)(i) * ogs) + TT(v) : TT(v))
#define BACKWARD_ROWS(DONE)                                                   \
  {                                                                           \
    const CoefConst<RS> CC{F.cl1, F.cl2, F.cu1, F.cu2, F.cu3};                \
    const CoefTable<RS> CT{F.l1, F.l2, F.u1, F.u2, F.u3};                     \
    RS cp1 = CT.U1(N) * RS(S(N));                                             \
    S(N) = OUT(N, cp1);                                                       \
    RS c = CT.U1(N - 1) * RS(S(N - 1)) - CT.U2(N - 1) * cp1;                  \
    S(N - 1) = OUT(N - 1, c);                                                 \
    RS cp2 = cp1;                                                             \
    cp1 = c;                                                                  \
    int i = N - 2;                                                            \
    for (int ch = CI.NC - 1; ch >= 0; --ch) {                                 \
      const int lo = ch * CI.CR;                                              \
      BWD_RUN(BR_TOP, CT, false)                                              \
      {                                                                       \
        const int ce = max(F.c0, lo);                                         \
        BWD_RUN(BR_CE, CC, true)                                              \
      }                                                                       \
      BWD_RUN(BR_LO, CT, false)                                               \
      for (; i >= lo; --i) {                                                  \
        c = (CT.U1(i) * RS(S(i)) - CT.U2(i) * cp1) - CT.U3(i) * cp2;          \
        S(i) = OUT(i, c);                                                     \
        cp2 = cp1;                                                            \
        cp1 = c;                                                              \
      }                                                                       \
      DONE(ch);                                                               \
    }                                                                         \
  }

// Compact first derivative of one line held in shared memory with element
// stride ST (src/mo_numerics.f90:742-792). On return the line holds the
// derivative; Done(ch) is called as chunks become final. Returns false if a
// bounded wait gave up.
template <int ST, class TT, class RS, class Done>
__device__ __forceinline__ bool sweep_deriv(TT* __restrict__ s, int L, const LuRows<RS>& F, int ndf0, int ndf1,
                                            const DevScheme* __restrict__ sc, TT r00, TT r10, TT r01, TT r11,
                                            ChunkIn& CI, int* err, Done&& done) {
#define S(i) s[(i)*ST]
  constexpr int ADD = 0;
  const TT* og = nullptr;
  const int ogs = 0;
  const int N = L - 1;
  TT b0, b1, bn1, bn;
  if (ndf0 == 0) {
    const TT s0 = S(0), s1 = S(1), s2 = S(2), s3 = S(3), s4 = S(4);
    b0 = ((TT(CA_A01) * (s1 - s0) + TT(CA_A02) * (s2 - s0)) + TT(CA_A03) * (s3 - s0)) + TT(CA_A04) * (s4 - s0);
    b1 = ((TT(CA_A10) * (s0 - s1) + TT(CA_A12) * (s2 - s1)) + TT(CA_A13) * (s3 - s1)) + TT(CA_A14) * (s4 - s1);
  } else {
    TT t0 = 0, t1 = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      const TT v = S(i);
      t0 = t0 + TT(sc->pbci[0][0][i]) * v;
      t1 = t1 + TT(sc->pbci[0][1][i]) * v;
    }
    b0 = t0 + r00;
    b1 = t1 + r10;
  }
  if (ndf1 == 0) {
    const TT e0 = S(N), e1 = S(N - 1), e2 = S(N - 2), e3 = S(N - 3), e4 = S(N - 4);
    bn = ((TT(CA_A01) * (e0 - e1) + TT(CA_A02) * (e0 - e2)) + TT(CA_A03) * (e0 - e3)) + TT(CA_A04) * (e0 - e4);
    bn1 = ((TT(CA_A10) * (e1 - e0) + TT(CA_A12) * (e1 - e2)) + TT(CA_A13) * (e1 - e3)) + TT(CA_A14) * (e1 - e4);
  } else {
    TT t0 = 0, t1 = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      const TT v = S(N - i);
      t0 = t0 + TT(sc->pbci[0][0][i]) * v;
      t1 = t1 + TT(sc->pbci[0][1][i]) * v;
    }
    bn = -t0 - r01;
    bn1 = -t1 - r11;
  }
  // forward elimination, in place; originals kept in a register window
  TT w0 = S(0), w1 = S(1), w2 = S(2), w3 = S(3);
  RS am2 = RS(b0);
  RS am1 = RS(b1) - __ldg(F.l2 + 1) * am2;
  S(0) = TT(am2);
  S(1) = TT(am1);
#define FWD(L1, L2)                                                 \
  {                                                                 \
    const TT w4 = S(i + 2);                                         \
    const TT rhs = TT(CA_AA) * (w3 - w1) + TT(CA_AB) * (w4 - w0);   \
    const RS a = (RS(rhs) - (L1) * am2) - (L2) * am1;               \
    S(i) = TT(a);                                                   \
    w0 = w1; w1 = w2; w2 = w3; w3 = w4;                             \
    am2 = am1; am1 = a;                                             \
  }
#define RHS8(I, R) rhs8_deriv<ST, TT>(s, I, w0, w1, w2, w3, R)
  FORWARD_ROWS(2, N - 2, 2, RHS8, FWD)
#undef RHS8
#undef FWD
  {
    const RS a = (RS(bn1) - __ldg(F.l1 + N - 1) * am2) - __ldg(F.l2 + N - 1) * am1;
    S(N - 1) = TT(a);
    am2 = am1; am1 = a;
    const RS an = (RS(bn) - __ldg(F.l1 + N) * am2) - __ldg(F.l2 + N) * am1;
    S(N) = TT(an);
  }
  TRACE(3)
  BACKWARD_ROWS(done)
#undef S
  return true;
}

// Compact filter of one line (src/mo_numerics.f90:922-977): the increment is
// solved for and each row stored as original + increment, the original read
// from og[row * ogs] (this lane's line in the unfiltered field).
// ADD 1: every row is stored as original (og, stride ogs) + increment; ADD 0:
// the tile receives the increment alone (the caller adds it to the field).
template <int ST, class TT, class RS, int ADD, class Done>
__device__ __forceinline__ bool sweep_filter(TT* __restrict__ s, int L, const LuRows<RS>& F, int ndf0, int ndf1,
                                             const DevScheme* __restrict__ sc, TT r00, TT r10, TT r20, TT r01,
                                             TT r11, TT r21, const TT* __restrict__ og, int ogs,
                                             ChunkIn& CI, int* err, Done&& done) {
#define S(i) s[(i)*ST]
  const int N = L - 1;
  const TT fa = TT(sc->fa), fb = TT(sc->fb), fc = TT(sc->fc);
  auto fbc = [&](int r, int k) { return TT(sc->fbc[r][k]); };
  TT b0, b1, b2, bn2, bn1, bn;
  if (ndf0 == 0) {
    const TT s0 = S(0), s1 = S(1), s2 = S(2), s3 = S(3), s4 = S(4), s5 = S(5);
    b0 = (((fbc(0, 0) * (s1 - s0) + fbc(0, 1) * (s2 - s0)) + fbc(0, 2) * (s3 - s0)) + fbc(0, 3) * (s4 - s0)) +
         fbc(0, 4) * (s5 - s0);
    b1 = (((fbc(1, 0) * (s0 - s1) + fbc(1, 1) * (s2 - s1)) + fbc(1, 2) * (s3 - s1)) + fbc(1, 3) * (s4 - s1)) +
         fbc(1, 4) * (s5 - s1);
    b2 = (((fbc(2, 0) * (s0 - s2) + fbc(2, 1) * (s1 - s2)) + fbc(2, 2) * (s3 - s2)) + fbc(2, 3) * (s4 - s2)) +
         fbc(2, 4) * (s5 - s2);
  } else {
    TT t0 = 0, t1 = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      const TT v = S(i);
      t0 = t0 + TT(sc->pbci[1][0][i]) * v;
      t1 = t1 + TT(sc->pbci[1][1][i]) * v;
    }
    const TT s0 = S(0), s1 = S(1), s2 = S(2), s3 = S(3), s4 = S(4), s5 = S(5);
    const TT ra2 = s2 + s2;
    b0 = t0 + r00;
    b1 = t1 + r10;
    b2 = (fa * ((s1 + s3) - ra2) + fb * ((s0 + s4) - ra2)) + fc * ((r20 + s5) - ra2);
  }
  if (ndf1 == 0) {
    const TT e0 = S(N), e1 = S(N - 1), e2 = S(N - 2), e3 = S(N - 3), e4 = S(N - 4), e5 = S(N - 5);
    bn = (((fbc(0, 0) * (e1 - e0) + fbc(0, 1) * (e2 - e0)) + fbc(0, 2) * (e3 - e0)) + fbc(0, 3) * (e4 - e0)) +
         fbc(0, 4) * (e5 - e0);
    bn1 = (((fbc(1, 0) * (e0 - e1) + fbc(1, 1) * (e2 - e1)) + fbc(1, 2) * (e3 - e1)) + fbc(1, 3) * (e4 - e1)) +
          fbc(1, 4) * (e5 - e1);
    bn2 = (((fbc(2, 0) * (e0 - e2) + fbc(2, 1) * (e1 - e2)) + fbc(2, 2) * (e3 - e2)) + fbc(2, 3) * (e4 - e2)) +
          fbc(2, 4) * (e5 - e2);
  } else {
    TT t0 = 0, t1 = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      const TT v = S(N - i);
      t0 = t0 + TT(sc->pbci[1][0][i]) * v;
      t1 = t1 + TT(sc->pbci[1][1][i]) * v;
    }
    const TT e0 = S(N), e1 = S(N - 1), e2 = S(N - 2), e3 = S(N - 3), e4 = S(N - 4), e5 = S(N - 5);
    const TT ra2 = e2 + e2;
    bn = t0 + r01;
    bn1 = t1 + r11;
    bn2 = (fa * ((e3 + e1) - ra2) + fb * ((e4 + e0) - ra2)) + fc * ((e5 + r21) - ra2);
  }
  // forward elimination: rows 0..2 from the closures, 3..N-3 interior
  TT w0 = S(0), w1 = S(1), w2 = S(2), w3 = S(3), w4 = S(4), w5 = S(5);  // s[i-3..i+2] at i = 3
  RS am2 = RS(b0);
  RS am1 = RS(b1) - __ldg(F.l2 + 1) * am2;
  const RS a2 = (RS(b2) - __ldg(F.l1 + 2) * am2) - __ldg(F.l2 + 2) * am1;
  S(0) = TT(am2);
  S(1) = TT(am1);
  S(2) = TT(a2);
  am2 = am1;
  am1 = a2;
#define FWD(L1, L2)                                                                                       \
  {                                                                                                       \
    const TT w6 = S(i + 3);                                                                               \
    const TT rk = w3 + w3;                                                                                \
    const TT rhs = (fa * ((w2 + w4) - rk) + fb * ((w1 + w5) - rk)) + fc * ((w0 + w6) - rk);               \
    const RS a = (RS(rhs) - (L1) * am2) - (L2) * am1;                                                     \
    S(i) = TT(a);                                                                                         \
    w0 = w1; w1 = w2; w2 = w3; w3 = w4; w4 = w5; w5 = w6;                                                 \
    am2 = am1; am1 = a;                                                                                   \
  }
#define RHS8(I, R) rhs8_filter<ST, TT>(s, I, fa, fb, fc, w0, w1, w2, w3, w4, w5, R)
  FORWARD_ROWS(3, N - 3, 3, RHS8, FWD)
#undef RHS8
#undef FWD
  {
    RS a = (RS(bn2) - __ldg(F.l1 + N - 2) * am2) - __ldg(F.l2 + N - 2) * am1;
    S(N - 2) = TT(a);
    am2 = am1; am1 = a;
    a = (RS(bn1) - __ldg(F.l1 + N - 1) * am2) - __ldg(F.l2 + N - 1) * am1;
    S(N - 1) = TT(a);
    am2 = am1; am1 = a;
    a = (RS(bn) - __ldg(F.l1 + N) * am2) - __ldg(F.l2 + N) * am1;
    S(N) = TT(a);
  }
  TRACE(3)
  BACKWARD_ROWS(done)
#undef S
  return true;
}
#undef FORWARD_ROWS
#undef BACKWARD_ROWS
#undef OUT
#undef FWD_RUN
#undef BWD_RUN
#undef FR_H
#undef FR_CE
#undef FR_E
#undef BR_TOP
#undef BR_CE
#undef BR_LO

// The task of this CTA's tile: tdiv > 0 when every task of the launch has
// tdiv tiles (no table read on the CTA's start-up path), else the table.
__device__ __forceinline__ int tile_of(const int* __restrict__ tile_task, int tdiv) {
  return tdiv > 0 ? (int)(blockIdx.x / (unsigned)tdiv) : __ldg(tile_task + blockIdx.x);
}

__device__ __forceinline__ int find_task(const int* __restrict__ tile0, int ntasks, int tile) {
  int lo = 0, hi = ntasks - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(tile0 + mid) <= tile) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Line pitch (elements) of the row-major xi tile, whose rows arrive by one
// bulk copy per line: rows start 16-byte aligned; FP64: = 2 (mod 4) doubles,
// so 64-bit column walks see at most 2-way bank conflicts; FP32: an odd number
// of 16-byte units (4-way for 32-bit walks, which measured faster than
// element-wise copies into a conflict-free transposed tile).
template <class TT>
__host__ __device__ __forceinline__ int dir1_pitch(int L) {
  if (sizeof(TT) == 8) {
    int p = (L + 1) / 2 * 2;
    if (p % 4 == 0) p += 2;
    return p;
  }
  int p = (L + 3) / 4 * 4;
  if ((p / 4) % 2 == 0) p += 4;
  return p;
}

// One CTA = one warp = 32 lines. DIR: 1 xi, 2 eta, 3 zeta. OP: 0 derivative,
// 1 filter (in place, f += increment). TT: field and tile type, RS: type of
// the elimination. The tile moves in chunks (see ChunkIn): loads overlap the
// forward sweep, stores the back substitution.
template <int DIR, int OP, class TT, class RS>
__global__ void __maxnreg__(200) k_line(const LineTask* __restrict__ tasks, const int* __restrict__ tile_task,
                                             int tdiv, const CUtensorMap* __restrict__ maps,
                                             int* __restrict__ err) {
  constexpr int kVec = 16 / (int)sizeof(TT);  // elements per 16 bytes
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);
  TT* s = reinterpret_cast<TT*>(smem_raw + 128);
  const int lane = threadIdx.x;
  TRACE(0)
  // the tile's task and the error flag load together (independent)
  const int ti = tile_of(tile_task, tdiv);
  const int eflag = error_flag_early(err);
  const LineTask& T = tasks[ti];
  const TT* in = static_cast<const TT*>(T.in);
  TT* out = static_cast<TT*>(T.out);
  const int lt = blockIdx.x - T.tile0;
  const int L = T.L;
  const int X = T.X, Y = T.Y, Z = T.Z, Xp = T.Xp;
  const int NC = T.nbox, CR = T.by;
  int nval, x0 = 0, r0 = 0, fix = 0;  // fix: z for dir 2, y for dir 3
  if (DIR == 1) {
    r0 = lt * kLanes;
    nval = min(kLanes, Y * Z - r0);
  } else {
    fix = lt / T.ntx;
    x0 = (lt % T.ntx) * kLanes;
    nval = min(kLanes, X - x0);
  }
  const int P = dir1_pitch<TT>(L);
  const long long pstride = (DIR == 2) ? (long long)Xp : (long long)Xp * Y;  // dir 2/3 position stride
  const long long base = (DIR == 1) ? (long long)r0 * Xp
                                    : ((DIR == 2) ? (long long)fix * Y * Xp + x0 : (long long)fix * Xp + x0);
  const CUtensorMap* map_in = maps + 2 * ti;
  const CUtensorMap* map_out = maps + 2 * ti + 1;
  auto chunk_len = [&](int c) { return min(CR, L - c * CR); };
  if (lane == 0) {
    for (int c = 0; c < NC; ++c) mbar_init(bars + c, 1);
    mbar_init_done();
  }
  // a kernel launched after a bounded wait gave up does no work
  if (__shfl_sync(0xffffffffu, eflag, 0) != 0) return;
  __syncwarp();
  // issue the loads: chunk 0, the last chunk, then the middle ones
  for (int k = 0; k < NC; ++k) {
    const int c = (k == 0) ? 0 : (k == 1 ? NC - 1 : k - 1);
    if (DIR == 1) {
      const uint32_t bytes = (uint32_t)((chunk_len(c) + kVec - 1) / kVec * kVec * sizeof(TT));
      if (lane == 0) mbar_expect_tx(bars + c, bytes * nval);
      __syncwarp();
      if (lane < nval)
        bulk_g2s(s + lane * P + c * CR, in + base + (long long)lane * Xp + c * CR, bytes, bars + c);
    } else if (lane == 0) {
      mbar_expect_tx(bars + c, (uint32_t)(CR * kLanes * sizeof(TT)));
      if (DIR == 2) tma_load_3d(s + c * CR * kLanes, map_in, x0, c * CR, fix, bars + c);
      else tma_load_3d(s + c * CR * kLanes, map_in, x0, fix, c * CR, bars + c);
    }
  }
  prefetch_sweep_start(T.sc, static_cast<const RS*>(T.lu), L, lane);
  TRACE(1)
  // the received interface sums load while the tile's copies are in flight
  // (the periodic contraction below reads the tile instead)
  const bool has = lane < nval;
  int jk = 0;
  if (DIR == 1) jk = r0 + lane;
  else if (DIR == 2) jk = (x0 + lane) * Z + fix;
  else jk = fix * X + x0 + lane;
  const int nbs = T.nbs;
  const TT* recv = static_cast<const TT*>(T.recv);
  TT r00 = 0, r10 = 0, r20 = 0, r01 = 0, r11 = 0, r21 = 0;
  if (OP == 0 && !T.selfp) {
    if (has && T.ndf0) { r00 = recv[jk]; r10 = recv[nbs + jk]; }
    if (has && T.ndf1) { r01 = recv[2 * nbs + jk]; r11 = recv[3 * nbs + jk]; }
  }
  if (OP == 1) {
    if (has && T.ndf0) { r00 = recv[jk]; r10 = recv[nbs + jk]; r20 = recv[2 * nbs + jk]; }
    if (has && T.ndf1) { r01 = recv[3 * nbs + jk]; r11 = recv[4 * nbs + jk]; r21 = recv[5 * nbs + jk]; }
  }
  if (!mbar_wait(bars, 0) || !mbar_wait(bars + NC - 1, 0)) {
    if (lane == 0) atomicExch(err, kErrTimeout);
    // copies may still be landing: wait for the other chunks (bounded) before exit
    for (int c = 1; c < NC - 1; ++c) mbar_wait(bars + c, 0);
    return;
  }
  __syncwarp();
  TRACE(2)
  ChunkIn CI{bars, CR, NC, L, 1, (NC > 1 ? CR : L)};
  if (NC <= 2) CI.ready = L;
#ifdef CANARD_TRACE_WAITALL
  while (CI.ready < L) CI.wait_next(err);
  TRACE(7)
#endif
  // The xi filter of FP64 fields (in place) leaves the increment in the tile
  // and adds it to the field with one bulk FP64 reduce-add per line chunk; the
  // eta/zeta filters add the originals row by row (a reduce-add per 256-byte
  // row costs more than the re-read, measured).
  constexpr bool kRedAdd = OP == 1 && sizeof(TT) == 8 && DIR == 1;
  if (kRedAdd && (L & 1)) s[lane * P + L] = TT(0);  // the 16-byte tail's pad element adds 0
  // chunk c is final: store it
  auto done = [&](int c) {
    const int lo = c * CR, len = chunk_len(c);
    fence_proxy_async();
    __syncwarp();
    if (kRedAdd) {
      if (lane < nval) {
        bulk_s2g_add_f64(out + base + (long long)lane * Xp + lo, s + lane * P + lo,
                         (uint32_t)((len + kVec - 1) / kVec * kVec * sizeof(TT)));
        bulk_commit();
      }
    } else if (DIR == 1) {
      if (lane < nval) {
        bulk_s2g(out + base + (long long)lane * Xp + lo, s + lane * P + lo,
                 (uint32_t)((len + kVec - 1) / kVec * kVec * sizeof(TT)));
        bulk_commit();
      }
    } else if (lane == 0) {
      // positions past the block edge (and x past X) are not written
      if (DIR == 2) tma_store_3d(map_out, x0, lo, fix, s + lo * kLanes);
      else tma_store_3d(map_out, x0, fix, lo, s + lo * kLanes);
      bulk_commit();
    }
  };
  bool ok = true;
  // every lane runs the sweep (lanes past the tile edge on zero-filled or
  // stale columns) so the chunk hand-offs stay warp-uniform; only lanes with a
  // line read the receive buffers or write drva
  constexpr int ST = (DIR == 1) ? 1 : kLanes;
  TT* sl = (DIR == 1) ? s + lane * P : s + lane;
  const LuRows<RS> F(static_cast<const RS*>(T.lu), L, RS(T.cl1), RS(T.cl2), RS(T.cu1), RS(T.cu2), RS(T.cu3), T.c0);
  if (OP == 0) {
    if (T.selfp) {
      // The line is periodic onto itself, so the interface contraction the
      // other end would send (src/mo_numerics.f90:503-518 with n45 = 0) is
      // formed here from the tile: side 0 receives the sums over positions
      // N-1..N-12, side 1 over positions 1..12, accumulated in the same order.
      const DevScheme* sc = T.sc;
      const int N = L - 1;
#pragma unroll
      for (int i = 0; i < 12; ++i) {
        const TT v = sl[(N - 1 - i) * ST], w = sl[(1 + i) * ST];
        r00 = r00 + TT(sc->pbco[0][0][i]) * v;
        r10 = r10 + TT(sc->pbco[0][1][i]) * v;
        r01 = r01 + TT(sc->pbco[0][0][i]) * w;
        r11 = r11 + TT(sc->pbco[0][1][i]) * w;
      }
    }
    ok = sweep_deriv<ST, TT, RS>(sl, L, F, T.ndf0, T.ndf1, T.sc, r00, r10, r01, r11, CI, err, done);
    if (ok && has && T.drva) {
      TT* drva = static_cast<TT*>(T.drva);
      drva[jk + (long long)nbs * (T.m - 1)] = sl[0];
      drva[jk + (long long)nbs * ((T.m - 1) + 5)] = sl[(L - 1) * ST];
    }
  } else {
    // this lane's line of the unfiltered field (lanes without a line read
    // lane 0's, whose results are not stored)
    const TT* og = (DIR == 1) ? in + base + (long long)(has ? lane : 0) * Xp : in + base + (has ? lane : 0);
    const int ogs = (DIR == 1) ? 1 : (int)pstride;
    ok = sweep_filter<ST, TT, RS, kRedAdd ? 0 : 1>(sl, L, F, T.ndf0, T.ndf1, T.sc, r00, r10, r20, r01, r11, r21,
                                                   og, ogs, CI, err, done);
  }
  // every issued bulk store has to finish reading shared memory before exit;
  // after a timeout, wait for the chunks still in flight (bounded) instead
  if (!ok) {
    for (int c = CI.next; c < NC - 1; ++c) mbar_wait(bars + c, 0);
    return;
  }
  TRACE(4)
  bulk_wait_read0();
  TRACE(5)
#ifdef CANARD_TRACE
  if (threadIdx.x == 0) {
    unsigned smid;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
    g_trace[(long long)blockIdx.x * 8 + 6] = smid;
  }
#endif
}

// ---------------------------------------------------------------------------
// Split line solves of the FP32 path. One warp holds 16 lines; lane l owns
// rows [0, h) of line l and lane l+16 rows [h, L) of the same line, and both
// halves run the same instruction stream over their own rows, so each
// dependent recurrence is about half as long as in k_line and a warp's tile
// needs half the shared memory. The second half eliminates forward from a
// zero start and substitutes backward from its true end; the first half
// eliminates forward exactly and substitutes backward from a zero start.
// By linearity the true solution is then
//   rows >= h:  c = c_part + H0 a(h-2) + H1 a(h-1)
//   rows <  h:  c = c_part + E0 c(h) + E1 c(h+1)
// where H0, H1 are the second half's back substitution of the homogeneous
// forward solutions started at rows h-2, h-1, and E0, E1 the homogeneous
// backward solutions started at rows h, h+1. They depend only on the LU
// factors and decay geometrically away from h; the host tabulates them in
// FP64 as far as they exceed a threshold below the elimination type's
// rounding (stored FP32 for the FP32 eliminations, FP64 for the fast FP64
// mode). Algebraically this is the same elimination; the rounding differs
// from the one-lane order, which is why the bit-exact FP64 path does not use
// it.
constexpr int kHalf = 16;

// Correction tables of one (block, direction, system): H0, H1 indexed by
// row - h, E0, E1 indexed by h-1-row, each L + 8 long (zero past kh / ke,
// so blocks of eight read past the end without a bound).
template <class RS>
struct SplitTab {
  const RS* __restrict__ h0;
  const RS* __restrict__ h1;
  const RS* __restrict__ e0;
  const RS* __restrict__ e1;
  int kh, ke;
  int kf;  // rows the forward homogeneous solutions from h span (register recurrence)
};
using SplitTables = SplitTab<float>;

// Forward elimination of rows [ib, ie) with per-lane bounds (window w0..w3 =
// s[i-2..i+1] on entry), blocks of eight, software-pipelined: the next block's
// factors and right-hand sides are formed while the current block's chain runs
// (they read rows the chain does not write).
template <int ST, class TT, class RS, class CF>
__device__ __forceinline__ void fwd_rows_deriv(TT* s, int ib, int ie, const CF& cf, TT& w0, TT& w1, TT& w2,
                                               TT& w3, RS& am2, RS& am1) {
  int i = ib;
  if (i + 7 < ie) {
    F8<RS> nx;
    nx.load(cf, i);
    TT rr[8];
    rhs8_deriv<ST, TT>(s, i, w0, w1, w2, w3, rr);
    while (i + 15 < ie) {
      const F8<RS> cu = nx;
      TT rc[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) rc[k] = rr[k];
      nx.load(cf, i + 8);
      rhs8_deriv<ST, TT>(s, i + 8, w0, w1, w2, w3, rr);
      chain8_fwd<ST, TT, RS>(s, i, cu, rc, am2, am1);
      i += 8;
    }
    chain8_fwd<ST, TT, RS>(s, i, nx, rr, am2, am1);
    i += 8;
  }
  for (; i < ie; ++i) {
    const TT w4 = s[(i + 2) * ST];
    const TT rhs = TT(CA_AA) * (w3 - w1) + TT(CA_AB) * (w4 - w0);
    const RS a = (RS(rhs) - cf.L1(i) * am2) - cf.L2(i) * am1;
    s[i * ST] = TT(a);
    w0 = w1; w1 = w2; w2 = w3; w3 = w4;
    am2 = am1; am1 = a;
  }
}

template <int ST, class TT, class RS, class CF, bool DIRECT = false>
__device__ __forceinline__ void fwd_rows_filter(TT* s, int ib, int ie, const CF& cf, TT fa, TT fb, TT fc, TT& w0,
                                                TT& w1, TT& w2, TT& w3, TT& w4, TT& w5, RS& am2, RS& am1,
                                                TT al = 0, TT be = 0) {
  int i = ib;
  if (i + 7 < ie) {
    F8<RS> nx;
    nx.load(cf, i);
    TT rr[8];
    rhs8_filter<ST, TT, DIRECT>(s, i, fa, fb, fc, w0, w1, w2, w3, w4, w5, rr, al, be);
    while (i + 15 < ie) {
      const F8<RS> cu = nx;
      TT rc[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) rc[k] = rr[k];
      nx.load(cf, i + 8);
      rhs8_filter<ST, TT, DIRECT>(s, i + 8, fa, fb, fc, w0, w1, w2, w3, w4, w5, rr, al, be);
      chain8_fwd<ST, TT, RS>(s, i, cu, rc, am2, am1);
      i += 8;
    }
    chain8_fwd<ST, TT, RS>(s, i, nx, rr, am2, am1);
    i += 8;
  }
  for (; i < ie; ++i) {
    const TT w6 = s[(i + 3) * ST];
    const TT rk = w3 + w3;
    TT rhs = (fa * ((w2 + w4) - rk) + fb * ((w1 + w5) - rk)) + fc * ((w0 + w6) - rk);
    if (DIRECT) rhs = rhs + ((w3 + al * (w2 + w4)) + be * (w1 + w5));
    const RS a = (RS(rhs) - cf.L1(i) * am2) - cf.L2(i) * am1;
    s[i * ST] = TT(a);
    w0 = w1; w1 = w2; w2 = w3; w3 = w4; w4 = w5; w5 = w6;
    am2 = am1; am1 = a;
  }
}

// back substitution of rows ihi down to ilo (inclusive), per-lane bounds;
// the next block's factors and u1 products are formed during the current
// block's chain (they read rows below the ones it writes)
template <int ST, class TT, class RS, class CF>
__device__ __forceinline__ void bwd_rows(TT* s, int ihi, int ilo, const CF& cf, RS& cp1, RS& cp2) {
  int i = ihi;
  if (i - 7 >= ilo) {
    B8<RS> bn;
    O8<TT> on;
    RS pn[8];
    bn.load(cf, i);
    bwd_p8<ST, TT, RS>(s, i, bn, pn);
    while (i - 15 >= ilo) {
      const B8<RS> bu = bn;
      RS pu[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) pu[k] = pn[k];
      bn.load(cf, i - 8);
      bwd_p8<ST, TT, RS>(s, i - 8, bn, pn);
      bwd_chain8<ST, TT, RS, 0>(s, i, bu, pu, on, cp1, cp2);
      i -= 8;
    }
    bwd_chain8<ST, TT, RS, 0>(s, i, bn, pn, on, cp1, cp2);
    i -= 8;
  }
  for (; i >= ilo; --i) {
    const RS c = (cf.U1(i) * RS(s[i * ST]) - cf.U2(i) * cp1) - cf.U3(i) * cp2;
    s[i * ST] = TT(c);
    cp2 = cp1;
    cp1 = c;
  }
}

// Rows [ib, ie) in three per-lane segments: table factors below c0, the
// register constants on [c0, c1], table factors above c1.
template <int OP, int ST, class TT, class RS>
__device__ __forceinline__ void fwd3(TT* s, int ib, int ie, int c0, int c1, const CoefTable<RS>& ct,
                                     const CoefConst<RS>& cc, TT fa, TT fb, TT fc, TT& w0, TT& w1, TT& w2, TT& w3,
                                     TT& w4, TT& w5, RS& am2, RS& am1) {
  const int m0 = max(ib, c0), m1 = min(ie, c1 + 1);
  if (OP == 0) {
    fwd_rows_deriv<ST, TT, RS>(s, ib, min(ie, m0), ct, w0, w1, w2, w3, am2, am1);
    fwd_rows_deriv<ST, TT, RS>(s, m0, m1, cc, w0, w1, w2, w3, am2, am1);
    fwd_rows_deriv<ST, TT, RS>(s, max(ib, c1 + 1), ie, ct, w0, w1, w2, w3, am2, am1);
  } else {
    fwd_rows_filter<ST, TT, RS>(s, ib, min(ie, m0), ct, fa, fb, fc, w0, w1, w2, w3, w4, w5, am2, am1);
    fwd_rows_filter<ST, TT, RS>(s, m0, m1, cc, fa, fb, fc, w0, w1, w2, w3, w4, w5, am2, am1);
    fwd_rows_filter<ST, TT, RS>(s, max(ib, c1 + 1), ie, ct, fa, fb, fc, w0, w1, w2, w3, w4, w5, am2, am1);
  }
}

// rows ihi down to ilo in the same three segments
template <int ST, class TT, class RS>
__device__ __forceinline__ void bwd3(TT* s, int ihi, int ilo, int c0, int c1, const CoefTable<RS>& ct,
                                     const CoefConst<RS>& cc, RS& cp1, RS& cp2) {
  bwd_rows<ST, TT, RS>(s, ihi, max(ilo, c1 + 1), ct, cp1, cp2);
  bwd_rows<ST, TT, RS>(s, min(ihi, c1), max(ilo, c0), cc, cp1, cp2);
  bwd_rows<ST, TT, RS>(s, min(ihi, c0 - 1), ilo, ct, cp1, cp2);
}

// OP 0: derivative, OP 1: filter increment, of the lane's half of its line.
// On return (after a warp-wide barrier) the tile holds the derivative or the
// increment. q0, q1 (, q2): interface values received by the lane's own end
// (side 0 for the first half, side 1 for the second).
template <int OP, int ST, class TT, class RS = float>
__device__ __forceinline__ void sweep2(TT* __restrict__ s, int L, int h, int half, const CoefTable<RS>& cf,
                                       const CoefConst<RS>& cc, int c0, const SplitTab<RS>& H, int ndf0,
                                       int ndf1, const DevScheme* __restrict__ sc, TT q0, TT q1, TT q2) {
  constexpr int NE = OP == 0 ? 2 : 3;  // closure rows at each end
  const int N = L - 1;
  const unsigned full = 0xffffffffu;
  const TT fa = TT(sc->fa), fb = TT(sc->fb), fc = TT(sc->fc);
  auto fbc = [&](int r, int k) { return TT(sc->fbc[r][k]); };
  // ---- reads of the original line, before any row is overwritten
  TT b[3] = {0, 0, 0};           // closure right-hand sides of the own end (second half: bn, bn1, bn2)
  TT w0, w1, w2, w3, w4 = 0, w5 = 0;
  TT x[3] = {0, 0, 0};           // first half: originals at h, h+1 (, h+2)
  if (half == 0) {
    if (OP == 0) {
      if (ndf0 == 0) {
        const TT s0 = s[0], s1 = s[ST], s2 = s[2 * ST], s3 = s[3 * ST], s4 = s[4 * ST];
        b[0] = ((TT(CA_A01) * (s1 - s0) + TT(CA_A02) * (s2 - s0)) + TT(CA_A03) * (s3 - s0)) + TT(CA_A04) * (s4 - s0);
        b[1] = ((TT(CA_A10) * (s0 - s1) + TT(CA_A12) * (s2 - s1)) + TT(CA_A13) * (s3 - s1)) + TT(CA_A14) * (s4 - s1);
      } else {
        TT t0 = 0, t1 = 0;
#pragma unroll
        for (int i = 0; i < 12; ++i) {
          const TT v = s[i * ST];
          t0 = t0 + TT(sc->pbci[0][0][i]) * v;
          t1 = t1 + TT(sc->pbci[0][1][i]) * v;
        }
        b[0] = t0 + q0;
        b[1] = t1 + q1;
      }
      w0 = s[0]; w1 = s[ST]; w2 = s[2 * ST]; w3 = s[3 * ST];
    } else {
      const TT s0 = s[0], s1 = s[ST], s2 = s[2 * ST], s3 = s[3 * ST], s4 = s[4 * ST], s5 = s[5 * ST];
      if (ndf0 == 0) {
        b[0] = (((fbc(0, 0) * (s1 - s0) + fbc(0, 1) * (s2 - s0)) + fbc(0, 2) * (s3 - s0)) + fbc(0, 3) * (s4 - s0)) +
               fbc(0, 4) * (s5 - s0);
        b[1] = (((fbc(1, 0) * (s0 - s1) + fbc(1, 1) * (s2 - s1)) + fbc(1, 2) * (s3 - s1)) + fbc(1, 3) * (s4 - s1)) +
               fbc(1, 4) * (s5 - s1);
        b[2] = (((fbc(2, 0) * (s0 - s2) + fbc(2, 1) * (s1 - s2)) + fbc(2, 2) * (s3 - s2)) + fbc(2, 3) * (s4 - s2)) +
               fbc(2, 4) * (s5 - s2);
      } else {
        TT t0 = 0, t1 = 0;
#pragma unroll
        for (int i = 0; i < 12; ++i) {
          const TT v = s[i * ST];
          t0 = t0 + TT(sc->pbci[1][0][i]) * v;
          t1 = t1 + TT(sc->pbci[1][1][i]) * v;
        }
        const TT ra2 = s2 + s2;
        b[0] = t0 + q0;
        b[1] = t1 + q1;
        b[2] = (fa * ((s1 + s3) - ra2) + fb * ((s0 + s4) - ra2)) + fc * ((q2 + s5) - ra2);
      }
      w0 = s0; w1 = s1; w2 = s2; w3 = s3; w4 = s4; w5 = s5;
      x[2] = s[(h + 2) * ST];
    }
    x[0] = s[h * ST];
    x[1] = s[(h + 1) * ST];
  } else {
    if (OP == 0) {
      if (ndf1 == 0) {
        const TT e0 = s[N * ST], e1 = s[(N - 1) * ST], e2 = s[(N - 2) * ST], e3 = s[(N - 3) * ST],
                 e4 = s[(N - 4) * ST];
        b[0] = ((TT(CA_A01) * (e0 - e1) + TT(CA_A02) * (e0 - e2)) + TT(CA_A03) * (e0 - e3)) + TT(CA_A04) * (e0 - e4);
        b[1] = ((TT(CA_A10) * (e1 - e0) + TT(CA_A12) * (e1 - e2)) + TT(CA_A13) * (e1 - e3)) + TT(CA_A14) * (e1 - e4);
      } else {
        TT t0 = 0, t1 = 0;
#pragma unroll
        for (int i = 0; i < 12; ++i) {
          const TT v = s[(N - i) * ST];
          t0 = t0 + TT(sc->pbci[0][0][i]) * v;
          t1 = t1 + TT(sc->pbci[0][1][i]) * v;
        }
        b[0] = -t0 - q0;
        b[1] = -t1 - q1;
      }
      w0 = s[(h - 2) * ST]; w1 = s[(h - 1) * ST]; w2 = s[h * ST]; w3 = s[(h + 1) * ST];
    } else {
      const TT e0 = s[N * ST], e1 = s[(N - 1) * ST], e2 = s[(N - 2) * ST], e3 = s[(N - 3) * ST],
               e4 = s[(N - 4) * ST], e5 = s[(N - 5) * ST];
      if (ndf1 == 0) {
        b[0] = (((fbc(0, 0) * (e1 - e0) + fbc(0, 1) * (e2 - e0)) + fbc(0, 2) * (e3 - e0)) + fbc(0, 3) * (e4 - e0)) +
               fbc(0, 4) * (e5 - e0);
        b[1] = (((fbc(1, 0) * (e0 - e1) + fbc(1, 1) * (e2 - e1)) + fbc(1, 2) * (e3 - e1)) + fbc(1, 3) * (e4 - e1)) +
               fbc(1, 4) * (e5 - e1);
        b[2] = (((fbc(2, 0) * (e0 - e2) + fbc(2, 1) * (e1 - e2)) + fbc(2, 2) * (e3 - e2)) + fbc(2, 3) * (e4 - e2)) +
               fbc(2, 4) * (e5 - e2);
      } else {
        TT t0 = 0, t1 = 0;
#pragma unroll
        for (int i = 0; i < 12; ++i) {
          const TT v = s[(N - i) * ST];
          t0 = t0 + TT(sc->pbci[1][0][i]) * v;
          t1 = t1 + TT(sc->pbci[1][1][i]) * v;
        }
        const TT ra2 = e2 + e2;
        b[0] = t0 + q0;
        b[1] = t1 + q1;
        b[2] = (fa * ((e3 + e1) - ra2) + fb * ((e4 + e0) - ra2)) + fc * ((e5 + q2) - ra2);
      }
      w0 = s[(h - 3) * ST]; w1 = s[(h - 2) * ST]; w2 = s[(h - 1) * ST];
      w3 = s[h * ST]; w4 = s[(h + 1) * ST]; w5 = s[(h + 2) * ST];
    }
  }
  __syncwarp();
  // ---- forward elimination: closure rows (first half), the shared interior
  // loop, then NE tail rows whose right-hand sides come from registers
  RS am2 = 0, am1 = 0;
  if (half == 0) {
    am2 = RS(b[0]);
    am1 = RS(b[1]) - cf.L2(1) * am2;
    s[0] = TT(am2);
    s[ST] = TT(am1);
    if (OP == 1) {
      const RS a2 = (RS(b[2]) - cf.L1(2) * am2) - cf.L2(2) * am1;
      s[2 * ST] = TT(a2);
      am2 = am1;
      am1 = a2;
    }
  }
  const int fb0 = half == 0 ? NE : h;          // interior rows [fb0, fe0)
  const int fe0 = half == 0 ? h - NE : N + 1 - NE;
  const int c1 = L - 4;
  fwd3<OP, ST, TT, RS>(s, fb0, fe0, c0, c1, cf, cc, fa, fb, fc, w0, w1, w2, w3, w4, w5, am2, am1);
#pragma unroll
  for (int k = 0; k < NE; ++k) {
    const int i = fe0 + k;
    TT rhs;
    if (OP == 0) {
      const TT w4n = x[k];
      rhs = TT(CA_AA) * (w3 - w1) + TT(CA_AB) * (w4n - w0);
      w0 = w1; w1 = w2; w2 = w3; w3 = w4n;
    } else {
      const TT w6 = x[k];
      const TT rk = w3 + w3;
      rhs = (fa * ((w2 + w4) - rk) + fb * ((w1 + w5) - rk)) + fc * ((w0 + w6) - rk);
      w0 = w1; w1 = w2; w2 = w3; w3 = w4; w4 = w5; w5 = w6;
    }
    if (half == 1) rhs = b[NE - 1 - k];
    const RS a = (RS(rhs) - cf.L1(i) * am2) - cf.L2(i) * am1;
    s[i * ST] = TT(a);
    am2 = am1;
    am1 = a;
  }
  // the first half's a(h-2), a(h-1), needed by the second half's correction
  const int src = threadIdx.x & (kHalf - 1);
  const RS A0 = __shfl_sync(full, am2, src), A1 = __shfl_sync(full, am1, src);
  __syncwarp();
  TRACE(3)
  // ---- second half: its forward values from the zero start plus the
  // homogeneous forward solution g(i) = -l1 g(i-2) - l2 g(i-1) started from
  // the first half's a(h-2), a(h-1), over the rows where it has not decayed
  // (the recurrence in registers: no table reads); its back substitution
  // below then runs on the true forward values
  if (half == 1) {
    RS g2 = A0, g1 = A1;
    const int ie = min(h + H.kf, L);
    int i = h;
    for (; i < min(ie, c0); ++i) {  // rows below the constant range (short lines)
      const RS g = -(cf.L1(i) * g2) - cf.L2(i) * g1;
      s[i * ST] = TT(RS(s[i * ST]) + g);
      g2 = g1;
      g1 = g;
    }
#pragma unroll 4
    for (; i < min(ie, c1 + 1); ++i) {  // the constant interior factors
      const RS g = -(cc.L1(i) * g2) - cc.L2(i) * g1;
      s[i * ST] = TT(RS(s[i * ST]) + g);
      g2 = g1;
      g1 = g;
    }
    for (; i < ie; ++i) {
      const RS g = -(cf.L1(i) * g2) - cf.L2(i) * g1;
      s[i * ST] = TT(RS(s[i * ST]) + g);
      g2 = g1;
      g1 = g;
    }
  }
  __syncwarp();
  // ---- back substitution: two end rows (second half), then the shared loop
  RS cp1 = 0, cp2 = 0;
  if (half == 1) {
    cp1 = cf.U1(N) * RS(s[N * ST]);
    s[N * ST] = TT(cp1);
    const RS c = cf.U1(N - 1) * RS(s[(N - 1) * ST]) - cf.U2(N - 1) * cp1;
    s[(N - 1) * ST] = TT(c);
    cp2 = cp1;
    cp1 = c;
  }
  bwd3<ST, TT, RS>(s, half == 0 ? h - 1 : N - 2, half == 0 ? 0 : h, c0, c1, cf, cc, cp1, cp2);
  TRACE(4)
  // the second half's c(h), c(h+1) are final: the first half adds the
  // homogeneous backward solution e(i) = -u2 e(i+1) - u3 e(i+2) started from
  // them to its rows from the zero start, down to where it has decayed
  const RS C0 = __shfl_sync(full, cp1, src + kHalf), C1 = __shfl_sync(full, cp2, src + kHalf);
  __syncwarp();
  if (half == 0) {
    RS e1 = C0, e2 = C1;
    const int ib = max(h - H.ke, 0);
    int i = h - 1;
    for (; i > c1 && i >= ib; --i) {  // rows above the constant range (short lines)
      const RS e = -(cf.U2(i) * e1) - cf.U3(i) * e2;
      s[i * ST] = TT(RS(s[i * ST]) + e);
      e2 = e1;
      e1 = e;
    }
#pragma unroll 4
    for (; i >= max(ib, c0); --i) {  // the constant interior factors
      const RS e = -(cc.U2(i) * e1) - cc.U3(i) * e2;
      s[i * ST] = TT(RS(s[i * ST]) + e);
      e2 = e1;
      e1 = e;
    }
    for (; i >= ib; --i) {
      const RS e = -(cf.U2(i) * e1) - cf.U3(i) * e2;
      s[i * ST] = TT(RS(s[i * ST]) + e);
      e2 = e1;
      e1 = e;
    }
  }
  __syncwarp();
}

// One CTA = one warp = 16 lines, split solve (see above). DIR: 1 xi, 2 eta,
// 3 zeta. OP: 0 derivative, 1 filter (in place). TT: field and tile type;
// RS: elimination type (FP32 for the mixed path; FP64 for the fast FP64
// mode, whose factors and correction tables are FP64).
template <int DIR, int OP, class TT, class RS = float>
__global__ void __launch_bounds__(32) k_line2(const LineTask* __restrict__ tasks, const int* __restrict__ tile_task,
                                              int tdiv, const CUtensorMap* __restrict__ maps,
                                              int* __restrict__ err) {
  static_assert(OP == 0 || sizeof(TT) == 8, "the split filter acts on FP64 fields (reduce-add stores)");
  constexpr int kVec = 16 / (int)sizeof(TT);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);
  TT* s = reinterpret_cast<TT*>(smem_raw + 128);
  const int lane = threadIdx.x;
  const int half = lane >> 4, li = lane & (kHalf - 1);
  TRACE(0)
  // the tile's task and the error flag load together (independent)
  const int ti = tile_of(tile_task, tdiv);
  const int eflag = error_flag_early(err);
  const LineTask& T = tasks[ti];
  const TT* in = static_cast<const TT*>(T.in);
  TT* out = static_cast<TT*>(T.out);
  const int lt = blockIdx.x - T.tile0;
  const int L = T.L, h = T.h;
  const int X = T.X, Y = T.Y, Z = T.Z, Xp = T.Xp;
  const int NC = T.nbox, CR = T.by;
  int nval, x0 = 0, r0 = 0, fix = 0;
  if (DIR == 1) {
    r0 = lt * kHalf;
    nval = min(kHalf, Y * Z - r0);
  } else {
    fix = lt / T.ntx;
    x0 = (lt % T.ntx) * kHalf;
    nval = min(kHalf, X - x0);
  }
  const int P = dir1_pitch<TT>(L);
  const long long pstride = (DIR == 2) ? (long long)Xp : (long long)Xp * Y;
  const long long base = (DIR == 1) ? (long long)r0 * Xp
                                    : ((DIR == 2) ? (long long)fix * Y * Xp + x0 : (long long)fix * Xp + x0);
  const CUtensorMap* map_in = maps + 2 * ti;
  const CUtensorMap* map_out = maps + 2 * ti + 1;
  auto chunk_len = [&](int c) { return min(CR, L - c * CR); };
  if (lane == 0) {
    for (int c = 0; c < NC; ++c) mbar_init(bars + c, 1);
    mbar_init_done();
  }
  // a kernel launched after a bounded wait gave up does no work
  if (__shfl_sync(0xffffffffu, eflag, 0) != 0) return;
  __syncwarp();
  for (int c = 0; c < NC; ++c) {
    if (DIR == 1) {
      const uint32_t bytes = (uint32_t)((chunk_len(c) + kVec - 1) / kVec * kVec * sizeof(TT));
      if (lane == 0) mbar_expect_tx(bars + c, bytes * nval);
      __syncwarp();
      if (lane < nval) bulk_g2s(s + lane * P + c * CR, in + base + (long long)lane * Xp + c * CR, bytes, bars + c);
    } else if (lane == 0) {
      mbar_expect_tx(bars + c, (uint32_t)(CR * kHalf * sizeof(TT)));
      if (DIR == 2) tma_load_3d(s + c * CR * kHalf, map_in, x0, c * CR, fix, bars + c);
      else tma_load_3d(s + c * CR * kHalf, map_in, x0, fix, c * CR, bars + c);
    }
  }
  prefetch_sweep_start(T.sc, static_cast<const RS*>(T.lu), L, lane);
  TRACE(1)
  bool ok = true;
  for (int c = 0; c < NC; ++c) ok = mbar_wait(bars + c, 0) && ok;
  if (!ok) {
    if (lane == 0) atomicExch(err, kErrTimeout);
    return;
  }
  __syncwarp();
  TRACE(2)
  constexpr int ST = (DIR == 1) ? 1 : kHalf;
  TT* sl = (DIR == 1) ? s + li * P : s + li;
  const bool has = li < nval;
  int jk = 0;
  if (DIR == 1) jk = r0 + li;
  else if (DIR == 2) jk = (x0 + li) * Z + fix;
  else jk = fix * X + x0 + li;
  const int nbs = T.nbs, N = L - 1;
  const RS* lu = static_cast<const RS*>(T.lu);
  const CoefTable<RS> cf{lu, lu + L, lu + 2 * L, lu + 3 * L, lu + 4 * L};
  const RS* hb = lu + 5 * L;  // correction tables follow the factors
  const int LT = L + 8;
  const SplitTab<RS> H{hb, hb + LT, hb + 2 * LT, hb + 3 * LT, T.kg, T.ke, T.kf};
  const TT* recv = static_cast<const TT*>(T.recv);
  // interface sums received by the own end
  TT q0 = 0, q1 = 0, q2 = 0;
  if (OP == 0 && T.selfp) {
    // periodic onto itself: the contraction the other end would send (see k_line)
    const DevScheme* sc = T.sc;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      const TT v = half == 0 ? sl[(N - 1 - i) * ST] : sl[(1 + i) * ST];
      q0 = q0 + TT(sc->pbco[0][0][i]) * v;
      q1 = q1 + TT(sc->pbco[0][1][i]) * v;
    }
  } else if (has) {
    const int nc = OP == 0 ? 2 : 3;
    if (half == 0 && T.ndf0) {
      q0 = recv[jk]; q1 = recv[nbs + jk];
      if (OP == 1) q2 = recv[2 * nbs + jk];
    }
    if (half == 1 && T.ndf1) {
      q0 = recv[nc * nbs + jk]; q1 = recv[(nc + 1) * nbs + jk];
      if (OP == 1) q2 = recv[(nc + 2) * nbs + jk];
    }
  }
  const CoefConst<RS> cc{RS(T.cl1), RS(T.cl2), RS(T.cu1), RS(T.cu2), RS(T.cu3)};
  sweep2<OP, ST, TT, RS>(sl, L, h, half, cf, cc, T.c0, H, T.ndf0, T.ndf1, T.sc, q0, q1, q2);
  TRACE(5)
  if (OP == 0 && has && T.drva) {
    TT* drva = static_cast<TT*>(T.drva);
    if (half == 0) drva[jk + (long long)nbs * (T.m - 1)] = sl[0];
    else drva[jk + (long long)nbs * ((T.m - 1) + 5)] = sl[N * ST];
  }
  // filter (in place on FP64 fields): along xi the tile keeps the increment,
  // added to the field by one bulk FP64 reduce-add per line chunk; along
  // eta/zeta the lanes of both halves add the originals to the 16 columns
  // (coalesced 128-byte rows, still in L2), then the chunks are stored
  if (OP == 1 && DIR != 1) {
    if (has) {
      const TT* g = in + base + li;
      TT* col = s + li;
      const int lo = half == 0 ? 0 : h, hi = half == 0 ? h : L;
      int i = lo;
      // two batches of 16 rows in flight: the next batch loads while the
      // current one is added (the originals have usually left L2 by now)
      if (i + 16 <= hi) {
        TT v[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = __ldg(g + (long long)(i + k) * pstride);
        for (; i + 32 <= hi; i += 16) {
          TT w[16];
#pragma unroll
          for (int k = 0; k < 16; ++k) w[k] = __ldg(g + (long long)(i + 16 + k) * pstride);
#pragma unroll
          for (int k = 0; k < 16; ++k) col[(i + k) * kHalf] = v[k] + col[(i + k) * kHalf];
#pragma unroll
          for (int k = 0; k < 16; ++k) v[k] = w[k];
        }
#pragma unroll
        for (int k = 0; k < 16; ++k) col[(i + k) * kHalf] = v[k] + col[(i + k) * kHalf];
        i += 16;
      }
      for (; i < hi; ++i) col[i * kHalf] = __ldg(g + (long long)i * pstride) + col[i * kHalf];
    }
    __syncwarp();
  }
  if (OP == 1 && DIR == 1 && (L & 1)) s[li * P + L] = TT(0);  // the 16-byte tail's pad element adds 0
  fence_proxy_async();
  __syncwarp();
  for (int c = 0; c < NC; ++c) {
    const int lo = c * CR, len = chunk_len(c);
    if (DIR == 1) {
      if (lane < nval) {
        const uint32_t nb = (uint32_t)((len + kVec - 1) / kVec * kVec * sizeof(TT));
        if (OP == 1) bulk_s2g_add_f64(out + base + (long long)lane * Xp + lo, s + lane * P + lo, nb);
        else bulk_s2g(out + base + (long long)lane * Xp + lo, s + lane * P + lo, nb);
      }
    } else if (lane == 0) {
      if (DIR == 2) tma_store_3d(map_out, x0, lo, fix, s + lo * kHalf);
      else tma_store_3d(map_out, x0, fix, lo, s + lo * kHalf);
    }
  }
  bulk_commit();
  bulk_wait_read0();
  TRACE(7)
#ifdef CANARD_TRACE
  if (threadIdx.x == 0) {
    unsigned smid;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
    g_trace[(long long)blockIdx.x * 8 + 6] = smid;
  }
#endif
}

// ---------------------------------------------------------------------------
// Two-ended ("twisted") line solve: two warps per tile of 32 lines, one lane
// per line in each. Warp 0 runs the LU elimination of the line from row 0 to
// row h-1. Warp 1 runs the LU elimination of the reversed line (the system
// with its two ends swapped, factored by the host the same way) from row L-1
// to row h. The first rows of U are rows of U of the whole system, so the
// last two forward values of each warp give four equations in x(h-2..h+1),
// which a 4 x 4 inverse from the host solves; each warp then substitutes back
// towards its own end. Exact up to rounding: no homogeneous corrections, and
// each chain is half a line long. Warp 1 works on a reversed view of its
// lines (negative row stride from row L-1), on which the derivative's
// right-hand sides change sign; its U1 factors carry that sign.

// Rows [ib, ie) in four per-lane segments: shared-memory factors below
// k0 = min(ks, c0), table factors on [k0, c0), the register constants on
// [c0, c1], table factors above c1.
template <int OP, int ST, class TT, class RS, bool DIRECT = false>
__device__ __forceinline__ void fwd4(TT* s, int ib, int ie, int ks, int c0, int c1, const CoefShared<RS>& sh,
                                     const CoefTable<RS>& ct, const CoefConst<RS>& cc, TT fa, TT fb, TT fc, TT& w0,
                                     TT& w1, TT& w2, TT& w3, TT& w4, TT& w5, RS& am2, RS& am1, TT al = 0,
                                     TT be = 0) {
  const int k0 = min(ks, c0);
  const int a1 = min(ie, k0), b0 = max(ib, k0), b1 = min(ie, c0), m0 = max(ib, c0), m1 = min(ie, c1 + 1),
            d0 = max(ib, c1 + 1);
  if (OP == 0) {
    fwd_rows_deriv<ST, TT, RS>(s, ib, a1, sh, w0, w1, w2, w3, am2, am1);
    fwd_rows_deriv<ST, TT, RS>(s, b0, b1, ct, w0, w1, w2, w3, am2, am1);
    fwd_rows_deriv<ST, TT, RS>(s, m0, m1, cc, w0, w1, w2, w3, am2, am1);
    fwd_rows_deriv<ST, TT, RS>(s, d0, ie, ct, w0, w1, w2, w3, am2, am1);
  } else {
    fwd_rows_filter<ST, TT, RS, CoefShared<RS>, DIRECT>(s, ib, a1, sh, fa, fb, fc, w0, w1, w2, w3, w4, w5, am2,
                                                        am1, al, be);
    fwd_rows_filter<ST, TT, RS, CoefTable<RS>, DIRECT>(s, b0, b1, ct, fa, fb, fc, w0, w1, w2, w3, w4, w5, am2, am1,
                                                       al, be);
    fwd_rows_filter<ST, TT, RS, CoefConst<RS>, DIRECT>(s, m0, m1, cc, fa, fb, fc, w0, w1, w2, w3, w4, w5, am2, am1,
                                                       al, be);
    fwd_rows_filter<ST, TT, RS, CoefTable<RS>, DIRECT>(s, d0, ie, ct, fa, fb, fc, w0, w1, w2, w3, w4, w5, am2, am1,
                                                       al, be);
  }
}

// rows ihi down to ilo in the same four segments
template <int ST, class TT, class RS>
__device__ __forceinline__ void bwd4(TT* s, int ihi, int ilo, int ks, int c0, int c1, const CoefShared<RS>& sh,
                                     const CoefTable<RS>& ct, const CoefConst<RS>& cc, RS& cp1, RS& cp2) {
  const int k0 = min(ks, c0);
  bwd_rows<ST, TT, RS>(s, ihi, max(ilo, c1 + 1), ct, cp1, cp2);
  bwd_rows<ST, TT, RS>(s, min(ihi, c1), max(ilo, c0), cc, cp1, cp2);
  bwd_rows<ST, TT, RS>(s, min(ihi, c0 - 1), max(ilo, k0), ct, cp1, cp2);
  bwd_rows<ST, TT, RS>(s, min(ihi, k0 - 1), ilo, sh, cp1, cp2);
}

// Reads of the original line (view rows 0..11 for the closures of the own
// end, rows hw..hw+2 next to the half), made before either warp writes.
template <class TT>
struct TwState {
  TT b[3];  // closure right-hand sides of the own end
  TT w[6];  // the window s[0..5] that the forward sweep starts with
  TT x[3];  // originals at view rows hw, hw+1, hw+2 (the other half's first rows)
};

template <int OP, int ST, class TT, bool DIRECT = false>
__device__ __forceinline__ void twist_read(const TT* __restrict__ s, int hw, int ndf,
                                           const DevScheme* __restrict__ sc, TT q0, TT q1, TT q2, TwState<TT>& t) {
  const TT fa = TT(sc->fa), fb = TT(sc->fb), fc = TT(sc->fc);
  auto fbc = [&](int r, int k) { return TT(sc->fbc[r][k]); };
  t.b[2] = 0;
  t.x[2] = 0;
  t.w[4] = t.w[5] = 0;
  if (OP == 0) {
    if (ndf == 0) {
      const TT s0 = s[0], s1 = s[ST], s2 = s[2 * ST], s3 = s[3 * ST], s4 = s[4 * ST];
      t.b[0] = ((TT(CA_A01) * (s1 - s0) + TT(CA_A02) * (s2 - s0)) + TT(CA_A03) * (s3 - s0)) + TT(CA_A04) * (s4 - s0);
      t.b[1] = ((TT(CA_A10) * (s0 - s1) + TT(CA_A12) * (s2 - s1)) + TT(CA_A13) * (s3 - s1)) + TT(CA_A14) * (s4 - s1);
    } else {
      TT t0 = 0, t1 = 0;
#pragma unroll
      for (int i = 0; i < 12; ++i) {
        const TT v = s[i * ST];
        t0 = t0 + TT(sc->pbci[0][0][i]) * v;
        t1 = t1 + TT(sc->pbci[0][1][i]) * v;
      }
      t.b[0] = t0 + q0;
      t.b[1] = t1 + q1;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) t.w[k] = s[k * ST];
  } else {
    const TT s0 = s[0], s1 = s[ST], s2 = s[2 * ST], s3 = s[3 * ST], s4 = s[4 * ST], s5 = s[5 * ST];
    if (ndf == 0) {
      t.b[0] = (((fbc(0, 0) * (s1 - s0) + fbc(0, 1) * (s2 - s0)) + fbc(0, 2) * (s3 - s0)) + fbc(0, 3) * (s4 - s0)) +
               fbc(0, 4) * (s5 - s0);
      t.b[1] = (((fbc(1, 0) * (s0 - s1) + fbc(1, 1) * (s2 - s1)) + fbc(1, 2) * (s3 - s1)) + fbc(1, 3) * (s4 - s1)) +
               fbc(1, 4) * (s5 - s1);
      t.b[2] = (((fbc(2, 0) * (s0 - s2) + fbc(2, 1) * (s1 - s2)) + fbc(2, 2) * (s3 - s2)) + fbc(2, 3) * (s4 - s2)) +
               fbc(2, 4) * (s5 - s2);
    } else {
      TT t0 = 0, t1 = 0;
#pragma unroll
      for (int i = 0; i < 12; ++i) {
        const TT v = s[i * ST];
        t0 = t0 + TT(sc->pbci[1][0][i]) * v;
        t1 = t1 + TT(sc->pbci[1][1][i]) * v;
      }
      const TT ra2 = s2 + s2;
      t.b[0] = t0 + q0;
      t.b[1] = t1 + q1;
      t.b[2] = (fa * ((s1 + s3) - ra2) + fb * ((s0 + s4) - ra2)) + fc * ((q2 + s5) - ra2);
    }
    if (DIRECT) {  // (A x) of the three closure rows: the filtered values' right-hand sides
      const double* a = &sc->albef[ndf][0][0];
      t.b[0] = t.b[0] + ((s0 + TT(a[3]) * s1) + TT(a[4]) * s2);
      t.b[1] = t.b[1] + (((TT(a[6]) * s0 + s1) + TT(a[8]) * s2) + TT(a[9]) * s3);
      t.b[2] = t.b[2] + ((((TT(a[10]) * s0 + TT(a[11]) * s1) + s2) + TT(a[13]) * s3) + TT(a[14]) * s4);
    }
    t.w[0] = s0; t.w[1] = s1; t.w[2] = s2; t.w[3] = s3; t.w[4] = s4; t.w[5] = s5;
    t.x[2] = s[(hw + 2) * ST];
  }
  t.x[0] = s[hw * ST];
  t.x[1] = s[(hw + 1) * ST];
}

// Forward elimination of view rows 0..hw-1: the closure rows, the interior
// (three segments, as fwd3), then the last NE rows, whose look-ahead rows
// belong to the other half and come from the values read before.
template <int OP, int ST, class TT, class RS, bool DIRECT = false>
__device__ __forceinline__ void twist_fwd(TT* __restrict__ s, int L, int hw, const CoefShared<RS>& sh, int ks,
                                          const CoefTable<RS>& cf, const CoefConst<RS>& cc, int c0,
                                          const DevScheme* __restrict__ sc, const TwState<TT>& t) {
  constexpr int NE = OP == 0 ? 2 : 3;
  const TT fa = TT(sc->fa), fb = TT(sc->fb), fc = TT(sc->fc);
  const TT al = DIRECT ? TT(sc->alphf) : TT(0), be = DIRECT ? TT(sc->betf) : TT(0);
  TT w0 = t.w[0], w1 = t.w[1], w2 = t.w[2], w3 = t.w[3], w4 = t.w[4], w5 = t.w[5];
  // rows 1 and 2 lie below the constant range, so among the staged factors
  RS am2 = RS(t.b[0]);
  RS am1 = RS(t.b[1]) - sh.L2(1) * am2;
  s[0] = TT(am2);
  s[ST] = TT(am1);
  if (OP == 1) {
    const RS a2 = (RS(t.b[2]) - sh.L1(2) * am2) - sh.L2(2) * am1;
    s[2 * ST] = TT(a2);
    am2 = am1;
    am1 = a2;
  }
  fwd4<OP, ST, TT, RS, DIRECT>(s, NE, hw - NE, ks, c0, L - 4, sh, cf, cc, fa, fb, fc, w0, w1, w2, w3, w4, w5, am2,
                               am1, al, be);
#pragma unroll
  for (int k = 0; k < NE; ++k) {
    const int i = hw - NE + k;
    TT rhs;
    if (OP == 0) {
      const TT w4n = t.x[k];
      rhs = TT(CA_AA) * (w3 - w1) + TT(CA_AB) * (w4n - w0);
      w0 = w1; w1 = w2; w2 = w3; w3 = w4n;
    } else {
      const TT w6 = t.x[k];
      const TT rk = w3 + w3;
      rhs = (fa * ((w2 + w4) - rk) + fb * ((w1 + w5) - rk)) + fc * ((w0 + w6) - rk);
      if (DIRECT) rhs = rhs + ((w3 + al * (w2 + w4)) + be * (w1 + w5));
      w0 = w1; w1 = w2; w2 = w3; w3 = w4; w4 = w5; w5 = w6;
    }
    const RS a = (RS(rhs) - cf.L1(i) * am2) - cf.L2(i) * am1;
    s[i * ST] = TT(a);
    am2 = am1;
    am1 = a;
  }
}

// Factor table of a twisted solve: the LU factors of the line (5 L), those of
// the reversed line (5 L, U1 negated for the derivative), the 4 x 4 inverse
// of the meeting equations with the U1 factors of their rows folded in (row
// k gives x(h-2+k) from the forward values at rows h-2, h-1, h, h+1), and the
// reversed system's bitwise-constant interior factors (5).
constexpr int kTwistExtra = 16 + 5;
// factor rows per warp staged in shared memory behind the tile: the closure
// rows below the constant range (at most 64 rows in FP64, 34 in FP32, for the
// schemes' 8th-order derivative and filter), read there instead of from L2
constexpr int kTwistSh = 64;
// shared-memory offset of the staged factors: the tile, rounded up to 16 bytes
__host__ __device__ __forceinline__ size_t twist_tile_bytes(int dir, int L, int nbox, int by, size_t es, int pitch) {
  const size_t t = dir == 0 ? (size_t)32 * pitch * es : (size_t)nbox * by * 32 * es;
  return (t + 15) / 16 * 16;
}

// One CTA = two warps = 32 lines. DIR: 1 xi, 2 eta, 3 zeta. OP: 0
// derivative, 1 filter (in place). TT: field and tile type; RS: elimination
// type. T.h: first row of the reversed half; T.kg: first row of the reversed
// system's constant factor range.
template <int DIR, int OP, class TT, class RS>
__global__ void __launch_bounds__(64) k_line2t(const LineTask* __restrict__ tasks, const int* __restrict__ tile_task,
                                               int tdiv, const CUtensorMap* __restrict__ maps,
                                               int* __restrict__ err) {
  static_assert(OP == 0 || sizeof(TT) == 8, "the filter acts on FP64 fields (reduce-add stores)");
  constexpr int kVec = 16 / (int)sizeof(TT);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);
  TT* s = reinterpret_cast<TT*>(smem_raw + 128);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool rev = warp == 1;
  TRACE(0)
  const int ti = tile_of(tile_task, tdiv);
  const int eflag = error_flag_early(err);
  const LineTask& T = tasks[ti];
  const TT* in = static_cast<const TT*>(T.in);
  TT* out = static_cast<TT*>(T.out);
  const int lt = blockIdx.x - T.tile0;
  const int L = T.L, h = T.h, N = L - 1;
  const int X = T.X, Y = T.Y, Z = T.Z, Xp = T.Xp;
  const int NC = T.nbox, CR = T.by;
  int nval, x0 = 0, r0 = 0, fix = 0;
  if (DIR == 1) {
    r0 = lt * kLanes;
    nval = min(kLanes, Y * Z - r0);
  } else {
    fix = lt / T.ntx;
    x0 = (lt % T.ntx) * kLanes;
    nval = min(kLanes, X - x0);
  }
  const int P = dir1_pitch<TT>(L);
  const long long pstride = (DIR == 2) ? (long long)Xp : (long long)Xp * Y;
  const long long base = (DIR == 1) ? (long long)r0 * Xp
                                    : ((DIR == 2) ? (long long)fix * Y * Xp + x0 : (long long)fix * Xp + x0);
  const CUtensorMap* map_in = maps + 2 * ti;
  const CUtensorMap* map_out = maps + 2 * ti + 1;
  auto chunk_len = [&](int c) { return min(CR, L - c * CR); };
  if (threadIdx.x == 0) {
    for (int c = 0; c < NC; ++c) mbar_init(bars + c, 1);
    mbar_init_done();
  }
  // one decision for both warps (they meet at CTA barriers below): a kernel
  // launched after a bounded wait gave up does no work
  if (__syncthreads_or(eflag != 0)) return;
  if (!rev) {
    for (int c = 0; c < NC; ++c) {
      if (DIR == 1) {
        const uint32_t bytes = (uint32_t)((chunk_len(c) + kVec - 1) / kVec * kVec * sizeof(TT));
        if (lane == 0) mbar_expect_tx(bars + c, bytes * nval);
        __syncwarp();
        if (lane < nval)
          bulk_g2s(s + lane * P + c * CR, in + base + (long long)lane * Xp + c * CR, bytes, bars + c);
      } else if (lane == 0) {
        mbar_expect_tx(bars + c, (uint32_t)(CR * kLanes * sizeof(TT)));
        if (DIR == 2) tma_load_3d(s + c * CR * kLanes, map_in, x0, c * CR, fix, bars + c);
        else tma_load_3d(s + c * CR * kLanes, map_in, x0, fix, c * CR, bars + c);
      }
    }
  }
  if (lane < 10) prefetch_l1(reinterpret_cast<const char*>(T.sc) + 128 * lane);
  TRACE(1)
  // while the tile's copies are in flight: the factors, the staged closure
  // factors and the received interface sums (none of them read the tile)
  constexpr int ST = (DIR == 1) ? 1 : kLanes;
  TT* sl = (DIR == 1) ? s + lane * P : s + lane;
  TT* sv = rev ? sl + N * ST : sl;  // the warp's view of its line (warp 1: reversed)
  const bool has = lane < nval;
  int jk = 0;
  if (DIR == 1) jk = r0 + lane;
  else if (DIR == 2) jk = (x0 + lane) * Z + fix;
  else jk = fix * X + x0 + lane;
  const int nbs = T.nbs;
  const RS* lu = static_cast<const RS*>(T.lu);
  const RS* tb = rev ? lu + 5 * L : lu;
  const RS* Wt = lu + 10 * L;
  const CoefTable<RS> cf{tb, tb + L, tb + 2 * L, tb + 3 * L, tb + 4 * L};
  const CoefConst<RS> cc = rev ? CoefConst<RS>{__ldg(Wt + 16), __ldg(Wt + 17), __ldg(Wt + 18), __ldg(Wt + 19),
                                               __ldg(Wt + 20)}
                               : CoefConst<RS>{RS(T.cl1), RS(T.cl2), RS(T.cu1), RS(T.cu2), RS(T.cu3)};
  const int c0 = rev ? T.kg : T.c0;
  const int hw = rev ? L - h : h;  // rows of the warp's half
  // the warp's closure-row factors into shared memory (read below c0 only)
  const int ks = min(min(c0, hw), kTwistSh);
  RS* fsh = reinterpret_cast<RS*>(smem_raw + 128 + twist_tile_bytes(DIR - 1, L, NC, CR, sizeof(TT), P)) +
            warp * 5 * kTwistSh;
#pragma unroll
  for (int k = 0; k < 5; ++k)
    for (int r = lane; r < ks; r += 32) fsh[k * kTwistSh + r] = __ldg(tb + k * L + r);
  const CoefShared<RS> sh{fsh, fsh + kTwistSh, fsh + 2 * kTwistSh, fsh + 3 * kTwistSh, fsh + 4 * kTwistSh};
  const TT* recv = static_cast<const TT*>(T.recv);
  // interface sums received by the warp's own end
  TT q0 = 0, q1 = 0, q2 = 0;
  if (!(OP == 0 && T.selfp) && has) {
    const int nc = OP == 0 ? 2 : 3;
    if (!rev && T.ndf0) {
      q0 = recv[jk]; q1 = recv[nbs + jk];
      if (OP == 1) q2 = recv[2 * nbs + jk];
    }
    if (rev && T.ndf1) {
      q0 = recv[nc * nbs + jk]; q1 = recv[(nc + 1) * nbs + jk];
      if (OP == 1) q2 = recv[(nc + 2) * nbs + jk];
    }
  }
  bool ok = true;
  for (int c = 0; c < NC; ++c) ok = mbar_wait(bars + c, 0) && ok;
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) atomicExch(err, kErrTimeout);
    return;
  }
  TRACE(2)
  if (OP == 0 && T.selfp) {
    // periodic onto itself: the contraction the other end would send (see k_line)
    const DevScheme* sc = T.sc;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      const TT v = !rev ? sl[(N - 1 - i) * ST] : sl[(1 + i) * ST];
      q0 = q0 + TT(sc->pbco[0][0][i]) * v;
      q1 = q1 + TT(sc->pbco[0][1][i]) * v;
    }
  }
  // FP64 eliminations of the filter solve for the filtered values directly
  // (right-hand side B x): no originals to add afterwards (the FP32 one keeps
  // the increment, whose rounding is then relative to the increment)
  constexpr bool kDirect = OP == 1 && sizeof(RS) == 8;
  TwState<TT> tw;
  if (!rev) twist_read<OP, ST, TT, kDirect>(sv, hw, T.ndf0, T.sc, q0, q1, q2, tw);
  else twist_read<OP, -ST, TT, kDirect>(sv, hw, T.ndf1, T.sc, q0, q1, q2, tw);
  __syncthreads();
  if (!rev) twist_fwd<OP, ST, TT, RS, kDirect>(sv, L, hw, sh, ks, cf, cc, c0, T.sc, tw);
  else twist_fwd<OP, -ST, TT, RS, kDirect>(sv, L, hw, sh, ks, cf, cc, c0, T.sc, tw);
  __syncthreads();
  TRACE(3)
  // the four meeting unknowns; warp 0 keeps x(h-2), x(h-1), warp 1 x(h), x(h+1)
  RS xa, xb;
  {
    const RS y0 = RS(sl[(h - 2) * ST]), y1 = RS(sl[(h - 1) * ST]), z0 = RS(sl[h * ST]), z1 = RS(sl[(h + 1) * ST]);
    const RS* w = Wt + (rev ? 8 : 0);
    xa = ((__ldg(w + 0) * y0 + __ldg(w + 1) * y1) + __ldg(w + 2) * z0) + __ldg(w + 3) * z1;
    xb = ((__ldg(w + 4) * y0 + __ldg(w + 5) * y1) + __ldg(w + 6) * z0) + __ldg(w + 7) * z1;
  }
  __syncthreads();
  if (!rev) {
    sv[(hw - 2) * ST] = TT(xa);
    sv[(hw - 1) * ST] = TT(xb);
    RS cp1 = xa, cp2 = xb;
    bwd4<ST, TT, RS>(sv, hw - 3, 0, ks, c0, L - 4, sh, cf, cc, cp1, cp2);
  } else {
    sv[(hw - 1) * -ST] = TT(xa);
    sv[(hw - 2) * -ST] = TT(xb);
    RS cp1 = xb, cp2 = xa;
    bwd4<-ST, TT, RS>(sv, hw - 3, 0, ks, c0, L - 4, sh, cf, cc, cp1, cp2);
  }
  TRACE(4)
  if (OP == 0 && has && T.drva) {
    TT* drva = static_cast<TT*>(T.drva);
    if (!rev) drva[jk + (long long)nbs * (T.m - 1)] = sl[0];
    else drva[jk + (long long)nbs * ((T.m - 1) + 5)] = sl[N * ST];
  }
  // filter (in place on FP64 fields): along xi the tile keeps the increment,
  // added to the field by one bulk FP64 reduce-add per line; along eta/zeta
  // each warp adds the originals to its half of the 32 columns (coalesced
  // rows), then the chunks are stored
  if (OP == 1 && !kDirect && DIR != 1 && has) {
    const TT* g = in + base + lane;
    TT* col = s + lane;
    const int lo = !rev ? 0 : h, hi = !rev ? h : L;
    int i = lo;
    if (i + 16 <= hi) {
      TT v[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) v[k] = __ldg(g + (long long)(i + k) * pstride);
      for (; i + 32 <= hi; i += 16) {
        TT w[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) w[k] = __ldg(g + (long long)(i + 16 + k) * pstride);
#pragma unroll
        for (int k = 0; k < 16; ++k) col[(i + k) * kLanes] = v[k] + col[(i + k) * kLanes];
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = w[k];
      }
#pragma unroll
      for (int k = 0; k < 16; ++k) col[(i + k) * kLanes] = v[k] + col[(i + k) * kLanes];
      i += 16;
    }
    for (; i < hi; ++i) col[i * kLanes] = __ldg(g + (long long)i * pstride) + col[i * kLanes];
  }
  if (OP == 1 && !kDirect && DIR == 1 && (L & 1) && !rev) s[lane * P + L] = TT(0);  // the 16-byte tail's pad adds 0
  fence_proxy_async();
  __syncthreads();
  TRACE(5)
  if (rev) return;
  for (int c = 0; c < NC; ++c) {
    const int lo = c * CR, len = chunk_len(c);
    if (DIR == 1) {
      if (lane < nval) {
        const uint32_t nb = (uint32_t)((len + kVec - 1) / kVec * kVec * sizeof(TT));
        if (OP == 1 && !kDirect) bulk_s2g_add_f64(out + base + (long long)lane * Xp + lo, s + lane * P + lo, nb);
        else bulk_s2g(out + base + (long long)lane * Xp + lo, s + lane * P + lo, nb);
      }
    } else if (lane == 0) {
      if (DIR == 2) tma_store_3d(map_out, x0, lo, fix, s + lo * kLanes);
      else tma_store_3d(map_out, x0, fix, lo, s + lo * kLanes);
    }
  }
  bulk_commit();
  bulk_wait_read0();
  TRACE(7)
#ifdef CANARD_TRACE
  if (threadIdx.x == 0) {
    unsigned smid;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
    g_trace[(long long)blockIdx.x * 8 + 6] = smid;
  }
#endif
}

// ---------------------------------------------------------------------------
// Quad split derivative: 8 lines per warp, four lanes per line. Lane (seg =
// lane / 8, li = lane % 8) owns rows [q_seg, q_seg+1) of line li (q_0 = 0,
// q_4 = L; q_1..q_3 from the task). Every segment eliminates forward from its
// own start (the first from its closure rows, the others from a zero start)
// and substitutes backward from its own end (the last from the true end, the
// others from a zero start). By linearity segment s then adds to its forward
// values the homogeneous forward solution started from segment s-1's last two
// forward values, and to its results the homogeneous backward solution
// started from segment s+1's first two results, both as register recurrences
// (as in the two-lane split solve). The host places the boundaries so that
// every segment is longer than both solutions take to fall below the solve
// type's rounding, so a segment's end values are final without a chain across
// segments and the four segments correct at once.
constexpr int kQuad = 8;

template <int DIR, class TT, class RS>
__global__ void __maxnreg__(168) k_line4(const LineTask* __restrict__ tasks, const int* __restrict__ tile_task,
                                              int tdiv, const CUtensorMap* __restrict__ maps,
                                              int* __restrict__ err) {
  constexpr int kVec = 16 / (int)sizeof(TT);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw);
  TT* s = reinterpret_cast<TT*>(smem_raw + 128);
  const int lane = threadIdx.x;
  const int seg = lane >> 3, li = lane & (kQuad - 1);
  const unsigned full = 0xffffffffu;
  TRACE(0)
  const int ti = tile_of(tile_task, tdiv);
  if (error_pending(err)) return;
  const LineTask& T = tasks[ti];
  const TT* in = static_cast<const TT*>(T.in);
  TT* out = static_cast<TT*>(T.out);
  const int lt = blockIdx.x - T.tile0;
  const int L = T.L, N = L - 1;
  const int X = T.X, Y = T.Y, Z = T.Z, Xp = T.Xp;
  const int NC = T.nbox, CR = T.by;
  int nval, x0 = 0, r0 = 0, fix = 0;
  if (DIR == 1) {
    r0 = lt * kQuad;
    nval = min(kQuad, Y * Z - r0);
  } else {
    fix = lt / T.ntx;
    x0 = (lt % T.ntx) * kQuad;
    nval = min(kQuad, X - x0);
  }
  const int P = dir1_pitch<TT>(L);
  const long long base = (DIR == 1) ? (long long)r0 * Xp
                                    : ((DIR == 2) ? (long long)fix * Y * Xp + x0 : (long long)fix * Xp + x0);
  const CUtensorMap* map_in = maps + 2 * ti;
  const CUtensorMap* map_out = maps + 2 * ti + 1;
  auto chunk_len = [&](int c) { return min(CR, L - c * CR); };
  if (lane == 0) {
    for (int c = 0; c < NC; ++c) mbar_init(bars + c, 1);
    mbar_init_done();
  }
  __syncwarp();
  for (int c = 0; c < NC; ++c) {
    if (DIR == 1) {
      const uint32_t bytes = (uint32_t)((chunk_len(c) + kVec - 1) / kVec * kVec * sizeof(TT));
      if (lane == 0) mbar_expect_tx(bars + c, bytes * nval);
      __syncwarp();
      if (lane < nval) bulk_g2s(s + lane * P + c * CR, in + base + (long long)lane * Xp + c * CR, bytes, bars + c);
    } else if (lane == 0) {
      mbar_expect_tx(bars + c, (uint32_t)(CR * kQuad * sizeof(TT)));
      if (DIR == 2) tma_load_3d(s + c * CR * kQuad, map_in, x0, c * CR, fix, bars + c);
      else tma_load_3d(s + c * CR * kQuad, map_in, x0, fix, c * CR, bars + c);
    }
  }
  TRACE(1)
  bool ok = true;
  for (int c = 0; c < NC; ++c) ok = mbar_wait(bars + c, 0) && ok;
  if (!ok) {
    if (lane == 0) atomicExch(err, kErrTimeout);
    return;
  }
  __syncwarp();
  TRACE(2)
  constexpr int ST = (DIR == 1) ? 1 : kQuad;
  TT* sl = (DIR == 1) ? s + li * P : s + li;
  const bool has = li < nval;
  int jk = 0;
  if (DIR == 1) jk = r0 + li;
  else if (DIR == 2) jk = (x0 + li) * Z + fix;
  else jk = fix * X + x0 + li;
  const int nbs = T.nbs;
  const RS* lu = static_cast<const RS*>(T.lu);
  const CoefTable<RS> cf{lu, lu + L, lu + 2 * L, lu + 3 * L, lu + 4 * L};
  const CoefConst<RS> cc{RS(T.cl1), RS(T.cl2), RS(T.cu1), RS(T.cu2), RS(T.cu3)};
  const int c0 = T.c0, c1 = L - 4;
  const int q1 = T.h, q2 = T.q2, q3 = T.q3;
  const int lo = seg == 0 ? 0 : (seg == 1 ? q1 : (seg == 2 ? q2 : q3));
  const int hi = seg == 0 ? q1 : (seg == 1 ? q2 : (seg == 2 ? q3 : L));
  const DevScheme* __restrict__ sc = T.sc;
  const TT* recv = static_cast<const TT*>(T.recv);
  // interface sums received by the own end (first and last segment)
  TT q0v = 0, q1v = 0;
  if (T.selfp) {
    // periodic onto itself: the contraction the other end would send (see k_line)
    if (seg == 0 || seg == 3) {
#pragma unroll
      for (int i = 0; i < 12; ++i) {
        const TT v = seg == 0 ? sl[(N - 1 - i) * ST] : sl[(1 + i) * ST];
        q0v = q0v + TT(sc->pbco[0][0][i]) * v;
        q1v = q1v + TT(sc->pbco[0][1][i]) * v;
      }
    }
  } else if (has) {
    if (seg == 0 && T.ndf0) { q0v = recv[jk]; q1v = recv[nbs + jk]; }
    if (seg == 3 && T.ndf1) { q0v = recv[2 * nbs + jk]; q1v = recv[3 * nbs + jk]; }
  }
  // ---- reads of the original line, before any row is overwritten
  TT b[2] = {0, 0};  // closure right-hand sides of the own end (last segment: bn, bn1)
  TT x[2] = {0, 0};  // originals at hi, hi + 1 (the stencil of the own last two rows)
  TT w0, w1, w2, w3;
  if (seg == 0) {
    if (T.ndf0 == 0) {
      const TT s0 = sl[0], s1 = sl[ST], s2 = sl[2 * ST], s3 = sl[3 * ST], s4 = sl[4 * ST];
      b[0] = ((TT(CA_A01) * (s1 - s0) + TT(CA_A02) * (s2 - s0)) + TT(CA_A03) * (s3 - s0)) + TT(CA_A04) * (s4 - s0);
      b[1] = ((TT(CA_A10) * (s0 - s1) + TT(CA_A12) * (s2 - s1)) + TT(CA_A13) * (s3 - s1)) + TT(CA_A14) * (s4 - s1);
    } else {
      TT t0 = 0, t1 = 0;
#pragma unroll
      for (int i = 0; i < 12; ++i) {
        const TT v = sl[i * ST];
        t0 = t0 + TT(sc->pbci[0][0][i]) * v;
        t1 = t1 + TT(sc->pbci[0][1][i]) * v;
      }
      b[0] = t0 + q0v;
      b[1] = t1 + q1v;
    }
    w0 = sl[0]; w1 = sl[ST]; w2 = sl[2 * ST]; w3 = sl[3 * ST];
  } else {
    if (seg == 3) {
      if (T.ndf1 == 0) {
        const TT e0 = sl[N * ST], e1 = sl[(N - 1) * ST], e2 = sl[(N - 2) * ST], e3 = sl[(N - 3) * ST],
                 e4 = sl[(N - 4) * ST];
        b[0] = ((TT(CA_A01) * (e0 - e1) + TT(CA_A02) * (e0 - e2)) + TT(CA_A03) * (e0 - e3)) + TT(CA_A04) * (e0 - e4);
        b[1] = ((TT(CA_A10) * (e1 - e0) + TT(CA_A12) * (e1 - e2)) + TT(CA_A13) * (e1 - e3)) + TT(CA_A14) * (e1 - e4);
      } else {
        TT t0 = 0, t1 = 0;
#pragma unroll
        for (int i = 0; i < 12; ++i) {
          const TT v = sl[(N - i) * ST];
          t0 = t0 + TT(sc->pbci[0][0][i]) * v;
          t1 = t1 + TT(sc->pbci[0][1][i]) * v;
        }
        b[0] = -t0 - q0v;
        b[1] = -t1 - q1v;
      }
    }
    w0 = sl[(lo - 2) * ST]; w1 = sl[(lo - 1) * ST]; w2 = sl[lo * ST]; w3 = sl[(lo + 1) * ST];
  }
  if (seg != 3) {
    x[0] = sl[hi * ST];
    x[1] = sl[(hi + 1) * ST];
  }
  __syncwarp();
  // ---- forward elimination: the first segment's closure rows, the interior
  // rows of every segment, then its last two rows (right-hand sides from x or,
  // in the last segment, the closures)
  RS am2 = 0, am1 = 0;
  if (seg == 0) {
    am2 = RS(b[0]);
    am1 = RS(b[1]) - cf.L2(1) * am2;
    sl[0] = TT(am2);
    sl[ST] = TT(am1);
  }
  const int fb = seg == 0 ? 2 : lo;
  const int fe = seg == 3 ? N - 1 : hi - 2;
  {
    TT w4 = 0, w5 = 0;
    fwd3<0, ST, TT, RS>(sl, fb, fe, c0, c1, cf, cc, TT(0), TT(0), TT(0), w0, w1, w2, w3, w4, w5, am2, am1);
  }
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int i = fe + k;
    TT rhs;
    {
      const TT w4n = x[k];
      rhs = TT(CA_AA) * (w3 - w1) + TT(CA_AB) * (w4n - w0);
      w0 = w1; w1 = w2; w2 = w3; w3 = w4n;
    }
    if (seg == 3) rhs = b[1 - k];
    const RS a = (RS(rhs) - cf.L1(i) * am2) - cf.L2(i) * am1;
    sl[i * ST] = TT(a);
    am2 = am1;
    am1 = a;
  }
  // ---- the previous segment's last two forward values start each segment's
  // homogeneous forward correction
  const int srcp = (lane + 24) & 31, srcn = (lane + 8) & 31;
  const RS A0 = __shfl_sync(full, am2, srcp), A1 = __shfl_sync(full, am1, srcp);
  __syncwarp();
  TRACE(3)
  if (seg >= 1) {
    RS g2 = A0, g1 = A1;
    const int ie = min(lo + T.kf, hi);
    int i = lo;
    for (; i < min(ie, c0); ++i) {
      const RS g = -(cf.L1(i) * g2) - cf.L2(i) * g1;
      sl[i * ST] = TT(RS(sl[i * ST]) + g);
      g2 = g1;
      g1 = g;
    }
#pragma unroll 4
    for (; i < min(ie, c1 + 1); ++i) {
      const RS g = -(cc.L1(i) * g2) - cc.L2(i) * g1;
      sl[i * ST] = TT(RS(sl[i * ST]) + g);
      g2 = g1;
      g1 = g;
    }
    for (; i < ie; ++i) {
      const RS g = -(cf.L1(i) * g2) - cf.L2(i) * g1;
      sl[i * ST] = TT(RS(sl[i * ST]) + g);
      g2 = g1;
      g1 = g;
    }
  }
  __syncwarp();
  // ---- back substitution: the last segment from the true end, the others
  // from a zero start at their own end
  RS cp1 = 0, cp2 = 0;
  if (seg == 3) {
    cp1 = cf.U1(N) * RS(sl[N * ST]);
    sl[N * ST] = TT(cp1);
    const RS c = cf.U1(N - 1) * RS(sl[(N - 1) * ST]) - cf.U2(N - 1) * cp1;
    sl[(N - 1) * ST] = TT(c);
    cp2 = cp1;
    cp1 = c;
  }
  bwd3<ST, TT, RS>(sl, seg == 3 ? N - 2 : hi - 1, lo, c0, c1, cf, cc, cp1, cp2);
  TRACE(4)
  // ---- the next segment's first two results start each segment's
  // homogeneous backward correction
  const RS C0 = __shfl_sync(full, cp1, srcn), C1 = __shfl_sync(full, cp2, srcn);
  __syncwarp();
  if (seg <= 2) {
    RS e1 = C0, e2 = C1;
    const int ib = max(hi - T.ke, lo);
    int i = hi - 1;
    for (; i > c1 && i >= ib; --i) {
      const RS e = -(cf.U2(i) * e1) - cf.U3(i) * e2;
      sl[i * ST] = TT(RS(sl[i * ST]) + e);
      e2 = e1;
      e1 = e;
    }
#pragma unroll 4
    for (; i >= max(ib, c0); --i) {
      const RS e = -(cc.U2(i) * e1) - cc.U3(i) * e2;
      sl[i * ST] = TT(RS(sl[i * ST]) + e);
      e2 = e1;
      e1 = e;
    }
    for (; i >= ib; --i) {
      const RS e = -(cf.U2(i) * e1) - cf.U3(i) * e2;
      sl[i * ST] = TT(RS(sl[i * ST]) + e);
      e2 = e1;
      e1 = e;
    }
  }
  __syncwarp();
  TRACE(5)
  if (has && T.drva) {
    TT* drva = static_cast<TT*>(T.drva);
    if (seg == 0) drva[jk + (long long)nbs * (T.m - 1)] = sl[0];
    if (seg == 3) drva[jk + (long long)nbs * ((T.m - 1) + 5)] = sl[N * ST];
  }
  fence_proxy_async();
  __syncwarp();
  for (int c = 0; c < NC; ++c) {
    const int clo = c * CR, len = chunk_len(c);
    if (DIR == 1) {
      if (lane < nval)
        bulk_s2g(out + base + (long long)lane * Xp + clo, s + lane * P + clo,
                 (uint32_t)((len + kVec - 1) / kVec * kVec * sizeof(TT)));
    } else if (lane == 0) {
      if (DIR == 2) tma_store_3d(map_out, x0, clo, fix, s + clo * kQuad);
      else tma_store_3d(map_out, x0, fix, clo, s + clo * kQuad);
    }
  }
  bulk_commit();
  bulk_wait_read0();
  TRACE(7)
}

// ---------------------------------------------------------------------------
// Mixed-precision filter of the FP64 state on an FP32 tile (split solve, 16
// lines per warp, two lanes per line as in k_line2). The FP64 field never
// sits in shared memory: each lane streams its half of its line from global
// memory (16 lines of one x-tile: 128-byte rows for eta and zeta), forms the
// filter's right-hand sides in FP64 from a 7-point register window and the
// closures (src/mo_numerics.f90:922-950), and stores them rounded to FP32 in
// the tile, which is half the size of an FP64 tile. The FP32 split
// elimination then runs on the tile (as sweep2, right-hand sides given), and
// each row is written back as original (FP64, read again: it was read moments
// before and is still in L2) + increment.

// forward elimination of rows [ib, ie) from right-hand sides held in the tile
template <int ST, class CF>
__device__ __forceinline__ void fwd_rows_rhs(float* s, int ib, int ie, const CF& cf, float& am2, float& am1) {
  int i = ib;
  for (; i + 7 < ie; i += 8) {
    float r[8], l1[8], l2[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) { r[k] = s[(i + k) * ST]; l1[k] = cf.L1(i + k); l2[k] = cf.L2(i + k); }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const float a = (r[k] - l1[k] * am2) - l2[k] * am1;
      s[(i + k) * ST] = a;
      am2 = am1;
      am1 = a;
    }
  }
  for (; i < ie; ++i) {
    const float a = (s[i * ST] - cf.L1(i) * am2) - cf.L2(i) * am1;
    s[i * ST] = a;
    am2 = am1;
    am1 = a;
  }
}

template <int DIR>
__global__ void __launch_bounds__(32) k_filt2s(const LineTask* __restrict__ tasks, const int* __restrict__ tile_task,
                                               int tdiv, int* __restrict__ err) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float* s = reinterpret_cast<float*>(smem_raw);
  const int lane = threadIdx.x;
  const int half = lane >> 4, li = lane & (kHalf - 1);
  const unsigned full = 0xffffffffu;
  if (error_pending(err)) return;
  const int ti = tile_of(tile_task, tdiv);
  const LineTask& T = tasks[ti];
  const double* __restrict__ in = static_cast<const double*>(T.in);
  double* out = static_cast<double*>(T.out);
  const int lt = blockIdx.x - T.tile0;
  const int L = T.L, h = T.h, N = L - 1;
  const int X = T.X, Y = T.Y, Z = T.Z, Xp = T.Xp;
  int nval, x0 = 0, r0 = 0, fix = 0;
  if (DIR == 1) {
    r0 = lt * kHalf;
    nval = min(kHalf, Y * Z - r0);
  } else {
    fix = lt / T.ntx;
    x0 = (lt % T.ntx) * kHalf;
    nval = min(kHalf, X - x0);
  }
  const bool has = li < nval;
  const int P = dir1_pitch<float>(L);
  constexpr int ST = (DIR == 1) ? 1 : kHalf;
  float* sl = (DIR == 1) ? s + li * P : s + li;
  // element r of this lane's line: in[lb + r * rs] (lanes past the block's
  // edge read line 0 of the tile and store nothing)
  const long long rs = (DIR == 1) ? 1 : ((DIR == 2) ? (long long)Xp : (long long)Xp * Y);
  const int lc = has ? li : 0;
  const long long lb = (DIR == 1) ? (long long)(r0 + lc) * Xp
                                  : ((DIR == 2) ? (long long)fix * Y * Xp + x0 + lc : (long long)fix * Xp + x0 + lc);
  auto F = [&](int r) { return __ldg(in + lb + (long long)r * rs); };
  int jk = 0;
  if (DIR == 1) jk = r0 + lc;
  else if (DIR == 2) jk = (x0 + lc) * Z + fix;
  else jk = fix * X + x0 + lc;
  const int nbs = T.nbs;
  const DevScheme* __restrict__ sc = T.sc;
  const double fa = sc->fa, fb = sc->fb, fc = sc->fc;
  const double* recv = static_cast<const double*>(T.recv);
  // ---- right-hand sides in FP64, stored as FP32
  const int ndf = half == 0 ? T.ndf0 : T.ndf1;
  {
    // the three closure rows of the own end: rows 0, 1, 2 (first half) or
    // N, N-1, N-2 (second half), e(k) = the k-th value from that end
    const int e0 = half == 0 ? 0 : N, de = half == 0 ? 1 : -1;
    auto E = [&](int k) { return F(e0 + de * k); };
    double b0, b1, b2;
    if (ndf == 0) {
      const double v0 = E(0), v1 = E(1), v2 = E(2), v3 = E(3), v4 = E(4), v5 = E(5);
      auto fbc = [&](int r, int k) { return sc->fbc[r][k]; };
      b0 = (((fbc(0, 0) * (v1 - v0) + fbc(0, 1) * (v2 - v0)) + fbc(0, 2) * (v3 - v0)) + fbc(0, 3) * (v4 - v0)) +
           fbc(0, 4) * (v5 - v0);
      b1 = (((fbc(1, 0) * (v0 - v1) + fbc(1, 1) * (v2 - v1)) + fbc(1, 2) * (v3 - v1)) + fbc(1, 3) * (v4 - v1)) +
           fbc(1, 4) * (v5 - v1);
      b2 = (((fbc(2, 0) * (v0 - v2) + fbc(2, 1) * (v1 - v2)) + fbc(2, 2) * (v3 - v2)) + fbc(2, 3) * (v4 - v2)) +
           fbc(2, 4) * (v5 - v2);
    } else {
      // interface closure: contraction with pbci plus the received sums; the
      // third row takes the neighbour's raw value in place of the missing one
      const int so = half == 0 ? 0 : 3;  // recv components of the side
      const double q0 = recv[(so + 0) * nbs + jk], q1 = recv[(so + 1) * nbs + jk], q2 = recv[(so + 2) * nbs + jk];
      double v[12];
#pragma unroll
      for (int k = 0; k < 12; ++k) v[k] = E(k);
      double t0 = 0, t1 = 0;
#pragma unroll
      for (int k = 0; k < 12; ++k) {
        t0 = t0 + sc->pbci[1][0][k] * v[k];
        t1 = t1 + sc->pbci[1][1][k] * v[k];
      }
      const double ra2 = v[2] + v[2];
      b0 = t0 + q0;
      b1 = t1 + q1;
      b2 = (fa * ((v[1] + v[3]) - ra2) + fb * ((v[0] + v[4]) - ra2)) + fc * ((q2 + v[5]) - ra2);
    }
    sl[e0 * ST] = float(b0);
    sl[(e0 + de) * ST] = float(b1);
    sl[(e0 + 2 * de) * ST] = float(b2);
  }
  {
    // interior rows [a, b) of the own half: rows 3..h-1 or h..N-3
    const int a = half == 0 ? 3 : h, b = half == 0 ? h : N - 2;
    double w0 = F(a - 3), w1 = F(a - 2), w2 = F(a - 1), w3 = F(a), w4 = F(a + 1), w5 = F(a + 2);
    auto rhs8 = [&](int r, const double (&v)[8]) {
      double win[14] = {w0, w1, w2, w3, w4, w5, v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7]};
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const double rk = win[k + 3] + win[k + 3];
        const double q = (fa * ((win[k + 2] + win[k + 4]) - rk) + fb * ((win[k + 1] + win[k + 5]) - rk)) +
                         fc * ((win[k] + win[k + 6]) - rk);
        sl[(r + k) * ST] = float(q);
      }
      w0 = win[8]; w1 = win[9]; w2 = win[10]; w3 = win[11]; w4 = win[12]; w5 = win[13];
    };
    int r = a;
    if (r + 8 <= b) {
      double nx[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) nx[k] = F(r + 3 + k);  // rows up to b + 2 <= N
      while (r + 16 <= b) {
        double cu[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) cu[k] = nx[k];
#pragma unroll
        for (int k = 0; k < 8; ++k) nx[k] = F(r + 11 + k);
        rhs8(r, cu);
        r += 8;
      }
      rhs8(r, nx);
      r += 8;
    }
    for (; r < b; ++r) {
      const double w6 = F(r + 3);
      const double rk = w3 + w3;
      const double q = (fa * ((w2 + w4) - rk) + fb * ((w1 + w5) - rk)) + fc * ((w0 + w6) - rk);
      sl[r * ST] = float(q);
      w0 = w1; w1 = w2; w2 = w3; w3 = w4; w4 = w5; w5 = w6;
    }
  }
  __syncwarp();
  // ---- FP32 split elimination (see sweep2)
  const float* lu = static_cast<const float*>(T.lu);
  const CoefTable<float> ct{lu, lu + L, lu + 2 * L, lu + 3 * L, lu + 4 * L};
  const CoefConst<float> cc{float(T.cl1), float(T.cl2), float(T.cu1), float(T.cu2), float(T.cu3)};
  const float* hb = lu + 5 * L;
  const int LT = L + 8;
  const SplitTables H{hb, hb + LT, hb + 2 * LT, hb + 3 * LT, T.kg, T.ke};
  const int c0 = T.c0, c1 = L - 4;
  float am2 = 0.f, am1 = 0.f;
  int fb0;
  if (half == 0) {
    am2 = sl[0];
    am1 = sl[ST] - ct.L2(1) * am2;
    sl[ST] = am1;
    fb0 = 2;
  } else {
    fb0 = h;
  }
  const int fe0 = half == 0 ? h : L;
  {
    const int m0 = max(fb0, c0), m1 = min(fe0, c1 + 1);
    fwd_rows_rhs<ST>(sl, fb0, min(fe0, m0), ct, am2, am1);
    fwd_rows_rhs<ST>(sl, m0, m1, cc, am2, am1);
    fwd_rows_rhs<ST>(sl, max(fb0, c1 + 1), fe0, ct, am2, am1);
  }
  const int src = lane & (kHalf - 1);
  const float A0 = __shfl_sync(full, am2, src), A1 = __shfl_sync(full, am1, src);
  __syncwarp();
  float cp1 = 0.f, cp2 = 0.f;
  if (half == 1) {
    cp1 = ct.U1(N) * sl[N * ST];
    sl[N * ST] = cp1;
    const float c = ct.U1(N - 1) * sl[(N - 1) * ST] - ct.U2(N - 1) * cp1;
    sl[(N - 1) * ST] = c;
    cp2 = cp1;
    cp1 = c;
  }
  bwd3<ST, float, float>(sl, half == 0 ? h - 1 : N - 2, half == 0 ? 0 : h, c0, c1, ct, cc, cp1, cp2);
  float ch0 = 0.f, ch1 = 0.f;
  if (half == 1) {
    ch0 = cp1 + (__ldg(H.h0) * A0 + __ldg(H.h1) * A1);
    ch1 = cp2 + (__ldg(H.h0 + 1) * A0 + __ldg(H.h1 + 1) * A1);
  }
  const float C0 = __shfl_sync(full, ch0, src + kHalf), C1 = __shfl_sync(full, ch1, src + kHalf);
  __syncwarp();
  {
    const float* t0 = half == 0 ? H.e0 : H.h0;
    const float* t1 = half == 0 ? H.e1 : H.h1;
    const float s0 = half == 0 ? C0 : A0, s1 = half == 0 ? C1 : A1;
    const int cnt = half == 0 ? min(H.ke, h) : min(H.kh, L - h);
    const int i0 = half == 0 ? h - 1 : h, di = half == 0 ? -1 : 1;
    for (int j = 0; j < cnt; ++j) {
      const int i = i0 + di * j;
      sl[i * ST] = sl[i * ST] + (__ldg(t0 + j) * s0 + __ldg(t1 + j) * s1);
    }
  }
  // ---- originals + increments of the own half, written back
  if (has) {
    const int lo = half == 0 ? 0 : h, hi = half == 0 ? h : L;
    int r = lo;
    for (; r + 8 <= hi; r += 8) {
      double v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] = F(r + k);
#pragma unroll
      for (int k = 0; k < 8; ++k) out[lb + (long long)(r + k) * rs] = v[k] + double(sl[(r + k) * ST]);
    }
    for (; r < hi; ++r) out[lb + (long long)r * rs] = F(r) + double(sl[r * ST]);
  }
}

// ---------------------------------------------------------------------------
__device__ __forceinline__ void line_xyz(int nn, int pos, int j, int k, int& x, int& y, int& z) {
  if (nn == 1) { x = pos; y = j; z = k; }
  else if (nn == 2) { x = k; y = pos; z = j; }
  else { x = j; y = k; z = pos; }
}

// t_numerics%mpigo for a list of faces (src/mo_numerics.f90:429-565), in the
// field type T.
template <class T>
__global__ void k_mpigo(const FaceTask* __restrict__ tasks, const int* __restrict__ line0s, int ntasks,
                        int nlines) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nlines; g += gridDim.x * blockDim.x) {
    const int ti = find_task(line0s, ntasks, g);
    const FaceTask& F = tasks[ti];
    const T* src = static_cast<const T*>(F.src);
    // eta faces run x fastest across threads so their reads coalesce; the
    // other faces already do (zeta) or read 12 contiguous values (xi)
    const int gl = g - F.line0;
    int j, k, jk;
    if (F.nn == 2) {
      k = gl % F.X;
      j = gl / F.X;
      jk = j + F.nj * k;
    } else {
      jk = gl;
      j = jk % F.nj;
      k = jk / F.nj;
    }
    const int istart = F.sb * F.N, step = 1 - 2 * F.sb;
    int x, y, z;
    line_xyz(F.nn, istart, j, k, x, y, z);
    const T resk = T(F.ra0k) * src[((long long)z * F.Y + y) * F.Xp + x];
    const DevScheme* sc = F.sc;
    const int nt = F.nt;
    T t0 = 0, t1 = 0, sap0 = 0;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      line_xyz(F.nn, istart + step * (i + F.iik), j, k, x, y, z);
      const T v = src[((long long)z * F.Y + y) * F.Xp + x];
      if (i == 0) sap0 = v;
      t0 = t0 + T(sc->pbco[nt][0][i]) * v;
      t1 = t1 + T(sc->pbco[nt][1][i]) * v;
    }
    T snd0 = t0 - resk * T(sc->pbcot[nt][0]);
    T snd1 = t1 - resk * T(sc->pbcot[nt][1]);
    T snd2 = 0;
    if (nt == 1) {
      if (F.chain) {
        const T old = T(F.chain[jk]);
        snd2 = old + ((sap0 - resk) - old);
        F.chain[jk] = double(snd2);
      } else {
        snd2 = sap0 - resk;  // the chain's exact value, without its rounding
      }
    }
    if (F.exch) {
      T* recv = static_cast<T*>(F.recv);
      if (F.corr) {  // receiver side is periodic and n45 = n45go
        line_xyz(F.nn, (1 - F.sb) * F.NA, j, k, x, y, z);
        const T f = static_cast<const T*>(F.dstf)[((long long)z * F.YA + y) * F.XpA + x];
        snd0 = snd0 + f * T(sc->pbcot[nt][0]);
        snd1 = snd1 + f * T(sc->pbcot[nt][1]);
        if (nt == 1) snd2 = snd2 + f; else snd1 = snd1 + T(0) * f;
      }
      recv[jk] = snd0;
      recv[F.nbs + jk] = snd1;
      if (nt == 1) recv[2 * F.nbs + jk] = snd2;
    }
  }
}

// ---------------------------------------------------------------------------
// element-wise kernels: blockIdx.y = block
// Grid-stride loop over the stored points of one block (pad columns x >= X
// skipped). The column x is found by one division per thread and then
// advanced with the stride, so no point pays an integer division.
#define FOR_POINTS(BD)                                                                \
  const BlockDev& B = BD;                                                             \
  const long long fp_stride_ = (long long)gridDim.x * blockDim.x;                     \
  const int fp_sx_ = (int)(fp_stride_ % B.Xp);                                        \
  int fp_x_ = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) % B.Xp);       \
  for (long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x; l < B.npad;   \
       l += fp_stride_, fp_x_ = (fp_x_ + fp_sx_ >= B.Xp) ? fp_x_ + fp_sx_ - B.Xp : fp_x_ + fp_sx_) \
    if (fp_x_ < B.X)

constexpr double kGam = 1.4;
#define KGAMM1 (kGam - 1.0)

// primitives, pressure, Sutherland viscosity of one point from its state
// (src/mo_canard_driver.f90:267-275), evaluated in FP64, stored in the flux type R
template <class R>
__device__ __forceinline__ void prim_point(const Work<R>& W, const CaseConst& C, long long l, long long n, double q0,
                                           double q1, double q2, double q3, double q4) {
  R* de = W.de;
  const double d1 = 1.0 / q0;
  const double d2 = q1 * d1, d3 = q2 * d1, d4 = q3 * d1;
  const double p = KGAMM1 * (q4 - 0.5 * ((q1 * d2 + q2 * d3) + q3 * d4));
  const double d5 = (kGam * p) * d1;
  de[l] = R(d1); de[l + n] = R(d2); de[l + 2 * n] = R(d3); de[l + 3 * n] = R(d4); de[l + 4 * n] = R(d5);
  W.p[l] = R(p);
  W.mu[l] = R((C.srefp1dre * pow15(d5)) / (d5 + C.srefoo));
}

// STORE_QO (the step's first stage): also qo = qa (src/mo_canard_driver.f90:
// 252) from the values this pass reads anyway, instead of a separate copy
template <class R, bool STORE_QO = false>
__global__ void k_prim(const BlockDev* __restrict__ bd, const CaseConst* __restrict__ cc) {
  FOR_POINTS(bd[blockIdx.y]) {
    const long long n = B.npad;
    const double* q = B.qa;
    const double q0 = q[l], q1 = q[l + n], q2 = q[l + 2 * n], q3 = q[l + 3 * n], q4 = q[l + 4 * n];
    if (STORE_QO) {
      double* o = B.qo;
      o[l] = q0; o[l + n] = q1; o[l + 2 * n] = q2; o[l + 3 * n] = q3; o[l + 4 * n] = q4;
    }
    prim_point<R>(work<R>(B), cc[B.case_id], l, n, q0, q1, q2, q3, q4);
  }
}

// the primitives again at the points junction averaging changed (targets of
// the three averaging plans), after a fused RK + primitives update
template <class R>
__global__ void k_prim_points(const BlockDev* __restrict__ bd, const CaseConst* __restrict__ cc,
                              const int* __restrict__ tb, const long long* __restrict__ tl, int ntg) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntg; t += gridDim.x * blockDim.x) {
    const BlockDev& B = bd[tb[t]];
    const long long l = tl[t], n = B.npad;
    const double* q = B.qa;
    prim_point<R>(work<R>(B), cc[B.case_id], l, n, q[l], q[l + n], q[l + 2 * n], q[l + 3 * n], q[l + 4 * n]);
  }
}

// time-step maxima (src/mo_physics.f90:185-207) in FP64 from the FP64 metrics;
// values are >= 0, so their bit patterns order like the values and atomicMax
// on them is exact. fmax drops NaN, so a non-finite state is flagged apart
// (err = kErrOverflow): the reference's overflow stop only sees dt == 0.
template <class R>
__global__ void k_dtmax(const BlockDev* __restrict__ bd, const StageParams* __restrict__ sp,
                        const CaseConst* __restrict__ cc, unsigned long long* __restrict__ out,
                        int* __restrict__ err) {
  const BlockDev& B0 = bd[blockIdx.y];
  const StageParams S = sp[B0.case_id];
  const int visc = cc[B0.case_id].viscous;
  double m1 = 0.0, m2 = 0.0;
  bool bad = false;
  FOR_POINTS(B0) {
    const Work<R> W = work<R>(B);
    const long long n = B.npad;
    const double *xi = B.xim, *et = B.etm, *ze = B.zem;
    const R* de = W.de;
    double r1 = xi[l] * xi[l];
    r1 = r1 + xi[l + n] * xi[l + n];
    r1 = r1 + xi[l + 2 * n] * xi[l + 2 * n];
    r1 = r1 + et[l] * et[l];
    r1 = r1 + et[l + n] * et[l + n];
    r1 = r1 + et[l + 2 * n] * et[l + 2 * n];
    r1 = r1 + ze[l] * ze[l];
    r1 = r1 + ze[l + n] * ze[l + n];
    r1 = r1 + ze[l + 2 * n] * ze[l + 2 * n];
    const double u = double(de[l + n]) + S.umf[0], v = double(de[l + 2 * n]) + S.umf[1],
                 w = double(de[l + 3 * n]) + S.umf[2];
    double r2 = fabs((xi[l] * u + xi[l + n] * v) + xi[l + 2 * n] * w) +
                fabs((et[l] * u + et[l + n] * v) + et[l + 2 * n] * w);
    r2 = r2 + fabs((ze[l] * u + ze[l + n] * v) + ze[l + 2 * n] * w);
    const double ssi = fabs(B.yaco[l]);
    const double v1 = (sqrt(double(de[l + 4 * n]) * r1) + r2) * ssi;
    bad = bad || !isfinite(v1);
    m1 = fmax(m1, v1);
    if (visc) m2 = fmax(m2, (((double(de[l]) * double(W.mu[l])) * r1) * ssi) * ssi);
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicExch(err, kErrOverflow);
  for (int o = 16; o > 0; o >>= 1) {
    m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
    m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out + 2 * B0.case_id, (unsigned long long)__double_as_longlong(m1));
    atomicMax(out + 2 * B0.case_id + 1, (unsigned long long)__double_as_longlong(m2));
  }
}

// viscous stresses and heat flux of one point from the 12 gradients in scr
// (src/mo_physics.f90:245-299); scr field g*3+d = d/d(xi_d) of u, v, w, T.
// t = txx tyy tzz txy tyz tzx hxx hyy hzz; d5 = (2/3) div u.
template <class R>
__host__ __device__ __forceinline__ void visc_point(const Work<R>& W, long long l, long long n, R mu, R t[9],
                                                    R& d5) {
  const R *xi = W.xim, *et = W.etm, *ze = W.zem, *g = W.scr;
  auto met = [&](int d, int c) { return (d == 0 ? xi : d == 1 ? et : ze)[l + c * n]; };
  auto comb = [&](int f, int c) {
    return (met(0, c) * g[l + (3 * f) * n] + met(1, c) * g[l + (3 * f + 1) * n]) + met(2, c) * g[l + (3 * f + 2) * n];
  };
  R txx = comb(0, 0), hzz = comb(0, 1), tzx = comb(0, 2);
  R txy = comb(1, 0), tyy = comb(1, 1), hxx = comb(1, 2);
  R hyy = comb(2, 0), tyz = comb(2, 1), tzz = comb(2, 2);
  const R s1 = comb(3, 0), s2 = comb(3, 1), s3 = comb(3, 2);
  const R rr1 = mu * W.yaco[l];
  const R rr2 = R(1.0 / (KGAMM1 * 0.71)) * rr1;
  d5 = R(2.0 / 3.0) * ((txx + tyy) + tzz);
  txx = rr1 * ((txx + txx) - d5);
  tyy = rr1 * ((tyy + tyy) - d5);
  tzz = rr1 * ((tzz + tzz) - d5);
  txy = rr1 * (txy + hzz);
  tyz = rr1 * (tyz + hxx);
  tzx = rr1 * (tzx + hyy);
  const R u = W.de[l + n], v = W.de[l + 2 * n], w = W.de[l + 3 * n];
  hxx = ((rr2 * s1 + u * txx) + v * txy) + w * tzx;
  hyy = ((rr2 * s2 + u * txy) + v * tyy) + w * tyz;
  hzz = ((rr2 * s3 + u * tzx) + v * tyz) + w * tzz;
  t[0] = txx; t[1] = tyy; t[2] = tzz; t[3] = txy; t[4] = tyz; t[5] = tzx; t[6] = hxx; t[7] = hyy; t[8] = hzz;
}

// flux components rr(:,d,m) of one point into scr field (m-1)*3 + d and
// de(:,5) = qa(:,5) + p (src/mo_physics.f90:319-382); t as from visc_point
// pre (optional): p and the five state values as loaded by the caller ahead
// of the viscous terms, so that their loads overlap the others'
template <class R>
__host__ __device__ __forceinline__ void flux_point(const Work<R>& W, const BlockDev& B, const StageParams& S,
                                                    bool visc, long long l, long long n, const R t[9],
                                                    const R* pre = nullptr) {
  const double* q = B.qa;
  R* de = W.de;
  const R p = pre ? pre[0] : W.p[l];
  R qv[5];
  if (pre) {
#pragma unroll
    for (int c = 0; c < 5; ++c) qv[c] = pre[1 + c];
  } else {
#pragma unroll
    for (int c = 0; c < 5; ++c) qv[c] = R(q[l + c * n]);
  }
  const R* mt[3] = {W.xim, W.etm, W.zem};
  const R um0 = R(S.umf[0]), um1 = R(S.umf[1]), um2 = R(S.umf[2]);
  const R u = de[l + n] + um0, v = de[l + 2 * n] + um1, w = de[l + 3 * n] + um2;
  R ssd[3], m[3][3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    m[d][0] = mt[d][l]; m[d][1] = mt[d][l + n]; m[d][2] = mt[d][l + 2 * n];
    ssd[d] = (m[d][0] * u + m[d][1] * v) + m[d][2] * w;
  }
  R* r = W.scr;
  const R q0 = qv[0];
#pragma unroll
  for (int d = 0; d < 3; ++d) r[l + d * n] = q0 * ssd[d];
  R tau[3][3];
  R hx = 0, hy = 0, hz = 0;
  if (visc) {
    tau[0][0] = t[0]; tau[0][1] = t[3]; tau[0][2] = t[5];
    tau[1][0] = t[3]; tau[1][1] = t[1]; tau[1][2] = t[4];
    tau[2][0] = t[5]; tau[2][1] = t[4]; tau[2][2] = t[2];
    hx = t[6]; hy = t[7]; hz = t[8];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const R qc = qv[c + 1];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      R v1 = qc * ssd[d] + m[d][c] * p;
      if (visc) {
        v1 = v1 - m[d][0] * tau[c][0];
        v1 = v1 - m[d][1] * tau[c][1];
        v1 = v1 - m[d][2] * tau[c][2];
      }
      r[l + (3 * (c + 1) + d) * n] = v1;
    }
  }
  const R d5 = qv[4] + p;
  de[l + 4 * n] = d5;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    R v1 = d5 * ssd[d] - p * ((um0 * m[d][0] + um1 * m[d][1]) + um2 * m[d][2]);
    if (visc) {
      v1 = v1 - m[d][0] * hx;
      v1 = v1 - m[d][1] * hy;
      v1 = v1 - m[d][2] * hz;
    }
    r[l + (12 + d) * n] = v1;
  }
}

// calc_viscous_shear_stress on its own (the phase of the C ABI): tau and
// de(:,5); de(:,1) holds ss(:,1)
template <class R>
__global__ void k_viscous_assemble(const BlockDev* __restrict__ bd) {
  FOR_POINTS(bd[blockIdx.y]) {
    const Work<R> W = work<R>(B);
    const long long n = B.npad;
    R t[9], d5;
    visc_point<R>(W, l, n, W.de[l], t, d5);
    W.de[l + 4 * n] = d5;
#pragma unroll
    for (int k = 0; k < 9; ++k) W.tau[l + k * n] = t[k];
  }
}

// de(:,1) = ss(:,1) before the viscous gradients (src/mo_physics.f90:228)
template <class R>
__global__ void k_copy_mu(const BlockDev* __restrict__ bd) {
  FOR_POINTS(bd[blockIdx.y]) {
    const Work<R> W = work<R>(B);
    W.de[l] = W.mu[l];
  }
}

// calc_fluxes on its own (the phase of the C ABI), from the stored tau
template <class R>
__global__ void k_flux(const BlockDev* __restrict__ bd, const StageParams* __restrict__ sp,
                       const CaseConst* __restrict__ cc) {
  FOR_POINTS(bd[blockIdx.y]) {
    const Work<R> W = work<R>(B);
    const long long n = B.npad;
    const bool visc = cc[B.case_id].viscous != 0;
    R t[9] = {};
    if (visc) {
#pragma unroll
      for (int k = 0; k < 9; ++k) t[k] = W.tau[l + k * n];
    }
    flux_point<R>(W, B, sp[B.case_id], visc, l, n, t);
  }
}

// The step path's fusion of the two: stresses stay in registers instead of a
// 9-field round trip through memory. Same operations in the same order, so
// the results are bit-identical to k_viscous_assemble followed by k_flux
// (de(:,1) = ss(:,1) is read from ss directly).
// FP64, two 256-thread blocks per SM (128 registers); the FP32 step path runs
// k_flux_visc_pairs.
template <class R>
__global__ void __launch_bounds__(256, 2)
    k_flux_visc(const BlockDev* __restrict__ bd, const StageParams* __restrict__ sp, const CaseConst* __restrict__ cc) {
  static_assert(sizeof(R) == 8, "the FP32 step path runs k_flux_visc_pairs");
  FOR_POINTS(bd[blockIdx.y]) {
    const Work<R> W = work<R>(B);
    const long long n = B.npad;
    const bool visc = cc[B.case_id].viscous != 0;
    // p and the state load with the viscous terms' inputs
    R pre[6];
    pre[0] = W.p[l];
#pragma unroll
    for (int c = 0; c < 5; ++c) pre[1 + c] = R(B.qa[l + c * n]);
    R t[9] = {};
    if (visc) {
      R d5;
      visc_point<R>(W, l, n, W.mu[l], t, d5);
    }
    flux_point<R>(W, B, sp[B.case_id], visc, l, n, t, pre);
  }
}

// One point of the FP32 fused kernel from values already in registers: the
// stresses and heat flux (src/mo_physics.f90:245-299) and the flux components
// (src/mo_physics.f90:319-382) in the order of visc_point and flux_point, with
// the conserved values formed from the primitives instead of read.
// a: 12 gradients, 9 metric terms [d][c], mu, yaco, p, then the primitives
// in de(:,1:4): 1/rho, u, v, w. out: the 15 flux components, then de(:,5).
// Host-callable too, so that a CPU test can check it point by point.
__host__ __device__ __forceinline__ void flux_visc_values(const float a[28], bool visc, float um0, float um1, float um2,
                                                 float out[16]) {
  const float* g = a;
  const float* mt = a + 12;
  const float mu = a[21], yaco = a[22], p = a[23], rhop = a[24], uu = a[25], vv = a[26], ww = a[27];
  float t[9] = {};
  if (visc) {
    auto comb = [&](int f, int c) {
      return (mt[c] * g[3 * f] + mt[3 + c] * g[3 * f + 1]) + mt[6 + c] * g[3 * f + 2];
    };
    float txx = comb(0, 0), hzz = comb(0, 1), tzx = comb(0, 2);
    float txy = comb(1, 0), tyy = comb(1, 1), hxx = comb(1, 2);
    float hyy = comb(2, 0), tyz = comb(2, 1), tzz = comb(2, 2);
    const float s1 = comb(3, 0), s2 = comb(3, 1), s3 = comb(3, 2);
    const float rr1 = mu * yaco;
    const float rr2 = float(1.0 / (KGAMM1 * 0.71)) * rr1;
    const float d5 = float(2.0 / 3.0) * ((txx + tyy) + tzz);
    txx = rr1 * ((txx + txx) - d5);
    tyy = rr1 * ((tyy + tyy) - d5);
    tzz = rr1 * ((tzz + tzz) - d5);
    txy = rr1 * (txy + hzz);
    tyz = rr1 * (tyz + hxx);
    tzx = rr1 * (tzx + hyy);
    t[0] = txx; t[1] = tyy; t[2] = tzz; t[3] = txy; t[4] = tyz; t[5] = tzx;
    t[6] = ((rr2 * s1 + uu * txx) + vv * txy) + ww * tzx;
    t[7] = ((rr2 * s2 + uu * txy) + vv * tyy) + ww * tyz;
    t[8] = ((rr2 * s3 + uu * tzx) + vv * tyz) + ww * tzz;
  }
  const float rho = 1.0f / rhop;
  float qv[5];
  qv[0] = rho;
  qv[1] = rho * uu;
  qv[2] = rho * vv;
  qv[3] = rho * ww;
  qv[4] = p * float(1.0 / KGAMM1) + 0.5f * rho * ((uu * uu + vv * vv) + ww * ww);
  const float u = uu + um0, v = vv + um1, w = ww + um2;
  float ssd[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) ssd[d] = (mt[3 * d] * u + mt[3 * d + 1] * v) + mt[3 * d + 2] * w;
#pragma unroll
  for (int d = 0; d < 3; ++d) out[d] = qv[0] * ssd[d];
  const float tau[3][3] = {{t[0], t[3], t[5]}, {t[3], t[1], t[4]}, {t[5], t[4], t[2]}};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      float v1 = qv[c + 1] * ssd[d] + mt[3 * d + c] * p;
      if (visc) {
        v1 = v1 - mt[3 * d] * tau[c][0];
        v1 = v1 - mt[3 * d + 1] * tau[c][1];
        v1 = v1 - mt[3 * d + 2] * tau[c][2];
      }
      out[3 * (c + 1) + d] = v1;
    }
  }
  const float d5 = qv[4] + p;
  out[15] = d5;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    float v1 = d5 * ssd[d] - p * ((um0 * mt[3 * d] + um1 * mt[3 * d + 1]) + um2 * mt[3 * d + 2]);
    if (visc) {
      v1 = v1 - mt[3 * d] * t[6];
      v1 = v1 - mt[3 * d + 1] * t[7];
      v1 = v1 - mt[3 * d + 2] * t[8];
    }
    out[12 + d] = v1;
  }
}

// The FP32 fused kernel over pairs of neighbouring points (x even, x + 1):
// every access is 8 bytes per thread, the width of the FP64 kernel's. The x
// pitch is a multiple of 4, so a pair never straddles two rows; the second
// point of a pair at the last x of an odd row is padding, computed and not
// stored. Each thread reads all 28 inputs of both points before its first
// store. Two blocks per SM (126 registers, no spill): with three, the spills
// cost what the wider accesses gain.
template <int MINB>
__global__ void __launch_bounds__(256, MINB)
    k_flux_visc_pairs(const BlockDev* __restrict__ bd, const StageParams* __restrict__ sp,
                      const CaseConst* __restrict__ cc) {
  const BlockDev& B = bd[blockIdx.y];
  const Work<float> W = B.f;
  const long long n = B.npad;
  const bool visc = cc[B.case_id].viscous != 0;
  const StageParams& S = sp[B.case_id];
  const float um0 = float(S.umf[0]), um1 = float(S.umf[1]), um2 = float(S.umf[2]);
  const long long stride = (long long)gridDim.x * blockDim.x;   // in pairs
  const int sx = (int)((2 * stride) % B.Xp);
  long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  int x = (int)((2 * j) % B.Xp);
  for (; 2 * j < n; j += stride, x = (x + sx >= B.Xp) ? x + sx - B.Xp : x + sx) {
    if (x >= B.X) continue;
    const long long l = 2 * j;
    auto ld = [&](const float* f, int c) { return *reinterpret_cast<const float2*>(f + l + c * n); };
    float2 v[28];
#pragma unroll
    for (int k = 0; k < 12; ++k) v[k] = visc ? ld(W.scr, k) : make_float2(0.f, 0.f);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      v[12 + c] = ld(W.xim, c);
      v[15 + c] = ld(W.etm, c);
      v[18 + c] = ld(W.zem, c);
    }
    v[21] = visc ? ld(W.mu, 0) : make_float2(0.f, 0.f);
    v[22] = visc ? ld(W.yaco, 0) : make_float2(0.f, 0.f);
    v[23] = ld(W.p, 0);
#pragma unroll
    for (int c = 0; c < 4; ++c) v[24 + c] = ld(W.de, c);
    float a0[28], a1[28], o0[16], o1[16];
#pragma unroll
    for (int k = 0; k < 28; ++k) {
      a0[k] = v[k].x;
      a1[k] = v[k].y;
    }
    flux_visc_values(a0, visc, um0, um1, um2, o0);
    flux_visc_values(a1, visc, um0, um1, um2, o1);
    if (x + 1 < B.X) {
#pragma unroll
      for (int k = 0; k < 15; ++k) *reinterpret_cast<float2*>(W.scr + l + k * n) = make_float2(o0[k], o1[k]);
      *reinterpret_cast<float2*>(W.de + l + 4 * n) = make_float2(o0[15], o1[15]);
    } else {
#pragma unroll
      for (int k = 0; k < 15; ++k) W.scr[l + k * n] = o0[k];
      W.de[l + 4 * n] = o0[15];
    }
  }
}

// de(:,m) = sum of the three flux derivatives (src/mo_physics.f90:399)
template <class R>
__global__ void k_flux_sum(const BlockDev* __restrict__ bd) {
  FOR_POINTS(bd[blockIdx.y]) {
    const Work<R> W = work<R>(B);
    const long long n = B.npad;
    const R* r = W.scr;
#pragma unroll
    for (int m = 0; m < 5; ++m)
      W.de[l + m * n] = (r[l + (3 * m) * n] + r[l + (3 * m + 1) * n]) + r[l + (3 * m + 2) * n];
  }
}

// RK stage update of the step path, with two optional fusions: sum > 0 forms
// de = sum of the three flux derivatives on the fly (no GCBC or sponge
// changes de in between; sum == 2 also stores it, so that de holds the last
// stage's right-hand side after a step), prim computes the next stage's
// primitives from the new state. Same operations in the same order as k_flux_sum, k_rk and
// k_prim, so bit-identical to running them one after the other. STORE_Q
// false: the stage state is not stored (k_rk_faces stores it on the block
// faces, the junction points); the FP32 fluxes of the next stage read the
// primitives, and nothing else reads the interior state before the last stage
// rewrites it.
template <class R, bool STORE_Q = true>
__global__ void k_rk_next(const BlockDev* __restrict__ bd, const StageParams* __restrict__ sp,
                          const CaseConst* __restrict__ cc, int sum, int prim) {
  FOR_POINTS(bd[blockIdx.y]) {
    const Work<R> W = work<R>(B);
    const long long n = B.npad;
    const double r1 = sp[B.case_id].dtk * B.yaco[l];
    // every input is read before the first store: the compiler cannot tell
    // that the stores (de, qa) touch nothing the loads read, and a store
    // between two loads would hold the second behind the first's latency
    R dv[5];
    double qo[5];
    if (sum) {
      const R* r = W.scr;
      R f[15];
#pragma unroll
      for (int k = 0; k < 15; ++k) f[k] = r[l + k * n];
#pragma unroll
      for (int c = 0; c < 5; ++c) dv[c] = (f[3 * c] + f[3 * c + 1]) + f[3 * c + 2];
    } else {
#pragma unroll
      for (int c = 0; c < 5; ++c) dv[c] = W.de[l + c * n];
    }
#pragma unroll
    for (int c = 0; c < 5; ++c) qo[c] = B.qo[l + c * n];
    double q[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      if (sum == 2) W.de[l + c * n] = dv[c];
      q[c] = qo[c] - r1 * double(dv[c]);
      if (STORE_Q) B.qa[l + c * n] = q[c];
    }
    if (prim) prim_point<R>(W, cc[B.case_id], l, n, q[0], q[1], q[2], q[3], q[4]);
  }
}

// RK stage update in FP64 (src/mo_canard_driver.f90:329-334)
template <class R>
__global__ void k_rk(const BlockDev* __restrict__ bd, const StageParams* __restrict__ sp) {
  FOR_POINTS(bd[blockIdx.y]) {
    const Work<R> W = work<R>(B);
    const long long n = B.npad;
    const double r1 = sp[B.case_id].dtk * B.yaco[l];
#pragma unroll
    for (int c = 0; c < 5; ++c) B.qa[l + c * n] = B.qo[l + c * n] - r1 * double(W.de[l + c * n]);
  }
}

// ---------------------------------------------------------------------------
// GCBC (src/mo_gcbc.f90:133-340, 506-611) in the flux type R
template <class R>
struct Elem { R ao, aoi, ve[3], hv2, vn, vs; };

template <class R>
__device__ __forceinline__ Elem<R> eleme(const R cm[3], R q1, R q2, R q3, R q4, R pp, const double umf[3]) {
  Elem<R> e;
  const R rhoi = R(1) / q1;
  e.ao = sqrt((R(kGam) * rhoi) * pp);
  e.aoi = R(1) / e.ao;
  e.ve[0] = rhoi * q2; e.ve[1] = rhoi * q3; e.ve[2] = rhoi * q4;
  e.hv2 = R(0.5) * ((e.ve[0] * e.ve[0] + e.ve[1] * e.ve[1]) + e.ve[2] * e.ve[2]);
  e.vn = (cm[0] * e.ve[0] + cm[1] * e.ve[1]) + cm[2] * e.ve[2];
  e.vs = (cm[0] * R(umf[0]) + cm[1] * R(umf[1])) + cm[2] * R(umf[2]);
  return e;
}

// r = X_{q->r} v (src/mo_gcbc.f90:506-548)
template <class R>
__device__ __forceinline__ void q2r_apply(const Elem<R>& e, const R cm[3], const R v[5], R r[5]) {
  const R ho = (R(KGAMM1) * e.aoi) * e.aoi;
  const R bo = R(1) - ho * e.hv2;
  const R co = e.aoi * e.vn;
  R dm[3], rv[3];
  for (int d = 0; d < 3; ++d) { dm[d] = e.aoi * cm[d]; rv[d] = ho * e.ve[d]; }
  const R* ve = e.ve;
  R xt[5][5];
  xt[0][0] = (bo * cm[0] + dm[1] * ve[2]) - dm[2] * ve[1];
  xt[0][1] = cm[0] * rv[0]; xt[0][2] = cm[0] * rv[1] + dm[2]; xt[0][3] = cm[0] * rv[2] - dm[1]; xt[0][4] = -ho * cm[0];
  xt[1][0] = (bo * cm[1] + dm[2] * ve[0]) - dm[0] * ve[2];
  xt[1][1] = cm[1] * rv[0] - dm[2]; xt[1][2] = cm[1] * rv[1]; xt[1][3] = cm[1] * rv[2] + dm[0]; xt[1][4] = -ho * cm[1];
  xt[2][0] = (bo * cm[2] + dm[0] * ve[1]) - dm[1] * ve[0];
  xt[2][1] = cm[2] * rv[0] + dm[1]; xt[2][2] = cm[2] * rv[1] - dm[0]; xt[2][3] = cm[2] * rv[2]; xt[2][4] = -ho * cm[2];
  xt[3][0] = (R(1) - bo) - co; xt[3][1] = dm[0] - rv[0]; xt[3][2] = dm[1] - rv[1]; xt[3][3] = dm[2] - rv[2];
  xt[3][4] = ho;
  xt[4][0] = (R(1) - bo) + co; xt[4][1] = -dm[0] - rv[0]; xt[4][2] = -dm[1] - rv[1]; xt[4][3] = -dm[2] - rv[2];
  xt[4][4] = ho;
  for (int i = 0; i < 5; ++i) {
    R s = 0;
    for (int c = 0; c < 5; ++c) s = s + xt[i][c] * v[c];
    r[i] = s;
  }
}

// r = X_{r->q} v (src/mo_gcbc.f90:552-591)
template <class R>
__device__ __forceinline__ void r2q_apply(const Elem<R>& e, const R cm[3], const R v[5], R r[5]) {
  const R bo = e.hv2 + (R(1.0 / KGAMM1) * e.ao) * e.ao;
  const R co = e.ao * e.vn;
  R dm[3];
  for (int d = 0; d < 3; ++d) dm[d] = e.ao * cm[d];
  const R* ve = e.ve;
  R xt[5][5];
  xt[0][0] = cm[0]; xt[0][1] = cm[1]; xt[0][2] = cm[2]; xt[0][3] = R(0.5); xt[0][4] = R(0.5);
  xt[1][0] = cm[0] * ve[0]; xt[1][1] = cm[1] * ve[0] - dm[2]; xt[1][2] = cm[2] * ve[0] + dm[1];
  xt[1][3] = R(0.5) * (ve[0] + dm[0]); xt[1][4] = xt[1][3] - dm[0];
  xt[2][0] = cm[0] * ve[1] + dm[2]; xt[2][1] = cm[1] * ve[1]; xt[2][2] = cm[2] * ve[1] - dm[0];
  xt[2][3] = R(0.5) * (ve[1] + dm[1]); xt[2][4] = xt[2][3] - dm[1];
  xt[3][0] = cm[0] * ve[2] - dm[1]; xt[3][1] = cm[1] * ve[2] + dm[0]; xt[3][2] = cm[2] * ve[2];
  xt[3][3] = R(0.5) * (ve[2] + dm[2]); xt[3][4] = xt[3][3] - dm[2];
  xt[4][0] = (e.hv2 * cm[0] + dm[2] * ve[1]) - dm[1] * ve[2];
  xt[4][1] = (e.hv2 * cm[1] + dm[0] * ve[2]) - dm[2] * ve[0];
  xt[4][2] = (e.hv2 * cm[2] + dm[1] * ve[0]) - dm[0] * ve[1];
  xt[4][3] = R(0.5) * (bo + co); xt[4][4] = xt[4][3] - co;
  for (int i = 0; i < 5; ++i) {
    R s = 0;
    for (int c = 0; c < 5; ++c) s = s + xt[i][c] * v[c];
    r[i] = s;
  }
}

template <class R>
__global__ void k_gcbc_setup(const BlockDev* __restrict__ bd, const GcbcTask* __restrict__ tasks,
                             const int* __restrict__ line0s, int ntasks, int nlines,
                             const StageParams* __restrict__ sp) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nlines; g += gridDim.x * blockDim.x) {
    const GcbcTask& T = tasks[find_task(line0s, ntasks, g)];
    const BlockDev& B = bd[T.b];
    const Work<R> W = work<R>(B);
    const StageParams S = sp[B.case_id];
    const int jk = g - T.line0, j = jk % T.nj, k = jk / T.nj;
    int x, y, z;
    line_xyz(T.nn, T.side * T.N, j, k, x, y, z);
    const long long n = B.npad;
    const long long l = ((long long)z * B.Y + y) * B.Xp + x;
    const R cm[3] = {R(T.cm[jk]), R(T.cm[T.nbs + jk]), R(T.cm[2 * T.nbs + jk])};
    const Elem<R> e =
        eleme<R>(cm, R(B.qa[l]), R(B.qa[l + n]), R(B.qa[l + 2 * n]), R(B.qa[l + 3 * n]), W.p[l], S.umf);
    const R ra0 = R(((20 - T.bc) * (25 - T.bc) * (30 - T.bc)) / 3000);
    const R ra1 = R(1) - ra0;
    R* drva = static_cast<R*>(T.drva);
    R v[5], r[5];
    for (int c = 0; c < 5; ++c) {
      const R cha = ra0 * drva[(long long)c * T.nbs + jk] + ra1 * W.de[l + c * n];
      v[c] = W.yaco[l] * cha;
    }
    q2r_apply<R>(e, cm, v, r);
    for (int c = 0; c < 5; ++c) drva[(long long)c * T.nbs + jk] = r[c];
  }
}

template <class R>
__global__ void k_gcbc_update(const BlockDev* __restrict__ bd, const GcbcTask* __restrict__ tasks,
                              const int* __restrict__ line0s, int ntasks, int nlines,
                              const StageParams* __restrict__ sp) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nlines; g += gridDim.x * blockDim.x) {
    const GcbcTask& T = tasks[find_task(line0s, ntasks, g)];
    const BlockDev& B = bd[T.b];
    const Work<R> W = work<R>(B);
    const StageParams S = sp[B.case_id];
    const int jk = g - T.line0, j = jk % T.nj, k = jk / T.nj;
    int x, y, z;
    line_xyz(T.nn, T.side * T.N, j, k, x, y, z);
    const long long n = B.npad;
    const long long l = ((long long)z * B.Y + y) * B.Xp + x;
    const R cm[3] = {R(T.cm[jk]), R(T.cm[T.nbs + jk]), R(T.cm[2 * T.nbs + jk])};
    const R q1 = R(B.qa[l]);
    const Elem<R> e = eleme<R>(cm, q1, R(B.qa[l + n]), R(B.qa[l + 2 * n]), R(B.qa[l + 3 * n]), W.p[l], S.umf);
    const R ra0 = R(1 - 2 * T.side);
    const R* drva = static_cast<const R*>(T.drva);
    const R* drvb = static_cast<const R*>(T.drvb);
    R cha[5], dha[5], drv[5];
    for (int c = 0; c < 5; ++c) {
      drv[c] = drva[(long long)c * T.nbs + jk];
      cha[c] = drv[c];
      dha[c] = drvb ? drvb[(long long)c * T.nbs + jk] : R(0);
    }
    if (T.bc == 10) {
      if (ra0 * ((e.vn + e.vs) + e.ao) > R(0)) cha[3] = 0;
      if (ra0 * ((e.vn + e.vs) - e.ao) > R(0)) cha[4] = 0;
    } else if (T.bc == 20 || T.bc == 25) {
      const R dtwi = R(1.0 / (4 * S.dt + 1.0e-8));
      R sd = 0;
      for (int d = 0; d < 3; ++d) sd = sd + cm[d] * R(S.dudtmf[d]);
      cha[3 + T.side] = cha[4 - T.side] + (((R(2) * ra0) * e.aoi) * q1) * (sd + dtwi * (e.vn + e.vs));
    } else {
      if (ra0 * (e.vn + e.vs) > R(0)) { cha[0] = dha[0]; cha[1] = dha[1]; cha[2] = dha[2]; }
      if (ra0 * ((e.vn + e.vs) + e.ao) > R(0)) cha[3] = dha[3];
      if (ra0 * ((e.vn + e.vs) - e.ao) > R(0)) cha[4] = dha[4];
    }
    R v[5];
    for (int c = 0; c < 5; ++c) v[c] = cha[c] - drv[c];
    r2q_apply<R>(e, cm, v, dha);
    // the five points of the line are distinct: their 25 values load before
    // any of them is stored (a store between two loads would make the second
    // wait for the first's latency, since the compiler cannot tell they differ)
    long long pts[5];
    R ws[5], dv[5][5];
#pragma unroll
    for (int ii = 0; ii <= 4; ++ii) {
      pts[ii] = T.pts[(long long)jk * 5 + ii];
      ws[ii] = R(T.w[(long long)jk * 5 + ii]);
    }
#pragma unroll
    for (int ii = 0; ii <= 4; ++ii)
#pragma unroll
      for (int c = 0; c < 5; ++c) dv[ii][c] = W.de[pts[ii] + c * n];
#pragma unroll
    for (int ii = 0; ii <= 4; ++ii)
#pragma unroll
      for (int c = 0; c < 5; ++c) W.de[pts[ii] + c * n] = dv[ii][c] + ws[ii] * dha[c];
  }
}

// sponge (src/mo_sponge.f90:75-88): the forcing is formed in FP64 from the
// FP64 state and added to de in the flux type
template <class R>
__global__ void k_sponge(const BlockDev* __restrict__ bd, const SpongeTask* __restrict__ tasks,
                         const int* __restrict__ first, int ntasks, int total) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
    const SpongeTask& T = tasks[find_task(first, ntasks, g)];
    const BlockDev& B = bd[T.b];
    R* de = work<R>(B).de;
    const int e = g - T.first;
    const long long l = T.pts[e], n = B.npad;
    const double a = T.asz[e], bb = T.bsz[e];
    // every input before the first store (see k_rk_next)
    R dv[5];
    double q[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      dv[c] = de[l + c * n];
      q[c] = B.qa[l + c * n];
    }
    de[l] = R(double(dv[0]) + a * (q[0] - 1.0));
    for (int d = 1; d <= 3; ++d) de[l + d * n] = R(double(dv[d]) + bb * (q[d] - 0.0));
    de[l + 4 * n] = R(double(dv[4]) + a * (q[4] - (1.0 / kGam) * (1.0 / KGAMM1)));
  }
}

// drvb <- drva of the partner face (gcbc_comm, src/mo_gcbc.f90:186-220)
template <class R>
__global__ void k_face_copy(const void* const* __restrict__ src, void* const* __restrict__ dst,
                            const int* __restrict__ counts, int nfaces) {
  const int f = blockIdx.y;
  if (f >= nfaces) return;
  const R* s = static_cast<const R*>(src[f]);
  R* d = static_cast<R*>(dst[f]);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < counts[f]; i += gridDim.x * blockDim.x) d[i] = s[i];
}

// ---------------------------------------------------------------------------
// Host launchers. The FP64 translation unit instantiates them for double; the
// float instantiations are made once, by the FMA-enabled FP32 translation
// unit, and declared extern everywhere else (kernels_f32.h).
template <class R>
void launch_prim(dim3 g, cudaStream_t st, const BlockDev* bd, const CaseConst* cc, int store_qo) {
  if (store_qo) k_prim<R, true><<<g, 256, 0, st>>>(bd, cc);
  else k_prim<R, false><<<g, 256, 0, st>>>(bd, cc);
}
template <class R>
void launch_dtmax(dim3 g, cudaStream_t st, const BlockDev* bd, const StageParams* sp, const CaseConst* cc,
                  unsigned long long* out, int* err) {
  k_dtmax<R><<<g, 256, 0, st>>>(bd, sp, cc, out, err);
}
template <class R>
void launch_copy_mu(dim3 g, cudaStream_t st, const BlockDev* bd) {
  k_copy_mu<R><<<g, 256, 0, st>>>(bd);
}
template <class R>
void launch_viscous_assemble(dim3 g, cudaStream_t st, const BlockDev* bd) {
  k_viscous_assemble<R><<<g, 256, 0, st>>>(bd);
}
template <class R>
void launch_flux(dim3 g, cudaStream_t st, const BlockDev* bd, const StageParams* sp, const CaseConst* cc) {
  k_flux<R><<<g, 256, 0, st>>>(bd, sp, cc);
}
template <class R>
void launch_flux_visc(dim3 g, cudaStream_t st, const BlockDev* bd, const StageParams* sp, const CaseConst* cc) {
  if constexpr (sizeof(R) == 4) {
    k_flux_visc_pairs<2><<<g, 256, 0, st>>>(bd, sp, cc);
  } else {
    k_flux_visc<R><<<g, 256, 0, st>>>(bd, sp, cc);
  }
}
template <class R>
void launch_flux_sum(dim3 g, cudaStream_t st, const BlockDev* bd) {
  k_flux_sum<R><<<g, 256, 0, st>>>(bd);
}
// the stage state of k_rk_next<R, false> at the listed points (the block
// faces), with the same expression
template <class R>
__global__ void k_rk_faces(const BlockDev* __restrict__ bd, const StageParams* __restrict__ sp,
                           const int* __restrict__ tb, const long long* __restrict__ tl, int ntg) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntg; t += gridDim.x * blockDim.x) {
    const BlockDev& B = bd[tb[t]];
    const Work<R> W = work<R>(B);
    const long long l = tl[t], n = B.npad;
    const double r1 = sp[B.case_id].dtk * B.yaco[l];
    const R* r = W.scr;
    // inputs first, then the stores (see k_rk_next)
    R f[15];
    double qo[5];
#pragma unroll
    for (int k = 0; k < 15; ++k) f[k] = r[l + k * n];
#pragma unroll
    for (int c = 0; c < 5; ++c) qo[c] = B.qo[l + c * n];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      const R dv = (f[3 * c] + f[3 * c + 1]) + f[3 * c + 2];
      B.qa[l + c * n] = qo[c] - r1 * double(dv);
    }
  }
}
template <class R>
void launch_rk_next(dim3 g, cudaStream_t st, const BlockDev* bd, const StageParams* sp, const CaseConst* cc, int sum,
                    int prim, int store_q) {
  if (store_q) k_rk_next<R, true><<<g, 256, 0, st>>>(bd, sp, cc, sum, prim);
  else k_rk_next<R, false><<<g, 256, 0, st>>>(bd, sp, cc, sum, prim);
}
template <class R>
void launch_rk_faces(int grid, cudaStream_t st, const BlockDev* bd, const StageParams* sp, const int* tb,
                     const long long* tl, int ntg) {
  k_rk_faces<R><<<grid, 256, 0, st>>>(bd, sp, tb, tl, ntg);
}
template <class R>
void launch_prim_points(int grid, cudaStream_t st, const BlockDev* bd, const CaseConst* cc, const int* tb,
                        const long long* tl, int ntg) {
  k_prim_points<R><<<grid, 256, 0, st>>>(bd, cc, tb, tl, ntg);
}
template <class R>
void launch_rk(dim3 g, cudaStream_t st, const BlockDev* bd, const StageParams* sp) {
  k_rk<R><<<g, 256, 0, st>>>(bd, sp);
}
template <class R>
void launch_gcbc_setup(int grid, cudaStream_t st, const BlockDev* bd, const GcbcTask* t, const int* f, int nt,
                       int total, const StageParams* sp) {
  k_gcbc_setup<R><<<grid, 128, 0, st>>>(bd, t, f, nt, total, sp);
}
template <class R>
void launch_gcbc_update(int grid, cudaStream_t st, const BlockDev* bd, const GcbcTask* t, const int* f, int nt,
                        int total, const StageParams* sp) {
  k_gcbc_update<R><<<grid, 128, 0, st>>>(bd, t, f, nt, total, sp);
}
template <class R>
void launch_sponge(int grid, cudaStream_t st, const BlockDev* bd, const SpongeTask* t, const int* f, int nt,
                   int total) {
  k_sponge<R><<<grid, 256, 0, st>>>(bd, t, f, nt, total);
}
template <class R>
void launch_face_copy(dim3 g, cudaStream_t st, const void* const* src, void* const* dst, const int* cnt, int n) {
  k_face_copy<R><<<g, 256, 0, st>>>(src, dst, cnt, n);
}
template <class T>
void launch_mpigo_t(int grid, cudaStream_t st, const FaceTask* t, const int* f, int nt, int total) {
  k_mpigo<T><<<grid, 128, 0, st>>>(t, f, nt, total);
}
template <int DIR, int OP, class TT, class RS>
void launch_line_t(int grid, size_t smem, cudaStream_t st, const LineTask* t, const int* f, int nt,
                   const CUtensorMap* maps, int* err) {
  k_line<DIR, OP, TT, RS><<<grid, kLanes, smem, st>>>(t, f, nt, maps, err);
}
template <int DIR, int OP, class TT, class RS = float>
void launch_line2_t(int grid, size_t smem, cudaStream_t st, const LineTask* t, const int* f, int nt,
                    const CUtensorMap* maps, int* err) {
  k_line2<DIR, OP, TT, RS><<<grid, kLanes, smem, st>>>(t, f, nt, maps, err);
}
template <int DIR, int OP, class TT, class RS>
void launch_line2t_t(int grid, size_t smem, cudaStream_t st, const LineTask* t, const int* f, int nt,
                     const CUtensorMap* maps, int* err) {
  k_line2t<DIR, OP, TT, RS><<<grid, 2 * kLanes, smem, st>>>(t, f, nt, maps, err);
}
template <int DIR, int OP, class TT, class RS>
cudaError_t line2t_smem_limit(int bytes) {
  return cudaFuncSetAttribute(k_line2t<DIR, OP, TT, RS>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}
template <int DIR, class TT, class RS>
void launch_line4_t(int grid, size_t smem, cudaStream_t st, const LineTask* t, const int* f, int nt,
                    const CUtensorMap* maps, int* err) {
  k_line4<DIR, TT, RS><<<grid, kLanes, smem, st>>>(t, f, nt, maps, err);
}
template <int DIR, class TT, class RS>
cudaError_t line4_smem_limit(int bytes) {
  return cudaFuncSetAttribute(k_line4<DIR, TT, RS>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}
template <int DIR>
void launch_filt2s_t(int grid, size_t smem, cudaStream_t st, const LineTask* t, const int* f, int nt, int* err) {
  k_filt2s<DIR><<<grid, kLanes, smem, st>>>(t, f, nt, err);
}
template <int DIR>
cudaError_t filt2s_smem_limit(int bytes) {
  return cudaFuncSetAttribute(k_filt2s<DIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}
template <int DIR, int OP, class TT, class RS = float>
cudaError_t line2_smem_limit(int bytes) {
  return cudaFuncSetAttribute(k_line2<DIR, OP, TT, RS>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}
template <int DIR, int OP, class TT, class RS>
cudaError_t line_smem_limit(int bytes) {
  return cudaFuncSetAttribute(k_line<DIR, OP, TT, RS>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

}  // namespace canard
