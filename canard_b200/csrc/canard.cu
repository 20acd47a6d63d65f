// Context, set-up and time-loop orchestration of the Canard hot path, behind
// the C ABI of include/canard_gpu.h. One context = one CUDA stream; all device
// memory is allocated at canard_ctx_create / canard_setup, never on the step
// path.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "canard_gpu.h"
#include "host.h"
#include "kernels.cuh"
#include "kernels_f32.h"
#include "kernels_setup.cuh"
#include "kernels_tm.cuh"

using namespace canard;

namespace {

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct ApiError : std::runtime_error {
  int code;
  ApiError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CK(x)                                                                                   \
  do {                                                                                          \
    cudaError_t e_ = (x);                                                                       \
    if (e_ != cudaSuccess)                                                                      \
      throw CudaError(std::string(#x) + ": " + cudaGetErrorString(e_));                       \
  } while (0)

// Allocation is set-up only. The zero fill is ordered on the context stream:
// that stream is non-blocking, so a fill on the legacy default stream could
// land after later uploads.
template <class T>
T* dalloc(size_t n, cudaStream_t st) {
  void* p = nullptr;
  if (n == 0) n = 1;
  CK(cudaMalloc(&p, n * sizeof(T)));
  CK(cudaMemsetAsync(p, 0, n * sizeof(T), st));
  return static_cast<T*>(p);
}

template <class T>
T* dupload(const std::vector<T>& v, cudaStream_t st) {
  T* p = dalloc<T>(v.size(), st);
  if (!v.empty()) CK(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return p;
}

const int kNnf[3] = {2, 3, 1};  // filter direction order (src/mo_numerics.f90:22)

// A task table resident on the device.
template <class T>
struct Table {
  T* tasks = nullptr;
  int* first = nullptr;  // line tables: the task of every tile; others: each task's first line
  int ntasks = 0;
  int total = 0;  // tiles or lines
  size_t smem = 0;
  double bytes = 0;  // algorithmic bytes of one launch
  CUtensorMap* maps = nullptr;  // line tables: TMA descriptors (in, out) per task
  int kind = 0;  // line tables: a LineKind; face tables: 0 FP64 fields, 1 FP32 fields
  int tdiv = 0;  // line tables: tiles per task when every task has as many (the kernels divide), else 0
};

// Element types of a line launch: tile (field) type and elimination type.
// Element types and solve form of a line launch: FP64 one-lane sweeps
// (bit-exact); FP32 fields; FP64 fields with an FP32 elimination. The FP32
// eliminations come as the split solve (16 lines per tile) or the one-lane
// sweeps (32 lines); the autotuner picks per direction.
enum LineKind {
  LK_F64 = 0,
  LK_F32 = 1,                  // split
  LK_F64_TILE_F32_SOLVE = 2,   // split
  LK_F32_1L = 3,
  LK_F64_TILE_F32_SOLVE_1L = 4,
  LK_F64_TM = 5,               // FP64, elimination results in TMEM (eta/zeta, 16 <= L <= 257)
  LK_F64_STREAM_F32 = 6,       // filter: FP64 field streamed into FP32 right-hand sides, split FP32 solve
  LK_F64_SPLIT = 7,            // FP64 fields, split FP64 solve with FMA (fast FP64 mode)
  LK_F64_QUAD = 8,             // derivative: FP64 fields, four lanes per line, FP64 solve with FMA
  LK_F32_QUAD = 9,             // derivative: FP32 fields, four lanes per line
  LK_F64_TWIST = 10,           // FP64 fields, two-ended FP64 solve with FMA (two warps per 32 lines)
  LK_F32_TWIST = 11,           // derivative: FP32 fields, two-ended FP32 solve
  LK_F64_TILE_F32_TWIST = 12   // filter: FP64 field, two-ended FP32 solve
};
inline bool kind_quad(int kind) { return kind == LK_F64_QUAD || kind == LK_F32_QUAD; }
inline bool kind_twist(int kind) {
  return kind == LK_F64_TWIST || kind == LK_F32_TWIST || kind == LK_F64_TILE_F32_TWIST;
}
inline bool kind_f32_fields(int kind) {
  return kind == LK_F32 || kind == LK_F32_1L || kind == LK_F32_QUAD || kind == LK_F32_TWIST;
}
inline size_t tile_elem(int kind) { return kind_f32_fields(kind) ? sizeof(float) : sizeof(double); }
inline int tile_lanes(int kind) {
  if (kind_quad(kind)) return kQuad;
  return (kind == LK_F32 || kind == LK_F64_TILE_F32_SOLVE || kind == LK_F64_STREAM_F32 || kind == LK_F64_SPLIT)
             ? kHalf
             : kLanes;
}

// Segment boundaries of the quad split along a line of L points: four
// segments of about L/4 rows, each at least the decay lengths kf, ke of the
// homogeneous solutions plus two rows, so that the segments' end values are
// final without a chain across segments. Returns false where L is too short.
bool quad_rows(int L, int kf, int ke, int& q1, int& q2, int& q3) {
  const int need = std::max(kf, ke) + 2;
  q1 = (L + 2) / 4;
  q2 = L / 2;
  q3 = (3 * L) / 4;
  const int len[4] = {q1, q2 - q1, q3 - q2, L - q3};
  for (int k = 0; k < 4; ++k)
    if (len[k] < std::max(need, 16)) return false;
  return true;
}

// First row of the second half of a split solve: balances the two halves'
// register-constant rows (the first half's rows below c0 use the tables
// alone), with a parity that puts their lock-step rows into different banks
// (es: tile element size).
int split_row(int L, int dir, int nt, int c0, int es = 4) {
  const int first = nt == 0 ? 2 : 3;   // first interior row of the elimination
  int h = (L - 3 + first + std::max(c0, first)) / 2;
  auto good = [&](int x) {
    if (es == 8) {
      // row-major FP64 tile (pitch 2 mod 4): an odd offset puts the second
      // half on the odd 8-byte words; a [row][16] FP64 row fills all banks
      return dir != 0 || ((x - first) % 2 + 2) % 2 == 1;
    }
    if (dir == 0) return ((x - first) % 4 + 4) % 4 == 2;  // row-major tile, 16-byte units of 4 floats
    return ((x - first) % 2 + 2) % 2 == 1;                // [row][16] tile
  };
  while (!good(h)) ++h;
  const int lo = nt == 0 ? 4 : 6, hi = L - (nt == 0 ? 2 : 3);
  return std::max(lo, std::min(h, hi));
}

// Correction tables of the split solve (see sweep2), from the FP64 factors:
// H0, H1 = the second half's back substitution (rows L-1..h) of the
// homogeneous forward solutions started at rows h-2, h-1 (index row - h);
// E0, E1 = the homogeneous backward solutions started at rows h, h+1 (index
// h-1-row); each L + 8 entries of type T; returns the lengths beyond which
// every entry stays below thr (set to zero): 1e-12 for the FP32
// eliminations, 1e-18 for the FP64 ones; kf: the same length for the
// forward homogeneous solutions G0, G1 themselves (index row - h), which the
// split kernel forms by their recurrence in registers.
template <class T>
void split_tables(const std::vector<double>& lu, int L, int h, double thr, std::vector<T>& out, int& kg, int& ke,
                  int& kf) {
  const double* l1 = lu.data();
  const double* l2 = l1 + L;
  const double* u1 = l1 + 2 * L;
  const double* u2 = l1 + 3 * L;
  const double* u3 = l1 + 4 * L;
  const int N = L - 1;
  std::vector<double> G0(L, 0.0), G1(L, 0.0), H0(L + 2, 0.0), H1(L + 2, 0.0), E0(L + 2, 0.0), E1(L + 2, 0.0);
  // forward homogeneous: G[i] = -l1[i] G[i-2] - l2[i] G[i-1], started at rows h-2, h-1
  double p2a = 1.0, p1a = 0.0, p2b = 0.0, p1b = 1.0;
  for (int i = h; i < L; ++i) {
    const double ga = -l1[i] * p2a - l2[i] * p1a, gb = -l1[i] * p2b - l2[i] * p1b;
    G0[i] = ga; G1[i] = gb;
    p2a = p1a; p1a = ga; p2b = p1b; p1b = gb;
  }
  // the second half's back substitution of G (rows N..h)
  auto back = [&](const std::vector<double>& g, std::vector<double>& hh) {
    double c1 = u1[N] * g[N];
    hh[N - h] = c1;
    double c = u1[N - 1] * g[N - 1] - u2[N - 1] * c1;
    hh[N - 1 - h] = c;
    double c2 = c1;
    c1 = c;
    for (int i = N - 2; i >= h; --i) {
      c = u1[i] * g[i] - u2[i] * c1 - u3[i] * c2;
      hh[i - h] = c;
      c2 = c1;
      c1 = c;
    }
  };
  back(G0, H0);
  back(G1, H1);
  // backward homogeneous: E[i] = -u2[i] E[i+1] - u3[i] E[i+2], started at rows h, h+1
  double n1a = 1.0, n2a = 0.0, n1b = 0.0, n2b = 1.0;
  for (int i = h - 1; i >= 0; --i) {
    const double ea = -u2[i] * n1a - u3[i] * n2a, eb = -u2[i] * n1b - u3[i] * n2b;
    E0[h - 1 - i] = ea; E1[h - 1 - i] = eb;
    n2a = n1a; n1a = ea; n2b = n1b; n1b = eb;
  }
  auto len = [&](const std::vector<double>& a, const std::vector<double>& b, int n) {
    int k = 0;
    for (int j = 0; j < n; ++j)
      if (std::fabs(a[j]) > thr || std::fabs(b[j]) > thr) k = j + 1;
    return k;
  };
  kg = std::max(2, len(H0, H1, L - h));  // c(h), c(h+1) always read H at 0 and 1
  ke = len(E0, E1, h);
  {
    std::vector<double> g0(G0.begin() + h, G0.end()), g1(G1.begin() + h, G1.end());
    kf = len(g0, g1, L - h);
  }
  const int LT = L + 8;  // padded: the kernel reads the tables in blocks of eight
  out.assign((size_t)4 * LT, T(0));
  for (int j = 0; j < kg; ++j) { out[j] = (T)H0[j]; out[LT + j] = (T)H1[j]; }
  for (int j = 0; j < ke; ++j) { out[2 * LT + j] = (T)E0[j]; out[3 * LT + j] = (T)E1[j]; }
}

// First row of the reversed half of a two-ended solve: the middle of the line.
int twist_row(int L) { return L / 2; }
// the two-ended solve needs halves of at least 16 rows
constexpr int kTwistMinL = 32;

// First row of the range [c0, L-4] over which a factor table's five factors
// are bit-identical to those of row L-4 (as T), and those factors.
template <class T>
int constant_rows(const std::vector<T>& lu, int L, T* cst) {
  const int e = L - 4;
  if (e < 0) return L - 3;
  auto same = [&](int r) {
    for (int k = 0; k < 5; ++k)
      if (std::memcmp(&lu[(size_t)k * L + r], &lu[(size_t)k * L + e], sizeof(T)) != 0) return false;
    return true;
  };
  int c0 = e;
  while (c0 - 1 >= 3 && same(c0 - 1)) --c0;
  for (int k = 0; k < 5; ++k) cst[k] = lu[(size_t)k * L + e];
  return c0;
}

// Factor table of the two-ended solve (k_line2t), as T: the line's factors
// (5 L, from lu), the reversed line's (the system with its ends swapped,
// U1 negated for the derivative, whose right-hand sides change sign on the
// reversed line), the 4 x 4 inverse of the meeting equations times the U1
// factors of their rows, and the reversed factors' constant interior values.
// Returns the first row of that constant range (reversed rows), or -1 where
// the meeting equations are singular.
template <class T>
int twist_tables(const Scheme& sch, const std::vector<double>& lu, int L, int n0, int n1, int nt, int h,
                 std::vector<T>& out) {
  std::vector<double> rl((size_t)5 * L);
  sch.lu(L, n1, n0, nt, rl.data());
  if (nt == 0)
    for (int i = 0; i < L; ++i) rl[(size_t)2 * L + i] = -rl[(size_t)2 * L + i];
  const int N = L - 1;
  auto U1 = [&](const std::vector<double>& f, int i) { return f[(size_t)2 * L + i]; };
  auto U2 = [&](const std::vector<double>& f, int i) { return f[(size_t)3 * L + i]; };
  auto U3 = [&](const std::vector<double>& f, int i) { return f[(size_t)4 * L + i]; };
  // unknowns x(h-2), x(h-1), x(h), x(h+1): rows h-2, h-1 of U, and rows N-h,
  // N-h-1 of the reversed U (the rows of x(h), x(h+1))
  double M[4][8] = {{1, U2(lu, h - 2), U3(lu, h - 2), 0},
                    {0, 1, U2(lu, h - 1), U3(lu, h - 1)},
                    {U3(rl, N - h), U2(rl, N - h), 1, 0},
                    {0, U3(rl, N - h - 1), U2(rl, N - h - 1), 1}};
  const double D[4] = {U1(lu, h - 2), U1(lu, h - 1), U1(rl, N - h), U1(rl, N - h - 1)};
  for (int r = 0; r < 4; ++r)
    for (int k = 0; k < 4; ++k) M[r][4 + k] = r == k ? 1.0 : 0.0;
  for (int col = 0; col < 4; ++col) {  // Gauss-Jordan with partial pivoting
    int p = col;
    for (int r = col + 1; r < 4; ++r)
      if (std::fabs(M[r][col]) > std::fabs(M[p][col])) p = r;
    if (std::fabs(M[p][col]) < 1e-12) return -1;  // not for this system (the kind is then unavailable)
    if (p != col)
      for (int k = 0; k < 8; ++k) std::swap(M[p][k], M[col][k]);
    const double inv = 1.0 / M[col][col];
    for (int k = 0; k < 8; ++k) M[col][k] *= inv;
    for (int r = 0; r < 4; ++r)
      if (r != col) {
        const double f = M[r][col];
        for (int k = 0; k < 8; ++k) M[r][k] -= f * M[col][k];
      }
  }
  out.assign(lu.begin(), lu.end());
  out.insert(out.end(), rl.begin(), rl.end());
  for (int r = 0; r < 4; ++r)
    for (int k = 0; k < 4; ++k) out.push_back((T)(M[r][4 + k] * D[k]));
  std::vector<T> rt(rl.begin(), rl.end());
  T cst[5];
  const int c0 = constant_rows(rt, L, cst);
  for (int k = 0; k < 5; ++k) out.push_back(cst[k]);
  return c0;
}

struct CaseState {
  canard_case_desc d;
  Scheme sch;
  DevScheme* dsch = nullptr;
  int b0 = 0, nb = 0;
  double reoo, srefoo, srefp1dre, uoo[3];
  long long n = 0;  // host mirror of the device step counter (decides the dt-reduction launch)
  // the case's blocks are sub-domains of split blocks (canard_set_subdomains)
  bool split = false;
  Decomp dec;
};

struct BlockState {
  BlockGeom g;
  double* arena = nullptr;
  double* qb = nullptr;  // time-averaged recording (5 fields, padded rows), while recording is on
  BlockDev dev;  // host copy of the device descriptor
  double *lu[2][3] = {};       // [nt][dir]: 5 * L
  double luc[2][3][5] = {};    // bitwise-constant interior factors
  int luc0[2][3] = {};         // first row of the constant range [luc0, L-4]
  double *recv[2][3] = {};     // [nt][dir]: 5 fields x 2 sides x ncomp x nbs
  double* chain[3] = {};       // [dir]: 2 sides x nbs
  double* drva[3] = {};        // (nbs,5,0:1)
  double* drvb[3] = {};
  double* cm[3] = {};          // (nbs,3,0:1)
  long long* gc_pts = nullptr;
  double* gc_w = nullptr;
  std::vector<GcbcFace> gc_faces;
  long long* sp_pts = nullptr;
  double *sp_a = nullptr, *sp_b = nullptr;
  int sp_n = 0;
  std::vector<double> xyz_host;  // reference layout, kept for the sponge set-up
  // mixed precision: FP32 work fields, factors and line-end buffers
  float* arena32 = nullptr;
  float* lu32[2][3] = {};   // FP32 factors (5 L) followed by the split-solve tables (4 (L + 8))
  int h32[2][3] = {}, kg32[2][3] = {}, ke32[2][3] = {}, kf32[2][3] = {};
  float luc32[2][3][5] = {};  // bitwise-constant interior FP32 factors
  int luc032[2][3] = {};      // first row of that range
  float* recv32[3] = {};  // derivative receive buffers of the FP32 fields
  float* drva32[3] = {};
  float* drvb32[3] = {};
  // FP64 factors (5 L) followed by the FP64 split-solve tables (4 (L + 8)):
  // the fast FP64 mode's line kind, also a filter candidate of the mixed path
  double* lu64s[2][3] = {};
  int h64[2][3] = {}, kg64[2][3] = {}, ke64[2][3] = {}, kf64[2][3] = {};
  // two-ended solves: factor tables (twist_tables) in FP64 and FP32, the first
  // row of the reversed half (0: unavailable for this system) and the first
  // row of the reversed factors' constant range
  double* lu64t[2][3] = {};
  float* lu32t[2][3] = {};
  int ht[2][3] = {}, c0r64[2][3] = {}, c0r32[2][3] = {};
  double* recv_ptr(int nt, int dir, int m, int side) const {
    const int nc = nt == 0 ? 2 : 3;
    return recv[nt][dir] + ((size_t)(m - 1) * 2 + side) * nc * g.nbs[dir];
  }
  float* recv32_ptr(int dir, int m, int side) const {
    return recv32[dir] + ((size_t)(m - 1) * 2 + side) * 2 * g.nbs[dir];
  }
};

// field offsets inside a block arena (in units of npad)
enum { F_QA = 0, F_QO = 5, F_DE = 10, F_P = 15, F_MU = 16, F_XIM = 17, F_ETM = 20, F_ZEM = 23, F_YACO = 26,
       F_TAU = 27, F_SCR = 36, F_XYZ = 51, F_COUNT = 54 };
// FP32 field offsets inside the mixed-precision arena (in units of npad)
enum { G_DE = 0, G_P = 5, G_MU = 6, G_TAU = 7, G_SCR = 16, G_XIM = 31, G_ETM = 34, G_ZEM = 37, G_YACO = 40,
       G_COUNT = 41 };

enum TimerFamily {
  T_DERIV_XI = 0, T_DERIV_ETA, T_DERIV_ZETA, T_FILTER_XI, T_FILTER_ETA, T_FILTER_ZETA, T_MPIGO, T_PRIM,
  T_FLUXCOMP, T_VISCASM, T_FLUXSUM, T_RK, T_GCBC, T_SPONGE, T_AVERAGE, T_TIMESTEP, T_COPY, T_NFAM
};
const char* kTimerNames[T_NFAM] = {"deriv_xi", "deriv_eta", "deriv_zeta", "filter_xi", "filter_eta", "filter_zeta",
                                   "mpigo", "primitives", "flux_components", "viscous_assemble", "flux_sum",
                                   "rk_update", "gcbc", "sponge", "averaging", "timestep", "copy_qo"};

struct AvgDev {
  int ntg = 0, nsrc = 0;
  int *tb = nullptr, *tfirst = nullptr, *tcount = nullptr, *sb = nullptr;
  long long *tl = nullptr, *sl = nullptr;
  double* snap = nullptr;
};

}  // namespace

struct canard_ctx {
  std::string err;
  int precision = CANARD_FP64;
  bool f32() const { return precision == CANARD_FP32_MIXED; }
  // fast FP64 mode: FP64 fields with the split FP64 line solves (FMA)
  bool fast() const { return precision == CANARD_FP64_FAST; }
  // the filter runs direction by direction over all five fields (one
  // contraction and one line launch per direction; the send chain's third
  // value is the field value itself, which the reference's running update
  // equals up to one rounding): every context except the bit-exact FP64 one
  bool filter5() const { return precision != CANARD_FP64; }
  cudaStream_t own = nullptr, st = nullptr;
  std::vector<CaseState> cases;
  std::vector<BlockState> blocks;
  std::vector<FaceLink> links;  // global block indices
  BlockDev* dbd = nullptr;
  CaseConst* dcc = nullptr;
  StageParams* dsp = nullptr;       // [5 slots][ncases]: stages 1..4, then the dt reduction / phase calls
  TimeDev* dtime = nullptr;         // [ncases] time-loop state
  double* dsn2 = nullptr;           // ramp factors sin(0.05 pi k)^2, k < kRampTable
  unsigned long long* ddt = nullptr;  // [ncases][2]
  // one step as a CUDA graph, without [0] and with [1] the dt reduction
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  long long graph_launches[2] = {0, 0};
  bool use_graphs = true;
  double* stage = nullptr;  // contiguous staging of host copies (reference layout)
  // canard_step_host: staging of every listed block's state and the two copy streams
  double* hs_stage = nullptr;
  size_t hs_n = 0;
  cudaStream_t s_in = nullptr, s_out = nullptr;
  size_t stage_n = 0;
  int* derr = nullptr;
  bool setup_done = false;
  // hot-path tables
  // filt[m][inn]: the filter of conserved field m along direction kNnf[inn].
  // Field-major as in the reference: every interface contraction advances the
  // persistent send chains of all three directions, so field m+1's filter
  // depends on field m's face values between its sweeps.
  Table<LineTask> filt[5][3], visc[3], flux[3];
  // FP32-mixed: the five fields filtered together along each direction (in
  // kNnf order). The fields are independent; the one change is the third
  // contracted value, which takes the send chain's exact value instead of
  // its rounded running update (a last-bit difference in FP64 face values).
  Table<LineTask> filt5[3];
  Table<FaceTask> mp_filt5[3];
  // line-tile choice per [group: 0 filter, 1 viscous gradients, 2 fluxes][direction]
  // (kind < 0: the precision's default); set by canard_autotune
  struct TuneChoice { int kind = -1; int nc = 0; } tune[3][3];
  Table<FaceTask> mp_filt[5][3], mp_visc, mp_flux;
  Table<GcbcTask> gc_setup, gc_upd[3][2];
  void** fc_src = nullptr;
  void** fc_dst = nullptr;
  int* fc_cnt = nullptr;
  int fc_n = 0, fc_max = 0;
  Table<SpongeTask> sponge;
  AvgDev avg_pt, avg_ln, avg_sf;
  // union of the three plans' target points: the primitives are recomputed
  // there after averaging when the RK update already formed them
  int prim_n = 0;
  int* prim_tb = nullptr;
  long long* prim_tl = nullptr;
  // step-path fusions: flux sum inside the RK update (no GCBC, no sponge in
  // the context), next stage's primitives inside the RK update
  bool fuse_sum = false, fuse_prim = true;
  // wall_condition_update: wall-face points, packed reset kinds (k_wall_update)
  double* dtsum = nullptr;  // [ncases] recording interval, while recording is on
  // every block-face point (k_rk_faces)
  int face_n = 0;
  int* face_tb = nullptr;
  long long* face_tl = nullptr;
  int wall_n = 0;
  int* wall_tb = nullptr;
  long long* wall_tl = nullptr;
  int* wall_tk = nullptr;
  // timers (mo_timer equivalent) and launch counter
  bool timers = false;
  long long launches = 0;
  double t_ms[T_NFAM] = {}, t_n[T_NFAM] = {}, t_bytes[T_NFAM] = {};
  struct Pending { int fam; cudaEvent_t a, b; };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> ev_pool;
  double ew_bytes_per_pt = 0;  // sum over blocks of valid points (for element-wise bytes)
  // scratch for set-up / unit calls
  std::vector<void*> transient;
  int cur_slot_base = 0;
  size_t max_smem_line = 0;
};

namespace {

void set_err(canard_ctx* c, const std::string& m) {
  if (c) c->err = m;
}

int nblk(const canard_ctx* c) { return (int)c->blocks.size(); }

cudaEvent_t pool_event(canard_ctx* c) {
  if (c->ev_pool.empty()) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    return e;
  }
  cudaEvent_t e = c->ev_pool.back();
  c->ev_pool.pop_back();
  return e;
}

// Brackets one launch of family `fam`; `bytes` = algorithmic bytes moved.
struct Timed {
  canard_ctx* c;
  int fam;
  cudaEvent_t b = nullptr;
  Timed(canard_ctx* c_, int fam_, double bytes) : c(c_), fam(fam_) {
    c->launches += 1;
    c->t_n[fam] += 1;
    c->t_bytes[fam] += bytes;
    if (c->timers) {
      cudaEvent_t a = pool_event(c);
      b = pool_event(c);
      CK(cudaEventRecord(a, c->st));
      c->pending.push_back({fam, a, b});
    }
  }
  ~Timed() noexcept(false) {
    if (b) CK(cudaEventRecord(b, c->st));
  }
};

void collect_timers(canard_ctx* c) {
  for (auto& p : c->pending) {
    float ms = 0;
    CK(cudaEventSynchronize(p.b));
    CK(cudaEventElapsedTime(&ms, p.a, p.b));
    c->t_ms[p.fam] += ms;
    c->ev_pool.push_back(p.a);
    c->ev_pool.push_back(p.b);
  }
  c->pending.clear();
}

double valid_points(const canard_ctx* c) {
  double s = 0;
  for (auto& b : c->blocks) s += (double)b.g.X * b.g.Y * b.g.Z;
  return s;
}

double* fptr(const BlockState& b, int f) { return b.arena + (size_t)f * b.g.npad; }
float* gptr(const BlockState& b, int f) { return b.arena32 + (size_t)f * b.g.npad; }

// A tile moves in nc chunks of cr positions: about 64 positions each (2..8
// chunks), cr even (16-byte aligned bulk copies) and at most 256 (a TMA box),
// and the first and the last chunk keep at least 13 positions, so the end
// closures and the in-kernel periodic contraction only need those two.
void chunking(int L, int& nc, int& cr, int nc_req = 0) {
  nc = std::max(1, std::min(kMaxChunks, nc_req > 0 ? nc_req : L / 64));
  for (;; --nc) {
    cr = ((L + nc - 1) / nc + 1) / 2 * 2;
    if (nc <= 2 || (L - (nc - 1) * cr >= 13 && cr >= 13)) break;
  }
  if (nc == 1) cr = (L + 1) / 2 * 2;
}

// xi lines (dir 0) move as one bulk copy per line: per-lane copy instructions
// are costly enough that chunking them does not pay.
void chunking_dir(int dir, int L, int& nc, int& cr, int nc_req = 0) {
  if (dir == 0) {
    nc = 1;
    cr = (L + 1) / 2 * 2;
  } else {
    chunking(L, nc, cr, nc_req);
  }
}

// ---- line task construction ----------------------------------------------------
// Both ends of direction dir periodic onto the block itself: the interface
// contraction of a derivative pass can be formed inside the line kernel.
bool self_periodic(const BlockGeom& g, int dir) {
  return g.nbc[dir][0] == BC_PERIODIC && g.nbc[dir][1] == BC_PERIODIC && g.nbr[dir][0] == g.block_in_case &&
         g.nbr[dir][1] == g.block_in_case;
}

void fill_line_task(const canard_ctx* c, const BlockState& B, int dir /*0..2*/, int nt, const void* in,
                    void* out, int m, bool with_drva, LineTask& t, int kind = LK_F64, bool allow_selfp = false,
                    int nc_req = 0) {
  const BlockGeom& g = B.g;
  // the filter kernels add the increment to the field they read (FP64
  // reduce-add stores): in place only
  if (nt == 1 && in != out) throw ApiError(CANARD_ERR_ARG, "the filter runs in place");
  t.selfp = (allow_selfp && nt == 0 && self_periodic(g, dir)) ? 1 : 0;
  t.in = in;
  t.out = out;
  const bool f64solve = kind == LK_F64 || kind == LK_F64_TM || kind == LK_F64_SPLIT || kind == LK_F64_QUAD ||
                        kind == LK_F64_TWIST;
  t.lu = (kind == LK_F64_SPLIT || kind == LK_F64_QUAD) ? static_cast<const void*>(B.lu64s[nt][dir])
         : kind == LK_F64_TWIST                        ? static_cast<const void*>(B.lu64t[nt][dir])
         : kind_twist(kind)                            ? static_cast<const void*>(B.lu32t[nt][dir])
         : f64solve                                    ? static_cast<const void*>(B.lu[nt][dir])
                                                       : static_cast<const void*>(B.lu32[nt][dir]);
  t.cl1 = B.luc[nt][dir][0]; t.cl2 = B.luc[nt][dir][1]; t.cu1 = B.luc[nt][dir][2];
  t.cu2 = B.luc[nt][dir][3]; t.cu3 = B.luc[nt][dir][4];
  t.c0 = B.luc0[nt][dir];
  t.recv = kind_f32_fields(kind) ? static_cast<const void*>(B.recv32_ptr(dir, m, 0))
                                 : static_cast<const void*>(B.recv_ptr(nt, dir, m, 0));
  t.drva = !with_drva ? nullptr
                      : (kind_f32_fields(kind) ? static_cast<void*>(B.drva32[dir]) : static_cast<void*>(B.drva[dir]));
  t.sc = c->cases[g.case_id].dsch;
  t.X = g.X; t.Y = g.Y; t.Z = g.Z; t.Xp = g.Xp;
  t.L = g.ijk[0][dir] + 1;
  t.nbs = g.nbs[dir];
  t.m = m;
  t.ndf0 = bc_interface(g.nbc[dir][0]) ? 1 : 0;
  t.ndf1 = bc_interface(g.nbc[dir][1]) ? 1 : 0;
  t.h = t.kg = t.ke = t.kf = t.q2 = t.q3 = 0;
  if (!f64solve) {  // FP32 elimination: rounded factors and their constant range
    t.cl1 = B.luc32[nt][dir][0]; t.cl2 = B.luc32[nt][dir][1]; t.cu1 = B.luc32[nt][dir][2];
    t.cu2 = B.luc32[nt][dir][3]; t.cu3 = B.luc32[nt][dir][4];
    t.c0 = B.luc032[nt][dir];
  }
  if (kind_twist(kind)) {
    if (!B.ht[nt][dir] || !t.lu) throw ApiError(CANARD_ERR_ARG, "lines too short for the two-ended solve");
    t.h = B.ht[nt][dir];
    t.kg = kind == LK_F64_TWIST ? B.c0r64[nt][dir] : B.c0r32[nt][dir];
  } else if (kind_quad(kind)) {
    const bool q64 = kind == LK_F64_QUAD;
    t.kf = q64 ? B.kf64[nt][dir] : B.kf32[nt][dir];
    t.ke = q64 ? B.ke64[nt][dir] : B.ke32[nt][dir];
    if (!quad_rows(t.L, t.kf, t.ke, t.h, t.q2, t.q3))
      throw ApiError(CANARD_ERR_ARG, "lines too short for the quad split solve");
  } else if (kind == LK_F64_SPLIT) {
    t.h = B.h64[nt][dir];
    t.kg = B.kg64[nt][dir];
    t.ke = B.ke64[nt][dir];
    t.kf = B.kf64[nt][dir];
  } else if (tile_lanes(kind) == kHalf) {
    t.h = B.h32[nt][dir];
    t.kg = B.kg32[nt][dir];
    t.ke = B.ke32[nt][dir];
    t.kf = B.kf32[nt][dir];
  }
  chunking_dir(dir, t.L, t.nbox, t.by, nc_req);
  if (kind == LK_F64_TM) {  // 32-row boxes streamed through the ring
    t.by = kTmChunk;
    t.nbox = (t.L + kTmChunk - 1) / kTmChunk;
  }
  if (dir != 0) {
    // every chunk's box starts 128-byte aligned in shared memory (a tensor
    // copy's requirement): rows of lanes x element bytes, so FP32 tiles of
    // 8 lanes (32-byte rows) take chunks of a multiple of 4 rows
    const int rb = tile_lanes(kind) * (int)tile_elem(kind);
    const int m = rb >= 128 ? 1 : 128 / rb;
    if (t.by % m) {
      t.by = (t.by + m - 1) / m * m;
      t.nbox = (t.L + t.by - 1) / t.by;
    }
  }
  const int lanes = tile_lanes(kind);
  if (dir == 0) {
    t.ntx = 1;
    t.ntiles = (g.Y * g.Z + lanes - 1) / lanes;
  } else {
    t.ntx = (g.X + lanes - 1) / lanes;
    t.ntiles = t.ntx * (dir == 1 ? g.Z : g.Y);
  }
}

// the largest dynamic shared memory a line kernel's CTA may request (sm_100a:
// 227 KiB per block)
constexpr int kLineSmemMax = 227 * 1024;

// dynamic shared memory of one task's tile
size_t line_smem(int dir, const LineTask& t, int kind) {
  if (kind == LK_F64_TM) return kTmSmem;
  if (kind == LK_F64_STREAM_F32)  // FP32 right-hand-side tile only (no copies in flight)
    return (size_t)kHalf * (dir == 0 ? dir1_pitch<float>(t.L) : t.L) * sizeof(float);
  const size_t es = tile_elem(kind);
  const int lanes = tile_lanes(kind);
  if (kind_twist(kind)) {  // the tile, then both warps' staged closure factors
    const size_t rs = kind == LK_F64_TWIST ? sizeof(double) : sizeof(float);
    const int P = kind_f32_fields(kind) ? dir1_pitch<float>(t.L) : dir1_pitch<double>(t.L);
    return 128 + twist_tile_bytes(dir, t.L, t.nbox, t.by, es, P) + (size_t)2 * 5 * kTwistSh * rs;
  }
  if (dir == 0)
    return 128 + (size_t)lanes * (kind_f32_fields(kind) ? dir1_pitch<float>(t.L) : dir1_pitch<double>(t.L)) * es;
  return 128 + (size_t)t.nbox * t.by * lanes * es;
}

// shared memory of a default-chunked tile of lines of L points
size_t tile_smem_for(int dir, int L, int kind) {
  LineTask t{};
  t.L = L;
  chunking_dir(dir, L, t.nbox, t.by);
  return line_smem(dir, t, kind);
}

// the longest line of direction dir whose tile of this kind fits in a CTA
int max_tile_points(int dir, int kind) {
  int L = 13;
  while (L < 8192 && tile_smem_for(dir, L + 1, kind) <= (size_t)kLineSmemMax) ++L;
  return L;
}

// Lines too long for the shared-memory tile of any kind the context's step
// uses are rejected up front (a launch would fail and lose the context).
void check_line_lengths(const BlockGeom& g, int precision) {
  static const char* dn[3] = {"xi", "eta", "zeta"};
  const bool f32 = precision == CANARD_FP32_MIXED;
  for (int dir = 0; dir < 3; ++dir) {
    const int L = g.ijk[0][dir] + 1;
    const int kinds64[1] = {precision == CANARD_FP64_FAST ? LK_F64_SPLIT : LK_F64};
    const int kinds32[2] = {LK_F64_TILE_F32_SOLVE, LK_F32};
    const int* ks = f32 ? kinds32 : kinds64;
    const int nk = f32 ? 2 : 1;
    for (int i = 0; i < nk; ++i)
      if (tile_smem_for(dir, L, ks[i]) > (size_t)kLineSmemMax)
        throw ApiError(CANARD_ERR_UNSUPPORTED,
                       std::string("lines of ") + std::to_string(L) + " points along " + dn[dir] +
                           " do not fit the shared-memory line tile (at most " +
                           std::to_string(max_tile_points(dir, ks[i])) + " points in this precision)");
  }
}

// cuTensorMapEncodeTiled from the driver, found at run time (the library does
// not link libcuda, so it loads on machines without a GPU).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (!p || q != cudaDriverEntryPointSuccess) throw CudaError("cuTensorMapEncodeTiled not available");
    fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// 3-D map over a padded field (X, Y, Z) with box (32, by, 1) for eta lines or
// (32, 1, by) for zeta lines.
CUtensorMap field_map(const void* base, int X, int Y, int Z, int Xp, int dir, int by, size_t es = sizeof(double),
                      int lanes = kLanes) {
  CUtensorMap m;
  cuuint64_t dims[3] = {(cuuint64_t)X, (cuuint64_t)Y, (cuuint64_t)Z};
  cuuint64_t strides[2] = {(cuuint64_t)Xp * es, (cuuint64_t)Xp * Y * es};
  cuuint32_t box[3] = {(cuuint32_t)lanes, (cuuint32_t)(dir == 1 ? by : 1), (cuuint32_t)(dir == 2 ? by : 1)};
  cuuint32_t estr[3] = {1, 1, 1};
  const CUtensorMapDataType ty = es == sizeof(float) ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  CUresult r = encode_fn()(&m, ty, 3, const_cast<void*>(base), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw CudaError("cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return m;
}

Table<LineTask> make_line_table(canard_ctx* c, std::vector<LineTask> v, int dir, bool transient,
                                int kind = LK_F64) {
  Table<LineTask> T;
  T.kind = kind;
  const size_t es = tile_elem(kind);
  // line tables: `first` holds the task of every tile (one load per CTA
  // instead of a search over the tasks' first tiles)
  std::vector<int> tile_task;
  int tot = 0;
  size_t sm = 0;
  for (size_t i = 0; i < v.size(); ++i) {
    LineTask& t = v[i];
    t.tile0 = tot;
    tile_task.insert(tile_task.end(), (size_t)t.ntiles, (int)i);
    tot += t.ntiles;
    sm = std::max(sm, line_smem(dir, t, kind));
    T.bytes += 2.0 * es * t.X * t.Y * t.Z;  // read the field, write the result
  }
  if (tile_task.empty()) tile_task.push_back(0);
  T.tdiv = v.empty() ? 0 : v[0].ntiles;
  for (const LineTask& t : v)
    if (t.ntiles != T.tdiv) T.tdiv = 0;
  T.ntasks = (int)v.size();
  T.total = tot;
  T.smem = sm;
  T.tasks = dupload(v, c->st);
  T.first = dupload(tile_task, c->st);
  std::vector<CUtensorMap> maps(2 * v.size());
  if (dir != 0)
    for (size_t i = 0; i < v.size(); ++i) {
      maps[2 * i] = field_map(v[i].in, v[i].X, v[i].Y, v[i].Z, v[i].Xp, dir, v[i].by, es, tile_lanes(kind));
      maps[2 * i + 1] = field_map(v[i].out, v[i].X, v[i].Y, v[i].Z, v[i].Xp, dir, v[i].by, es, tile_lanes(kind));
    }
  else
    std::memset(maps.data(), 0, maps.size() * sizeof(CUtensorMap));
  T.maps = dupload(maps, c->st);
  if (transient) {
    c->transient.push_back(T.tasks);
    c->transient.push_back(T.first);
    c->transient.push_back(T.maps);
  }
  return T;
}

template <class T>
Table<T> make_lines_table(canard_ctx* c, std::vector<T> v, bool transient, int T::*count_field,
                          int T::*first_field) {
  Table<T> Tb;
  std::vector<int> first;
  int tot = 0;
  for (auto& t : v) {
    t.*first_field = tot;
    first.push_back(tot);
    tot += t.*count_field;
  }
  Tb.ntasks = (int)v.size();
  Tb.total = tot;
  Tb.tasks = dupload(v, c->st);
  Tb.first = dupload(first, c->st);
  if (transient) {
    c->transient.push_back(Tb.tasks);
    c->transient.push_back(Tb.first);
  }
  return Tb;
}

template <int DIR, int OP, class TT, class RS>
void launch_line_dir(canard_ctx* c, const Table<LineTask>& T) {
  if (T.ntasks == 0 || T.total == 0) return;
  Timed tm(c, (OP == 0 ? T_DERIV_XI : T_FILTER_XI) + DIR - 1, T.bytes);
  launch_line_t<DIR, OP, TT, RS>(T.total, T.smem, c->st, T.tasks, T.first, T.tdiv, T.maps, c->derr);
  CK(cudaGetLastError());
}

template <int DIR, int OP, class TT, class RS = float>
void launch_line2_dir(canard_ctx* c, const Table<LineTask>& T) {
  if (T.ntasks == 0 || T.total == 0) return;
  Timed tm(c, (OP == 0 ? T_DERIV_XI : T_FILTER_XI) + DIR - 1, T.bytes);
  launch_line2_t<DIR, OP, TT, RS>(T.total, T.smem, c->st, T.tasks, T.first, T.tdiv, T.maps, c->derr);
  CK(cudaGetLastError());
}

int num_sms() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
  }
  return n;
}

// persistent: one CTA of kTmWarps tiles per SM
template <int DIR, int OP>
void launch_line_tm_dir(canard_ctx* c, const Table<LineTask>& T) {
  if (T.ntasks == 0 || T.total == 0) return;
  Timed tm(c, (OP == 0 ? T_DERIV_XI : T_FILTER_XI) + DIR - 1, T.bytes);
  const int grid = std::max(1, std::min(num_sms(), (T.total + kTmWarps - 1) / kTmWarps));
  launch_line_tm_t<DIR, OP>(grid, c->st, T.tasks, T.first, T.ntasks, T.total, T.maps, c->derr);
  CK(cudaGetLastError());
}

template <int DIR, int OP, class TT, class RS>
void launch_line2t_dir(canard_ctx* c, const Table<LineTask>& T) {
  if (T.ntasks == 0 || T.total == 0) return;
  Timed tm(c, (OP == 0 ? T_DERIV_XI : T_FILTER_XI) + DIR - 1, T.bytes);
  launch_line2t_t<DIR, OP, TT, RS>(T.total, T.smem, c->st, T.tasks, T.first, T.tdiv, T.maps, c->derr);
  CK(cudaGetLastError());
}

template <int DIR, class TT, class RS>
void launch_line4_dir(canard_ctx* c, const Table<LineTask>& T) {
  if (T.ntasks == 0 || T.total == 0) return;
  Timed tm(c, T_DERIV_XI + DIR - 1, T.bytes);
  launch_line4_t<DIR, TT, RS>(T.total, T.smem, c->st, T.tasks, T.first, T.tdiv, T.maps, c->derr);
  CK(cudaGetLastError());
}

template <int DIR>
void launch_filt2s_dir(canard_ctx* c, const Table<LineTask>& T) {
  if (T.ntasks == 0 || T.total == 0) return;
  Timed tm(c, T_FILTER_XI + DIR - 1, T.bytes);
  launch_filt2s_t<DIR>(T.total, T.smem, c->st, T.tasks, T.first, T.tdiv, c->derr);
  CK(cudaGetLastError());
}

template <int DIR, int OP>
void launch_line_kind(canard_ctx* c, const Table<LineTask>& T) {
  if (T.kind == LK_F64) launch_line_dir<DIR, OP, double, double>(c, T);
  else if (DIR != 1 && T.kind == LK_F64_TM) launch_line_tm_dir<(DIR == 1 ? 2 : DIR), OP>(c, T);
  else if (OP == 0 && T.kind == LK_F32) launch_line2_dir<DIR, 0, float>(c, T);
  else if (OP == 1 && T.kind == LK_F64_TILE_F32_SOLVE) launch_line2_dir<DIR, 1, double>(c, T);
  else if (OP == 0 && T.kind == LK_F32_1L) launch_line_dir<DIR, 0, float, float>(c, T);
  else if (OP == 1 && T.kind == LK_F64_TILE_F32_SOLVE_1L) launch_line_dir<DIR, 1, double, float>(c, T);
  else if (OP == 1 && T.kind == LK_F64_STREAM_F32) launch_filt2s_dir<DIR>(c, T);
  else if (T.kind == LK_F64_SPLIT) launch_line2_dir<DIR, OP, double, double>(c, T);
  else if (OP == 0 && T.kind == LK_F64_QUAD) launch_line4_dir<DIR, double, double>(c, T);
  else if (OP == 0 && T.kind == LK_F32_QUAD) launch_line4_dir<DIR, float, float>(c, T);
  else if (T.kind == LK_F64_TWIST) launch_line2t_dir<DIR, OP, double, double>(c, T);
  else if (OP == 0 && T.kind == LK_F32_TWIST) launch_line2t_dir<DIR, 0, float, float>(c, T);
  else if (OP == 1 && T.kind == LK_F64_TILE_F32_TWIST) launch_line2t_dir<DIR, 1, double, float>(c, T);
  else throw ApiError(CANARD_ERR_ARG, "line table of an unsupported element type");
}

void launch_line(canard_ctx* c, const Table<LineTask>& T, int dir, int op) {
  if (op == 0) {
    if (dir == 0) launch_line_kind<1, 0>(c, T);
    else if (dir == 1) launch_line_kind<2, 0>(c, T);
    else launch_line_kind<3, 0>(c, T);
  } else {
    if (dir == 0) launch_line_kind<1, 1>(c, T);
    else if (dir == 1) launch_line_kind<2, 1>(c, T);
    else launch_line_kind<3, 1>(c, T);
  }
}

// The dynamic shared memory limit is a per-device function attribute: it is
// raised once for every device this process uses (with that device current).
void set_line_smem_limits() {
  static std::mutex mu;
  static bool done_dev[256] = {};
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) throw ApiError(CANARD_ERR_ARG, "device index out of range");
  std::lock_guard<std::mutex> lk(mu);
  if (done_dev[dev]) return;
  const int lim = kLineSmemMax;
  CK((line_smem_limit<1, 0, double, double>(lim)));
  CK((line_smem_limit<2, 0, double, double>(lim)));
  CK((line_smem_limit<3, 0, double, double>(lim)));
  CK((line_smem_limit<1, 1, double, double>(lim)));
  CK((line_smem_limit<2, 1, double, double>(lim)));
  CK((line_smem_limit<3, 1, double, double>(lim)));
  CK((line2_smem_limit<1, 0, float>(lim)));
  CK((line2_smem_limit<2, 0, float>(lim)));
  CK((line2_smem_limit<3, 0, float>(lim)));
  CK((line2_smem_limit<1, 1, double>(lim)));
  CK((line2_smem_limit<2, 1, double>(lim)));
  CK((line2_smem_limit<3, 1, double>(lim)));
  CK((line_smem_limit<1, 0, float, float>(lim)));
  CK((line_smem_limit<2, 0, float, float>(lim)));
  CK((line_smem_limit<3, 0, float, float>(lim)));
  CK((line_smem_limit<1, 1, double, float>(lim)));
  CK((line_smem_limit<2, 1, double, float>(lim)));
  CK((line_smem_limit<3, 1, double, float>(lim)));
  CK((line_tm_smem_limit<2, 0>()));
  CK((line_tm_smem_limit<3, 0>()));
  CK((line_tm_smem_limit<2, 1>()));
  CK((line_tm_smem_limit<3, 1>()));
  CK((line2_smem_limit<1, 0, double, double>(lim)));
  CK((line2_smem_limit<2, 0, double, double>(lim)));
  CK((line2_smem_limit<3, 0, double, double>(lim)));
  CK((line2_smem_limit<1, 1, double, double>(lim)));
  CK((line2_smem_limit<2, 1, double, double>(lim)));
  CK((line2_smem_limit<3, 1, double, double>(lim)));
  CK((line2t_smem_limit<1, 0, double, double>(lim)));
  CK((line2t_smem_limit<2, 0, double, double>(lim)));
  CK((line2t_smem_limit<3, 0, double, double>(lim)));
  CK((line2t_smem_limit<1, 1, double, double>(lim)));
  CK((line2t_smem_limit<2, 1, double, double>(lim)));
  CK((line2t_smem_limit<3, 1, double, double>(lim)));
  CK((line2t_smem_limit<1, 0, float, float>(lim)));
  CK((line2t_smem_limit<2, 0, float, float>(lim)));
  CK((line2t_smem_limit<3, 0, float, float>(lim)));
  CK((line2t_smem_limit<1, 1, double, float>(lim)));
  CK((line2t_smem_limit<2, 1, double, float>(lim)));
  CK((line2t_smem_limit<3, 1, double, float>(lim)));
  CK((line4_smem_limit<1, double, double>(lim)));
  CK((line4_smem_limit<2, double, double>(lim)));
  CK((line4_smem_limit<3, double, double>(lim)));
  CK((line4_smem_limit<1, float, float>(lim)));
  CK((line4_smem_limit<2, float, float>(lim)));
  CK((line4_smem_limit<3, float, float>(lim)));
  CK((filt2s_smem_limit<1>(lim)));
  CK((filt2s_smem_limit<2>(lim)));
  CK((filt2s_smem_limit<3>(lim)));
  done_dev[dev] = true;
}

// ---- mpigo face tasks ----------------------------------------------------------
// One task per sending face (block, dir, side) with ndf = 1. `col(b, dir)`
// gives the field column the block uses for that direction.
template <class ColFn>
std::vector<FaceTask> face_tasks(const canard_ctx* c, int nt, int n45, int m, int exch_dir, ColFn col,
                                 int only_case = -1, bool f32 = false, bool skip_selfp = false) {
  std::vector<FaceTask> out;
  int line0 = 0;
  for (const FaceLink& L : c->links) {
    if (only_case >= 0 && c->blocks[L.src_b].g.case_id != only_case) continue;
    const BlockState& S = c->blocks[L.src_b];
    const BlockState& R = c->blocks[L.dst_b];
    const int d = L.nn;
    if (!bc_interface(S.g.nbc[d][L.src_side])) continue;
    if (skip_selfp && L.src_b == L.dst_b && self_periodic(S.g, d)) continue;  // formed in the line kernel
    FaceTask t{};
    t.src = col(L.src_b, d);
    t.dstf = col(L.dst_b, d);
    t.recv = f32 ? static_cast<void*>(R.recv32_ptr(d, m, L.dst_side))
                 : static_cast<void*>(R.recv_ptr(nt, d, m, L.dst_side));
    t.chain = S.chain[d] + (size_t)L.src_side * S.g.nbs[d];
    t.sc = c->cases[S.g.case_id].dsch;
    t.nn = d + 1;
    t.sb = L.src_side;
    t.nt = nt;
    t.exch = (exch_dir < 0 || exch_dir == d) ? 1 : 0;
    const int np = S.g.nbc[d][L.src_side];
    t.iik = (np == BC_SUBDOM) ? 0 : 1;
    t.ra0k = (np == BC_PERIODIC) ? (double)n45 : 0.0;
    t.corr = (n45 == 1 && R.g.nbc[d][L.dst_side] == BC_PERIODIC) ? 1 : 0;
    t.X = S.g.X; t.Y = S.g.Y; t.Z = S.g.Z; t.Xp = S.g.Xp; t.N = S.g.ijk[0][d];
    t.XA = R.g.X; t.YA = R.g.Y; t.ZA = R.g.Z; t.XpA = R.g.Xp; t.NA = R.g.ijk[0][d];
    t.nbs = S.g.nbs[d];
    t.nj = S.g.ijk[1][d] + 1;
    t.line0 = line0;
    line0 += t.nbs;
    out.push_back(t);
  }
  return out;
}

Table<FaceTask> make_face_table(canard_ctx* c, std::vector<FaceTask> v, bool transient, int kind = 0) {
  Table<FaceTask> T;
  T.kind = kind;
  std::vector<int> first;
  int tot = 0;
  for (auto& t : v) { t.line0 = tot; first.push_back(tot); tot += t.nbs; }
  T.ntasks = (int)v.size();
  T.total = tot;
  T.bytes = (double)tot * (12 + (v.empty() ? 0 : (v[0].nt ? 3 : 2))) * (kind ? sizeof(float) : sizeof(double));
  T.tasks = dupload(v, c->st);
  T.first = dupload(first, c->st);
  if (transient) { c->transient.push_back(T.tasks); c->transient.push_back(T.first); }
  return T;
}

void launch_mpigo(canard_ctx* c, const Table<FaceTask>& T) {
  if (T.ntasks == 0) return;
  const int thr = 128;
  const int grid = std::min((T.total + thr - 1) / thr, 148 * 16);
  Timed tm(c, T_MPIGO, T.bytes);
  if (T.kind) launch_mpigo_t<float>(grid, c->st, T.tasks, T.first, T.ntasks, T.total);
  else launch_mpigo_t<double>(grid, c->st, T.tasks, T.first, T.ntasks, T.total);
  CK(cudaGetLastError());
}

dim3 ew_grid(const canard_ctx* c) {
  long long mx = 0;
  for (auto& b : c->blocks) mx = std::max<long long>(mx, (long long)b.g.npad);
  long long gx = std::min<long long>((mx + 255) / 256, 148 * 8);
  return dim3((unsigned)std::max<long long>(gx, 1), (unsigned)c->blocks.size());
}

void free_transient(canard_ctx* c) {
  for (void* p : c->transient) cudaFree(p);
  c->transient.clear();
}

void collect_timers(canard_ctx* c);
void sync_check(canard_ctx* c) {
  CK(cudaStreamSynchronize(c->st));
  collect_timers(c);
  int e = 0;
  CK(cudaMemcpy(&e, c->derr, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    CK(cudaMemset(c->derr, 0, sizeof(int)));
    if (e == kErrOverflow)
      throw ApiError(CANARD_ERR_NAN, "Canard: Overflow. (dt == 0 after step 2, or a non-finite state)");
    throw ApiError(CANARD_ERR_TIMEOUT, "a bounded device wait gave up (error flag set by a kernel)");
  }
}

constexpr int kRampTable = 64;

StageParams* dev_slot(canard_ctx* c, int slot) {  // slot 0..3 = stages, 4 = dt reduction / phase calls
  return c->dsp + (size_t)slot * c->cases.size();
}

int ncase(const canard_ctx* c) { return (int)c->cases.size(); }

// stage scalars of stages nk0..nk1 into slots nk0-1..nk1-1 (or, with
// to_slot >= 0, of one stage into that slot), from the device time state
void stage_params(canard_ctx* c, int nk0, int nk1, int to_slot = -1) {
  const int n = (nk1 - nk0 + 1) * ncase(c);
  StageParams* out = to_slot >= 0 ? dev_slot(c, to_slot) : dev_slot(c, nk0 - 1);
  c->launches += 1;
  k_stage_params<<<(n + 127) / 128, 128, 0, c->st>>>(c->dtime, c->dcc, out, nk0, nk1, ncase(c));
  CK(cudaGetLastError());
}

// ---- phases --------------------------------------------------------------------
// filtering (src/mo_canard_driver.f90:232-251): for each field, the
// interface contraction and the filter sweep along each direction in turn
void ph_filter(canard_ctx* c) {
  if (c->filter5()) {
    for (int inn = 1; inn <= 3; ++inn) {
      launch_mpigo(c, c->mp_filt5[inn - 1]);
      launch_line(c, c->filt5[inn - 1], kNnf[inn - 1] - 1, 1);
    }
    return;
  }
  for (int m = 1; m <= 5; ++m)
    for (int inn = 1; inn <= 3; ++inn) {
      launch_mpigo(c, c->mp_filt[m - 1][inn - 1]);
      launch_line(c, c->filt[m - 1][inn - 1], kNnf[inn - 1] - 1, 1);
    }
}

void ph_copyqo(canard_ctx* c) {
  Timed tm(c, T_COPY, 80.0 * valid_points(c));
  k_copy5<<<ew_grid(c), 256, 0, c->st>>>(c->dbd);
  CK(cudaGetLastError());
}

// Algorithmic bytes per point of an element-wise kernel: n64 FP64 values and
// nr values of the flux type.
double ew_bytes(const canard_ctx* c, int n64, int nr) {
  return (8.0 * n64 + (c->f32() ? 4.0 : 8.0) * nr) * valid_points(c);
}

// with store_qo (the step's first stage) the pass also copies qa to qo
void ph_prim(canard_ctx* c, bool store_qo = false) {
  Timed tm(c, T_PRIM, ew_bytes(c, store_qo ? 10 : 5, 7));
  if (c->f32()) launch_prim<float>(ew_grid(c), c->st, c->dbd, c->dcc, store_qo ? 1 : 0);
  else launch_prim<double>(ew_grid(c), c->st, c->dbd, c->dcc, store_qo ? 1 : 0);
  CK(cudaGetLastError());
}

bool any_viscous(const canard_ctx* c) {
  for (auto& cs : c->cases)
    if (cs.d.viscous) return true;
  return false;
}

// interface contraction and the 12 derivative sweeps of u, v, w, T
void viscous_gradients(canard_ctx* c) {
  launch_mpigo(c, c->mp_visc);
  launch_line(c, c->visc[2], 2, 0);
  launch_line(c, c->visc[1], 1, 0);
  launch_line(c, c->visc[0], 0, 0);
}

// flux interface contraction, the 15 derivative sweeps and (unless the RK
// update forms it) their sum into de
void flux_derivatives(canard_ctx* c, bool sum = true) {
  launch_mpigo(c, c->mp_flux);
  launch_line(c, c->flux[0], 0, 0);
  launch_line(c, c->flux[1], 1, 0);
  launch_line(c, c->flux[2], 2, 0);
  if (!sum) return;
  Timed tm(c, T_FLUXSUM, ew_bytes(c, 0, 20));
  if (c->f32()) launch_flux_sum<float>(ew_grid(c), c->st, c->dbd);
  else launch_flux_sum<double>(ew_grid(c), c->st, c->dbd);
  CK(cudaGetLastError());
}

// calc_viscous_shear_stress as the phase of the C ABI (tau stored)
void ph_viscous(canard_ctx* c) {
  if (!any_viscous(c)) return;
  {
    Timed tm(c, T_COPY, ew_bytes(c, 0, 2));
    if (c->f32()) launch_copy_mu<float>(ew_grid(c), c->st, c->dbd);
    else launch_copy_mu<double>(ew_grid(c), c->st, c->dbd);
    CK(cudaGetLastError());
  }
  viscous_gradients(c);
  Timed tm(c, T_VISCASM, ew_bytes(c, 0, 12 + 9 + 1 + 4 + 9 + 1));
  if (c->f32()) launch_viscous_assemble<float>(ew_grid(c), c->st, c->dbd);
  else launch_viscous_assemble<double>(ew_grid(c), c->st, c->dbd);
  CK(cudaGetLastError());
}

// calc_fluxes as the phase of the C ABI (reads the stored tau)
void ph_fluxes(canard_ctx* c, const StageParams* sp) {
  {
    Timed tm(c, T_FLUXCOMP, ew_bytes(c, 5, 1 + 3 + 9 + 9 + 15 + 1));
    if (c->f32()) launch_flux<float>(ew_grid(c), c->st, c->dbd, sp, c->dcc);
    else launch_flux<double>(ew_grid(c), c->st, c->dbd, sp, c->dcc);
    CK(cudaGetLastError());
  }
  flux_derivatives(c);
}

// The step path: viscous stresses formed inside the flux kernel (no tau
// round trip, no ss copy into de(:,1)); bit-identical to ph_viscous + ph_fluxes.
void ph_visc_fluxes(canard_ctx* c, const StageParams* sp) {
  const bool visc = any_viscous(c);
  if (visc) viscous_gradients(c);
  {
    // reads: qa 5 (FP64; FP32 forms the state from 1/rho, u, v, w, p instead);
    // p, u, v, w, metrics 9, and if viscous 12 gradients, ss, yaco;
    // writes: 15 flux components, de(:,5)
    const int rd = 1 + 3 + 9 + (visc ? 12 + 1 + 1 : 0) + 15 + 1;
    Timed tm(c, T_FLUXCOMP, c->f32() ? ew_bytes(c, 0, rd + 1) : ew_bytes(c, 5, rd));
    if (c->f32()) launch_flux_visc<float>(ew_grid(c), c->st, c->dbd, sp, c->dcc);
    else launch_flux_visc<double>(ew_grid(c), c->st, c->dbd, sp, c->dcc);
    CK(cudaGetLastError());
  }
  flux_derivatives(c, !c->fuse_sum);
}

void ph_gcbc(canard_ctx* c, const StageParams* sp) {
  if (c->gc_setup.ntasks == 0) return;
  const int thr = 128;
  auto grid = [](int n) { return std::max(1, std::min((n + 127) / 128, 148 * 8)); };
  Timed tm(c, T_GCBC, 0.0);
  (void)thr;
  if (c->f32())
    launch_gcbc_setup<float>(grid(c->gc_setup.total), c->st, c->dbd, c->gc_setup.tasks, c->gc_setup.first,
                             c->gc_setup.ntasks, c->gc_setup.total, sp);
  else
    launch_gcbc_setup<double>(grid(c->gc_setup.total), c->st, c->dbd, c->gc_setup.tasks, c->gc_setup.first,
                              c->gc_setup.ntasks, c->gc_setup.total, sp);
  CK(cudaGetLastError());
  for (int d = 0; d < 3; ++d)
    for (int s = 0; s < 2; ++s) c->launches += c->gc_upd[d][s].ntasks > 0 ? 1 : 0;
  if (c->fc_n > 0) {
    c->launches += 1;
    const dim3 g(std::max(1, std::min((c->fc_max + 255) / 256, 1024)), c->fc_n);
    if (c->f32()) launch_face_copy<float>(g, c->st, c->fc_src, c->fc_dst, c->fc_cnt, c->fc_n);
    else launch_face_copy<double>(g, c->st, c->fc_src, c->fc_dst, c->fc_cnt, c->fc_n);
    CK(cudaGetLastError());
  }
  for (int d = 0; d < 3; ++d)
    for (int s = 0; s < 2; ++s) {
      const auto& T = c->gc_upd[d][s];
      if (T.ntasks == 0) continue;
      if (c->f32()) launch_gcbc_update<float>(grid(T.total), c->st, c->dbd, T.tasks, T.first, T.ntasks, T.total, sp);
      else launch_gcbc_update<double>(grid(T.total), c->st, c->dbd, T.tasks, T.first, T.ntasks, T.total, sp);
      CK(cudaGetLastError());
    }
}

void ph_sponge(canard_ctx* c) {
  if (c->sponge.ntasks == 0 || c->sponge.total == 0) return;
  const int grid = std::max(1, std::min((c->sponge.total + 255) / 256, 148 * 8));
  Timed tm(c, T_SPONGE, 8.0 * 22 * c->sponge.total);
  if (c->f32())
    launch_sponge<float>(grid, c->st, c->dbd, c->sponge.tasks, c->sponge.first, c->sponge.ntasks, c->sponge.total);
  else
    launch_sponge<double>(grid, c->st, c->dbd, c->sponge.tasks, c->sponge.first, c->sponge.ntasks, c->sponge.total);
  CK(cudaGetLastError());
}

void ph_rk(canard_ctx* c, const StageParams* sp) {
  Timed tm(c, T_RK, ew_bytes(c, 11, 5));
  if (c->f32()) launch_rk<float>(ew_grid(c), c->st, c->dbd, sp);
  else launch_rk<double>(ew_grid(c), c->st, c->dbd, sp);
  CK(cudaGetLastError());
}

// the step path's RK update: flux sum and next primitives fused as the
// context allows (k_rk_next)
void ph_rk_next(canard_ctx* c, const StageParams* sp, bool prim) {
  // the last stage stores the summed right-hand side (readable after a step)
  const int sum = c->fuse_sum ? (prim ? 1 : 2) : 0;
  // FP32 stages 1-3 without GCBC, sponge or walls: the stage state only on the
  // block faces (the FP32 fluxes read the primitives), stored by k_rk_faces;
  // worth it while the face points are few (large blocks)
  const bool faces = c->f32() && prim && c->fuse_sum && c->wall_n == 0 && c->face_n > 0 &&
                     c->face_n < 0.05 * valid_points(c);
  Timed tm(c, T_RK, ew_bytes(c, 11 - (faces ? 5 : 0), (sum ? 15 : 5) + (sum == 2 ? 5 : 0) + (prim ? 7 : 0)));
  if (c->f32()) launch_rk_next<float>(ew_grid(c), c->st, c->dbd, sp, c->dcc, sum, prim, faces ? 0 : 1);
  else launch_rk_next<double>(ew_grid(c), c->st, c->dbd, sp, c->dcc, sum, prim, 1);
  CK(cudaGetLastError());
  if (faces) {
    c->launches += 1;
    launch_rk_faces<float>(std::max(1, std::min((c->face_n + 255) / 256, 1184)), c->st, c->dbd, sp, c->face_tb,
                           c->face_tl, c->face_n);
  }
  CK(cudaGetLastError());
}

// primitives at the averaged points (after ph_rk_next formed them everywhere)
void ph_prim_points(canard_ctx* c) {
  if (c->prim_n == 0) return;
  Timed tm(c, T_PRIM, (8.0 * 5 + (c->f32() ? 4.0 : 8.0) * 7) * c->prim_n);
  const int grid = std::max(1, std::min((c->prim_n + 255) / 256, 1184));
  if (c->f32()) launch_prim_points<float>(grid, c->st, c->dbd, c->dcc, c->prim_tb, c->prim_tl, c->prim_n);
  else launch_prim_points<double>(grid, c->st, c->dbd, c->dcc, c->prim_tb, c->prim_tl, c->prim_n);
  CK(cudaGetLastError());
}

void ph_wall(canard_ctx* c, const StageParams* sp) {
  if (c->wall_n == 0) return;
  Timed tm(c, T_RK, 8.0 * 10 * c->wall_n);
  k_wall_update<<<std::max(1, std::min((c->wall_n + 255) / 256, 1184)), 256, 0, c->st>>>(
      c->dbd, sp, c->wall_tb, c->wall_tl, c->wall_tk, c->wall_n);
  CK(cudaGetLastError());
}

void run_avg(canard_ctx* c, const AvgDev& A, int mode) {
  if (A.ntg == 0) return;
  Timed tm(c, T_AVERAGE, 8.0 * 5 * (A.nsrc + A.ntg));
  c->launches += 1;  // snapshot + combine
  k_avg_snapshot<<<std::max(1, std::min((A.nsrc + 255) / 256, 1184)), 256, 0, c->st>>>(c->dbd, A.sb, A.sl,
                                                                                       A.nsrc, A.snap);
  CK(cudaGetLastError());
  k_avg_combine<<<std::max(1, std::min((A.ntg + 255) / 256, 1184)), 256, 0, c->st>>>(
      c->dbd, A.tb, A.tl, A.tfirst, A.tcount, A.ntg, A.snap, mode);
  CK(cudaGetLastError());
}

void ph_average(canard_ctx* c) {
  run_avg(c, c->avg_pt, 0);
  run_avg(c, c->avg_ln, 0);
  run_avg(c, c->avg_sf, 1);
}

bool needs_dt_reduction(const canard_ctx* c) {
  for (auto& cs : c->cases)
    if (cs.n % 10 == 1) return true;
  return false;
}

// time step reduction (src/mo_physics.f90:171-211) every tenth step and the dt
// ramp (src/mo_canard_driver.f90:278-294), all on the device
void timestep(canard_ctx* c) {
  if (needs_dt_reduction(c)) {
    stage_params(c, 1, 1, 4);  // stage-1 moving frame (dtko = dtk = 0)
    CK(cudaMemsetAsync(c->ddt, 0, 2 * c->cases.size() * sizeof(unsigned long long), c->st));
    Timed tm(c, T_TIMESTEP, ew_bytes(c, 10, 7));
    if (c->f32()) launch_dtmax<float>(ew_grid(c), c->st, c->dbd, dev_slot(c, 4), c->dcc, c->ddt, c->derr);
    else launch_dtmax<double>(ew_grid(c), c->st, c->dbd, dev_slot(c, 4), c->dcc, c->ddt, c->derr);
    CK(cudaGetLastError());
  }
  c->launches += 1;
  k_time_dt<<<(ncase(c) + 127) / 128, 128, 0, c->st>>>(c->dtime, c->ddt, c->dcc, c->dsn2, kRampTable, ncase(c),
                                                       c->derr);
  CK(cudaGetLastError());
}

void time_advance(canard_ctx* c) {
  c->launches += 1;
  k_time_advance<<<(ncase(c) + 127) / 128, 128, 0, c->st>>>(c->dtime, ncase(c));
  CK(cudaGetLastError());
  for (auto& cs : c->cases) cs.n = cs.n + 1;
}

// The time-loop body (src/mo_canard_driver.f90:226-370): every launch on c->st,
// no host synchronisation, so it can be captured as a graph.
void step_body(canard_ctx* c) {
  ph_filter(c);
  ph_prim(c, true);  // and qo = qa
  timestep(c);
  stage_params(c, 1, 4);
  for (int nk = 1; nk <= 4; ++nk) {
    const StageParams* sp = dev_slot(c, nk - 1);
    if (nk > 1 && !c->fuse_prim) ph_prim(c);
    ph_visc_fluxes(c, sp);
    ph_gcbc(c, sp);
    ph_sponge(c);
    const bool prim = c->fuse_prim && nk < 4;
    ph_rk_next(c, sp, prim);
    ph_wall(c, sp);
    ph_average(c);
    if (prim) ph_prim_points(c);
  }
  time_advance(c);
}

// One step: replays the captured graph of the step (captured on first use,
// per variant with and without the dt reduction), or launches the kernels
// directly while per-family timers are on.
void one_step(canard_ctx* c) {
  if (!c->use_graphs || c->timers) {
    step_body(c);
    return;
  }
  const int v = needs_dt_reduction(c) ? 1 : 0;
  if (!c->graph[v]) {
    // capture on the context's own stream (a legacy default stream cannot
    // capture); the graph then runs on whatever stream the context uses
    cudaStream_t user = c->st;
    CK(cudaStreamSynchronize(user));
    c->st = c->own;
    const long long l0 = c->launches;
    const long long n0 = c->cases.empty() ? 0 : c->cases[0].n;
    std::vector<long long> nsave;
    for (auto& cs : c->cases) nsave.push_back(cs.n);
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
    try {
      step_body(c);
    } catch (...) {
      cudaStreamEndCapture(c->st, &g);
      if (g) cudaGraphDestroy(g);
      c->st = user;
      throw;
    }
    CK(cudaStreamEndCapture(c->st, &g));
    c->st = user;
    (void)n0;
    for (size_t i = 0; i < c->cases.size(); ++i) c->cases[i].n = nsave[i];
    c->graph_launches[v] = c->launches - l0;
    c->launches = l0;
    cudaError_t e = cudaGraphInstantiate(&c->graph[v], g, 0);
    cudaGraphDestroy(g);
    CK(e);
  }
  CK(cudaGraphLaunch(c->graph[v], c->st));
  c->launches += c->graph_launches[v];
  for (auto& cs : c->cases) cs.n = cs.n + 1;
}

// ---- set-up ------------------------------------------------------------------------
// The line tasks of one group (0 filter of field m, 1 viscous gradients,
// 2 fluxes) and direction, for line kind `kind` and chunk count `nc`
// (0 = default). With `scratch`, filter tasks work on scratch fields instead
// of the state (autotuning).
std::vector<LineTask> group_tasks(canard_ctx* c, int grp, int dir, int m, int kind, int nc, bool scratch = false) {
  const int nb = nblk(c);
  const bool w32 = kind_f32_fields(kind);
  auto wf = [&](int b, int f64_field, int f32_field) -> void* {
    return w32 ? static_cast<void*>(gptr(c->blocks[b], f32_field)) : static_cast<void*>(fptr(c->blocks[b], f64_field));
  };
  std::vector<LineTask> v;
  for (int b = 0; b < nb; ++b) {
    if (grp == 0) {
      LineTask t;
      double* f = fptr(c->blocks[b], scratch ? F_SCR + m - 1 : F_QA + m - 1);
      fill_line_task(c, c->blocks[b], dir, 1, f, f, m, false, t, kind, false, nc);
      v.push_back(t);
    } else if (grp == 1) {
      // viscous gradients: de(:,m) m = 2..5 -> scr 3*(m-2) + dir
      if (!c->cases[c->blocks[b].g.case_id].d.viscous) continue;
      for (int mm = 2; mm <= 5; ++mm) {
        LineTask t;
        fill_line_task(c, c->blocks[b], dir, 0, wf(b, F_DE + mm - 1, G_DE + mm - 1),
                       wf(b, F_SCR + 3 * (mm - 2) + dir, G_SCR + 3 * (mm - 2) + dir), mm, false, t, kind, true, nc);
        v.push_back(t);
      }
    } else {
      // fluxes: scr 3*(m-1) + dir, in place
      for (int mm = 1; mm <= 5; ++mm) {
        LineTask t;
        void* f = wf(b, F_SCR + 3 * (mm - 1) + dir, G_SCR + 3 * (mm - 1) + dir);
        fill_line_task(c, c->blocks[b], dir, 0, f, f, mm, true, t, kind, true, nc);
        v.push_back(t);
      }
    }
  }
  return v;
}

// the TMEM line kernel takes eta/zeta lines of kTmMinL..kTmMaxL points
bool tm_ok(const canard_ctx* c, int dir) {
  if (dir == 0 || c->blocks.empty()) return false;
  for (const auto& b : c->blocks) {
    const int L = b.g.ijk[0][dir] + 1;
    if (L < kTmMinL || L > kTmMaxL) return false;
  }
  return true;
}

// the quad split solve takes derivative lines long enough for its four
// segments in every block (FP64 or FP32 decay lengths)
bool quad_ok(const canard_ctx* c, int dir, int kind) {
  if (c->blocks.empty()) return false;
  for (const auto& b : c->blocks) {
    const int L = b.g.ijk[0][dir] + 1;
    const bool q64 = kind == LK_F64_QUAD;
    const int kf = q64 ? b.kf64[0][dir] : b.kf32[0][dir], ke = q64 ? b.ke64[0][dir] : b.ke32[0][dir];
    int q1, q2, q3;
    if (!quad_rows(L, kf, ke, q1, q2, q3)) return false;
  }
  return true;
}

// the two-ended solve has its tables for direction dir in every block (lines
// of at least kTwistMinL points; FP32 tables in mixed-precision contexts)
bool twist_ok(const canard_ctx* c, int dir, int kind) {
  if (c->blocks.empty()) return false;
  for (const auto& b : c->blocks) {
    for (int nt = 0; nt < 2; ++nt) {
      if (!b.ht[nt][dir]) return false;
      if (kind != LK_F64_TWIST && !b.lu32t[nt][dir]) return false;
    }
    // the whole tile of 32 lines (and the staged factors) in one CTA's shared memory
    LineTask t{};
    t.L = b.g.ijk[0][dir] + 1;
    chunking_dir(dir, t.L, t.nbox, t.by);
    if (line_smem(dir, t, kind) > (size_t)kLineSmemMax) return false;
  }
  return true;
}

// Defaults without autotuning: the two-ended solve where the lines admit it
// (fast mode: the fastest FP64 filter and derivative at 257 points; mixed
// precision: the fastest filter), else the split solve
int default_kind(const canard_ctx* c, int grp, int dir) {
  if (c->fast()) return twist_ok(c, dir, LK_F64_TWIST) ? LK_F64_TWIST : LK_F64_SPLIT;
  if (!c->f32()) return LK_F64;
  if (grp == 0) return twist_ok(c, dir, LK_F64_TILE_F32_TWIST) ? LK_F64_TILE_F32_TWIST : LK_F64_TILE_F32_SOLVE;
  return LK_F32;
}

int group_kind(const canard_ctx* c, int grp, int dir) {
  const int k = c->tune[grp][dir].kind;
  return k >= 0 ? k : default_kind(c, grp, dir);
}

void free_line_table(Table<LineTask>& T) {
  cudaFree(T.tasks);
  cudaFree(T.first);
  cudaFree(T.maps);
  T = Table<LineTask>{};
}

// the filter tasks of the five fields along one direction (FP32-mixed step)
std::vector<LineTask> filter_tasks5(canard_ctx* c, int dir, int kind, int nc, bool scratch = false) {
  std::vector<LineTask> v;
  for (int m = 1; m <= 5; ++m) {
    auto w = group_tasks(c, 0, dir, m, kind, nc, scratch);
    v.insert(v.end(), w.begin(), w.end());
  }
  return v;
}

void build_line_tables(canard_ctx* c) {
  for (int inn = 1; inn <= 3; ++inn) {
    const int dir = kNnf[inn - 1] - 1, k = group_kind(c, 0, dir);
    if (c->filter5())
      c->filt5[inn - 1] = make_line_table(c, filter_tasks5(c, dir, k, c->tune[0][dir].nc), dir, false, k);
    else
      for (int m = 1; m <= 5; ++m)
        c->filt[m - 1][inn - 1] =
            make_line_table(c, group_tasks(c, 0, dir, m, k, c->tune[0][dir].nc), dir, false, k);
  }
  for (int dir = 0; dir < 3; ++dir) {
    int k = group_kind(c, 1, dir);
    c->visc[dir] = make_line_table(c, group_tasks(c, 1, dir, 0, k, c->tune[1][dir].nc), dir, false, k);
    k = group_kind(c, 2, dir);
    c->flux[dir] = make_line_table(c, group_tasks(c, 2, dir, 0, k, c->tune[2][dir].nc), dir, false, k);
  }
}

// the step tables with the current choices; the step graphs used the old ones
void rebuild_line_tables(canard_ctx* c) {
  for (int m = 0; m < 5; ++m)
    for (int i = 0; i < 3; ++i) free_line_table(c->filt[m][i]);
  for (int d = 0; d < 3; ++d) {
    free_line_table(c->filt5[d]);
    free_line_table(c->visc[d]);
    free_line_table(c->flux[d]);
  }
  for (auto& g : c->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  build_line_tables(c);
  CK(cudaStreamSynchronize(c->st));
}

void build_tables(canard_ctx* c) {
  const bool f32 = c->f32();
  auto wf = [&](int b, int f64_field, int f32_field) -> void* {
    return f32 ? static_cast<void*>(gptr(c->blocks[b], f32_field)) : static_cast<void*>(fptr(c->blocks[b], f64_field));
  };
  build_line_tables(c);
  for (int inn = 1; inn <= 3; ++inn) {
    const int dir = kNnf[inn - 1] - 1;
    if (c->filter5()) {
      // the faces of this direction only, no send chain
      std::vector<FaceTask> all;
      for (int m = 1; m <= 5; ++m)
        for (FaceTask t : face_tasks(c, 1, 0, m, dir, [&](int b, int) { return fptr(c->blocks[b], F_QA + m - 1); }))
          if (t.nn == dir + 1) {
            t.chain = nullptr;
            all.push_back(t);
          }
      c->mp_filt5[inn - 1] = make_face_table(c, all, false);
    } else {
      for (int m = 1; m <= 5; ++m)
        c->mp_filt[m - 1][inn - 1] = make_face_table(
            c, face_tasks(c, 1, 0, m, dir, [&](int b, int) { return fptr(c->blocks[b], F_QA + m - 1); }), false);
    }
  }
  {
    std::vector<FaceTask> all;
    for (int m = 2; m <= 5; ++m) {
      auto v = face_tasks(c, 0, 0, m, -1, [&](int b, int) { return wf(b, F_DE + m - 1, G_DE + m - 1); }, -1, f32,
                          true);
      all.insert(all.end(), v.begin(), v.end());
    }
    c->mp_visc = make_face_table(c, all, false, f32 ? 1 : 0);
  }
  {
    std::vector<FaceTask> all;
    for (int m = 1; m <= 5; ++m) {
      auto v = face_tasks(
          c, 0, 0, m, -1, [&](int b, int d) { return wf(b, F_SCR + 3 * (m - 1) + d, G_SCR + 3 * (m - 1) + d); }, -1,
          f32, true);
      all.insert(all.end(), v.begin(), v.end());
    }
    c->mp_flux = make_face_table(c, all, false, f32 ? 1 : 0);
  }
}

void build_gcbc_sponge_avg(canard_ctx* c) {
  const int nb = nblk(c);
  // GCBC tables need yaco (reference layout) on the host
  std::vector<GcbcTask> setup_tasks;
  std::vector<GcbcTask> upd[3][2];
  std::vector<void*> fsrc;
  std::vector<void*> fdst;
  std::vector<int> fcnt;
  std::vector<SpongeTask> sp_tasks;
  for (int b = 0; b < nb; ++b) {
    BlockState& B = c->blocks[b];
    const BlockGeom& g = B.g;
    const CaseState& cs = c->cases[g.case_id];
    const size_t Lr = (size_t)g.X * g.Y * g.Z;
    std::vector<double> ypad((size_t)g.npad), yref(Lr);
    CK(cudaMemcpyAsync(ypad.data(), fptr(B, F_YACO), g.npad * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    for (int z = 0; z < g.Z; ++z)
      for (int y = 0; y < g.Y; ++y)
        for (int x = 0; x < g.X; ++x) yref[g.ref_index(x, y, z)] = ypad[g.dev(x, y, z)];
    std::vector<int64_t> pts;
    std::vector<double> w;
    gcbc_tables(g, yref.data(), B.gc_faces, pts, w);
    if (!pts.empty()) {
      std::vector<long long> p2(pts.begin(), pts.end());
      B.gc_pts = dupload(p2, c->st);
      B.gc_w = dupload(w, c->st);
    }
    for (const GcbcFace& f : B.gc_faces) {
      const int d = f.nn - 1;
      GcbcTask t{};
      t.b = b; t.nn = f.nn; t.side = f.side; t.bc = f.bc;
      t.cm = B.cm[d] + (size_t)3 * f.side * g.nbs[d];
      const size_t off = (size_t)5 * f.side * g.nbs[d];
      if (c->f32()) {
        t.drva = B.drva32[d] + off;
        t.drvb = (f.bc == BC_CURV) ? B.drvb32[d] + off : nullptr;
      } else {
        t.drva = B.drva[d] + off;
        t.drvb = (f.bc == BC_CURV) ? B.drvb[d] + off : nullptr;
      }
      t.pts = B.gc_pts + f.first;
      t.w = B.gc_w + f.first;
      t.nbs = g.nbs[d];
      t.nj = g.ijk[1][d] + 1;
      t.X = g.X; t.Y = g.Y; t.Z = g.Z; t.Xp = g.Xp; t.N = g.ijk[0][d];
      setup_tasks.push_back(t);
      upd[d][f.side].push_back(t);
    }
    // sponge
    if (cs.d.szco != 0.0) {
      std::vector<int64_t> sp;
      std::vector<double> a, bb;
      sponge_list(g, cs.d, B.xyz_host.data(), yref.data(), sp, a, bb);
      if (!sp.empty()) {
        std::vector<long long> s2(sp.begin(), sp.end());
        B.sp_pts = dupload(s2, c->st);
        B.sp_a = dupload(a, c->st);
        B.sp_b = dupload(bb, c->st);
        B.sp_n = (int)sp.size();
        SpongeTask st{b, B.sp_pts, B.sp_a, B.sp_b, B.sp_n, 0};
        sp_tasks.push_back(st);
      }
    }
  }
  for (const FaceLink& L : c->links) {  // gcbc_comm: BC_INTER_CURV faces only
    const BlockState& R = c->blocks[L.dst_b];
    const BlockState& S = c->blocks[L.src_b];
    const int d = L.nn;
    if (R.g.nbc[d][L.dst_side] != BC_CURV) continue;
    if (c->f32()) {
      fsrc.push_back(S.drva32[d] + (size_t)5 * L.src_side * S.g.nbs[d]);
      fdst.push_back(R.drvb32[d] + (size_t)5 * L.dst_side * R.g.nbs[d]);
    } else {
      fsrc.push_back(S.drva[d] + (size_t)5 * L.src_side * S.g.nbs[d]);
      fdst.push_back(R.drvb[d] + (size_t)5 * L.dst_side * R.g.nbs[d]);
    }
    fcnt.push_back(5 * R.g.nbs[d]);
  }
  c->gc_setup = make_lines_table(c, setup_tasks, false, &GcbcTask::nbs, &GcbcTask::line0);
  for (int d = 0; d < 3; ++d)
    for (int s = 0; s < 2; ++s)
      c->gc_upd[d][s] = make_lines_table(c, upd[d][s], false, &GcbcTask::nbs, &GcbcTask::line0);
  c->fc_n = (int)fsrc.size();
  if (c->fc_n) {
    c->fc_src = dupload(fsrc, c->st);
    c->fc_dst = dupload(fdst, c->st);
    c->fc_cnt = dupload(fcnt, c->st);
    c->fc_max = *std::max_element(fcnt.begin(), fcnt.end());
  }
  c->sponge = make_lines_table(c, sp_tasks, false, &SpongeTask::count, &SpongeTask::first);
  // junction averaging plans (per case: blocks of one case only see each other)
  AvgPlan P, Lp, Sf;
  for (const CaseState& cs : c->cases) {
    std::vector<BlockGeom> gs;
    for (int b = cs.b0; b < cs.b0 + cs.nb; ++b) gs.push_back(c->blocks[b].g);
    std::vector<FaceLink> lk;
    std::string e = face_links(gs, lk);
    if (!e.empty()) throw ApiError(CANARD_ERR_UNSUPPORTED, e);
    AvgPlan p1, l1, s1;
    bool sub40 = false;
    for (const auto& g : gs)
      for (int d = 0; d < 3; ++d)
        for (int s = 0; s < 2; ++s) sub40 = sub40 || g.nbc[d][s] == BC_SUBDOM;
    if (sub40 && !cs.split)
      throw ApiError(CANARD_ERR_UNSUPPORTED, "faces with code 40 need the case's split (canard_set_subdomains)");
    e = cs.split ? junction_plans(gs, cs.dec, p1, l1) : junction_plans(gs, p1, l1);
    if (!e.empty()) throw ApiError(CANARD_ERR_UNSUPPORTED, e);
    e = surface_plan(gs, lk, s1);
    if (!e.empty()) throw ApiError(CANARD_ERR_UNSUPPORTED, e);
    auto append = [&](AvgPlan& dst, const AvgPlan& src) {
      const int off = (int)dst.src_b.size();
      for (AvgTarget t : src.targets) { t.b += cs.b0; t.first += off; dst.targets.push_back(t); }
      for (int b : src.src_b) dst.src_b.push_back(b + cs.b0);
      dst.src_l.insert(dst.src_l.end(), src.src_l.begin(), src.src_l.end());
    };
    append(P, p1); append(Lp, l1); append(Sf, s1);
  }
  auto upload_avg = [&](const AvgPlan& p, AvgDev& A) {
    A.ntg = (int)p.targets.size();
    A.nsrc = (int)p.src_b.size();
    if (A.ntg == 0) return;
    std::vector<int> tb, tf, tc;
    std::vector<long long> tl, sl(p.src_l.begin(), p.src_l.end());
    for (const auto& t : p.targets) { tb.push_back(t.b); tl.push_back(t.l); tf.push_back(t.first); tc.push_back(t.count); }
    A.tb = dupload(tb, c->st); A.tl = dupload(tl, c->st); A.tfirst = dupload(tf, c->st); A.tcount = dupload(tc, c->st);
    A.sb = dupload(p.src_b, c->st); A.sl = dupload(sl, c->st);
    A.snap = dalloc<double>((size_t)A.nsrc * 5, c->st);
  };
  upload_avg(P, c->avg_pt);
  upload_avg(Lp, c->avg_ln);
  upload_avg(Sf, c->avg_sf);
  // wall-face points with their resets in the reference's face order
  std::map<std::pair<int, long long>, int> wall;
  for (int b = 0; b < nb; ++b) {
    const BlockGeom& g = c->blocks[b].g;
    for (int nn = 1; nn <= 3; ++nn)
      for (int ip = 0; ip <= 1; ++ip) {
        const int np = g.nbc[nn - 1][ip];
        if (np != BC_WALLI && np != BC_WALLV) continue;
        const int pos = ip * g.ijk[0][nn - 1];
        for (int k = 0; k <= g.ijk[2][nn - 1]; ++k)
          for (int j = 0; j <= g.ijk[1][nn - 1]; ++j) {
            int x, y, z;
            g.line_xyz(nn, pos, j, k, x, y, z);
            int& kinds = wall[{b, (long long)g.dev(x, y, z)}];
            int s = 0;
            while ((kinds >> (2 * s)) & 3) ++s;
            kinds |= (np == BC_WALLI ? 1 : 2) << (2 * s);
          }
      }
  }
  c->wall_n = (int)wall.size();
  if (c->wall_n) {
    std::vector<int> wb, wk;
    std::vector<long long> wl;
    for (const auto& e : wall) { wb.push_back(e.first.first); wl.push_back(e.first.second); wk.push_back(e.second); }
    c->wall_tb = dupload(wb, c->st);
    c->wall_tl = dupload(wl, c->st);
    c->wall_tk = dupload(wk, c->st);
  }
  // every block-face point
  {
    std::vector<int> fb;
    std::vector<long long> fl;
    for (int b = 0; b < nb; ++b) {
      const BlockGeom& g = c->blocks[b].g;
      for (int z = 0; z < g.Z; ++z)
        for (int y = 0; y < g.Y; ++y)
          for (int x = 0; x < g.X; ++x)
            if (x == 0 || x == g.X - 1 || y == 0 || y == g.Y - 1 || z == 0 || z == g.Z - 1) {
              fb.push_back(b);
              fl.push_back((long long)g.dev(x, y, z));
            }
    }
    c->face_n = (int)fb.size();
    if (c->face_n) {
      c->face_tb = dupload(fb, c->st);
      c->face_tl = dupload(fl, c->st);
    }
  }
  // the primitives are recomputed at averaged and at reset wall points
  std::vector<std::pair<int, long long>> pts;
  for (const AvgPlan* p : {&P, &Lp, &Sf})
    for (const auto& t : p->targets) pts.emplace_back(t.b, (long long)t.l);
  for (const auto& e : wall) pts.push_back(e.first);
  std::sort(pts.begin(), pts.end());
  pts.erase(std::unique(pts.begin(), pts.end()), pts.end());
  c->prim_n = (int)pts.size();
  if (c->prim_n) {
    std::vector<int> pb;
    std::vector<long long> pl;
    for (const auto& q : pts) { pb.push_back(q.first); pl.push_back(q.second); }
    c->prim_tb = dupload(pb, c->st);
    c->prim_tl = dupload(pl, c->st);
  }
  c->fuse_sum = c->gc_setup.ntasks == 0 && c->sponge.total == 0;
}

// t_grid%grid_metrics on the device (src/mo_grid.f90:52-189)
void grid_metrics(canard_ctx* c) {
  const int nb = nblk(c);
  // coordinate derivatives: scr 3*(m-1) + dir
  for (int m = 1; m <= 3; ++m) {
    auto ft = face_tasks(c, 0, 1, m, -1, [&](int b, int) { return fptr(c->blocks[b], F_XYZ + m - 1); });
    launch_mpigo(c, make_face_table(c, ft, true));
    for (int dir = 2; dir >= 0; --dir) {
      std::vector<LineTask> v;
      for (int b = 0; b < nb; ++b) {
        LineTask t;
        fill_line_task(c, c->blocks[b], dir, 0, fptr(c->blocks[b], F_XYZ + m - 1),
                       fptr(c->blocks[b], F_SCR + 3 * (m - 1) + dir), m, true, t);
        v.push_back(t);
      }
      launch_line(c, make_line_table(c, v, dir, true), dir, 0);
    }
  }
  k_cofactors<<<ew_grid(c), 256, 0, c->st>>>(c->dbd);
  CK(cudaGetLastError());
  const int mets[3] = {F_XIM, F_ETM, F_ZEM};
  for (int m = 1; m <= 3; ++m)
    for (int w = 0; w < 3; ++w)
      for (int inn = 1; inn <= 3; ++inn) {
        const int dir = kNnf[inn - 1] - 1;
        auto col = [&](int b, int) { return fptr(c->blocks[b], mets[w] + m - 1); };
        launch_mpigo(c, make_face_table(c, face_tasks(c, 1, 0, m, dir, col), true));
        std::vector<LineTask> v;
        for (int b = 0; b < nb; ++b) {
          LineTask t;
          double* f = fptr(c->blocks[b], mets[w] + m - 1);
          fill_line_task(c, c->blocks[b], dir, 1, f, f, m, false, t);
          v.push_back(t);
        }
        launch_line(c, make_line_table(c, v, dir, true), dir, 1);
      }
  k_jacobian<<<ew_grid(c), 256, 0, c->st>>>(c->dbd);
  CK(cudaGetLastError());
  // face normals of all six faces
  std::vector<CmTask> cmt;
  std::vector<int> first;
  int tot = 0;
  for (int b = 0; b < nb; ++b)
    for (int d = 0; d < 3; ++d)
      for (int s = 0; s < 2; ++s) {
        const BlockState& B = c->blocks[b];
        CmTask t{b, d + 1, s, B.g.nbs[d], B.g.ijk[1][d] + 1, B.g.ijk[0][d], tot,
                 B.cm[d] + (size_t)3 * s * B.g.nbs[d]};
        first.push_back(tot);
        tot += t.nbs;
        cmt.push_back(t);
      }
  CmTask* dt = dupload(cmt, c->st);
  int* df = dupload(first, c->st);
  c->transient.push_back(dt);
  c->transient.push_back(df);
  k_face_normals<<<std::max(1, std::min((tot + 127) / 128, 1184)), 128, 0, c->st>>>(c->dbd, dt, df,
                                                                                     (int)cmt.size(), tot);
  CK(cudaGetLastError());
  if (c->f32()) {
    k_metrics_to_f32<<<ew_grid(c), 256, 0, c->st>>>(c->dbd);
    CK(cudaGetLastError());
  }
  sync_check(c);
  free_transient(c);
}

// copy between a host array in the reference layout (ncols x X*Y*Z) and a
// padded device field
// Copies between a host array in the reference layout (ncols x X*Y*Z) and a
// padded device field: one contiguous copy into the context's staging buffer
// and a repacking kernel (a strided 2-D copy of rows of a few KB reaches
// about half the link bandwidth).
void h2d_field(canard_ctx* c, const BlockState& B, double* dst, const double* src, int ncols) {
  const BlockGeom& g = B.g;
  const size_t n = (size_t)ncols * g.X * g.Y * g.Z;
  if (n > c->stage_n) {
    CK(cudaMemcpy2DAsync(dst, g.Xp * sizeof(double), src, g.X * sizeof(double), g.X * sizeof(double),
                         (size_t)g.Y * g.Z * ncols, cudaMemcpyHostToDevice, c->st));
    return;
  }
  CK(cudaMemcpyAsync(c->stage, src, n * sizeof(double), cudaMemcpyHostToDevice, c->st));
  const long long rows = (long long)g.Y * g.Z * ncols;
  k_rows_repack<<<(unsigned)std::min<long long>((rows * g.X + 255) / 256, 148 * 16), 256, 0, c->st>>>(
      c->stage, g.X, dst, g.Xp, g.X, rows);
  CK(cudaGetLastError());
}
void d2h_field(canard_ctx* c, const BlockState& B, double* dst, const double* src, int ncols) {
  const BlockGeom& g = B.g;
  const size_t n = (size_t)ncols * g.X * g.Y * g.Z;
  if (n > c->stage_n) {
    CK(cudaMemcpy2DAsync(dst, g.X * sizeof(double), src, g.Xp * sizeof(double), g.X * sizeof(double),
                         (size_t)g.Y * g.Z * ncols, cudaMemcpyDeviceToHost, c->st));
    return;
  }
  const long long rows = (long long)g.Y * g.Z * ncols;
  k_rows_repack<<<(unsigned)std::min<long long>((rows * g.X + 255) / 256, 148 * 16), 256, 0, c->st>>>(
      src, g.Xp, c->stage, g.X, g.X, rows);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(dst, c->stage, n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
}

int block_index(const canard_ctx* c, int icase, int iblock) {
  if (icase < 0 || icase >= (int)c->cases.size()) throw ApiError(CANARD_ERR_ARG, "case index out of range");
  const CaseState& cs = c->cases[icase];
  if (iblock < 0 || iblock >= cs.nb) throw ApiError(CANARD_ERR_ARG, "block index out of range");
  return cs.b0 + iblock;
}

template <class F>
int guarded(canard_ctx* c, F&& f) {
  if (!c) return CANARD_ERR_ARG;
  try {
    f();
    return CANARD_OK;
  } catch (const ApiError& e) {
    set_err(c, e.what());
    return e.code;
  } catch (const CudaError& e) {
    set_err(c, e.what());
    return CANARD_ERR_CUDA;
  } catch (const std::exception& e) {
    set_err(c, e.what());
    return CANARD_ERR_ARG;
  }
}

void destroy(canard_ctx* c) {
  for (auto& b : c->blocks) {
    cudaFree(b.arena);
    for (int nt = 0; nt < 2; ++nt)
      for (int d = 0; d < 3; ++d) { cudaFree(b.lu[nt][d]); cudaFree(b.recv[nt][d]); }
    for (int d = 0; d < 3; ++d) { cudaFree(b.chain[d]); cudaFree(b.drva[d]); cudaFree(b.drvb[d]); cudaFree(b.cm[d]); }
    cudaFree(b.arena32);
    for (int nt = 0; nt < 2; ++nt)
      for (int d = 0; d < 3; ++d) {
        cudaFree(b.lu32[nt][d]);
        cudaFree(b.lu64s[nt][d]);
        cudaFree(b.lu64t[nt][d]);
        cudaFree(b.lu32t[nt][d]);
      }
    for (int d = 0; d < 3; ++d) { cudaFree(b.recv32[d]); cudaFree(b.drva32[d]); cudaFree(b.drvb32[d]); }
    cudaFree(b.gc_pts); cudaFree(b.gc_w); cudaFree(b.sp_pts); cudaFree(b.sp_a); cudaFree(b.sp_b);
  }
  for (auto& cs : c->cases) cudaFree(cs.dsch);
  cudaFree(c->dbd); cudaFree(c->dcc); cudaFree(c->dsp); cudaFree(c->ddt); cudaFree(c->derr);
  cudaFree(c->dtime); cudaFree(c->dsn2); cudaFree(c->stage);
  for (auto g : c->graph) if (g) cudaGraphExecDestroy(g);
  for (auto& p : c->pending) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
  for (auto e : c->ev_pool) cudaEventDestroy(e);
  auto ft = [](auto& T) { cudaFree(T.tasks); cudaFree(T.first); };
  auto fl = [](Table<LineTask>& T) { cudaFree(T.maps); };
  for (int m = 0; m < 5; ++m) for (int i = 0; i < 3; ++i) fl(c->filt[m][i]);
  for (int d = 0; d < 3; ++d) { fl(c->filt5[d]); fl(c->visc[d]); fl(c->flux[d]); }
  for (int m = 0; m < 5; ++m) for (int i = 0; i < 3; ++i) { ft(c->filt[m][i]); ft(c->mp_filt[m][i]); }
  for (int d = 0; d < 3; ++d) { ft(c->filt5[d]); ft(c->mp_filt5[d]); ft(c->visc[d]); ft(c->flux[d]); }
  ft(c->mp_visc); ft(c->mp_flux); ft(c->gc_setup); ft(c->sponge);
  for (int d = 0; d < 3; ++d) for (int s = 0; s < 2; ++s) ft(c->gc_upd[d][s]);
  cudaFree(c->fc_src); cudaFree(c->fc_dst); cudaFree(c->fc_cnt);
  cudaFree(c->prim_tb); cudaFree(c->prim_tl);
  cudaFree(c->wall_tb); cudaFree(c->wall_tl); cudaFree(c->wall_tk);
  cudaFree(c->dtsum);
  cudaFree(c->face_tb); cudaFree(c->face_tl);
  for (auto& b : c->blocks) cudaFree(b.qb);
  for (AvgDev* A : {&c->avg_pt, &c->avg_ln, &c->avg_sf}) {
    cudaFree(A->tb); cudaFree(A->tl); cudaFree(A->tfirst); cudaFree(A->tcount); cudaFree(A->sb); cudaFree(A->sl);
    cudaFree(A->snap);
  }
  free_transient(c);
  cudaFree(c->hs_stage);
  if (c->s_in) cudaStreamDestroy(c->s_in);
  if (c->s_out) cudaStreamDestroy(c->s_out);
  if (c->own) cudaStreamDestroy(c->own);
}

void create(canard_ctx* c, const canard_case_desc* cases, int ncases, const canard_block_desc* blocks) {
  if (!cases || !blocks || ncases <= 0) throw ApiError(CANARD_ERR_ARG, "null or empty case list");
  int b0 = 0;
  for (int i = 0; i < ncases; ++i) {
    CaseState cs;
    cs.d = cases[i];
    if (cs.d.nblocks <= 0) throw ApiError(CANARD_ERR_ARG, "case without blocks");
    if (!(cs.d.fltrbc > 0.0)) throw ApiError(CANARD_ERR_ARG, "fltrbc must be positive");
    cs.sch.build(cs.d.fltk, cs.d.fltrbc);
    // src/mo_physics.f90:101-111
    const double am = std::sqrt((cs.d.amach1 * cs.d.amach1 + cs.d.amach2 * cs.d.amach2) + cs.d.amach3 * cs.d.amach3);
    cs.reoo = cs.d.reoo;
    if (am > 1.0e-8) cs.reoo = cs.reoo / am;
    cs.srefoo = 111 / cs.d.tempoo;
    cs.srefp1dre = (cs.srefoo + 1.0) / cs.reoo;
    cs.uoo[0] = cs.d.amach1; cs.uoo[1] = cs.d.amach2; cs.uoo[2] = cs.d.amach3;
    cs.b0 = b0;
    cs.nb = cs.d.nblocks;
    for (int k = 0; k < cs.nb; ++k) {
      BlockState B;
      const canard_block_desc& bd = blocks[b0 + k];
      if (bd.lxi < 12 || bd.let < 12 || bd.lze < 12)
        throw ApiError(CANARD_ERR_ARG, "every direction needs at least 13 points (interface closures read 13)");
      for (int d = 0; d < 3; ++d)
        for (int s = 0; s < 2; ++s) {
          const int np = bd.nbc[d][s];
          if (!(np == BC_SUBDOM || np == BC_NR || np == BC_WALLI || np == BC_WALLV || np == BC_CURV || np == BC_STRAIGHT ||
                np == BC_PERIODIC))
            throw ApiError(CANARD_ERR_ARG, "unknown boundary code " + std::to_string(np));
          if (np != BC_NR && np != BC_WALLI && np != BC_WALLV && (bd.mbcd[d][s] < 0 || bd.mbcd[d][s] >= cs.nb))
            throw ApiError(CANARD_ERR_ARG, "interface face without a neighbour block in the case");
        }
      make_geom(bd, i, k, B.g);
      check_line_lengths(B.g, c->precision);
      // remap neighbours to global indices for the links
      c->blocks.push_back(B);
    }
    b0 += cs.nb;
    c->cases.push_back(cs);
  }
  // face links per case
  for (const CaseState& cs : c->cases) {
    std::vector<BlockGeom> gs;
    for (int b = cs.b0; b < cs.b0 + cs.nb; ++b) gs.push_back(c->blocks[b].g);
    std::vector<FaceLink> lk;
    std::string e = face_links(gs, lk);
    if (!e.empty()) throw ApiError(CANARD_ERR_UNSUPPORTED, e);
    for (FaceLink L : lk) { L.dst_b += cs.b0; L.src_b += cs.b0; c->links.push_back(L); }
  }
  // device memory (everything above is host-side argument checking)
  CK(cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking));
  c->st = c->own;
  std::vector<BlockDev> bdv;
  for (auto& B : c->blocks) {
    const BlockGeom& g = B.g;
    B.arena = dalloc<double>((size_t)F_COUNT * g.npad, c->st);
    BlockDev& d = B.dev;
    d.X = g.X; d.Y = g.Y; d.Z = g.Z; d.Xp = g.Xp; d.npad = g.npad; d.case_id = g.case_id;
    d.qa = fptr(B, F_QA); d.qo = fptr(B, F_QO); d.de = fptr(B, F_DE); d.p = fptr(B, F_P); d.mu = fptr(B, F_MU);
    d.xim = fptr(B, F_XIM); d.etm = fptr(B, F_ETM); d.zem = fptr(B, F_ZEM); d.yaco = fptr(B, F_YACO);
    d.tau = fptr(B, F_TAU); d.scr = fptr(B, F_SCR); d.xyz = fptr(B, F_XYZ);
    d.f = Work<float>{};
    if (c->f32()) {
      B.arena32 = dalloc<float>((size_t)G_COUNT * g.npad, c->st);
      d.f.de = gptr(B, G_DE); d.f.p = gptr(B, G_P); d.f.mu = gptr(B, G_MU); d.f.tau = gptr(B, G_TAU);
      d.f.scr = gptr(B, G_SCR); d.f.xim = gptr(B, G_XIM); d.f.etm = gptr(B, G_ETM); d.f.zem = gptr(B, G_ZEM);
      d.f.yaco = gptr(B, G_YACO);
    }
    const Scheme& sch = c->cases[g.case_id].sch;
    for (int dir = 0; dir < 3; ++dir) {
      const int L = g.ijk[0][dir] + 1, nbs = g.nbs[dir];
      const int n0 = bc_interface(g.nbc[dir][0]) ? 1 : 0, n1 = bc_interface(g.nbc[dir][1]) ? 1 : 0;
      for (int nt = 0; nt < 2; ++nt) {
        std::vector<double> lu((size_t)5 * L);
        sch.lu(L, n0, n1, nt, lu.data());
        B.lu[nt][dir] = dupload(lu, c->st);
        if (c->f32()) {  // the FP64 factorisation, rounded for the FP32 eliminations
          std::vector<float> lu32(lu.begin(), lu.end()), hom;
          // rows [c0, L-4] whose rounded factors are bit-identical to row L-4
          const int e = L - 4;
          int c0f = e;
          auto same32 = [&](int r) {
            for (int k = 0; k < 5; ++k)
              if (std::memcmp(&lu32[(size_t)k * L + r], &lu32[(size_t)k * L + e], sizeof(float)) != 0) return false;
            return true;
          };
          while (c0f - 1 >= 3 && same32(c0f - 1)) --c0f;
          for (int k = 0; k < 5; ++k) B.luc32[nt][dir][k] = lu32[(size_t)k * L + e];
          B.luc032[nt][dir] = c0f;
          const int h = split_row(L, dir, nt, c0f);
          split_tables(lu, L, h, 1e-12, hom, B.kg32[nt][dir], B.ke32[nt][dir], B.kf32[nt][dir]);
          B.h32[nt][dir] = h;
          lu32.insert(lu32.end(), hom.begin(), hom.end());
          B.lu32[nt][dir] = dupload(lu32, c->st);
        }
        // rows [i0, L-4] whose five factors are bit-identical to row L-4
        const int e = L - 4;
        int i0 = e + 1;
        if (e >= 0) {
          i0 = e;
          auto same = [&](int r) {
            for (int k = 0; k < 5; ++k)
              if (std::memcmp(&lu[(size_t)k * L + r], &lu[(size_t)k * L + e], sizeof(double)) != 0) return false;
            return true;
          };
          while (i0 - 1 >= 3 && same(i0 - 1)) --i0;
          for (int k = 0; k < 5; ++k) B.luc[nt][dir][k] = lu[(size_t)k * L + e];
        }
        B.luc0[nt][dir] = i0;
        {  // the split FP64 solve: factors followed by FP64 correction tables
          std::vector<double> lus(lu), hom;
          const int h = split_row(L, dir, nt, i0, (int)sizeof(double));
          split_tables(lu, L, h, 1e-18, hom, B.kg64[nt][dir], B.ke64[nt][dir], B.kf64[nt][dir]);
          B.h64[nt][dir] = h;
          lus.insert(lus.end(), hom.begin(), hom.end());
          B.lu64s[nt][dir] = dupload(lus, c->st);
        }
        if (L >= kTwistMinL) {  // the two-ended solve's tables
          const int h = twist_row(L);
          std::vector<double> t64;
          const int r64 = twist_tables(sch, lu, L, n0, n1, nt, h, t64);
          int r32 = -1;
          std::vector<float> t32;
          if (r64 >= 0 && c->f32()) r32 = twist_tables(sch, lu, L, n0, n1, nt, h, t32);
          if (r64 >= 0 && (!c->f32() || r32 >= 0)) {
            B.ht[nt][dir] = h;
            B.c0r64[nt][dir] = r64;
            B.lu64t[nt][dir] = dupload(t64, c->st);
            if (c->f32()) {
              B.c0r32[nt][dir] = r32;
              B.lu32t[nt][dir] = dupload(t32, c->st);
            }
          }
        }
        B.recv[nt][dir] = dalloc<double>((size_t)5 * 2 * (nt == 0 ? 2 : 3) * nbs, c->st);
      }
      B.chain[dir] = dalloc<double>((size_t)2 * nbs, c->st);
      if (c->f32()) {
        B.recv32[dir] = dalloc<float>((size_t)5 * 2 * 2 * nbs, c->st);
        B.drva32[dir] = dalloc<float>((size_t)10 * nbs, c->st);
        B.drvb32[dir] = dalloc<float>((size_t)10 * nbs, c->st);
      }
      B.drva[dir] = dalloc<double>((size_t)10 * nbs, c->st);
      B.drvb[dir] = dalloc<double>((size_t)10 * nbs, c->st);
      B.cm[dir] = dalloc<double>((size_t)6 * nbs, c->st);
    }
    bdv.push_back(d);
  }
  c->dbd = dupload(bdv, c->st);
  std::vector<CaseConst> ccv;
  for (auto& cs : c->cases) {
    CaseConst k{};
    k.srefoo = cs.srefoo; k.srefp1dre = cs.srefp1dre; k.viscous = cs.d.viscous; k.nsmf = cs.d.nsmf;
    k.cfl = cs.d.cfl; k.timf = cs.d.timf;
    for (int d = 0; d < 3; ++d) k.uoo[d] = cs.uoo[d];
    ccv.push_back(k);
    DevScheme ds{};
    std::memcpy(ds.pbci, cs.sch.pbci, sizeof(ds.pbci));
    std::memcpy(ds.pbco, cs.sch.pbco, sizeof(ds.pbco));
    std::memcpy(ds.pbcot, cs.sch.pbcot, sizeof(ds.pbcot));
    ds.fa = cs.sch.fa; ds.fb = cs.sch.fb; ds.fc = cs.sch.fc;
    std::memcpy(ds.fbc, cs.sch.fbc, sizeof(ds.fbc));
    ds.alphf = cs.sch.alphf; ds.betf = cs.sch.betf;
    std::memcpy(ds.albef, cs.sch.albef, sizeof(ds.albef));
    cs.dsch = dupload(std::vector<DevScheme>{ds}, c->st);
  }
  c->dcc = dupload(ccv, c->st);
  c->dsp = dalloc<StageParams>(5 * c->cases.size(), c->st);
  c->dtime = dalloc<TimeDev>(c->cases.size(), c->st);  // n = ndt = 0, dt = dts = dte = timo = 0
  {
    // ramp factors with the host's libm, as the CPU code evaluates them
    const double pi = std::acos(-1.0);
    std::vector<double> sn2(kRampTable);
    for (int k = 0; k < kRampTable; ++k) {
      const double sn = std::sin((0.05 * pi) * k);
      sn2[k] = sn * sn;
    }
    c->dsn2 = dupload(sn2, c->st);
  }
  c->ddt = dalloc<unsigned long long>(2 * c->cases.size(), c->st);
  c->derr = dalloc<int>(1, c->st);
  // staging buffer of the host copies: the largest block's 5 state fields
  for (auto& B : c->blocks) c->stage_n = std::max(c->stage_n, (size_t)5 * B.g.X * B.g.Y * B.g.Z);
  c->stage = dalloc<double>(c->stage_n, c->st);
  set_line_smem_limits();
  build_tables(c);
  CK(cudaStreamSynchronize(c->st));
}

}  // namespace

// ==================================================================================
extern "C" {

int canard_version(void) { return 1; }

int canard_coeffs(double fltk, double fltrbc, double* out150) {
  if (!out150 || !(fltrbc > 0.0)) return CANARD_ERR_ARG;
  Scheme s;
  s.build(fltk, fltrbc);
  s.pack150(out150);
  return CANARD_OK;
}

int canard_penta(double fltk, double fltrbc, int32_t n, int32_t ns, int32_t ne, int32_t nt, double* xu,
                 double* xl) {
  if (!xu || !xl || n < 8 || ns < 0 || ns > 1 || ne < 0 || ne > 1 || nt < 0 || nt > 1) return CANARD_ERR_ARG;
  Scheme s;
  s.build(fltk, fltrbc);
  std::vector<double> o((size_t)5 * n);
  s.lu(n, ns, ne, nt, o.data());
  // xu (n,3) = u1,u2,u3 ; xl (n,2) = l1,l2 (column-major)
  for (int i = 0; i < n; ++i) {
    xl[i] = o[i]; xl[n + i] = o[n + i];
    xu[i] = o[2 * n + i]; xu[n + i] = o[3 * n + i]; xu[2 * n + i] = o[4 * n + i];
  }
  return CANARD_OK;
}

int canard_ctx_create(const canard_case_desc* cases, int32_t ncases, const canard_block_desc* blocks,
                      int32_t precision, canard_ctx** out) {
  if (!out) return CANARD_ERR_ARG;
  *out = nullptr;
  if (precision != CANARD_FP64 && precision != CANARD_FP32_MIXED && precision != CANARD_FP64_FAST)
    return CANARD_ERR_UNSUPPORTED;
  canard_ctx* c = new canard_ctx();
  c->precision = precision;
  int rc = guarded(c, [&] { create(c, cases, ncases, blocks); });
  if (rc != CANARD_OK) {
    std::fprintf(stderr, "canard_ctx_create: %s\n", c->err.c_str());
    destroy(c);
    delete c;
    return rc;
  }
  *out = c;
  return CANARD_OK;
}

void canard_ctx_destroy(canard_ctx* c) {
  if (!c) return;
  cudaStreamSynchronize(c->st);
  destroy(c);
  delete c;
}

const char* canard_last_error(const canard_ctx* c) { return c ? c->err.c_str() : "null context"; }

int canard_set_stream(canard_ctx* c, void* stream) {
  return guarded(c, [&] {
    CK(cudaStreamSynchronize(c->st));
    c->st = stream ? static_cast<cudaStream_t>(stream) : c->own;
  });
}

int canard_upload_grid(canard_ctx* c, int32_t icase, int32_t iblock, const double* xyz) {
  return guarded(c, [&] {
    if (!xyz) throw ApiError(CANARD_ERR_ARG, "null grid");
    BlockState& B = c->blocks[block_index(c, icase, iblock)];
    const size_t L = (size_t)B.g.X * B.g.Y * B.g.Z;
    B.xyz_host.assign(xyz, xyz + 3 * L);
    h2d_field(c, B, fptr(B, F_XYZ), xyz, 3);
    CK(cudaStreamSynchronize(c->st));
  });
}

int canard_set_subdomains(canard_ctx* c, int32_t icase, int32_t nblocks, const int32_t* nbpc, const int32_t* mbcd,
                          const int32_t* sub) {
  return guarded(c, [&] {
    if (c->setup_done) throw ApiError(CANARD_ERR_STATE, "canard_set_subdomains after canard_setup");
    if (icase < 0 || icase >= (int)c->cases.size() || nblocks < 1 || !nbpc || !mbcd || !sub)
      throw ApiError(CANARD_ERR_ARG, "bad sub-domain argument");
    CaseState& cs = c->cases[icase];
    Decomp d;
    int mo = 0;
    for (int m = 0; m < nblocks; ++m) {
      Decomp::Parent p;
      for (int a = 0; a < 3; ++a) {
        p.nbpc[a] = nbpc[3 * m + a];
        for (int s = 0; s < 2; ++s) p.nbr[a][s] = mbcd[6 * m + 2 * a + s];
      }
      p.mo = mo;
      mo += p.nbpc[0] * p.nbpc[1] * p.nbpc[2];
      d.parents.push_back(p);
    }
    for (int r = 0; r < cs.nb; ++r) {
      d.mb.push_back(sub[4 * r]);
      d.pos.push_back({sub[4 * r + 1], sub[4 * r + 2], sub[4 * r + 3]});
    }
    std::vector<BlockGeom> gs;
    for (int b = cs.b0; b < cs.b0 + cs.nb; ++b) gs.push_back(c->blocks[b].g);
    const std::string e = check_decomp(gs, d);
    if (!e.empty()) throw ApiError(CANARD_ERR_ARG, e);
    cs.dec = d;
    cs.split = true;
  });
}

int canard_setup(canard_ctx* c) {
  return guarded(c, [&] {
    for (auto& B : c->blocks)
      if (B.xyz_host.empty()) throw ApiError(CANARD_ERR_STATE, "canard_setup before every grid is uploaded");
    grid_metrics(c);
    build_gcbc_sponge_avg(c);
    CK(cudaStreamSynchronize(c->st));
    c->setup_done = true;
  });
}

int canard_set_state(canard_ctx* c, int32_t icase, int32_t iblock, const double* qa) {
  return guarded(c, [&] {
    if (!qa) throw ApiError(CANARD_ERR_ARG, "null state");
    BlockState& B = c->blocks[block_index(c, icase, iblock)];
    h2d_field(c, B, fptr(B, F_QA), qa, 5);
    CK(cudaStreamSynchronize(c->st));
  });
}

int canard_get_state(canard_ctx* c, int32_t icase, int32_t iblock, double* qa) {
  return guarded(c, [&] {
    if (!qa) throw ApiError(CANARD_ERR_ARG, "null state");
    BlockState& B = c->blocks[block_index(c, icase, iblock)];
    d2h_field(c, B, qa, fptr(B, F_QA), 5);
    CK(cudaStreamSynchronize(c->st));
  });
}

// Device location of a field. In a mixed-precision context the work fields
// (de, p, ss1, tau, drva) are FP32 and f32ptr is set instead of dptr.
static void field_info(const canard_ctx* c, const BlockState& B, int field, const double*& dptr, int& ncols,
                       bool& face, size_t& count, const float*& f32ptr) {
  face = false;
  f32ptr = nullptr;
  const bool w32 = c->f32();
  switch (field) {
    case CANARD_F_QA: dptr = fptr(B, F_QA); ncols = 5; break;
    case CANARD_F_QO: dptr = fptr(B, F_QO); ncols = 5; break;
    case CANARD_F_DE: dptr = fptr(B, F_DE); ncols = 5; if (w32) f32ptr = gptr(B, G_DE); break;
    case CANARD_F_P: dptr = fptr(B, F_P); ncols = 1; if (w32) f32ptr = gptr(B, G_P); break;
    case CANARD_F_SS1: dptr = fptr(B, F_MU); ncols = 1; if (w32) f32ptr = gptr(B, G_MU); break;
    case CANARD_F_XIM: dptr = fptr(B, F_XIM); ncols = 3; break;
    case CANARD_F_ETM: dptr = fptr(B, F_ETM); ncols = 3; break;
    case CANARD_F_ZEM: dptr = fptr(B, F_ZEM); ncols = 3; break;
    case CANARD_F_YACO: dptr = fptr(B, F_YACO); ncols = 1; break;
    case CANARD_F_TAU: dptr = fptr(B, F_TAU); ncols = 9; if (w32) f32ptr = gptr(B, G_TAU); break;
    case CANARD_F_DRVA1: case CANARD_F_DRVA2: case CANARD_F_DRVA3: {
      const int d = field - CANARD_F_DRVA1;
      dptr = B.drva[d]; face = true; count = (size_t)10 * B.g.nbs[d]; ncols = 0;
      if (w32) f32ptr = B.drva32[d];
      return;
    }
    case CANARD_F_CM1: case CANARD_F_CM2: case CANARD_F_CM3: {
      const int d = field - CANARD_F_CM1;
      dptr = B.cm[d]; face = true; count = (size_t)6 * B.g.nbs[d]; ncols = 0;
      return;
    }
    default: throw ApiError(CANARD_ERR_ARG, "unknown field id");
  }
  count = (size_t)ncols * B.g.X * B.g.Y * B.g.Z;
}

// element conversions between an FP32 field and its FP64 image (unit calls and
// field access of mixed-precision contexts; not on the step path)
void to_f64(canard_ctx* c, const float* a, double* b, size_t n) {
  k_f32_to_f64<<<std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 1184)), 256, 0, c->st>>>(a, b, (long long)n);
  CK(cudaGetLastError());
}
void to_f32(canard_ctx* c, const double* a, float* b, size_t n) {
  k_f64_to_f32<<<std::max<size_t>(1, std::min<size_t>((n + 255) / 256, 1184)), 256, 0, c->st>>>(a, b, (long long)n);
  CK(cudaGetLastError());
}

int canard_get_field(canard_ctx* c, int32_t icase, int32_t iblock, int32_t field, double* out, int64_t count) {
  return guarded(c, [&] {
    BlockState& B = c->blocks[block_index(c, icase, iblock)];
    const double* dp; int nc; bool face; size_t n; const float* fp;
    field_info(c, B, field, dp, nc, face, n, fp);
    if (!out || count != (int64_t)n) throw ApiError(CANARD_ERR_ARG, "count does not match the field size");
    if (fp) {  // FP32 work field: widen into the FP64 slot of the same field, then copy
      to_f64(c, fp, const_cast<double*>(dp), face ? n : (size_t)nc * B.g.npad);
    }
    if (face) CK(cudaMemcpyAsync(out, dp, n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    else d2h_field(c, B, out, dp, nc);
    CK(cudaStreamSynchronize(c->st));
  });
}

int canard_set_field(canard_ctx* c, int32_t icase, int32_t iblock, int32_t field, const double* in, int64_t count) {
  return guarded(c, [&] {
    BlockState& B = c->blocks[block_index(c, icase, iblock)];
    const double* dp; int nc; bool face; size_t n; const float* fp;
    field_info(c, B, field, dp, nc, face, n, fp);
    if (!in || count != (int64_t)n) throw ApiError(CANARD_ERR_ARG, "count does not match the field size");
    if (face) CK(cudaMemcpyAsync(const_cast<double*>(dp), in, n * sizeof(double), cudaMemcpyHostToDevice, c->st));
    else h2d_field(c, B, const_cast<double*>(dp), in, nc);
    if (fp) to_f32(c, dp, const_cast<float*>(fp), face ? n : (size_t)nc * B.g.npad);
    CK(cudaStreamSynchronize(c->st));
  });
}

int canard_step(canard_ctx* c, int32_t nsteps) {
  return guarded(c, [&] {
    if (!c->setup_done) throw ApiError(CANARD_ERR_STATE, "canard_step before canard_setup");
    if (nsteps < 0) throw ApiError(CANARD_ERR_ARG, "negative step count");
    for (int i = 0; i < nsteps; ++i) one_step(c);
    sync_check(c);
  });
}

// Steps through host memory, pipelined: each listed block's state is cut into
// chunks of rows of the reference layout; a chunk of step n's result goes out
// on s_out as soon as it is packed, and the same chunk of step n+1's input
// (the caller's array, which the call owns meanwhile) goes back in on s_in
// right after, so the two directions of the host link overlap. Same results
// as nsteps x (set_state, step, get_state).
int canard_step_host(canard_ctx* c, int32_t nsteps, int32_t nblocks, const int32_t* icase, const int32_t* iblock,
                     double* const* host) {
  return guarded(c, [&] {
    if (!c->setup_done) throw ApiError(CANARD_ERR_STATE, "canard_step_host before canard_setup");
    if (nsteps < 0 || nblocks < 1 || !icase || !iblock || !host) throw ApiError(CANARD_ERR_ARG, "bad argument");
    std::vector<int> bs((size_t)nblocks);
    std::vector<size_t> off((size_t)nblocks);
    size_t tot = 0;
    for (int k = 0; k < nblocks; ++k) {
      if (!host[k]) throw ApiError(CANARD_ERR_ARG, "null host state");
      bs[k] = block_index(c, icase[k], iblock[k]);
      for (int q = 0; q < k; ++q)
        if (bs[q] == bs[k]) throw ApiError(CANARD_ERR_ARG, "a block is listed twice");
      off[k] = tot;
      const BlockGeom& g = c->blocks[bs[k]].g;
      tot += (size_t)5 * g.X * g.Y * g.Z;
    }
    if (nsteps == 0) return;
    if (c->hs_n < tot) {
      CK(cudaStreamSynchronize(c->st));
      cudaFree(c->hs_stage);
      c->hs_stage = nullptr;
      c->hs_n = 0;
      c->hs_stage = dalloc<double>(tot, c->st);
      c->hs_n = tot;
    }
    if (!c->s_in) CK(cudaStreamCreateWithFlags(&c->s_in, cudaStreamNonBlocking));
    if (!c->s_out) CK(cudaStreamCreateWithFlags(&c->s_out, cudaStreamNonBlocking));
    struct Chunk { int k; long long r0, r1; };
    std::vector<Chunk> ch;
    constexpr int kChunks = 16;
    for (int k = 0; k < nblocks; ++k) {
      const BlockGeom& g = c->blocks[bs[k]].g;
      const long long rows = 5LL * g.Y * g.Z, per = (rows + kChunks - 1) / kChunks;
      for (long long r0 = 0; r0 < rows; r0 += per) ch.push_back({k, r0, std::min(rows, r0 + per)});
    }
    const size_t nc = ch.size();
    std::vector<cudaEvent_t> ev(3 * nc + 1, nullptr);
    struct EvGuard {
      std::vector<cudaEvent_t>& v;
      ~EvGuard() {
        for (auto e : v)
          if (e) cudaEventDestroy(e);
      }
    } guard{ev};
    for (auto& e : ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    cudaEvent_t* ev_in = ev.data();
    cudaEvent_t* ev_pack = ev.data() + nc;
    cudaEvent_t* ev_out = ev.data() + 2 * nc;
    auto grid_for = [](long long n) { return (unsigned)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148 * 16)); };
    for (int st = 0; st < nsteps; ++st) {
      for (size_t j = 0; j < nc; ++j) {
        const Chunk& q = ch[j];
        BlockState& B = c->blocks[bs[q.k]];
        const BlockGeom& g = B.g;
        double* sg = c->hs_stage + off[q.k] + q.r0 * g.X;
        const long long nr = q.r1 - q.r0;
        // the chunk's previous result has left the staging and landed in the host array
        if (st > 0) CK(cudaStreamWaitEvent(c->s_in, ev_out[j], 0));
        CK(cudaMemcpyAsync(sg, host[q.k] + q.r0 * g.X, (size_t)nr * g.X * sizeof(double), cudaMemcpyHostToDevice,
                           c->s_in));
        CK(cudaEventRecord(ev_in[j], c->s_in));
        CK(cudaStreamWaitEvent(c->st, ev_in[j], 0));
        k_rows_repack<<<grid_for(nr * g.X), 256, 0, c->st>>>(sg, g.X, fptr(B, F_QA) + q.r0 * g.Xp, g.Xp, g.X, nr);
        CK(cudaGetLastError());
      }
      one_step(c);
      for (size_t j = 0; j < nc; ++j) {
        const Chunk& q = ch[j];
        BlockState& B = c->blocks[bs[q.k]];
        const BlockGeom& g = B.g;
        double* sg = c->hs_stage + off[q.k] + q.r0 * g.X;
        const long long nr = q.r1 - q.r0;
        k_rows_repack<<<grid_for(nr * g.X), 256, 0, c->st>>>(fptr(B, F_QA) + q.r0 * g.Xp, g.Xp, sg, g.X, g.X, nr);
        CK(cudaGetLastError());
        CK(cudaEventRecord(ev_pack[j], c->st));
        CK(cudaStreamWaitEvent(c->s_out, ev_pack[j], 0));
        CK(cudaMemcpyAsync(host[q.k] + q.r0 * g.X, sg, (size_t)nr * g.X * sizeof(double), cudaMemcpyDeviceToHost,
                           c->s_out));
        CK(cudaEventRecord(ev_out[j], c->s_out));
      }
    }
    // the context's stream ends after the last copy out
    CK(cudaEventRecord(ev[3 * nc], c->s_out));
    CK(cudaStreamWaitEvent(c->st, ev[3 * nc], 0));
    c->launches += 2LL * (long long)nc * nsteps;
    sync_check(c);
  });
}

int canard_phase(canard_ctx* c, int32_t phase, int32_t nk) {
  return guarded(c, [&] {
    if (!c->setup_done) throw ApiError(CANARD_ERR_STATE, "canard_phase before canard_setup");
    if ((phase == CANARD_PH_MOVEF_A || phase == CANARD_PH_TIMESTEP || phase == CANARD_PH_VISCOUS ||
         phase == CANARD_PH_FLUXES || phase == CANARD_PH_GCBC || phase == CANARD_PH_RKUPDATE ||
         phase == CANARD_PH_WALL) &&
        (nk < 1 || nk > 4))
      throw ApiError(CANARD_ERR_ARG, "stage index nk must be 1..4");
    // parameters of stage nk for the current dt / timo
    auto params = [&]() {
      stage_params(c, nk, nk, 4);
      return dev_slot(c, 4);
    };
    switch (phase) {
      case CANARD_PH_FILTER: ph_filter(c); break;
      case CANARD_PH_COPYQO: ph_copyqo(c); break;
      case CANARD_PH_PRIM: ph_prim(c); break;
      case CANARD_PH_MOVEF_A: break;
      case CANARD_PH_TIMESTEP: if (nk == 1) timestep(c); break;
      case CANARD_PH_VISCOUS: ph_viscous(c); break;
      case CANARD_PH_FLUXES: ph_fluxes(c, params()); break;
      case CANARD_PH_GCBC: ph_gcbc(c, params()); break;
      case CANARD_PH_SPONGE: ph_sponge(c); break;
      case CANARD_PH_RKUPDATE: ph_rk(c, params()); break;
      case CANARD_PH_WALL: ph_wall(c, params()); break;
      case CANARD_PH_AVERAGE: ph_average(c); break;
      case CANARD_PH_ADVANCE: time_advance(c); break;
      default: throw ApiError(CANARD_ERR_ARG, "unknown phase");
    }
    sync_check(c);
  });
}

int canard_phase_with(canard_ctx* c, int32_t phase, int32_t nk, double dt, const double* umf,
                      const double* dudtmf) {
  return guarded(c, [&] {
    if (!c->setup_done) throw ApiError(CANARD_ERR_STATE, "canard_phase_with before canard_setup");
    if (!umf || !dudtmf) throw ApiError(CANARD_ERR_ARG, "null frame velocity or acceleration");
    if (nk < 1 || nk > 4) throw ApiError(CANARD_ERR_ARG, "stage index nk must be 1..4");
    if (phase != CANARD_PH_FLUXES && phase != CANARD_PH_GCBC && phase != CANARD_PH_RKUPDATE &&
        phase != CANARD_PH_WALL)
      throw ApiError(CANARD_ERR_ARG, "canard_phase_with takes the fluxes, GCBC, RK update and wall phases");
    // the stage scalars of every case as the caller's movef gave them
    // (src/mo_canard_driver.f90:261-263, 336-338): dtk = dt / (nkrk - nk + 1)
    StageParams sp{};
    for (int k = 0; k < 3; ++k) { sp.umf[k] = umf[k]; sp.dudtmf[k] = dudtmf[k]; sp.umfb[k] = umf[k]; }
    sp.dt = dt;
    sp.dtk = dt / (4 - nk + 1);
    std::vector<StageParams> v(c->cases.size(), sp);
    CK(cudaMemcpyAsync(dev_slot(c, 4), v.data(), v.size() * sizeof(StageParams), cudaMemcpyHostToDevice, c->st));
    const StageParams* d = dev_slot(c, 4);
    switch (phase) {
      case CANARD_PH_FLUXES: ph_fluxes(c, d); break;
      case CANARD_PH_GCBC: ph_gcbc(c, d); break;
      case CANARD_PH_RKUPDATE: ph_rk(c, d); break;
      default: ph_wall(c, d); break;
    }
    sync_check(c);
  });
}

int canard_get_time(canard_ctx* c, int32_t icase, double* t) {
  return guarded(c, [&] {
    if (!t || icase < 0 || icase >= (int)c->cases.size()) throw ApiError(CANARD_ERR_ARG, "bad case / pointer");
    TimeDev d;
    CK(cudaMemcpyAsync(&d, c->dtime + icase, sizeof(d), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    t[0] = (double)d.n; t[1] = (double)d.ndt; t[2] = d.dt; t[3] = d.dts; t[4] = d.dte; t[5] = d.timo;
  });
}

int canard_write_restart(canard_ctx* c, int32_t icase, int32_t iblock, const char* path) {
  return guarded(c, [&] {
    if (!path) throw ApiError(CANARD_ERR_ARG, "null path");
    const BlockState& B = c->blocks[block_index(c, icase, iblock)];
    const int64_t npts = (int64_t)B.g.X * B.g.Y * B.g.Z;
    std::vector<double> qa((size_t)5 * npts);
    double t[6];
    int rc = canard_get_state(c, icase, iblock, qa.data());
    if (rc == CANARD_OK) rc = canard_get_time(c, icase, t);
    if (rc != CANARD_OK) throw ApiError(rc, c->err);
    rc = canard_restart_write_file(path, t, qa.data(), npts);
    if (rc != CANARD_OK) throw ApiError(rc, std::string("cannot write restart file ") + path);
  });
}

int canard_read_restart(canard_ctx* c, int32_t icase, int32_t iblock, const char* path) {
  return guarded(c, [&] {
    if (!path) throw ApiError(CANARD_ERR_ARG, "null path");
    const BlockState& B = c->blocks[block_index(c, icase, iblock)];
    const int64_t npts = (int64_t)B.g.X * B.g.Y * B.g.Z;
    std::vector<double> qa((size_t)5 * npts);
    double t[6];
    int rc = canard_restart_read_file(path, t, qa.data(), npts);
    if (rc != CANARD_OK)
      throw ApiError(rc, std::string("cannot read restart file ") + path + " for a block of " +
                             std::to_string(npts) + " points");
    rc = canard_set_state(c, icase, iblock, qa.data());
    if (rc == CANARD_OK) rc = canard_set_time(c, icase, t);
    if (rc != CANARD_OK) throw ApiError(rc, c->err);
  });
}

int canard_record_enable(canard_ctx* c, int32_t on) {
  return guarded(c, [&] {
    CK(cudaStreamSynchronize(c->st));
    for (auto& b : c->blocks) {
      cudaFree(b.qb);
      b.qb = nullptr;
    }
    cudaFree(c->dtsum);
    c->dtsum = nullptr;
    if (!on) return;
    for (auto& b : c->blocks) {
      b.qb = dalloc<double>((size_t)5 * b.g.npad, c->st);
      CK(cudaMemsetAsync(b.qb, 0, (size_t)5 * b.g.npad * sizeof(double), c->st));
    }
    c->dtsum = dalloc<double>(c->cases.size(), c->st);
    CK(cudaMemsetAsync(c->dtsum, 0, c->cases.size() * sizeof(double), c->st));
    CK(cudaStreamSynchronize(c->st));
  });
}

int canard_record_accumulate(canard_ctx* c) {
  return guarded(c, [&] {
    if (!c->dtsum) throw ApiError(CANARD_ERR_STATE, "recording is off (canard_record_enable)");
    for (auto& b : c->blocks) {
      const long long n = 5 * b.g.npad;
      const int grid = (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148 * 8));
      k_record_acc<<<grid, 256, 0, c->st>>>(b.qb, fptr(b, F_QO), fptr(b, F_QA), b.g.npad, b.g.X, b.g.Xp, c->dtime,
                                            b.g.case_id);
      CK(cudaGetLastError());
    }
    k_record_dtsum<<<(ncase(c) + 127) / 128, 128, 0, c->st>>>(c->dtsum, c->dtime, ncase(c));
    CK(cudaGetLastError());
    c->launches += (long long)c->blocks.size() + 1;
  });
}

int canard_record_output(canard_ctx* c, int32_t icase, float* const* vart, double* time_out) {
  return guarded(c, [&] {
    if (!c->dtsum) throw ApiError(CANARD_ERR_STATE, "recording is off (canard_record_enable)");
    if (!vart || icase < 0 || icase >= (int)c->cases.size()) throw ApiError(CANARD_ERR_ARG, "bad case / pointer");
    const CaseState& cs = c->cases[icase];
    size_t most = 0;
    for (int b = cs.b0; b < cs.b0 + cs.nb; ++b) {
      if (!vart[b - cs.b0]) throw ApiError(CANARD_ERR_ARG, "null output array");
      const BlockGeom& g = c->blocks[b].g;
      most = std::max(most, (size_t)5 * g.X * g.Y * g.Z);
    }
    float* dout = dalloc<float>(most, c->st);
    c->transient.push_back(dout);
    for (int b = cs.b0; b < cs.b0 + cs.nb; ++b) {
      const BlockState& B = c->blocks[b];
      const BlockGeom& g = B.g;
      const int grid = (int)std::max<long long>(1, std::min<long long>((g.npad + 255) / 256, 148 * 8));
      k_record_out<<<grid, 256, 0, c->st>>>(B.qb, fptr(B, F_QO), dout, g.X, g.Y, g.Z, g.Xp, g.npad, c->dtime,
                                            c->dtsum, dev_slot(c, 3), icase);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(vart[b - cs.b0], dout, (size_t)5 * g.X * g.Y * g.Z * sizeof(float),
                         cudaMemcpyDeviceToHost, c->st));
    }
    TimeDev d;
    double dts = 0;
    CK(cudaMemcpyAsync(&d, c->dtime + icase, sizeof(d), cudaMemcpyDeviceToHost, c->st));
    CK(cudaMemcpyAsync(&dts, c->dtsum + icase, sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (time_out) *time_out = d.timo - 0.5 * dts;  // times(ndati) = timo - dtsum/2
    // reset the recording of this case (dtsum = 0, qb = 0)
    for (int b = cs.b0; b < cs.b0 + cs.nb; ++b)
      CK(cudaMemsetAsync(c->blocks[b].qb, 0, (size_t)5 * c->blocks[b].g.npad * sizeof(double), c->st));
    CK(cudaMemsetAsync(c->dtsum + icase, 0, sizeof(double), c->st));
    CK(cudaStreamSynchronize(c->st));
    free_transient(c);
  });
}

int canard_set_time(canard_ctx* c, int32_t icase, const double* t) {
  return guarded(c, [&] {
    if (!t || icase < 0 || icase >= (int)c->cases.size()) throw ApiError(CANARD_ERR_ARG, "bad case / pointer");
    TimeDev d;
    d.n = (long long)t[0]; d.ndt = (long long)t[1]; d.dt = t[2]; d.dts = t[3]; d.dte = t[4]; d.timo = t[5];
    CK(cudaMemcpyAsync(c->dtime + icase, &d, sizeof(d), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->cases[icase].n = d.n;
  });
}

// ---- unit operations (case 0) ------------------------------------------------------
int canard_mpigo(canard_ctx* c, const double* const* fields, int32_t ncols, int32_t nt, int32_t nrt, int32_t n45,
                 int32_t itag, int32_t m) {
  (void)itag;
  return guarded(c, [&] {
    if (!fields || ncols < 1 || ncols > 3 || nt < 0 || nt > 1 || nrt < 0 || nrt > 1 || n45 < 0 || n45 > 1 || m < 1 ||
        m > 5)
      throw ApiError(CANARD_ERR_ARG, "bad mpigo argument");
    if (nrt == 0 && ncols != 3) throw ApiError(CANARD_ERR_ARG, "nrall needs three columns");
    const CaseState& cs = c->cases[0];
    // stage the fields in the scratch columns 12..14 of every block; a
    // mixed-precision context contracts derivative inputs (nt = 0) in FP32
    const bool w32 = c->f32() && nt == 0;
    for (int b = cs.b0; b < cs.b0 + cs.nb; ++b) {
      if (!fields[b - cs.b0]) throw ApiError(CANARD_ERR_ARG, "null field");
      BlockState& B = c->blocks[b];
      h2d_field(c, B, fptr(B, F_SCR + 12), fields[b - cs.b0], ncols);
      if (w32) to_f32(c, fptr(B, F_SCR + 12), gptr(B, G_SCR + 12), (size_t)ncols * B.g.npad);
    }
    auto col = [&](int b, int d) -> const void* {
      const int k = 12 + (nrt == 0 ? d : 0);
      return w32 ? static_cast<const void*>(gptr(c->blocks[b], G_SCR + k))
                 : static_cast<const void*>(fptr(c->blocks[b], F_SCR + k));
    };
    launch_mpigo(c, make_face_table(c, face_tasks(c, nt, n45, m, -1, col, 0, w32), true, w32 ? 1 : 0));
    sync_check(c);
    free_transient(c);
  });
}

// One field through one line solve; in a mixed-precision context the
// derivative runs on an FP32 copy and the filter on the FP64 field with an
// FP32 elimination, as on the step path.
static void unit_line(canard_ctx* c, int iblock, const double* in, double* out, int dir, int nt, int m) {
  const int b = block_index(c, 0, iblock);
  BlockState& B = c->blocks[b];
  double* f = fptr(B, F_SCR + 11);
  h2d_field(c, B, f, in, 1);
  const int kind = c->fast() ? LK_F64_SPLIT : !c->f32() ? LK_F64 : (nt == 0 ? LK_F32 : LK_F64_TILE_F32_SOLVE);
  void* fd = f;
  if (kind_f32_fields(kind)) {
    fd = gptr(B, G_SCR + 11);
    to_f32(c, f, gptr(B, G_SCR + 11), (size_t)B.g.npad);
  }
  LineTask t;
  fill_line_task(c, B, dir, nt, fd, fd, m, nt == 0, t, kind);
  launch_line(c, make_line_table(c, {t}, dir, true, kind), dir, nt);
  if (kind_f32_fields(kind)) to_f64(c, gptr(B, G_SCR + 11), f, (size_t)B.g.npad);
  d2h_field(c, B, out, f, 1);
  sync_check(c);
  free_transient(c);
}

int canard_deriv(canard_ctx* c, int32_t iblock, const double* in, double* out, int32_t nn, int32_t m) {
  return guarded(c, [&] {
    if (!in || !out || nn < 1 || nn > 3 || m < 1 || m > 5) throw ApiError(CANARD_ERR_ARG, "bad deriv argument");
    unit_line(c, iblock, in, out, nn - 1, 0, m);
  });
}

int canard_filte(canard_ctx* c, int32_t iblock, double* f, int32_t inn, int32_t m) {
  return guarded(c, [&] {
    if (!f || inn < 1 || inn > 3 || m < 1 || m > 5) throw ApiError(CANARD_ERR_ARG, "bad filte argument");
    unit_line(c, iblock, f, f, kNnf[inn - 1] - 1, 1, m);
  });
}

int canard_line_bench(canard_ctx* c, int32_t op, int32_t nn, int32_t nfields, const double* in, double* out,
                      int32_t reps, double* ms_per_launch) {
  return guarded(c, [&] {
    if (!in || !out || !ms_per_launch || op < 0 || op > 1 || nn < 1 || nn > 3 || nfields < 1 || nfields > 5 ||
        reps < 1)
      throw ApiError(CANARD_ERR_ARG, "bad line bench argument");
    BlockState& B = c->blocks[block_index(c, 0, 0)];
    const int dir = nn - 1;
    const canard_ctx::TuneChoice& tc = c->tune[op == 0 ? 2 : 0][dir];
    const int kind = tc.kind >= 0 ? tc.kind : default_kind(c, op == 0 ? 2 : 0, dir);
    const size_t L = (size_t)B.g.X * B.g.Y * B.g.Z;
    std::vector<LineTask> tasks;
    for (int k = 0; k < nfields; ++k) {
      double* f = fptr(B, F_SCR + k);
      h2d_field(c, B, f, in + k * L, 1);
      void* src = f;
      void* dst = op == 0 ? static_cast<void*>(fptr(B, F_SCR + 5 + k)) : static_cast<void*>(f);
      if (kind_f32_fields(kind)) {
        to_f32(c, f, gptr(B, G_SCR + k), (size_t)B.g.npad);
        src = gptr(B, G_SCR + k);
        dst = gptr(B, G_SCR + 5 + k);
      }
      LineTask t;
      fill_line_task(c, B, dir, op, src, dst, k + 1, false, t, kind, true, tc.nc);
      tasks.push_back(t);
      // interface contraction of the faces not formed in the kernel
      const bool w32 = kind_f32_fields(kind);
      auto col = [&](int b, int) -> const void* {
        return w32 ? static_cast<const void*>(gptr(c->blocks[b], G_SCR + k))
                   : static_cast<const void*>(fptr(c->blocks[b], F_SCR + k));
      };
      launch_mpigo(c, make_face_table(c, face_tasks(c, op, 0, k + 1, dir, col, 0, w32, op == 0), true, w32 ? 1 : 0));
    }
    const Table<LineTask> T = make_line_table(c, tasks, dir, true, kind);
    launch_line(c, T, dir, op);
    for (int k = 0; k < nfields; ++k) {
      double* r = fptr(B, F_SCR + (op == 0 ? 5 : 0) + k);
      if (kind_f32_fields(kind)) to_f64(c, gptr(B, G_SCR + 5 + k), r, (size_t)B.g.npad);
      d2h_field(c, B, out + k * L, r, 1);
    }
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, c->st));
    for (int r = 0; r < reps; ++r) launch_line(c, T, dir, op);
    CK(cudaEventRecord(e1, c->st));
    CK(cudaEventSynchronize(e1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms_per_launch = ms / reps;
    sync_check(c);
    free_transient(c);
  });
}

int canard_autotune(canard_ctx* c, int32_t reps, double* report, int32_t nmax) {
  int rows = 0;
  const int rc = guarded(c, [&] {
    if (!c->setup_done) throw ApiError(CANARD_ERR_STATE, "canard_autotune before canard_setup");
    if (reps < 1) throw ApiError(CANARD_ERR_ARG, "reps must be positive");
    CK(cudaStreamSynchronize(c->st));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    auto time_table = [&](const Table<LineTask>& T, int dir, int op) {
      launch_line(c, T, dir, op);  // warm-up
      CK(cudaEventRecord(e0, c->st));
      for (int r = 0; r < reps; ++r) launch_line(c, T, dir, op);
      CK(cudaEventRecord(e1, c->st));
      CK(cudaEventSynchronize(e1));
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      return (double)ms / reps;
    };
    for (int grp = 0; grp < 3; ++grp)
      for (int dir = 0; dir < 3; ++dir) {
        const int op = grp == 0 ? 1 : 0;
        std::vector<std::pair<int, int>> cand;  // (kind, nc)
        std::vector<int> kinds{default_kind(c, grp, dir)};
        if (c->fast()) {  // the one-lane and split FP64 sweeps compete in the fast mode
          kinds.push_back(LK_F64);
          kinds.push_back(LK_F64_SPLIT);
        }
        if (grp != 0 && c->fast() && quad_ok(c, dir, LK_F64_QUAD)) kinds.push_back(LK_F64_QUAD);
        if (grp != 0 && c->f32() && quad_ok(c, dir, LK_F32_QUAD)) kinds.push_back(LK_F32_QUAD);
        if (c->f32()) kinds.push_back(grp == 0 ? LK_F64_TILE_F32_SOLVE_1L : LK_F32_1L);
        if (c->fast() && twist_ok(c, dir, LK_F64_TWIST)) kinds.push_back(LK_F64_TWIST);
        if (c->f32() && twist_ok(c, dir, LK_F32_TWIST)) kinds.push_back(grp == 0 ? LK_F64_TILE_F32_TWIST : LK_F32_TWIST);
        // the streamed filter reads a row of 32 lines per step: coalesced along
        // eta/zeta only (along xi each lane's row is a line length away)
        if (c->f32() && grp == 0) {
          if (dir != 0) kinds.push_back(LK_F64_STREAM_F32);
        } else if (tm_ok(c, dir)) kinds.push_back(LK_F64_TM);
        // the filter acts on the FP64 state with an FP64 right-hand side in every
        // kind; the FP64 eliminations (one-lane and split) compete with the FP32 ones there
        if (c->f32() && grp == 0) {
          kinds.push_back(LK_F64);
          kinds.push_back(LK_F64_SPLIT);
          if (twist_ok(c, dir, LK_F64_TWIST)) kinds.push_back(LK_F64_TWIST);
        }
        {  // each kind once, the default first
          std::vector<int> u;
          for (int k : kinds)
            if (std::find(u.begin(), u.end(), k) == u.end()) u.push_back(k);
          kinds.swap(u);
        }
        for (int k : kinds) {
          cand.push_back({k, 0});
          if (dir != 0 && k != LK_F64_TM && k != LK_F64_STREAM_F32)
            for (int nc : {2, 4, 8}) cand.push_back({k, nc});
        }
        double best = 1e300, def = 0;
        canard_ctx::TuneChoice pick;
        for (size_t i = 0; i < cand.size(); ++i) {
          // the step's launch shape: FP32-mixed filters the five fields at once
          auto v = (grp == 0 && c->filter5()) ? filter_tasks5(c, dir, cand[i].first, cand[i].second, true)
                                          : group_tasks(c, grp, dir, 1, cand[i].first, cand[i].second, true);
          if (v.empty()) continue;
          Table<LineTask> T = make_line_table(c, v, dir, true, cand[i].first);
          if (T.smem > 227 * 1024) continue;
          const double ms = time_table(T, dir, op);
          if (i == 0) def = ms;
          if (ms < best) { best = ms; pick.kind = cand[i].first; pick.nc = cand[i].second; }
          free_transient(c);
        }
        if (best < 1e300) c->tune[grp][dir] = pick;
        if (report && rows < nmax) {
          double* r = report + 6 * rows;
          r[0] = grp; r[1] = dir; r[2] = pick.kind; r[3] = pick.nc; r[4] = best < 1e300 ? best : 0; r[5] = def;
        }
        ++rows;
      }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    rebuild_line_tables(c);
  });
  return rc == CANARD_OK ? rows : -rc;
}

int canard_set_line_kind(canard_ctx* c, int32_t group, int32_t dir, int32_t kind, int32_t chunks) {
  return guarded(c, [&] {
    if (group < 0 || group > 2 || dir < 0 || dir > 2 || kind < -1 || kind > LK_F64_TILE_F32_TWIST || chunks < 0 ||
        chunks == 1 || chunks > kMaxChunks || (dir == 0 && chunks != 0))
      throw ApiError(CANARD_ERR_ARG, "bad line kind argument");
    if (kind >= 0) {
      bool fits;
      if (!c->f32())
        fits = kind == LK_F64 || kind == LK_F64_SPLIT || (kind == LK_F64_TM && tm_ok(c, dir) && chunks == 0) ||
               (kind == LK_F64_QUAD && group != 0 && quad_ok(c, dir, kind)) ||
               (kind == LK_F64_TWIST && twist_ok(c, dir, kind));
      else if (group == 0)
        fits = kind == LK_F64_TILE_F32_SOLVE || kind == LK_F64_TILE_F32_SOLVE_1L || kind == LK_F64 ||
               kind == LK_F64_SPLIT || (kind == LK_F64_STREAM_F32 && chunks == 0) ||
               ((kind == LK_F64_TWIST || kind == LK_F64_TILE_F32_TWIST) && twist_ok(c, dir, kind));
      else
        fits = kind == LK_F32 || kind == LK_F32_1L || (kind == LK_F32_QUAD && quad_ok(c, dir, kind)) ||
               (kind == LK_F32_TWIST && twist_ok(c, dir, kind));
      if (!fits) throw ApiError(CANARD_ERR_ARG, "line kind not available for this precision or line length");
    }
    CK(cudaStreamSynchronize(c->st));
    c->tune[group][dir].kind = kind;
    c->tune[group][dir].nc = kind >= 0 ? chunks : 0;
    if (c->setup_done) rebuild_line_tables(c);
  });
}

int canard_set_timers(canard_ctx* c, int32_t on) {
  return guarded(c, [&] {
    CK(cudaStreamSynchronize(c->st));
    collect_timers(c);
    c->timers = on != 0;
    for (int i = 0; i < T_NFAM; ++i) c->t_ms[i] = c->t_n[i] = c->t_bytes[i] = 0;
  });
}

int canard_get_timers(canard_ctx* c, double* ms, double* launches, double* bytes, int32_t nmax) {
  if (!c) return -CANARD_ERR_ARG;
  int rc = guarded(c, [&] {
    CK(cudaStreamSynchronize(c->st));
    collect_timers(c);
    for (int i = 0; i < T_NFAM && i < nmax; ++i) {
      if (ms) ms[i] = c->t_ms[i];
      if (launches) launches[i] = c->t_n[i];
      if (bytes) bytes[i] = c->t_bytes[i];
    }
  });
  return rc == CANARD_OK ? (int)T_NFAM : -rc;
}

const char* canard_timer_name(int32_t f) { return (f >= 0 && f < T_NFAM) ? kTimerNames[f] : ""; }

int canard_set_graphs(canard_ctx* c, int32_t on) {
  return guarded(c, [&] {
    CK(cudaStreamSynchronize(c->st));
    c->use_graphs = on != 0;
  });
}

int canard_launch_count(canard_ctx* c, int64_t* count) {
  if (!c || !count) return CANARD_ERR_ARG;
  *count = c->launches;
  return CANARD_OK;
}

#ifdef CANARD_TRACE
// Trace builds only (-DCANARD_TRACE): the device buffer of 8 int64 per CTA that
// the line kernels fill with clock64 stamps and the SM id.
int canard_trace_buffer(void* dev) {
  return cudaMemcpyToSymbol(g_trace, &dev, sizeof(dev)) == cudaSuccess ? CANARD_OK : CANARD_ERR_CUDA;
}
#endif

int canard_selftest_wait(canard_ctx* c, double* seconds) {
  return guarded(c, [&] {
    CK(cudaStreamSynchronize(c->st));
    const auto t0 = std::chrono::steady_clock::now();
    c->launches += 1;
    k_wait_selftest<<<1, 32, 0, c->st>>>(c->derr);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->st));
    if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    sync_check(c);  // reports the flag (CANARD_ERR_TIMEOUT) and clears it
  });
}

}  // extern "C"

// ==================================================================================
// Compact derivative without device allocation.
//
// For callers that cannot allocate device memory on the step path: solvers that
// own every device buffer themselves (a Fortran code whose arrays come from its
// own OpenACC/CUDA-Fortran pool), code running under a memory budget that
// forbids allocator calls between steps, or a host thread that must not block
// in the allocator. The caller passes device input and output; the scratch the
// derivative needs (task records, TMA descriptors, coefficients, LU factors and
// the periodic contraction buffers) lives in one file-scope device array of
// fixed size that every GPU loading this library holds until the process exits.
namespace {
constexpr int kNaMaxLines = 65536;   // lines of the direction (nbsize)
constexpr int kNaMaxPoints = 1024;   // points per line the scratch's factor table holds (the FP64
                                     // tile allows fewer: 906 along xi, 896 along eta or zeta)
constexpr size_t kNaTask = 0;        // LineTask
constexpr size_t kNaFace = 512;      // up to 2 FaceTask
constexpr size_t kNaIdx = 1536;      // (unused int), line0 of the 2 face tasks
constexpr size_t kNaErr = 1600;      // device error flag
constexpr size_t kNaChain = 1608;    // unused third send component (2 doubles)
constexpr size_t kNaMaps = 1664;     // 2 CUtensorMap, 64-byte aligned
constexpr size_t kNaScheme = 2048;   // DevScheme
constexpr size_t kNaLu = 4096;       // 5 x kNaMaxPoints doubles
constexpr size_t kNaRecv = kNaLu + 5 * kNaMaxPoints * sizeof(double);  // 2 sides x 2 comps x lines
// the line kernel's tile -> task index: every tile belongs to task 0, so this
// region is never written and keeps the zeros of static initialisation
constexpr int kNaMaxTiles = 8192;
constexpr size_t kNaTiles = kNaRecv + (size_t)4 * kNaMaxLines * sizeof(double);
constexpr size_t kNaBytes = kNaTiles + (size_t)kNaMaxTiles * sizeof(int);
static_assert(sizeof(LineTask) <= kNaFace - kNaTask, "LineTask slot");
static_assert(2 * sizeof(FaceTask) <= kNaIdx - kNaFace, "FaceTask slots");
static_assert(sizeof(DevScheme) <= kNaLu - kNaScheme, "scheme slot");
static_assert(kNaMaps % 64 == 0 && kNaLu % 256 == 0 && kNaRecv % 256 == 0, "alignment");
}  // namespace

// about 2.1 MiB per device (zero-initialised)
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

namespace {
std::mutex g_na_mu;
unsigned char* g_na_addr[256] = {};

// Device address of the scratch array for the current device. The symbol's
// host-side name is only a stand-in, so the address is looked up once per
// device (with that device current) and cached.
unsigned char* noalloc_scratch(int dev) {
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (dev < 0 || dev >= 256) throw ApiError(CANARD_ERR_ARG, "device index out of range");
  if (!g_na_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) throw CudaError(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    set_line_smem_limits();
    g_na_addr[dev] = static_cast<unsigned char*>(p);
  }
  return g_na_addr[dev];
}
}  // namespace

extern "C" int canard_deriv_noalloc(const double* d_in, double* d_out, int32_t lxi, int32_t let, int32_t lze,
                                    int32_t pitch, int32_t nn, int32_t nbc0, int32_t nbc1, double fltk,
                                    double fltrbc, void* stream) {
  auto fail = [](int code, const char* msg) {
    std::fprintf(stderr, "canard_deriv_noalloc: %s\n", msg);
    return code;
  };
  if (!d_in || !d_out) return fail(CANARD_ERR_ARG, "null field pointer");
  if ((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_out)) & 15)
    return fail(CANARD_ERR_ARG, "fields must be 16-byte aligned");
  if (lxi < 12 || let < 12 || lze < 12) return fail(CANARD_ERR_ARG, "every direction needs at least 13 points");
  if (pitch < lxi + 1 || pitch % 4 != 0) return fail(CANARD_ERR_ARG, "pitch must be >= lxi+1 and a multiple of 4");
  if (nn < 1 || nn > 3) return fail(CANARD_ERR_ARG, "direction nn must be 1, 2 or 3");
  auto closure_ok = [](int b) {
    return b == BC_NR || b == BC_WALLI || b == BC_WALLV || b == BC_CURV || b == BC_PERIODIC;
  };
  if (!closure_ok(nbc0) || !closure_ok(nbc1))
    return fail(CANARD_ERR_UNSUPPORTED, "end codes must be 10, 20, 25, 30 or 45 (periodic on the same line)");
  if ((nbc0 == BC_PERIODIC) != (nbc1 == BC_PERIODIC))
    return fail(CANARD_ERR_UNSUPPORTED, "a periodic line needs code 45 at both ends");
  if (!(fltrbc > 0.0)) return fail(CANARD_ERR_ARG, "fltrbc must be positive");
  const int dir = nn - 1;
  canard_block_desc bd{};
  bd.lxi = lxi; bd.let = let; bd.lze = lze;
  for (int d = 0; d < 3; ++d)
    for (int sd = 0; sd < 2; ++sd) { bd.nbc[d][sd] = BC_NR; bd.mbcd[d][sd] = -1; }
  bd.nbc[dir][0] = nbc0; bd.nbc[dir][1] = nbc1;
  if (nbc0 == BC_PERIODIC) { bd.mbcd[dir][0] = 0; bd.mbcd[dir][1] = 0; }
  BlockGeom g;
  make_geom(bd, 0, 0, g);
  g.Xp = pitch;
  g.npad = (int64_t)pitch * g.Y * g.Z;
  const int L = g.ijk[0][dir] + 1, nbs = g.nbs[dir];
  if (L > kNaMaxPoints || tile_smem_for(dir, L, LK_F64) > (size_t)kLineSmemMax)
    return fail(CANARD_ERR_ARG, "line too long for the shared-memory tile (at most 906 points along xi, "
                                "896 along eta or zeta)");
  if (nbs > kNaMaxLines) return fail(CANARD_ERR_ARG, "more than 65536 lines in this direction");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  try {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    unsigned char* base = noalloc_scratch(dev);
    Scheme sch;
    sch.build(fltk, fltrbc);
    const int n0 = nbc0 == BC_PERIODIC ? 1 : 0, n1 = n0;
    std::vector<double> lu((size_t)5 * L);
    sch.lu(L, n0, n1, 0, lu.data());
    LineTask t{};
    t.in = d_in;
    t.out = d_out;
    t.lu = base + kNaLu;
    {  // bitwise-constant interior rows, as for the context path
      const int e = L - 4;
      int i0 = e;
      auto same = [&](int r) {
        for (int k = 0; k < 5; ++k)
          if (std::memcmp(&lu[(size_t)k * L + r], &lu[(size_t)k * L + e], sizeof(double)) != 0) return false;
        return true;
      };
      while (i0 - 1 >= 3 && same(i0 - 1)) --i0;
      t.cl1 = lu[e]; t.cl2 = lu[(size_t)L + e]; t.cu1 = lu[(size_t)2 * L + e];
      t.cu2 = lu[(size_t)3 * L + e]; t.cu3 = lu[(size_t)4 * L + e];
      t.c0 = i0;
    }
    t.recv = base + kNaRecv;
    t.drva = nullptr;
    t.sc = reinterpret_cast<const DevScheme*>(base + kNaScheme);
    t.X = g.X; t.Y = g.Y; t.Z = g.Z; t.Xp = g.Xp;
    t.L = L; t.nbs = nbs; t.m = 1; t.ndf0 = n0; t.ndf1 = n1;
    chunking_dir(dir, L, t.nbox, t.by);
    if (dir == 0) {
      t.ntx = 1;
      t.ntiles = (g.Y * g.Z + kLanes - 1) / kLanes;
    } else {
      t.ntx = (g.X + kLanes - 1) / kLanes;
      t.ntiles = t.ntx * (dir == 1 ? g.Z : g.Y);
    }
    t.tile0 = 0;
    if (t.ntiles > kNaMaxTiles) return fail(CANARD_ERR_ARG, "more than 8192 tiles of 32 lines");
    // periodic on the line itself: each end's contraction feeds the other end
    FaceTask f[2];
    int nf = 0;
    if (n0) {
      for (int sb = 0; sb < 2; ++sb) {
        FaceTask& q = f[nf];
        q = FaceTask{};
        q.src = d_in;
        q.dstf = d_in;
        q.recv = reinterpret_cast<double*>(base + kNaRecv) + (size_t)(1 - sb) * 2 * nbs;
        q.chain = reinterpret_cast<double*>(base + kNaChain);
        q.sc = t.sc;
        q.nn = nn; q.sb = sb; q.nt = 0; q.exch = 1; q.corr = 0; q.iik = 1; q.ra0k = 0.0;
        q.X = g.X; q.Y = g.Y; q.Z = g.Z; q.Xp = g.Xp; q.N = L - 1;
        q.XA = g.X; q.YA = g.Y; q.ZA = g.Z; q.XpA = g.Xp; q.NA = L - 1;
        q.nbs = nbs; q.nj = g.ijk[1][dir] + 1; q.line0 = nf * nbs;
        ++nf;
      }
    }
    DevScheme ds{};
    std::memcpy(ds.pbci, sch.pbci, sizeof(ds.pbci));
    std::memcpy(ds.pbco, sch.pbco, sizeof(ds.pbco));
    std::memcpy(ds.pbcot, sch.pbcot, sizeof(ds.pbcot));
    ds.fa = sch.fa; ds.fb = sch.fb; ds.fc = sch.fc;
    std::memcpy(ds.fbc, sch.fbc, sizeof(ds.fbc));
    ds.alphf = sch.alphf; ds.betf = sch.betf;
    std::memcpy(ds.albef, sch.albef, sizeof(ds.albef));
    CUtensorMap maps[2];
    std::memset(maps, 0, sizeof(maps));
    if (dir != 0) {
      maps[0] = field_map(d_in, g.X, g.Y, g.Z, g.Xp, dir, t.by);
      maps[1] = field_map(d_out, g.X, g.Y, g.Z, g.Xp, dir, t.by);
    }
    const int idx[3] = {0, 0, nbs};
    CK(cudaMemcpyToSymbolAsync(g_noalloc_scratch, &t, sizeof(t), kNaTask, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyToSymbolAsync(g_noalloc_scratch, f, sizeof(f), kNaFace, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyToSymbolAsync(g_noalloc_scratch, idx, sizeof(idx), kNaIdx, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyToSymbolAsync(g_noalloc_scratch, maps, sizeof(maps), kNaMaps, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyToSymbolAsync(g_noalloc_scratch, &ds, sizeof(ds), kNaScheme, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyToSymbolAsync(g_noalloc_scratch, lu.data(), lu.size() * sizeof(double), kNaLu,
                               cudaMemcpyHostToDevice, st));
    if (nf) {
      const int tot = nf * nbs;
      launch_mpigo_t<double>(std::max(1, std::min((tot + 127) / 128, 148 * 16)), st,
                             reinterpret_cast<const FaceTask*>(base + kNaFace),
                             reinterpret_cast<const int*>(base + kNaIdx) + 1, nf, tot);
      CK(cudaGetLastError());
    }
    const size_t smem = line_smem(dir, t, LK_F64);
    const LineTask* dt = reinterpret_cast<const LineTask*>(base + kNaTask);
    const int* d0 = reinterpret_cast<const int*>(base + kNaTiles);  // zeros: tile -> task 0
    const CUtensorMap* dm = reinterpret_cast<const CUtensorMap*>(base + kNaMaps);
    int* de = reinterpret_cast<int*>(base + kNaErr);
    // one task: every tile's task is tile / ntiles = 0 (the zero table is not read)
    if (dir == 0) launch_line_t<1, 0, double, double>(t.ntiles, smem, st, dt, d0, t.ntiles, dm, de);
    else if (dir == 1) launch_line_t<2, 0, double, double>(t.ntiles, smem, st, dt, d0, t.ntiles, dm, de);
    else launch_line_t<3, 0, double, double>(t.ntiles, smem, st, dt, d0, t.ntiles, dm, de);
    CK(cudaGetLastError());
  } catch (const ApiError& e) {
    return fail(e.code, e.what());
  } catch (const std::exception& e) {
    return fail(CANARD_ERR_CUDA, e.what());
  }
  return CANARD_OK;
}

// Reads and clears the error flag of the allocation-free derivative after the
// work queued on `stream` has finished. The flag is raised by a line kernel
// whose bounded wait for its input copies gave up; it stays up, and makes later
// calls skip their work, until this function clears it.
extern "C" int canard_deriv_noalloc_status(void* stream) {
  try {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    unsigned char* base = noalloc_scratch(dev);
    CK(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    int flag = 0;
    CK(cudaMemcpy(&flag, base + kNaErr, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag == 0) return CANARD_OK;
    const int zero = 0;
    CK(cudaMemcpy(base + kNaErr, &zero, sizeof(int), cudaMemcpyHostToDevice));
    std::fprintf(stderr, "canard_deriv_noalloc_status: a bounded device wait gave up (flag %d)\n", flag);
    return (flag & kErrTimeout) ? CANARD_ERR_TIMEOUT : CANARD_ERR_CUDA;
  } catch (const ApiError& e) {
    std::fprintf(stderr, "canard_deriv_noalloc_status: %s\n", e.what());
    return e.code;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "canard_deriv_noalloc_status: %s\n", e.what());
    return CANARD_ERR_CUDA;
  }
}
