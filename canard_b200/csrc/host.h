// Host-side set-up of the Canard hot path: scheme coefficients, LU factors,
// exchange maps and the tables the device kernels consume. Everything here runs
// once per context; nothing here is on the time-step path.
#pragma once
#include <cstdint>
#include <string>
#include <array>
#include <vector>

#include "canard_gpu.h"

namespace canard {

constexpr int BC_NR = 10, BC_WALLI = 20, BC_WALLV = 25, BC_CURV = 30, BC_STRAIGHT = 35,
              BC_SUBDOM = 40, BC_PERIODIC = 45;

inline bool bc_gcbc(int np) { return np == BC_NR || np == BC_WALLI || np == BC_WALLV || np == BC_CURV; }
inline bool bc_interface(int np) { return np == BC_STRAIGHT || np == BC_SUBDOM || np == BC_PERIODIC; }
inline bool bc_averaged(int np) { return np == BC_CURV || np == BC_STRAIGHT || np == BC_PERIODIC; }

// Compact-scheme coefficients of one case (src/mo_numerics.f90:114-134).
struct Scheme {
  double alphf = 0, betf = 0, fa = 0, fb = 0, fc = 0;
  double albef[2][3][5] = {};  // [n][row][k+2]
  double fbc[3][5] = {};       // [row][k]
  double pbci[2][2][12] = {};  // [nt][side][i]
  double pbco[2][2][12] = {};
  double pbcot[2][2] = {};     // [nt][side]
  void build(double fltk_nml, double fltrbc);
  // LU of one line of n points: 5 arrays of n (xl1, xl2, xu1, xu2, xu3).
  void lu(int n, int ns, int ne, int nt, double* out5n) const;
  void pack150(double* o) const;
};

// Geometry of one block as the kernels see it.
struct BlockGeom {
  int lxi, let, lze;
  int X, Y, Z, Xp;  // points per direction, padded row length (multiple of 4)
  int64_t npad;     // Xp*Y*Z
  int nbc[3][2], nbr[3][2];
  int ijk[3][3];    // ijk[a][nn] as in t_domdcomp (a = line, 2nd, 3rd index)
  int nbs[3];       // lines per direction
  int case_id, block_in_case;
  int64_t dev(int x, int y, int z) const { return ((int64_t)z * Y + y) * Xp + x; }
  // point at position pos of line (j, k) along direction nn (src/mo_utils.f90:54-69)
  void line_xyz(int nn, int pos, int j, int k, int& x, int& y, int& z) const {
    if (nn == 1) { x = pos; y = j; z = k; }
    else if (nn == 2) { x = k; y = pos; z = j; }
    else { x = j; y = k; z = pos; }
  }
  int64_t ref_index(int x, int y, int z) const { return ((int64_t)z * Y + y) * X + x; }
};

void make_geom(const canard_block_desc& d, int case_id, int bic, BlockGeom& g);

// Face exchange map: recv face (b, nn, side) <- send face (src_b, nn, 1-side).
struct FaceLink { int dst_b, nn, dst_side, src_b, src_side; };
// Returns empty string on success, else an error message. Blocks are case-local.
std::string face_links(const std::vector<BlockGeom>& blocks, std::vector<FaceLink>& out);

// Junction averaging plans (average_point / average_line): per target point,
// the sources (own value first) summed in order, times 1/(count).
struct AvgTarget { int b; int64_t l; int first, count; };  // l = device index
struct AvgPlan {
  std::vector<AvgTarget> targets;
  std::vector<int> src_b;       // per source entry
  std::vector<int64_t> src_l;   // device index
};
// The blocks of a case split into sub-domains (nbpc > 1, src/mo_domdcomp.f90:
// 85-232): the BlockGeoms are then the ranks. parents[m]: the split of input
// block m and its neighbour blocks; mb[r], pos[r]: rank r's block and position.
struct Decomp {
  struct Parent { int nbpc[3]; int nbr[3][2]; int mo; };
  std::vector<Parent> parents;
  std::vector<int> mb;
  std::vector<std::array<int, 3>> pos;
  // rank of block mm's sub-domain at (i along nn, j along nn+1, k along nn+2)
  // (idsd3, src/mo_domdcomp.f90:588-605); nn = 1..3
  int idsd3(int i, int j, int k, int mm, int nn) const {
    const Parent& p = parents[mm];
    int q[3];
    q[nn - 1] = i; q[nn % 3] = j; q[(nn + 1) % 3] = k;
    return p.mo + (q[2] * p.nbpc[1] + q[1]) * p.nbpc[0] + q[0];
  }
};
// Every rank its own block (nbpc = 1): the decomposition of unsplit blocks.
Decomp unsplit(const std::vector<BlockGeom>& blocks);
// Checks a decomposition against the ranks' geometry; empty string if sound.
std::string check_decomp(const std::vector<BlockGeom>& ranks, const Decomp& d);

std::string junction_plans(const std::vector<BlockGeom>& blocks, AvgPlan& points, AvgPlan& lines);
std::string junction_plans(const std::vector<BlockGeom>& ranks, const Decomp& d, AvgPlan& points, AvgPlan& lines);

// average_surface plan: per averaged point, its ordered list of snapshot sources.
std::string surface_plan(const std::vector<BlockGeom>& blocks, const std::vector<FaceLink>& links,
                         AvgPlan& surf);

// GCBC weights (gcbc_init, src/mo_gcbc.f90:40-131): for each GCBC face of the
// block in reference order, per line 5 (device point, weight) entries.
struct GcbcFace { int nn, side, bc; int64_t first; };  // first entry = line 0, offset 0
void gcbc_tables(const BlockGeom& g, const double* yaco_ref, std::vector<GcbcFace>& faces,
                 std::vector<int64_t>& pts, std::vector<double>& w);

// Sponge list (spongeup, src/mo_sponge.f90:34-71).
void sponge_list(const BlockGeom& g, const canard_case_desc& c, const double* xyz_ref,
                 const double* yaco_ref, std::vector<int64_t>& pts, std::vector<double>& asz,
                 std::vector<double>& bsz);

}  // namespace canard
