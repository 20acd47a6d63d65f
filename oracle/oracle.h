/*
 * CPU oracle for the Canard per-step hot path — TEST INFRASTRUCTURE ONLY.
 *
 * This library is a plain C++ FP64 restatement of the reference Fortran
 * (EnricoDeg/Canard, src/mo_numerics.f90, mo_physics.f90, mo_gcbc.f90,
 * mo_sponge.f90, mo_grid.f90, mo_domdcomp.f90, mo_canard_driver.f90). It is
 * used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as
 * the checker, never by the product path (canard_b200/).
 *
 * Parity status: UNPINNED against the reference itself. The reference ships no
 * tests, golden vectors or fixtures, and it cannot be compiled here (Fortran
 * 2003 + MPI; no Fortran compiler in the image). The oracle is pinned instead
 * against known answers derived from the scheme's mathematics (modified
 * wavenumber, filter transfer function, constant preservation, coefficient
 * identities) in tests/test_oracle_kat.py.
 *
 * Every block is one "rank" of the reference (nbpc = 1 per block), or, after
 * orc_set_subdomains, every rank is a sub-domain of a split block; the MPI
 * point-to-point exchanges are reproduced by a message-matching simulator with
 * MPI's non-overtaking rule (per source/destination/tag FIFO).
 */
#ifndef CANARD_ORACLE_H
#define CANARD_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int32_t lxi, let, lze;   /* cells per direction; points = l + 1 */
  int32_t nbc[3][2];       /* boundary code per direction (xi, eta, zeta) and side */
  int32_t mbcd[3][2];      /* neighbour block per face, -1 = none */
} orc_block_desc;

typedef struct {
  int32_t nblocks;
  int32_t viscous;         /* the reference's -DVISCOUS build */
  double fltk, fltrbc;     /* namelist values (fltk is multiplied by pi) */
  double reoo, tempoo, amach1, amach2, amach3, timf;
  int32_t nsmf;
  double cfl;
  double szco, szth0, szth1, doml0, doml1; /* sponge */
} orc_case_desc;

typedef struct orc_solver orc_solver;

/* Coefficients: writes 2*12*2 pbci, 2*12*2 pbco, 4 pbcot, 5 filter scalars
 * (alphf, betf, fa, fb, fc), 5*3*2 albef, 5*3 fbc  => 48+48+4+5+30+15 = 150. */
int orc_coeffs(double fltk_nml, double fltrbc, double* out150);
/* LU factors of one line: xu (n,3) and xl (n,2) column-major, nt 0/1, ns/ne 0/1 */
int orc_penta(double fltk_nml, double fltrbc, int n, int ns, int ne, int nt,
              double* xu, double* xl);

orc_solver* orc_create(const orc_case_desc* c, const orc_block_desc* b);
void orc_destroy(orc_solver* s);
void orc_set_threads(int n);
int orc_lmx(orc_solver* s, int b);
int orc_set_grid(orc_solver* s, int b, const double* xyz);  /* (0:lmx,3) */
int orc_setup(orc_solver* s);   /* metrics, gcbc_init, junction search, sponge */
/* Ranks as sub-domains of split blocks (nbpc > 1; src/mo_domdcomp.f90:85-232):
 * the create call's blocks are then the ranks, with their BC 40 faces and
 * neighbour ranks; here the input's blocks: nbpc[m][3], mbcd[m][3][2] (block
 * neighbours), and per rank sub[r] = (block, position along xi, eta, zeta),
 * ranks numbered as the reference numbers them. Call before orc_setup. */
int orc_set_subdomains(orc_solver* s, int nblocks, const int32_t* nbpc, const int32_t* mbcd, const int32_t* sub);
int orc_set_state(orc_solver* s, int b, const double* qa);  /* (0:lmx,5) */
/* array ids: see ORC_A_* below; returns number of doubles written or <0 */
long orc_get_array(orc_solver* s, int b, int which, double* out);
int orc_set_array(orc_solver* s, int b, int which, const double* in);
int orc_step(orc_solver* s, int nsteps);
int orc_phase(orc_solver* s, int phase, int nk);
int orc_get_time(orc_solver* s, double* out6); /* n, ndt, dt, dts, dte, timo */
int orc_set_time(orc_solver* s, const double* in6);

/* Exchange hook, for tests that hold a case's ranks in several processes: it
 * is called where one rank's step reads another rank's data. kind 0: after
 * mpigo's messages arrived (a = nt, b = m), before the periodic correction;
 * kind 1: after gcbc_setup, before gcbc_comm; kind 2: before average_point
 * (a = 0), average_line (1) and average_surface (2); kind 3: in
 * calc_time_step, data = the per-rank maxima res1[0:n] then res2[0:n], which
 * the hook may overwrite before they are reduced. NULL removes the hook. */
typedef void (*orc_hook_fn)(void* user, int kind, int a, int b, double* data, int n);
void orc_set_hook(orc_solver* s, orc_hook_fn fn, void* user);

/* unit operations (mirror t_numerics) */
int orc_mpigo(orc_solver* s, double* const* fields, int ncols, int nt, int nrt,
              int n45, int itag, int m);
int orc_deriv(orc_solver* s, int b, const double* in, double* out, int nn, int m);
int orc_filte(orc_solver* s, int b, double* f, int inn, int m);

enum {
  ORC_A_QA = 0, ORC_A_QO = 1, ORC_A_DE = 2, ORC_A_P = 3, ORC_A_SS1 = 4,
  ORC_A_XIM = 5, ORC_A_ETM = 6, ORC_A_ZEM = 7, ORC_A_YACO = 8,
  ORC_A_TAU = 9,   /* txx tyy tzz txy tyz tzx hxx hyy hzz */
  ORC_A_DRVA1 = 10, ORC_A_DRVA2 = 11, ORC_A_DRVA3 = 12, /* (nbs,5,2) */
  ORC_A_CM1 = 13, ORC_A_CM2 = 14, ORC_A_CM3 = 15,       /* (nbs,3,2) */
  ORC_A_RECV0 = 16, /* recv0{1,2,3} concatenated, each (nbs,2,2,5) */
  ORC_A_RECV1 = 17, /* recv1{1,2,3} concatenated, each (nbs,3,2,5) */
  ORC_A_SEND1 = 18, /* send1{1,2,3} concatenated, each (nbs,3,2) */
  ORC_A_SBCC = 19, ORC_A_SPONGE = 20 /* lsz+1 entries of (l, asz, bsz) */
};

enum {
  ORC_PH_FILTER = 0, ORC_PH_COPYQO = 1, ORC_PH_PRIM = 2, ORC_PH_TIMESTEP = 3,
  ORC_PH_VISCOUS = 4, ORC_PH_FLUXES = 5, ORC_PH_GCBC = 6, ORC_PH_SPONGE = 7,
  ORC_PH_RKUPDATE = 8, ORC_PH_WALL = 9, ORC_PH_AVERAGE = 10, ORC_PH_ADVANCE = 11,
  ORC_PH_MOVEF_A = 12,
  ORC_PH_GCBC_SETUP = 13, ORC_PH_GCBC_COMM_UPDATE = 14 /* ORC_PH_GCBC in two parts */
};

#ifdef __cplusplus
}
#endif
#endif
