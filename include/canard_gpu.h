/*
 * canard_gpu.h — C ABI of the B200 implementation of Canard's per-step hot path.
 *
 * The entry points replace the reference's Fortran type-bound procedures on the
 * time-step path (EnricoDeg/Canard):
 *   t_numerics%mpigo / deriv / filte        src/mo_numerics.f90:429-987
 *   t_physics%calc_viscous_shear_stress     src/mo_physics.f90:216-301
 *   t_physics%calc_fluxes                   src/mo_physics.f90:306-402
 *   t_physics%calc_time_step                src/mo_physics.f90:171-211
 *   gcbc_setup / gcbc_comm / gcbc_update     src/mo_gcbc.f90:133-340
 *   average_surface                         src/mo_gcbc.f90:342-422
 *   t_domdcomp%average_point / average_line src/mo_domdcomp.f90:439-559
 *   spongego                                src/mo_sponge.f90:75-88
 *   the time loop body (filter, RK stages)  src/mo_canard_driver.f90:226-431
 * and the set-up they depend on (t_grid%grid_metrics src/mo_grid.f90:52-189,
 * gcbc_init src/mo_gcbc.f90:40-131, spongeup src/mo_sponge.f90:34-71,
 * search_point / search_line src/mo_domdcomp.f90:269-437, init_extra / init
 * src/mo_numerics.f90:114-249).
 *
 * Conventions: all integers are int32_t (the reference's ni), all reals double
 * (nr). Field arrays passed in or out are HOST pointers in the reference layout
 * q(0:lmx, ncols), column-major, l = (k*(let+1)+j)*(lxi+1)+i. Every block is
 * one sub-domain (the reference's nbpc = 1 per block). A context owns all device
 * memory; it is single-stream and not thread-safe (one context per host
 * thread), like the reference's t_numerics, which owns scratch lines.
 *
 * Every function returns CANARD_OK (0) or an error code; canard_last_error()
 * gives the message. A failed call leaves the context usable unless the code is
 * CANARD_ERR_CUDA.
 */
#ifndef CANARD_GPU_H
#define CANARD_GPU_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define CANARD_OK 0
#define CANARD_ERR_ARG 1         /* bad argument (index, size, NULL) */
#define CANARD_ERR_CUDA 2        /* CUDA runtime failure */
#define CANARD_ERR_NAN 3         /* dt == 0 after step 2 (the reference's "Canard: Overflow."), or a non-finite state */
#define CANARD_ERR_TIMEOUT 4     /* a bounded device wait gave up */
#define CANARD_ERR_UNSUPPORTED 5 /* configuration the path does not handle */
#define CANARD_ERR_STATE 6       /* call order (e.g. step before setup) */
#define CANARD_ERR_IO 7          /* a file could not be opened, read or written, or has another block's size */

#define CANARD_FP64 0            /* plain FP64 path, bit-identical to the reference's operation order */
#define CANARD_FP32_MIXED 1      /* FP32 line solves/fluxes, FP64 state, RK, metrics, LU */
#define CANARD_FP64_FAST 2       /* FP64 throughout, line solves split in two halves per line with FMA,
                                    the filter direction by direction over the five fields: not
                                    bit-identical, rounding-level differences (<= 1e-10 relative L2
                                    after 10 steps is the bound its tests hold) */

typedef struct canard_ctx canard_ctx;

/* One block: nml_domdcomp entries lximb/letmb/lzemb, nbbc, mbcd for block mb
 * (src/mo_domdcomp.f90:232-267). nbc[d][s], mbcd[d][s]: direction d = xi, eta,
 * zeta; side s = 0 (min), 1 (max). mbcd is the neighbour block within the same
 * case, -1 for none. */
typedef struct {
  int32_t lxi, let, lze;
  int32_t nbc[3][2];
  int32_t mbcd[3][2];
} canard_block_desc;

/* One case: nml_numerics (fltk, fltrbc), nml_physics (reoo, tempoo, amach1..3,
 * timf, nsmf), nml_canard (cfl), nml_sponge (szco) and the sponge geometry of
 * nml_gridgen (szth0, szth1, doml0, doml1); viscous selects the reference's
 * -DVISCOUS build. */
typedef struct {
  int32_t nblocks;
  int32_t viscous;
  double fltk, fltrbc;
  double reoo, tempoo, amach1, amach2, amach3, timf;
  int32_t nsmf;
  double cfl;
  double szco, szth0, szth1, doml0, doml1;
} canard_case_desc;

/* Field ids for canard_get_field / canard_set_field (ncols in brackets). */
enum {
  CANARD_F_QA = 0,    /* conserved state qa [5] */
  CANARD_F_QO = 1,    /* RK stage start qo [5] */
  CANARD_F_DE = 2,    /* de [5] */
  CANARD_F_P = 3,     /* pressure [1] */
  CANARD_F_SS1 = 4,   /* Sutherland viscosity ss(:,1) [1] */
  CANARD_F_XIM = 5,   /* metrics [3] */
  CANARD_F_ETM = 6,
  CANARD_F_ZEM = 7,
  CANARD_F_YACO = 8,  /* Jacobian [1] */
  CANARD_F_TAU = 9,   /* txx tyy tzz txy tyz tzx hxx hyy hzz [9] */
  CANARD_F_DRVA1 = 10, CANARD_F_DRVA2 = 11, CANARD_F_DRVA3 = 12, /* (nbsize,5,0:1) */
  CANARD_F_CM1 = 13, CANARD_F_CM2 = 14, CANARD_F_CM3 = 15         /* (nbsize,3,0:1) */
};

/* Phase ids for canard_phase (one piece of src/mo_canard_driver.f90:234-371). */
enum {
  CANARD_PH_FILTER = 0,   /* mpigo + filte, 5 fields x 3 directions (:234-250) */
  CANARD_PH_COPYQO = 1,   /* qo = qa (:252) */
  CANARD_PH_PRIM = 2,     /* primitives, p, Sutherland (:267-275) */
  CANARD_PH_TIMESTEP = 3, /* calc_time_step every 10th step + dt ramp (:278-294) */
  CANARD_PH_VISCOUS = 4,  /* calc_viscous_shear_stress (:297) */
  CANARD_PH_FLUXES = 5,   /* calc_fluxes (:301) */
  CANARD_PH_GCBC = 6,     /* gcbc_setup + gcbc_comm + gcbc_update (:307-315) */
  CANARD_PH_SPONGE = 7,   /* spongego (:321) */
  CANARD_PH_RKUPDATE = 8, /* movef + RK update (:325-334) */
  CANARD_PH_WALL = 9,     /* wall_condition_update (:342) */
  CANARD_PH_AVERAGE = 10, /* average_point, average_line, average_surface (:347-355) */
  CANARD_PH_ADVANCE = 11, /* n = n + 1, timo = timo + dt (:369-370) */
  CANARD_PH_MOVEF_A = 12  /* movef before time advancing (:261-263) */
};

/* Context life cycle. blocks holds the blocks of all cases back to back
 * (cases[0].nblocks entries first). Several cases make a batched context: the
 * cases advance together, each with its own dt. */
int canard_ctx_create(const canard_case_desc* cases, int32_t ncases,
                      const canard_block_desc* blocks, int32_t precision,
                      canard_ctx** out);
void canard_ctx_destroy(canard_ctx* ctx);
const char* canard_last_error(const canard_ctx* ctx);
/* Run all device work of this context on the given cudaStream_t (NULL = the
 * context's own stream). */
int canard_set_stream(canard_ctx* ctx, void* cuda_stream);

/* Grid, set-up, state. xyz is (0:lmx,3): x, y, z of every stored point
 * (replaces read_grid_parallel, src/mo_io.f90:151-180). canard_setup runs
 * grid_metrics on the device, then gcbc_init, the junction searches and
 * spongeup; call it once after every block's grid is uploaded. */
int canard_upload_grid(canard_ctx* ctx, int32_t icase, int32_t iblock, const double* xyz);
/* Sub-domains (the reference's nbpc > 1, src/mo_domdcomp.f90:85-232): the
 * case's blocks are then the ranks of its split input blocks, with code-40
 * faces between sub-domains of one block; nbpc[m][3] and mbcd[m][3][2] are the
 * input blocks' split and neighbours, sub[r] = (block, position along xi, eta,
 * zeta) of rank r, numbered as src/mo_domdcomp.f90:588-605 numbers them.
 * The junction averaging then follows search_point / search_line over the
 * input blocks. Call before canard_setup; a case with code-40 faces needs it. */
int canard_set_subdomains(canard_ctx* ctx, int32_t icase, int32_t nblocks, const int32_t* nbpc,
                          const int32_t* mbcd, const int32_t* sub);
int canard_setup(canard_ctx* ctx);
int canard_set_state(canard_ctx* ctx, int32_t icase, int32_t iblock, const double* qa);
int canard_get_state(canard_ctx* ctx, int32_t icase, int32_t iblock, double* qa);
int canard_get_field(canard_ctx* ctx, int32_t icase, int32_t iblock, int32_t field,
                     double* out, int64_t count);
int canard_set_field(canard_ctx* ctx, int32_t icase, int32_t iblock, int32_t field,
                     const double* in, int64_t count);

/* Time loop. canard_step advances every case nsteps full steps (filter, 4 RK
 * stages, junction averaging) with the reference's dt schedule; it returns
 * CANARD_ERR_NAN where the reference's loop would stop with "Overflow."
 * time6 = (n, ndt, dt, dts, dte, timo) of one case. */
int canard_step(canard_ctx* ctx, int32_t nsteps);
int canard_phase(canard_ctx* ctx, int32_t phase, int32_t nk);
/* nsteps time steps through host memory (no counterpart in the reference; a
 * driver that keeps the state on the host between steps, e.g. for a coupled
 * host-side code): before every step the state of each listed block (case
 * icase[k], block iblock[k]) is read from host[k], reference layout (0:lmx,5)
 * (pinned memory reaches the full link bandwidth), and after it the step's
 * result is written back to host[k]. The same as nsteps x (canard_set_state,
 * canard_step(1), canard_get_state), but the copies are pipelined: each block's
 * state moves in chunks on two streams of the context, and a chunk of one
 * step's result goes back in as the next step's input as soon as it has landed,
 * so both directions of the host link run at once. The arrays belong to the
 * call until it returns. */
int canard_step_host(canard_ctx* ctx, int32_t nsteps, int32_t nblocks, const int32_t* icase,
                     const int32_t* iblock, double* const* host);
/* The fluxes, GCBC, RK update or wall phase of stage nk with the stage's
 * scalars given by the caller, as the reference's routines receive them
 * (calc_fluxes reads this%umf, src/mo_physics.f90:319-321; gcbc_update takes
 * dt, umf, dudtmf, src/mo_gcbc.f90:222; the RK update uses dtk = dt/(5-nk),
 * src/mo_canard_driver.f90:336-345; wall_condition_update takes umf,
 * src/mo_gcbc.f90:424), for every case of the context, instead of the frame
 * motion and dt the device derives from its own time state. For per-routine
 * drop-in where the caller's time loop owns the time state. */
int canard_phase_with(canard_ctx* ctx, int32_t phase, int32_t nk, double dt, const double* umf,
                      const double* dudtmf);
int canard_get_time(canard_ctx* ctx, int32_t icase, double* time6);
int canard_set_time(canard_ctx* ctx, int32_t icase, const double* time6);

/* Restart files in the reference's format: one block per file, Fortran
 * direct-access records of 5 doubles (write_restart_file / read_restart_file,
 * src/mo_io.f90:184-271): record 1 = n, ndt, dt, dts, dte; record 2 = timo,
 * 0, 0, 0, 0; then one record qa(l, 1..5) per stored point l (i fastest,
 * then j, then k). time6 and qa(0:npts-1, 5) as elsewhere in this header.
 * canard_write_restart / canard_read_restart move one block's state and its
 * case's time state between the context and such a file; a file of another
 * block size returns CANARD_ERR_IO. */
int canard_restart_write_file(const char* path, const double* time6, const double* qa, int64_t npts);
int canard_restart_read_file(const char* path, double* time6, double* qa, int64_t npts);

/* Grid files in the reference's format (misc/gridZZZ.dat of block ZZZ): one
 * 24-byte record (x, y, z) per stored point, i fastest, then j, then k, as
 * the generators write them plane by plane (src/mo_gridgen.f90:536-570) and
 * read_grid_parallel reads them point by point (src/mo_io.f90:151-180, which
 * these replace on the host side; canard_upload_grid takes the result).
 * xyz is ss(0:npts-1, 3). A file of another size returns CANARD_ERR_IO. */
int canard_grid_write_file(const char* path, const double* xyz, int64_t npts);

/* Junction averaging of one case on the host (average_point, average_line,
 * average_surface: src/mo_domdcomp.f90:439-559, src/mo_gcbc.f90:342-422),
 * through the same averaging plans the device builds and applies, in the same
 * arithmetic; no device is used. ranks: the blocks, or with nbpc != NULL the
 * sub-domains of nblocks split blocks (nbpc[m][3], mbcd[m][3][2] of the
 * input's blocks, sub[r] = block, position along xi, eta, zeta; ranks
 * numbered as src/mo_domdcomp.f90:588-605 numbers them). qa[r]: rank r's state
 * (0:lmx, 5), averaged in place. For checking the plans without a GPU. */
int canard_average_host(int32_t nranks, const canard_block_desc* ranks, int32_t nblocks, const int32_t* nbpc,
                        const int32_t* mbcd, const int32_t* sub, double* const* qa);
/* The exchanges of one case as lists, for placing its ranks on several
 * devices (arguments as canard_average_host; no device is used). They are the
 * reference's message pattern between ranks: the interface contractions and
 * the drva exchange of mpigo / gcbc_comm (src/mo_numerics.f90:429-705,
 * src/mo_gcbc.f90:186-220) and the sources of average_point / average_line /
 * average_surface (src/mo_domdcomp.f90:439-559, src/mo_gcbc.f90:342-422).
 * kind 0: face links, 7 values each: receiving rank, direction nn (1..3),
 *   receiving side (0 start, 1 end), sending rank, sending side, lines, the
 *   sending face's boundary code;
 * kind 1, 2, 3: targets of the point, line and surface averaging, 4 values
 *   each: rank, point l (reference layout), first source, source count;
 * kind 4, 5, 6: their sources, 2 values each: rank, point l.
 * *n receives the number of values; with cap = 0 nothing else is written, else
 * out (cap values) receives them, CANARD_ERR_ARG if cap < *n. */
int canard_plan_export(int32_t nranks, const canard_block_desc* ranks, int32_t nblocks, const int32_t* nbpc,
                       const int32_t* mbcd, const int32_t* sub, int32_t kind, int64_t* out, int64_t cap,
                       int64_t* n);
int canard_grid_read_file(const char* path, double* xyz, int64_t npts);
int canard_write_restart(canard_ctx* ctx, int32_t icase, int32_t iblock, const char* path);
int canard_read_restart(canard_ctx* ctx, int32_t icase, int32_t iblock, const char* path);

/* Time-averaged recording and Tecplot output (src/mo_canard_driver.f90:373-425,
 * src/mo_io.f90:275-562). canard_record_enable(ctx, 1) allocates the average
 * qb of every block (5 FP64 fields, zeroed; 0 frees it). After each
 * canard_step(ctx, 1), canard_record_accumulate adds (dt/2)(qo + qa) to qb and
 * dt to the case's dtsum, as the reference's loop does every step. On an output
 * step, canard_record_output returns, per block of the case, the FP32 output
 * variables rho, u, v, w, p (vart[b]: 5 x (lxi+1)(let+1)(lze+1), variable by
 * variable, i fastest; velocities include the frame velocity) of qb / dtsum (of
 * qo after the first step) and the output time timo - dtsum/2, then resets qb
 * and dtsum. canard_plt_write writes one output in the reference's Tecplot
 * binary layout (data/nNNN.plt, n >= 0, 5 variables; n = -1: data/grid.plt
 * with x, y, z): dims holds (lxi+1, let+1, lze+1) per block, data[b] the
 * block's variables in the same layout as vart. The reference's names have
 * three digits: n <= 999 and at most 1000 blocks, else CANARD_ERR_ARG. */
int canard_record_enable(canard_ctx* ctx, int32_t on);
int canard_record_accumulate(canard_ctx* ctx);
int canard_record_output(canard_ctx* ctx, int32_t icase, float* const* vart, double* time_out);
int canard_plt_write(const char* path, int32_t n, int32_t nblocks, const int32_t* dims, double time,
                     const float* const* data);

/* The restart comparer (contrib/dcanard.f90:100-126): both files of npts
 * points are read and every value whose difference, relative to the first
 * file's value, exceeds wtol is counted in *nreported and, when report_path
 * is not NULL, written there as dcanard's line " i=<i8> j=<i8> v1=<e15.7>
 * v2=<e15.7> abs=<e15.7> rel=<e15.7>" (point index from 0, variable 1..5). */
int canard_restart_compare(const char* path1, const char* path2, int64_t npts, double wtol, const char* report_path,
                           int64_t* nreported);

/* Unit operations of t_numerics on host arrays, for case 0 (parity tests and
 * drop-in calls). fields[b] = rfield(0:lmx, ncols) of block b. mpigo computes
 * the interface contractions of every block face and exchanges them into the
 * receive buffers of field m (src/mo_numerics.f90:429-705); deriv and filte
 * then use them (src/mo_numerics.f90:709-987). deriv writes the line-end
 * values into drva (read them with CANARD_F_DRVA*). in and out may alias. */
int canard_mpigo(canard_ctx* ctx, const double* const* fields, int32_t ncols, int32_t nt,
                 int32_t nrt, int32_t n45, int32_t itag, int32_t m);
int canard_deriv(canard_ctx* ctx, int32_t iblock, const double* in, double* out,
                 int32_t nn, int32_t m);
int canard_filte(canard_ctx* ctx, int32_t iblock, double* f, int32_t inn, int32_t m);

/* Host-only coefficient tables (no GPU needed), as used by the kernels:
 * canard_coeffs writes pbci[nt][side][0:11], pbco[nt][side][0:11],
 * pbcot[nt][side], alphf, betf, fa, fb, fc, albef[n][row][-2:2],
 * fbc[row][0:4] (150 doubles; init_extracoeff_bounds, src/mo_numerics.f90:114-134).
 * canard_penta writes the LU factors of one line of n points, xu (n,3) and
 * xl (n,2) column-major (src/mo_numerics.f90:179-249). */
int canard_coeffs(double fltk, double fltrbc, double* out150);
int canard_penta(double fltk, double fltrbc, int32_t n, int32_t ns, int32_t ne, int32_t nt,
                 double* xu, double* xl);
int canard_version(void);

/* Isolated line-solve bench (no counterpart in the reference): nfields <= 5
 * fields of block 0 of case 0 (host arrays in the reference layout, field k
 * at in + k*(lxi+1)(let+1)(lze+1)) are copied to the device once; one launch
 * of the direction's derivative (op 0) or filter (op 1, in place) over all of
 * them runs after their interface contraction and its result is copied to
 * out; then `reps` more launches are timed with CUDA events on the context
 * stream and *ms_per_launch receives their average. In a mixed-precision
 * context the derivative runs on FP32 copies, the filter on the FP64 fields
 * with an FP32 elimination, as on the step path. */
int canard_line_bench(canard_ctx* ctx, int32_t op, int32_t nn, int32_t nfields, const double* in, double* out,
                      int32_t reps, double* ms_per_launch);

/* Line-tile autotuner (no counterpart in the reference). For each group of
 * line solves (0: the filter passes, 1: the viscous gradients, 2: the flux
 * derivatives) and direction, times the candidate tile shapes on the
 * context's own blocks (filter candidates on scratch copies, the state is not
 * touched): FP64 contexts try TMA staging depths (2, 4, 8 chunks per eta or
 * zeta line) and, on eta/zeta lines of 16..257 points, the kernel that keeps
 * the elimination results in tensor memory; mixed-precision contexts also try
 * the one-lane FP32 sweeps (32 lines per tile) against the split solve (16
 * lines per tile), and for the filter, which filters the FP64 state with an
 * FP64 right-hand side in every kind, the FP64 eliminations (one-lane and
 * split) as well; fast FP64 contexts try the split FP64 solve against the
 * one-lane FP64 sweeps. Where every block's lines along the direction have at
 * least 32 points, the two-ended solves (kinds 10-12) compete too. The
 * fastest choice is installed in the step tables. Returns the number of groups
 * (9) and fills up to nmax report rows of 6 doubles: group, direction
 * (0..2), chosen kind, chosen chunk count (0 = default), its ms per launch
 * and the default's. Call after canard_setup. */
int canard_autotune(canard_ctx* ctx, int32_t reps, double* report, int32_t nmax);

/* Pins the line kernel of one group (0 filter, 1 viscous gradients, 2 flux
 * derivatives) and direction (0..2), as canard_autotune would install it (no
 * counterpart in the reference): kind 0 FP64 tiles in shared memory (chunks:
 * 0 default or 2..8 TMA stages), 1 FP32 split, 2 FP64 tile / FP32 split, 3
 * FP32 one-lane, 4 FP64 tile / FP32 one-lane, 5 FP64 with the elimination
 * results in tensor memory (eta/zeta, 16..257 points per line), 6 the filter
 * of the FP64 state streamed into FP32 right-hand sides (mixed precision), 7
 * FP64 split solve with FMA (FP64 and fast FP64 contexts; the fast mode's
 * default on lines under 32 points), 8 and 9 the derivative's quad split solve (four lanes per line) on
 * FP64 fields (FP64 and fast FP64 contexts) and on FP32 fields (mixed
 * precision), for lines of at least about 4 x 60 points (FP64) or 4 x 40
 * (FP32); 10, 11 and 12 the two-ended solve (two warps per tile of 32 lines,
 * one eliminating from each end of the line, the four unknowns where they
 * meet from a 4 x 4 inverse; lines of at least 32 points) with FP64 fields and
 * elimination (FP64 and fast FP64 contexts, and the filter of mixed-precision
 * ones), FP32 fields (derivatives, mixed precision) and the FP64 state with an
 * FP32 elimination (filter, mixed precision); -1 restores the precision's
 * default. Kinds 0 and 5 give results bit-identical to the reference's
 * operation order; kinds 7, 8 and 10 differ from them at the rounding level.
 * A kind
 * the context's precision or line lengths do not admit returns
 * CANARD_ERR_ARG. Before canard_setup the choice only applies to
 * canard_line_bench (the step tables are built by canard_setup). */
int canard_set_line_kind(canard_ctx* ctx, int32_t group, int32_t dir, int32_t kind, int32_t chunks);

/* Observability (the reference's mo_timer, src/mo_timer.f90:84-133, as CUDA
 * events per kernel family). With timers on, every launch of the family is
 * bracketed by events; canard_get_timers returns per family the accumulated
 * device milliseconds, the number of launches and the algorithmic bytes moved
 * (unique reads + writes of the launch's fields), and the number of families.
 * canard_timer_name gives a family's name. canard_launch_count returns the
 * number of kernel launches this context issued since it was created. */
int canard_set_timers(canard_ctx* ctx, int32_t on);
int canard_get_timers(canard_ctx* ctx, double* ms, double* launches, double* bytes, int32_t nmax);
const char* canard_timer_name(int32_t family);
int canard_launch_count(canard_ctx* ctx, int64_t* count);

/* Self-test of the bounded device waits (no counterpart in the reference):
 * runs one kernel whose mbarrier wait can never complete. Like every wait of
 * the line kernels it gives up after 0.5 s and raises the context's error
 * flag, so the call returns CANARD_ERR_TIMEOUT, with *seconds (may be NULL)
 * the host time it took; the flag is cleared and the context stays usable.
 * Line kernels launched while the flag is up return without work. */
int canard_selftest_wait(canard_ctx* ctx, double* seconds);

/* Step execution. canard_step runs each time step as one CUDA graph (captured
 * on the first step of each kind: with and without the every-tenth-step dt
 * reduction) whose kernels read the device-resident time state, so a step
 * costs one host call and no host synchronisation. With graphs off (or the
 * timers on) the same kernels are launched one by one. The reference has no
 * counterpart; the results are identical either way. Default: on. */
int canard_set_graphs(canard_ctx* ctx, int32_t on);

/* Compact first derivative without device allocation. This entry point has no
 * counterpart in the reference. It serves callers that cannot allocate device
 * memory: solvers that own every device buffer themselves, code under a memory
 * budget that forbids allocator calls between steps, and host threads that
 * must not block in the allocator. It computes what canard_mpigo + canard_deriv
 * compute for one block, on DEVICE arrays, enqueued on `stream`:
 *   d_in, d_out   device fields, element (i,j,k) at (k*(let+1)+j)*pitch + i,
 *                 16-byte aligned, pitch >= lxi+1 and a multiple of 4; in may
 *                 equal out; pad columns of out may be overwritten
 *   nn            direction (1 xi, 2 eta, 3 zeta)
 *   nbc0, nbc1    end closures: 10/20/25/30 one-sided, 45 periodic on the line
 *                 itself (both ends)
 *   fltk, fltrbc  nml_numerics values (fix the interface coefficients)
 * Limits: a line of the direction must fit the FP64 shared-memory tile, at
 * most 906 points along xi and 896 along eta or zeta, and the direction may
 * have at most 65536 lines; larger sizes return CANARD_ERR_ARG before any
 * work is queued. The scratch is one static device array of about 2.1 MiB
 * that every GPU loading the library holds until the process exits. Every
 * call reuses it and leaves its last contents there, so calls that overlap on
 * the GPU (on different streams) race. The first call on a device looks up
 * the array's device address with that device current and caches it; make
 * that first call before any stream capture. No cudaMalloc, cudaFree or other
 * allocating routine is called. The return code covers the arguments and the
 * queuing; the kernels' own status is read with canard_deriv_noalloc_status. */
int canard_deriv_noalloc(const double* d_in, double* d_out, int32_t lxi, int32_t let, int32_t lze,
                         int32_t pitch, int32_t nn, int32_t nbc0, int32_t nbc1, double fltk,
                         double fltrbc, void* stream);
/* Status of the allocation-free derivative's kernels (no counterpart in the
 * reference): waits for `stream`, then returns CANARD_ERR_TIMEOUT if a line
 * kernel's bounded wait for its input copies gave up since the last status
 * call (its output is then incomplete), else CANARD_OK, and clears the flag.
 * While the flag is up, later canard_deriv_noalloc calls skip their line
 * solve. Allocates nothing. */
int canard_deriv_noalloc_status(void* stream);

#ifdef __cplusplus
}
#endif
#endif
