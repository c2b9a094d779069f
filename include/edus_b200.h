/*
 * edus_b200.h — C ABI of the B200-native k-space density-matrix propagator.
 *
 * Plain C types only (pointers, sizes, doubles). Complex numbers are passed
 * as interleaved (re, im) double pairs. Every function returns 0 on success
 * or a negative EDUS_E* code; edus_strerror() turns a code into text and
 * edus_last_error() gives the message of the last failure on this thread.
 *
 * Reference seams replaced (anpicon/EDUS, paths relative to its root):
 *   input.txt reader ............ headers/ReadInput.h:332-815 (Read_Input)
 *   k grid / b shells ........... headers/InitParameters.h:1-40, headers/CalculateWeigths.h:1-226
 *   k partition ................. headers/Organize_kspaceMPI.h:242-301 (one device-resident grid here)
 *   H, U, D tabulation .......... Source_Main/save_HUD.cpp:19-53, headers/HUD.h:5-20
 *   RHS ......................... headers/RungeKutta.h:7-297 (get_derivative_Df)
 *   stage updates ............... headers/RungeKutta.h:301-355 (Runge_Kutta_Ad / Runge_Kutta_Ac)
 *   RK4 / AB / Taylor drivers ... Source_Main/RungeKutta.cpp, Source_Main/Linear_Multistep_ODE_solvers.cpp,
 *                                 Source_Main/Taylor_DE_solver_deriv_Polynom.cpp, headers/ODE_solver.h
 *   time loops .................. Source_Main/const_dt_evolution.cpp, Source_Main/dyn_dt_evolution.cpp
 *   Coulomb mean field .......... headers/Coulomb.h:273-541, Source_Main/Fourier_Coulomb.cpp:505-622
 *   observables ................. headers/Observables_MPI.h:134-140,217-484,559-598,668-775
 */
#ifndef EDUS_B200_H
#define EDUS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EDUS_ABI_VERSION 1

/* ---------------------------------------------------------------- errors */
enum {
  EDUS_OK = 0,
  EDUS_EINVAL = -1,       /* bad argument / inconsistent problem */
  EDUS_ENOMEM = -2,       /* host or HBM allocation failed, or HBM budget exceeded */
  EDUS_ECUDA = -3,        /* CUDA runtime error */
  EDUS_ENONFINITE = -4,   /* health check: non-finite rho */
  EDUS_ETRACE = -5,       /* health check: trace drift above tolerance */
  EDUS_ETIMEOUT = -6,     /* bounded device wait ran out */
  EDUS_ECANCELLED = -7,   /* request cancelled */
  EDUS_EIO = -8,          /* file could not be read or written */
  EDUS_EPARSE = -9,       /* input.txt grammar error (the reference exits(1) there) */
  EDUS_EUNSUPPORTED = -10,/* option the reference has that is not built here */
  EDUS_ENOTREADY = -11    /* result not available yet (serving poll) */
};

/* ---------------------------------------------------------------- enums */
enum { EDUS_MODE_TB = 1, EDUS_MODE_WANNIER = 2, EDUS_MODE_CRYSTAL = 3 };
enum { EDUS_SOLVER_RK4 = 0, EDUS_SOLVER_AB = 1, EDUS_SOLVER_TAYLOR = 2 };
enum { EDUS_ENV_NONE = 0, EDUS_ENV_SIN2 = 1, EDUS_ENV_GAUSS = 2, EDUS_ENV_PW = 3 };
enum { EDUS_PREC_FP64 = 0, EDUS_PREC_MIXED = 1 };

#define EDUS_MAX_PUMPS 8
#define EDUS_MAX_HOPPING 8
#define EDUS_MAX_BANDS 16
#define EDUS_MAX_TABSK 64  /* k points of a TAbsK section */
#define EDUS_STRLEN 256

/* One laser pulse with every derived quantity resolved (headers/Laser.h:1-51).
 * Polarisation vectors are Cartesian and already Gram–Schmidt-orthogonalised
 * as Laser::set_pol does (headers/Laser.h:82-106). */
typedef struct {
  int32_t envelope_kind;  /* EDUS_ENV_* (Laser::gaussian / sin2 / PW) */
  int32_t envelope_only;  /* Laser::envelope: no carrier oscillation (probe) */
  double wl;              /* angular frequency, a.u. */
  double period;          /* 2 pi / wl */
  double lambdanm;
  double intensity;       /* W/cm^2 */
  double A0, E0;          /* a.u.; A0 = sqrt(I / 3.51e16) / wl, E0 = A0 wl */
  double t0, tf;          /* a.u. */
  double ncycle, sigma;   /* sin2 cycles / gaussian sigma (a.u.) */
  double w1, w2;          /* pseudo plane wave window */
  double phase;           /* carrier envelope phase */
  double pol1[3], pol2[3];
} edus_laser;

/* Everything input.txt says, resolved to atomic units (the reference's
 * globals after Read_Input + BZ_parameters). */
typedef struct {
  char ref_coord[EDUS_STRLEN];   /* first token; Wannier file stem <ref_coord>_tb.dat */
  int32_t mode;                  /* EDUS_MODE_* */
  char tb_type[64];              /* TightBinding::_name */
  double hopping[EDUS_MAX_HOPPING];
  int32_t n_hopping;
  double a[3][3];                /* direct lattice rows, a.u. */
  double b[3][3];                /* reciprocal lattice rows, a.u. */
  int32_t nk[3];                 /* Monkhorst–Pack grid */
  int32_t nb[3];                 /* core, valence, conduction band counts */
  double conduction_shift;       /* scissor, a.u. (bands{conduction_shift}) */
  double fermi_energy;
  /* tdse */
  double dt, t_fin;              /* a.u. */
  int32_t solver;                /* EDUS_SOLVER_* */
  int32_t order;                 /* Adams–Bashforth / Taylor order (SolverOrder) */
  int32_t dynamical_dt;
  double eps_step_abs;
  int32_t ab_rk4_startup;        /* extension: RK4 start-up for AB (reference: 0, zero history) */
  double gap_correction;
  /* lasers */
  int32_t n_pumps;
  edus_laser pump[EDUS_MAX_PUMPS];
  edus_laser probe;
  double delay;
  /* decoherence (headers/InitParameters.h:203-224) */
  double T1, T2, Tch;
  /* observables */
  int32_t current, tabs, it_resolution;
  int32_t print_population;
  double print_start, print_end, print_step;
  /* Coulomb */
  int32_t coulomb;
  int32_t ncut;
  double qTF, r0, epsilon_static, G_distance;
  int32_t rytova_keldysh, diag_basis, read_from_files, print_band_dispersion;
  char coulomb_label[EDUS_STRLEN];
  int32_t sample_110;            /* sample in xy ("110") instead of yz ("011") */
  int32_t vectorization;
  /* execution options (not in the reference) */
  int32_t precision;             /* EDUS_PREC_* */
  /* k-resolved transient absorption (observables{kTAbs} and the TAbsK
   * section): the reference reads the k points and opens one file per point,
   * Output/TAbsK_<k0>_<k1>_<k2>.txt, that nothing writes into */
  int32_t tabs_k;
  int32_t n_tabs_k;
  double tabs_k_pts[EDUS_MAX_TABSK][3];
  /* nkpt read: the k points are listed in the input file after the grid
   * sizes (headers/ReadInput.h:420-440); set-up reads them from input_path */
  int32_t kpt_read;
  int64_t kpt_offset;            /* byte offset of the first listed k point in input_path */
  char input_path[EDUS_STRLEN];
  /* extension (tdse{ velocity_gauge }): Wannier models integrated in the
   * frame that moves with the vector potential, rho'(k) = rho(k + A(t)), with
   * H and D evaluated at k + A(t) every stage and no k-gradient term; the
   * reference integrates the length gauge only */
  int32_t velocity_gauge;
} edus_params;

/* Observables at one output instant (headers/Observables_MPI.h). */
typedef struct {
  double t;                      /* a.u. */
  double EF_pump[3];             /* field printed to EF.txt */
  double EF_probe[3];            /* field printed to TransientAbs.txt */
  double J1[6];                  /* complex J1 x,y,z (re, im), Current1 */
  double J2[3];                  /* -2 Im(...), Current2 */
  double pop[EDUS_MAX_BANDS];    /* Losses.txt columns */
  double tabs[6];                /* complex TAbs / nktot */
  double trace_dev;              /* sum of populations - (Nch + Nv) */
  double p_cond_max;             /* P_cond_max_loc */
  double p_min;                  /* Coulomb_set.P_min */
  double n_cond;
  double dt;                     /* step used after this instant (adaptive dt) */
  double pol[6];                 /* extension: polarisation per cell, complex (1/Nk) sum_k Tr(D_x rho(k)),
                                    x,y,z (re, im), a.u.; the reference has no such output */
} edus_obs;

/* ------------------------------------------------------- input.txt layer */
/* Parse input.txt (headers/ReadInput.h:332-815 grammar, BZ_parameters laser
 * resolution headers/InitParameters.h:1-11). */
int edus_parse_input(const char* path, edus_params* out);
int edus_params_default(edus_params* out);   /* Source_Main/variables.cpp defaults */

/* ------------------------------------------------------- problem (host) */
typedef struct edus_problem edus_problem;

typedef struct {
  int32_t ncv, nch, nv, nc;
  int32_t nk;                /* k points */
  int32_t n1, n2;            /* in-plane grid (rows, columns) */
  int32_t nshell, nnb;       /* b-vector shells, total neighbours per k */
  int32_t nrpts;             /* Wannier R vectors (0 for TB) */
  int32_t n_diss;            /* non-zero dissipation entries */
  int32_t nsteps;            /* itfi + 1 for constant dt */
  int32_t nprint;            /* output instants for constant dt */
  double t_start;            /* -0.21 fs in a.u. */
  double det_a, jacobian;
  double dk[3];
} edus_problem_info;

/* Build the problem on the host: grid, shells, neighbour table, model tables
 * (H, U, D on the grid, GradientEnergy), dissipation tensor, initial state,
 * Coulomb coefficient files. workdir holds <ref>_tb.dat and Output/Coulomb/. */
int edus_problem_create(const edus_params* p, const char* workdir, edus_problem** out);
int edus_problem_info_get(const edus_problem* pb, edus_problem_info* out);
/* As edus_problem_create, but a Wannier model is not tabulated on the host:
 * H(k), D(k), U(k), dH/dk and the initial state are built on the device when
 * the problem is admitted to a batch (seconds of host work become
 * milliseconds of device work). Single-solve contexts need host tables and
 * refuse such a problem. Tight-binding models are tabulated as usual. */
int edus_problem_create_deferred(const edus_params* p, const char* workdir, edus_problem** out);
/* Remove the core bands when nothing in the run couples them to the other
 * bands (no probe, no dissipation, no Coulomb, no H / dH/dk entries and no
 * dipole component along the pump between core and the rest). The remaining
 * bands then evolve exactly as in the full problem, with fewer elements per
 * k point (the Haldane_CoreBN models with an in-plane pump become 2-band).
 * EDUS_EUNSUPPORTED (problem unchanged) when a coupling exists. No
 * counterpart in the reference. */
int edus_problem_drop_decoupled_core(edus_problem* pb);
/* Copy a named host array out (names: "kpt","H","U","D","GE","P0","nbr",
 * "weights","bvec","T","wq_A","wq_B","wq_C","wq_D","screen","vhartree",
 * "HR","rR","Rvec"); nbytes must match exactly. */
int edus_problem_get(const edus_problem* pb, const char* name, void* dst, size_t nbytes);
void edus_problem_free(edus_problem* pb);
/* Write outdir/k_grid.txt (outdir created if missing): the crystal
 * coordinates of every k point, one "k0 k1 k2" line each in the default C++
 * stream format, as the reference's print_k_MPI (headers/Observables_MPI.h:
 * 492-550) writes Output/k_grid.txt. edus_write_outputs writes it too. */
int edus_problem_write_kgrid(const edus_problem* pb, const char* outdir);
/* Write workdir/kpt.txt ("ik i0 i1 i2 k0 k1 k2" per k point), the grid listing
 * the reference's BZ_parameters leaves in its working directory
 * (headers/InitParameters.h:17-39); edus_run writes it at set-up. */
int edus_problem_write_kpt(const edus_problem* pb, const char* workdir);
/* Write workdir/Test_matrices.txt: H, U, U H U^dagger, U U^dagger and the
 * dipoles at crystal k = (0, 0.3, 0.1), as the reference's set-up prints them
 * (Source_Main/test_matrix_k.cpp); edus_run writes it at set-up. */
int edus_problem_write_test_matrices(const edus_problem* pb, const char* workdir);
/* H(k), U(k) and D(k) of the problem's model at one crystal k point, as
 * gHUD (headers/HUD.h:5-20) returns them: H, U [n][n], D [n][n][3] interleaved
 * complex. */
int edus_model_hud(const edus_problem* pb, const double kcrys[3], double* H, double* U, double* D);
/* sizeof of the ABI structs: params, obs, problem_info, options (for bindings). */
int edus_struct_sizes(int64_t out[4]);

/* --------------------------------------------- Coulomb coefficient generator */
typedef struct {
  int32_t device;        /* CUDA device ordinal */
  int32_t n_sum;         /* Simpson points per axis of the coefficient fit (reference: 4999) */
  int32_t n_sum_screen;  /* ... of the screening constant (reference: 39999) */
} edus_coulomb_gen_options;
int edus_coulomb_gen_options_default(edus_coulomb_gen_options* o);
/* Compute the Coulomb tables of a run on the GPU, as the reference does when
 * its Coulomb section has no Read_Coulomb_from_files
 * (Source_Main/Fourier_Coulomb.cpp:95-500): the Fourier coefficients A, B, C, D
 * of the lattice-summed Thomas-Fermi / Rytova-Keldysh interaction (Simpson
 * integrals over the zone, every reciprocal vector inside G_distance), the
 * Hartree table and the screening constant. Writes
 * workdir/Output/Coulomb/{A,B,C,D}_coeff<label>.txt, V_Hartree_<label>.txt and
 * Screen_const_<label>.txt in the reference's formats, label =
 * "G_num<G>_Ncut<Ncut><labelInput>" (returned in label_out, the number of G
 * vectors in g_num_out); a run reads them with Read_Coulomb_from_files and
 * labelInput <label>. Up to 4 bands; opt may be null (the reference's grids). */
int edus_coulomb_generate(const edus_params* p, const char* workdir, const edus_coulomb_gen_options* opt, char* label_out,
                          int32_t label_cap, int32_t* g_num_out);

/* ------------------------------------------------------- device context */
typedef struct edus_ctx edus_ctx;

typedef struct {
  int32_t device;            /* CUDA device ordinal */
  int32_t precision;         /* EDUS_PREC_*; overrides params.precision if >= 0 */
  int32_t use_graphs;        /* capture step chunks in CUDA graphs */
  int32_t health_checks;     /* device-side non-finite / trace checks */
  double trace_tol;
  int64_t hbm_budget_bytes;  /* 0 = unlimited */
} edus_options;

int edus_options_default(edus_options* o);
/* Upload the problem and allocate all device state. */
int edus_create(const edus_problem* pb, const edus_options* opt, edus_ctx** out);
void edus_destroy(edus_ctx* ctx);

/* Restore the initial state (ground-state projector, zero multistep history)
 * and the clock (it = 0, t = -0.21 fs); the next edus_run replays the CUDA
 * graph captured by the first one. */
int edus_reset(edus_ctx* ctx);

/* State in the reference layout P[k][i][j], interleaved complex128. */
int edus_set_state(edus_ctx* ctx, const double* rho);
int edus_get_state(edus_ctx* ctx, double* rho);

/* Advance nsteps of the configured integrator from the current (it, t, dt).
 * Reproduces one iteration of the reference time loop per step
 * (Source_Main/const_dt_evolution.cpp:10-55, dyn_dt_evolution.cpp:28-183),
 * including the output instants every it_resolution steps, which are
 * appended to the context's observable log. */
int edus_step(edus_ctx* ctx, int32_t nsteps);
/* Run the whole time loop (itfi+1 steps for constant dt). */
int edus_run(edus_ctx* ctx);
/* Clock of the loop: iteration index, time (a.u.), current dt. */
int edus_clock(edus_ctx* ctx, int32_t* it, double* t, double* dt);
/* Number of logged output instants and a copy of them. */
int edus_obs_count(edus_ctx* ctx, int32_t* n);
int edus_obs_get(edus_ctx* ctx, int32_t first, int32_t count, edus_obs* out);
/* Observables of the current state (does not append to the log). */
int edus_observables(edus_ctx* ctx, edus_obs* out);
/* Same result as edus_observables, but the call allocates no memory: the
 * reduction scratch (per-block partial sums, the arrival counter that starts
 * at zero, the output record) lives in a fixed device array inside the
 * library. For callers that cannot take an allocation at this point: a
 * serving loop whose HBM is fully committed to admitted solves, or a caller
 * that must not run into the device-wide synchronisation a device
 * free brings. No reference counterpart.
 * Limits: at most 524 288 k points (4096 partials of 128 k points), else
 * EDUS_EINVAL. The first call on a device looks the array up on that device
 * (make it outside any stream capture); the address is kept until the process
 * ends, so no call may follow a cudaDeviceReset of that device. The array is
 * shared by every context on a device: calls that overlap in time (two host
 * threads, or two streams) race on it and must be serialised by the caller. */
int edus_observables_static(edus_ctx* ctx, edus_obs* out);
/* Failure-path self-test of the kernels' bounded waits: one kernel waits, with
 * the same bounded wait the bulk-copy kernels use but cut to `iters` polls, on
 * an mbarrier nothing arrives on (no copy is issued), records the timeout in
 * the device error word and returns. Expected result EDUS_ETIMEOUT, with the
 * device still usable. No reference counterpart. */
int edus_selftest_bounded_wait(int32_t device, int32_t iters);
/* Write Output/{EF,J1,J2,Losses,TransientAbs,k_grid}.txt in the reference's
 * format, the per-k files of the first output step (H_Eigen_*, H_Wannier_cond,
 * P_initial_Wannier_, Uk_) and, when the input asks for them, the snapshot
 * files (P_*_in_Eigenstate_*, Edia_*, t_Ek.txt) taken during edus_run. */
int edus_write_outputs(edus_ctx* ctx, const char* outdir);
/* Device time (ms, CUDA events) of the last edus_step/edus_run call and the
 * number of kernel launches it issued. */
int edus_last_timing(edus_ctx* ctx, double* ms, int64_t* launches);
/* Run nsteps eagerly with CUDA events around every launch of the fused
 * RHS + stage-update kernel and of the Coulomb transform pair; returns their
 * summed device times (ms) and launch counts. */
int edus_profile(edus_ctx* ctx, int32_t nsteps, double* rhs_ms, int64_t* rhs_launches, double* coul_ms,
                 int64_t* coul_launches);
/* As edus_profile, with every RHS launch whose result does not depend on its
 * own output (AB, Taylor and Pv launches) repeated reps times back to back
 * between its events: the launch-count-weighted average is the kernel's
 * duration in a pipeline, without one event pair's overhead per launch. The
 * repeats leave the state as one launch would. */
int edus_profile_ex(edus_ctx* ctx, int32_t nsteps, int32_t reps, double* rhs_ms, int64_t* rhs_launches, double* coul_ms,
                    int64_t* coul_launches);

/* --------------------------------------------- ODE_solver-level mirror
 * Slots name device arrays of the state shape: 0 = P0, 1 = P1, 2 = P2,
 * 3 = Pv. These replace the reference's per-thread calls one for one. */
enum { EDUS_SLOT_P0 = 0, EDUS_SLOT_P1 = 1, EDUS_SLOT_P2 = 2, EDUS_SLOT_PV = 3 };
/* get_derivative_Df (headers/RungeKutta.h:7-297): Pv = RHS(P_slot).
 * EF = {pump x,y,z, probe x,y,z} as the reference's EF[0], EF[1]. */
int edus_get_derivative(edus_ctx* ctx, int32_t p_slot, const double EF[6], double wx2, int32_t e_non0);
/* Runge_Kutta_Ad (headers/RungeKutta.h:301-328): P_dst = P_src + dt * Pv. */
int edus_runge_kutta_ad(edus_ctx* ctx, int32_t src, int32_t dst, double dt);
/* Runge_Kutta_Ac (headers/RungeKutta.h:331-355): P_dst += dt * Pv. */
int edus_runge_kutta_ac(edus_ctx* ctx, int32_t dst, double dt);
/* Copy one slot to another (host-side bookkeeping the reference does by assignment). */
int edus_slot_copy(edus_ctx* ctx, int32_t src, int32_t dst);
int edus_slot_set(edus_ctx* ctx, int32_t slot, const double* rho);
int edus_slot_get(edus_ctx* ctx, int32_t slot, double* rho);
/* Coulomb mean field of slot P: X(k) as the reference adds it to H
 * (headers/Coulomb.h:273-541 + headers/RungeKutta.h:69-138): writes
 * Hk_renorm[k][n][n] (interleaved) to hk_out. */
int edus_coulomb_hk(edus_ctx* ctx, int32_t p_slot, double* hk_out);

/* ------------------------------------------------------- batches
 * Many independent solves (pulse sweeps, served requests) advanced together
 * on one GPU. No counterpart in the reference, which runs one solve per MPI
 * job. Every instance keeps its own state and tables in HBM; all active
 * instances step in lockstep, one RK4 step per tick, and a chunk of ticks is
 * replayed from one CUDA graph of persistent kernels. Instances join and
 * leave only between chunks. Supported per instance: RK4 at constant dt,
 * band counts 2, 3, 4, 5, 8, 16, no Coulomb mean field, no dissipation
 * (others: EDUS_EUNSUPPORTED). */
typedef struct edus_batch edus_batch;

typedef struct {
  int32_t device;
  int32_t precision;        /* EDUS_PREC_FP64 or EDUS_PREC_MIXED (FP32 H, D, commutator; FP64 rho) */
  int32_t max_instances;    /* slots */
  int32_t chunk_steps;      /* time steps per graph replay (even) */
  int32_t use_graphs;
  int32_t tile_k[EDUS_MAX_BANDS + 1]; /* k points per tile by band count; 0 = default */
  int32_t regs_profile[EDUS_MAX_BANDS + 1]; /* stage-kernel form by band count: 0 = element-parallel,
                                               56 registers; 1 = element-parallel, more registers;
                                               2 = matrix-product form (FP64; 8 and 16 bands);
                                               3 = staged (cp.async one tile ahead; mixed);
                                               4 = staged with the register-blocked commutator
                                               (mixed; 8 and 16 bands), 2 x 2 blocks of C per thread;
                                               5 = the same with 2 x 1 blocks. 3-5 fall back to 0 for
                                               an instance without a lattice stencil */
  int32_t tc_contraction;   /* mixed precision: deferred Wannier models contracted on the tensor
                               cores (exact BF16 slices, FP32 sums exact per segment, FP64 across
                               segments; band energies FP64) */
  int32_t pad;
  int64_t hbm_budget_bytes; /* admission limit; 0 = 90 % of the free device memory at create */
} edus_batch_options;

enum { EDUS_INST_FREE = 0, EDUS_INST_RUNNING = 1, EDUS_INST_DONE = 2 };

typedef struct {
  int64_t ticks;            /* time steps advanced by the batch */
  int32_t active, done, free_slots, pad;
  int64_t bytes_used, bytes_budget;
  double device_ms;         /* CUDA-event time of all chunk replays */
  double kpoint_steps;      /* k-point steps advanced (sum over instances) */
  int64_t launches;         /* kernel launches replayed */
  int64_t h2d_bytes;        /* bytes copied host -> device by admissions (tables, state, field, descriptor) */
  int64_t d2h_bytes;        /* bytes copied device -> host by edus_batch_obs_get / edus_batch_get_state */
} edus_batch_stats;

/* One kernel of a profiled advance: the band-count class, the kernel (0 =
 * observables, 1-4 = RK4 stage 0-3), its launches, their summed CUDA-event
 * time, and the k points of the class per launch. */
typedef struct {
  int32_t nbands, kind;
  int64_t launches;
  double total_ms;
  int64_t kpoints;
} edus_kernel_time;

int edus_batch_options_default(edus_batch_options* o);
int edus_batch_create(const edus_batch_options* o, edus_batch** out);
void edus_batch_destroy(edus_batch* b);
/* HBM bytes an instance of this problem takes in this batch. */
int edus_batch_footprint(edus_batch* b, const edus_problem* pb, int64_t* bytes);
/* Admit a solve: uploads its tables and initial state; it starts at the next
 * tick. EDUS_ENOMEM when the budget or the slots are used up (nothing is
 * changed then). */
int edus_batch_add(edus_batch* b, const edus_problem* pb, int64_t tag, int32_t* slot);
/* Advance every running instance by nsteps time steps (rounded up to whole
 * chunks); instances that reach the end of their time grid become DONE. */
int edus_batch_advance(edus_batch* b, int32_t nsteps);
int edus_batch_poll(edus_batch* b, int32_t slot, int32_t* status, int32_t* it, int64_t* tag);
int edus_batch_obs_count(edus_batch* b, int32_t slot, int32_t* n);
int edus_batch_obs_get(edus_batch* b, int32_t slot, int32_t first, int32_t count, edus_obs* out);
/* State of a slot in the reference layout P[k][i][j] (interleaved complex128). */
int edus_batch_get_state(edus_batch* b, int32_t slot, double* rho);
/* Free a slot and its device memory. */
int edus_batch_release(edus_batch* b, int32_t slot);
int edus_batch_stats_get(edus_batch* b, edus_batch_stats* out);
/* Tile length in use for a band count (after the autotuner). */
int edus_batch_tile_k(edus_batch* b, int32_t nbands, int32_t* kt);
/* Advance like edus_batch_advance, but launch every kernel eagerly (no graph)
 * between its own pair of CUDA events on the batch's stream; per (class,
 * kernel) totals go to out[0 .. *n), at most cap entries. For measurement:
 * the per-launch durations behind a roofline. No counterpart in the reference. */
int edus_batch_profile(edus_batch* b, int32_t nsteps, edus_kernel_time* out, int32_t cap, int32_t* n);

/* ------------------------------------------------------- serving
 * A request loop over one batch. Submitted solves are set up on host threads
 * (input -> grid, stencil, model tables), then admitted into the batch when
 * their HBM footprint fits, oldest first (a younger request may pass one that
 * does not fit yet, for at most max_bypass_s). Admitted solves keep their
 * state on the device and advance together with every other running solve;
 * each is retired when its time grid ends, its observables copied to the host
 * and its memory returned. The loop runs on its own thread; every function
 * here may be called from any thread. No counterpart in the reference. */
typedef struct edus_server edus_server;

typedef struct {
  edus_batch_options batch;
  int32_t setup_threads;        /* host threads building problems */
  int32_t drop_decoupled_core;  /* apply edus_problem_drop_decoupled_core where it holds */
  double max_bypass_s;          /* how long younger requests may pass one that does not fit */
  double trace_tol;             /* health check of every finished request's observable log:
                                   a non-finite record fails it with EDUS_ENONFINITE, a record with
                                   |trace - (Nch + Nv)| > trace_tol with EDUS_ETRACE (0: no trace
                                   check); default 1e-3 */
} edus_server_options;

enum { EDUS_REQ_QUEUED = 0, EDUS_REQ_SETUP = 1, EDUS_REQ_READY = 2, EDUS_REQ_RUNNING = 3, EDUS_REQ_DONE = 4, EDUS_REQ_FAILED = 5 };

typedef struct {
  int32_t status, error;        /* EDUS_REQ_*, EDUS_E* when FAILED */
  int32_t nbands, nobs;
  int64_t nk, steps;
  int64_t footprint_bytes;
  double t_submit, t_ready, t_admit, t_done;  /* seconds on the server clock */
} edus_request_info;

typedef struct {
  int64_t submitted, completed, failed, running, waiting;
  double span_s;                /* first submission to last completion */
  double solves_per_s;          /* completed / span_s */
  double kpoint_steps_per_s;    /* k-point steps of the completed solves / span_s */
  double p50_latency_s, p99_latency_s, max_latency_s;  /* t_done - t_submit */
  double device_ms;             /* CUDA-event time of the batch chunks */
  int64_t peak_bytes;           /* largest HBM footprint in use at once */
  int32_t peak_active, pad;
} edus_server_stats;

int edus_server_options_default(edus_server_options* o);
int edus_server_create(const edus_server_options* o, edus_server** out);
/* Queue a solve; returns at once. workdir holds its model files. */
int edus_server_submit(edus_server* s, const edus_params* p, const char* workdir, int64_t* id);
int edus_server_info(edus_server* s, int64_t id, edus_request_info* out);
/* Observables of a DONE request (EDUS_ENOTREADY before). */
int edus_server_obs(edus_server* s, int64_t id, int32_t first, int32_t count, edus_obs* out);
/* Drop a finished request's results. */
int edus_server_forget(edus_server* s, int64_t id);
/* Wait until every submitted request is DONE or FAILED (EDUS_ETIMEOUT otherwise). */
int edus_server_drain(edus_server* s, double timeout_s);
int edus_server_stats_get(edus_server* s, edus_server_stats* out);
/* Seconds on the server clock (the time base of edus_request_info). */
double edus_server_clock(edus_server* s);
void edus_server_destroy(edus_server* s);

/* ------------------------------------------------------- strings */
const char* edus_strerror(int code);
const char* edus_last_error(void);
int edus_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* EDUS_B200_H */
