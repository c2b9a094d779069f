/*
 * edus_oracle.h — CPU FP64 oracle for the EDUS k-space propagation.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain-C restatement of the
 * reference's algorithm (anpicon/EDUS) used as the checker for the CUDA
 * path. Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference arm may load it. The product never links or calls it.
 *
 * Parity pin: the oracle reproduces the reference's shipped Adams–Bashforth
 * run (example/Adams–Bashforth ODE Solver example/AB5_.../Output/{J1,J2,
 * Losses,EF,TransientAbs}.txt); see tests/test_oracle_golden.py.
 */
#ifndef EDUS_ORACLE_H
#define EDUS_ORACLE_H
#include <stddef.h>
#include "../include/edus_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc orc;

/* Build grid, shells, neighbour table, model tables, initial state and
 * Coulomb tables from resolved parameters (workdir holds <ref>_tb.dat and
 * Output/Coulomb/). */
int orc_create(const edus_params* p, const char* workdir, orc** out);
void orc_free(orc* o);
int orc_info(const orc* o, edus_problem_info* out);
int orc_get(const orc* o, const char* name, void* dst, size_t nbytes);
int orc_set(orc* o, const char* name, const void* src, size_t nbytes);

/* Run the reference time loop for at most max_steps iterations (<0: all).
 * Each output instant (it % it_resolution == 0) is written to log[]. */
int orc_run(orc* o, int max_steps, edus_obs* log, int log_cap, int* n_log);

/* Unit-level mirrors of the reference seam (state in reference layout). */
int orc_rhs(orc* o, const double* P, double* Pv, const double EF[6], double wx2, int e_non0);
int orc_coulomb_hk(orc* o, const double* P, double* hk);
int orc_observables(orc* o, const double* P, edus_obs* out);
/* Time loop clock after orc_run. */
int orc_clock(const orc* o, int* it, double* t, double* dt);
int orc_num_threads(void);
/* Coulomb coefficient generator (Source_Main/Fourier_Coulomb.cpp:95-500):
 * what = 1 Hartree table VH[n][n], 2 coefficients A..D [ncut^2][n^2] complex,
 * 4 screening constant [n^2] complex (with 2); grid points per axis n_sum,
 * n_sum_screen (the reference uses 4999 and 39999). */
int orc_coulomb_generate(const edus_params* p, const char* workdir, int what, int n_sum, int n_sum_screen, double* A,
                         double* B, double* C, double* D, double* screen, double* VH, int* g_num);

#ifdef __cplusplus
}
#endif
#endif
