/* ta3b_cma.h -- C ABI of the host CMA-ES used by the island trainer
 * (library tetris_ai3_b200/_lib/libta3b_host.so).
 *
 * Replaces the reference's pagmo user-defined algorithms
 *   ta3::trn::sep_cmaes (ta3_trainer/incl/ta3/trainer/pagmo/sep_cmaes.hpp,
 *                        ta3_trainer/src/pagmo/sep_cmaes.cpp:34-279)
 *   ta3::trn::dd_cmaes  (ta3_trainer/incl/ta3/trainer/pagmo/dd_cmaes.hpp,
 *                        ta3_trainer/src/pagmo/dd_cmaes.cpp:35-358)
 * as ask/tell optimisers: one ask + tell pair is one generation of the
 * reference's evolve() loop; ta3c_new_evolve marks the start of one evolve()
 * call (the reference draws from a fresh normal distribution per call).
 * Minimisation; NaN fitness ranks last. Host-only: no GPU needed. */
#ifndef TA3B_CMA_H
#define TA3B_CMA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ta3c_opt ta3c_opt;

enum { TA3C_SEP = 1, TA3C_DD = 2 };

/* sep_cmaes{gen, -1, -1, -1, -1, sigma0, ...} / dd_cmaes{gen, sigma0, ..., active_update, seed}
 * started at x0 (the reference starts at the population's best individual);
 * lb / ub: the problem's box, which sets the initial per-axis scale
 * (sigma0 * (ub - lb)). NULL on invalid arguments (ta3c_last_error). */
ta3c_opt* ta3c_create(int kind, uint32_t dim, const double* x0, const double* lb, const double* ub, double sigma0,
                      uint32_t seed, int active_update);
void ta3c_destroy(ta3c_opt* opt);

/* the evolve() boundary: drop the normal distribution's cached deviate */
int ta3c_new_evolve(ta3c_opt* opt);
/* sample lam candidates, row-major (candidate i at x_out[i * dim]) */
int ta3c_ask(ta3c_opt* opt, uint32_t lam, double* x_out);
/* ||step|| of the last asked candidate (the reference's dx exit statistic) */
double ta3c_last_dx(const ta3c_opt* opt);
/* adapt from k evaluated candidates of the last ask: fitness[j] belongs to
 * candidate idx[j] (idx NULL: candidates 0..k-1). k == lam is the reference's
 * update; k < lam (surrogate pre-screening) ranks only the evaluated subset. */
int ta3c_tell(ta3c_opt* opt, uint32_t k, const int32_t* idx, const double* fitness);
int ta3c_mean(const ta3c_opt* opt, double* out);
double ta3c_sigma(const ta3c_opt* opt);
int ta3c_axis_std(const ta3c_opt* opt, double* out);
/* k points (row-major) in the coordinates of the current search distribution,
 * the inverse of ask's sampling map (there the distribution is N(0, I)). No
 * reference counterpart. */
int ta3c_whiten(const ta3c_opt* opt, uint32_t k, const double* x, double* z_out);
uint32_t ta3c_dim(const ta3c_opt* opt);

/* Full adaptation state (paths, D, C, accumulated update, random engine) in a
 * documented binary format ("TA3CMAES", version, kind, dim, fields). Returns
 * the size; writes only when cap is large enough. Replaces the reference's
 * Boost archive of the algorithm (trainer2.cpp:226-232). */
uint64_t ta3c_save(const ta3c_opt* opt, void* buf, uint64_t cap);
ta3c_opt* ta3c_load(const void* buf, uint64_t len);

/* thread-local message of the last failure */
const char* ta3c_last_error(void);

/* Symmetric eigendecomposition (cyclic Jacobi) of the row-major n x n matrix a:
 * eigenvalues to w, eigenvectors to the columns of v (v may be NULL).
 * Returns 0, or 1 if the sweep limit was reached. */
int ta3c_sym_eig(uint32_t n, const double* a, double* w, double* v);

/* The reference's optimiser tests (ta3_trainer/tests/src/pagmo/dd_cmaes_test.cpp,
 * sep_cmaes_test.cpp, test_problems.hpp) run natively: problem 0 sphere,
 * 1 separable ellipsoid (condition 1e6), 2 rotated ellipsoid; box [-5, 5]^dim;
 * a population of `pop` uniform individuals from mt19937(seed), then one
 * evolve() of `gens` generations from its best individual.
 * Writes the champion's fitness and x. */
int ta3c_run_test_problem(int kind, int problem, uint32_t dim, uint32_t pop, uint32_t gens, double sigma0,
                          uint32_t seed, double ftol, double xtol, double* champion_f, double* champion_x);

#ifdef __cplusplus
}
#endif

#endif
