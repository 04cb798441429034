/* ta3b_trainer.h -- C ABI of the island CMA-ES trainer (library
 * tetris_ai3_b200/_lib/libta3b_host.so), the evaluator's caller.
 *
 * Restates ta3::trn::Trainer2 (ta3_trainer/incl/ta3/trainer/trainer2.hpp,
 * ta3_trainer/src/trainer2.cpp) with pagmo's archipelago replaced by a
 * lock-step island loop: in every generation each island asks its CMA-ES for
 * candidates, ALL islands' candidates are scored in ONE evaluator call
 * (islands share the cycle's game seeds, trainer2.cpp:150-157,316), then each
 * island tells its optimiser. Fitness = -(mean score over the games)
 * (tetris_problem2.cpp:44-72). Ring migration (trainer2.cpp:145-146, ring{1})
 * runs once per iteration; champions, best fitness and the saved state follow
 * trainer2.cpp:213-303.
 *
 * Optional surrogate pre-screening (no counterpart in the reference): from
 * generation `surrogate_start_gen` each island samples `surrogate_sample`
 * candidates, the surrogate ranks them, and only the best-predicted
 * `surrogate_top` plus `surrogate_random` random others are fully evaluated
 * and told to the optimiser. The surrogate is retrained every
 * `surrogate_retrain` generations on the fully evaluated (parameters -> mean
 * score) pairs of the last `surrogate_window` generations (all when 0) except
 * the latest generation, which is held out; while its
 * Spearman rho on that held-out slice is below `surrogate_min_rho` the
 * generation runs without pre-screening. Every fitness the trainer reports
 * comes from full evaluation. Without a caller-supplied surrogate the built-in
 * GPU model is used: 97 -> 128 -> 128 -> 2 (ta3s_*) for v11's 97 parameters,
 * num_params -> 256 -> 256 -> 2 (ta3w_*) for any other size. */
#ifndef TA3B_TRAINER_H
#define TA3B_TRAINER_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ta3t_trainer ta3t_trainer;

/* Per-(model, game) scores, model-major (m * num_games + g): every model plays
 * the same seeds. The semantics of ta3::gpu::simulate + ModelEvaluator::eval
 * (model_eval.hpp:46-51,84-103). pieces_out may be NULL. Returns 0 on success. */
typedef int (*ta3t_score_fn)(void* user, const float* weights, uint32_t num_models, uint32_t num_params,
                             const uint64_t* seeds, uint32_t num_games, uint32_t max_moves, float* score_out,
                             uint32_t* pieces_out);

/* A surrogate model of mean score from a parameter vector. */
typedef struct {
    void* user;
    /* fit to n pairs: x row-major (n x dim), y the mean score; 0 on success */
    int (*train)(void* user, const float* x, const float* y, uint32_t n, uint32_t dim);
    /* predicted mean score of n candidates; 0 on success */
    int (*predict)(void* user, const float* x, uint32_t n, uint32_t dim, float* mean_out);
} ta3t_surrogate;

typedef struct {
    uint32_t islands;            /* ISLANDS = 4 (runner main.cpp:20) */
    uint32_t population;         /* POPULATION_SIZE = 50 per island */
    uint32_t gens_per_iteration; /* GENS_PER_ITERATION = 10 */
    uint32_t iterations_per_cycle; /* ITERATIONS_PER_CYCLE = 10: one game seed per cycle */
    uint32_t games;              /* simulationsPerEval */
    uint32_t max_moves;
    uint32_t algo;               /* TA3C_SEP or TA3C_DD (ta3b_cma.h); the runner uses DD */
    uint32_t num_params;         /* 97 for the v11 evaluator */
    uint64_t training_seed;      /* TrainerConfig2::trainingSeed = 0x3e28df7b1811145b */
    double sigma0;               /* 1.3 (trainer2.cpp:122) */
    double lower, upper;         /* the model's parameter box, [-2, 2] */
    int device;                  /* CUDA device of the built-in evaluator */
    uint32_t surrogate_start_gen;   /* 0 = no pre-screening; else first generation (1-based) with it */
    uint32_t surrogate_sample;      /* candidates sampled per island */
    uint32_t surrogate_top;         /* best-predicted candidates fully evaluated per island */
    uint32_t surrogate_random;      /* extra random candidates fully evaluated per island */
    uint32_t surrogate_retrain;     /* retrain period in generations */
    double surrogate_min_rho;       /* Spearman gate on the held-out generation */
    uint32_t surrogate_epochs;      /* built-in GPU surrogate: epochs per retrain */
    uint32_t surrogate_batch;       /* built-in GPU surrogate: minibatch rows */
    double surrogate_lr;            /* built-in GPU surrogate: Adam learning rate */
    uint32_t surrogate_window;      /* train on the last N generations before the held-out one (0 = all) */
    uint32_t num_devices;           /* built-in evaluator: island groups on devices device .. device + n - 1 */
} ta3t_config;

typedef struct {
    uint64_t generation;         /* generations completed (all islands in lock step) */
    uint64_t iteration;          /* iterations completed */
    uint64_t evaluations;        /* fully evaluated candidates */
    uint64_t sims;               /* model x game simulations run */
    uint64_t pieces;             /* pieces placed by those simulations */
    uint64_t game_seed;          /* the current cycle's game seed */
    double best_fitness;         /* min over islands of the champion fitness (-mean score) */
    double eval_seconds;         /* wall time inside the score function */
    double host_seconds;         /* wall time in ask / tell / migration / bookkeeping */
    double surrogate_seconds;    /* wall time in surrogate train + predict */
    double last_rho;             /* Spearman rho of the last surrogate check (NaN before one) */
    uint32_t surrogate_active;   /* 1 while pre-screening is on */
    uint32_t surrogate_trainings;
} ta3t_stats;

/* fills the reference runner's configuration (runner main.cpp:20-34, trainer2.cpp:122-135) */
void ta3t_default_config(ta3t_config* cfg);

/* Build the archipelago (trainer2.cpp:144-171): islands of uniform random
 * populations, evaluated with game seed 0, optimisers seeded from the training
 * seed's xoshiro256** stream. score_fn NULL: the built-in GPU evaluator
 * (libta3b.so, ta3b_eval on cfg->device). surrogate NULL with
 * surrogate_start_gen > 0: the built-in GPU surrogate (ta3b_surrogate.h).
 * NULL on failure (message via ta3t_last_error(NULL)). */
ta3t_trainer* ta3t_create(const ta3t_config* cfg, ta3t_score_fn score_fn, void* user, const ta3t_surrogate* surrogate);
/* Island groups (the multi-GPU split of a training run): islands i with
 * i % num_groups == g are scored by score_fns[g] (with users[g]), every group
 * on its own host thread, concurrently; the built-in evaluator does the same
 * with one context per device when cfg->num_devices > 1 (ta3t_create). Every
 * generation stays one lock-step step of all islands, and as the evaluator is
 * deterministic a split run equals the single-device run bit for bit. The
 * reference runs its islands on host threads with one evaluator per
 * model-scheduler thread (ta3_trainer/src/trainer2.cpp:98-100,144-170,
 * ta3_gpu/incl/ta3/gpu/model_eval.hpp:21-26). */
ta3t_trainer* ta3t_create_groups(const ta3t_config* cfg, uint32_t num_groups, const ta3t_score_fn* score_fns,
                                 void* const* users, const ta3t_surrogate* surrogate);
/* Like ta3t_create, but every island's optimiser resumes from a saved state
 * (trainer2.cpp:178-212: the best island's optimiser, copied to all islands,
 * re-seeded per island). */
ta3t_trainer* ta3t_create_from_state(const ta3t_config* cfg, const char* state_path, ta3t_score_fn score_fn,
                                     void* user, const ta3t_surrogate* surrogate);
void ta3t_destroy(ta3t_trainer* t);
const char* ta3t_last_error(const ta3t_trainer* t);

/* Trainer2::nextGameSeed (trainer2.cpp:316): the next cycle's game seed */
int ta3t_next_game_seed(ta3t_trainer* t);
/* one generation on every island (ask, one evaluator call, tell) */
int ta3t_run_generation(ta3t_trainer* t);
/* Trainer2::runIteration (trainer2.cpp:317-331): migration, then gens_per_iteration generations */
int ta3t_run_iteration(ta3t_trainer* t);
/* Trainer2::run for a bounded number of iterations: a new game seed every
 * iterations_per_cycle iterations (trainer2.cpp:332-388) */
int ta3t_run(ta3t_trainer* t, uint32_t iterations);

int ta3t_get_stats(const ta3t_trainer* t, ta3t_stats* out);
/* island champion (best fully evaluated candidate so far): x (num_params doubles) and fitness */
int ta3t_champion(const ta3t_trainer* t, uint32_t island, double* x_out, double* f_out);
/* current CMA-ES mean of an island */
int ta3t_island_mean(const ta3t_trainer* t, uint32_t island, double* x_out);
/* n parameter vectors (row-major) in an island's own search coordinates: the map
 * under which its current sampling distribution is N(0, I) (dd-CMA-ES:
 * z = C^(-1/2) ((x - m) / (sigma d)); sep-CMA-ES: (x - m) / (sigma sqrt(diag))).
 * No reference counterpart (used to fit per-island surrogates). */
int ta3t_island_whiten(const ta3t_trainer* t, uint32_t island, const double* x, uint32_t n, double* z_out);

/* Trainer2::saveState (trainer2.cpp:213-268): the best island's optimiser state
 * to state_path, its champion to the same path with extension .champ */
int ta3t_save_state(const ta3t_trainer* t, const char* state_path);

/* .champ files (trainer2.cpp:252-265): uint64 count, then count doubles */
int ta3t_write_champ(const char* path, const double* x, uint64_t n);
/* returns the count (or 0 on error); writes min(count, cap) values */
uint64_t ta3t_read_champ(const char* path, double* x_out, uint64_t cap);

#ifdef __cplusplus
}
#endif

#endif
