/*
 * ta3b_host_ref.h -- the evaluator's CPU parity path, on the CALLER's side.
 *
 * ta3b_eval_host plays every game with the reference's own CPU beam search
 * (ta3::ai::search::search_move_beam over ta3::sim::TetrisEngine, scored by
 * stats_v4 / score_v1). It is the check a trainer runs at start-up to prove
 * the device evaluator is sound (ta3_trainer/src/trainer2.cpp:57-89 compares
 * ModelEvaluator::eval against ModelEvaluator::eval_host bit for bit), never a
 * fallback for it.
 *
 * It is NOT part of libta3b.so and the Python package never loads it: the
 * definition lives in integration/ta3b_eval_host.cpp, which the caller
 * compiles into its own binary against the reference's headers (ta3_sim/incl,
 * ta3_ai/incl, ta3_gpu/incl), in the place of the reference's
 * ta3_gpu/src/common/model_eval_host.cpp. include/ta3b.hpp forwards
 * ta3::gpu::ModelEvaluator::eval_host to it.
 */
#ifndef TA3B_HOST_REF_H
#define TA3B_HOST_REF_H

#include "ta3b.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One model played on num_games seeds on the CPU: weights holds the model's
 * TA3B_NUM_PARAMS v11 parameters (num_params >= 97; only the first 97 are read,
 * as the reference's subspan<0, NUM_PARAMS> does); score_out[g] is game g's
 * score_v1 (-1e6 when no piece was placed); pieces_out / lines_out may be NULL.
 * Returns TA3B_OK, or TA3B_ERR_ARG for num_params < 97 or a null pointer.
 * Replaces static std::vector<float> ModelEvaluator::eval_host(weights, seeds,
 * max_moves), ta3_gpu/incl/ta3/gpu/model_eval.hpp:62-67, defined in
 * ta3_gpu/src/common/model_eval_host.cpp:26-53. */
int ta3b_eval_host(const float* weights, uint32_t num_params, const uint64_t* seeds, uint32_t num_games,
                   uint32_t max_moves, float* score_out, uint32_t* pieces_out, uint32_t* lines_out);

#ifdef __cplusplus
}
#endif

#endif /* TA3B_HOST_REF_H */
