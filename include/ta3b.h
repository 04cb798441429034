/*
 * ta3b.h -- C ABI of the B200 model x game beam-search evaluator.
 *
 * Drop-in for the reference's evaluator seam: a population of value-model
 * weight vectors plus game seeds go in; per-(model, game) score, piece count
 * and line count come out. Every game is played with the reference's depth-4
 * beam search (widths 16/32/32) on the 10x23 bit-board with hold and a 5-piece
 * preview, bit-exact with the reference CPU path.
 *
 * Plain C types only (no CUDA or torch types), so cgo / JNI / ctypes / a C++
 * host can bind it directly. All functions return TA3B_OK (0) or a negative
 * TA3B_ERR_* code; the message is available from ta3b_last_error(ctx).
 *
 * Threading: a context is NOT thread-safe (same contract as the reference's
 * ta3::gpu::ModelEvaluator, ta3_gpu/incl/ta3/gpu/model_eval.hpp:21-26); use one
 * context per host thread. Separate contexts may run concurrently; each owns
 * its own CUDA stream and device buffers.
 */
#ifndef TA3B_H
#define TA3B_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TA3B_NUM_PARAMS 97 /* v11 value model, ta3_ai/incl/ta3/ai/models/models/model_v11.hpp:44 */
/* The reference's dense layers (ta3_ai/incl/ta3/ai/models/models/utility.hpp:29-46)
 * widened to 10 -> H ReLU -> H ReLU -> 1 over the same v11 inputs; per layer
 * [out][in] weights then [out] biases. The kernels are built for H = 64 (4,929
 * parameters) and H = 32 (1,441). Every evaluation entry point except
 * ta3b_eval_device_noalloc and ta3b_core_selftest accepts them as num_params. */
#define TA3B_NUM_PARAMS_WIDE 4929
#define TA3B_NUM_PARAMS_WIDE32 1441

enum {
    TA3B_OK = 0,
    TA3B_ERR_ARG = -1,     /* bad size, null pointer, parameter-count mismatch */
    TA3B_ERR_CUDA = -2,    /* a CUDA runtime call failed (message has the CUDA error string) */
    TA3B_ERR_NODEV = -3,   /* no usable sm_100 device */
    TA3B_ERR_DEVICE = -4,  /* the kernel reported an error status */
    TA3B_ERR_TIMEOUT = -5, /* the launch exceeded the context's time budget (ta3b_set_time_budget) */
};

typedef struct ta3b_ctx ta3b_ctx;

typedef struct {
    int device;                /* CUDA device ordinal */
    uint32_t warps_per_block;  /* 0 = tuned default; else pick the kernel variant with this shape */
    uint32_t blocks_per_sm;    /* 0 = tuned default; else the variant's minimum resident blocks per SM */
} ta3b_config;

/* Create an evaluation context (stream + grow-only device buffers).
 * Replaces ModelEvaluator::ModelEvaluator(), ta3_gpu/src/cuda/model_eval.cu:92.
 * Returns NULL on failure; ta3b_last_error(NULL) then holds the reason. */
ta3b_ctx* ta3b_create(const ta3b_config* cfg);

/* Release the context. Replaces ModelEvaluator::~ModelEvaluator, model_eval.cu:72-83,93. */
void ta3b_destroy(ta3b_ctx* ctx);

/* Message of the last failure on this context (or of ta3b_create when ctx is NULL). */
const char* ta3b_last_error(const ta3b_ctx* ctx);

/* Per-launch time budget for this context's evaluations (0 = none, the default).
 * Every warp compares the GPU's global timer with its launch start after each
 * move; past the budget it stops (no new game, no further move) and the call
 * returns TA3B_ERR_TIMEOUT, with incomplete results. The context stays usable.
 * While a budget is set, launches use a fixed launch shape (the checking
 * flavour of the kernel), not the one chosen by ta3b_select_variant.
 * No reference counterpart (the reference has no device-side limit). */
int ta3b_set_time_budget(ta3b_ctx* ctx, double seconds);

/* Batched evaluation with host buffers: num_models models, each played on the
 * SAME num_games seeds. weights is model-major, num_models * num_params floats
 * (num_params: TA3B_NUM_PARAMS, or TA3B_NUM_PARAMS_WIDE / TA3B_NUM_PARAMS_WIDE32 for
 * the widened networks).
 * Outputs are model-major: index
 * m * num_games + g holds model m on game g. pieces_out, lines_out may be NULL.
 * score is the reference's score_v1 (FP64, rounded to float); -1e6 when no
 * piece was placed.
 * Replaces std::vector<float> ModelEvaluator::eval(std::span<const float> weights,
 * uint32_t num_models, std::span<const uint64_t> seeds, uint32_t max_moves),
 * ta3_gpu/incl/ta3/gpu/model_eval.hpp:46-51 / ta3_gpu/src/cuda/model_eval.cu:97-153. */
int ta3b_eval(ta3b_ctx* ctx, const float* weights, uint32_t num_models, uint32_t num_params,
              const uint64_t* seeds, uint32_t num_games, uint32_t max_moves,
              float* score_out, uint32_t* pieces_out, uint32_t* lines_out);

/* Island-batched evaluation in ONE launch: island i owns models
 * [i*models_per_island, (i+1)*models_per_island) and plays seeds
 * [i*num_games, (i+1)*num_games). Identical results to one ta3b_eval per
 * island. This is how one CMA-ES generation of several islands is scored
 * (ta3_trainer/src/tetris_problem2.cpp:29-72 calls eval once per island batch). */
int ta3b_eval_islands(ta3b_ctx* ctx, const float* weights, uint32_t num_islands, uint32_t models_per_island,
                      uint32_t num_params, const uint64_t* seeds, uint32_t num_games, uint32_t max_moves,
                      float* score_out, uint32_t* pieces_out, uint32_t* lines_out);

/* Device-resident variant of ta3b_eval_islands: every pointer is device memory;
 * enqueued on `stream` (a cudaStream_t, NULL = the context's stream, a
 * non-blocking stream that does not wait for the legacy default stream: inputs
 * written elsewhere must be complete first) and NOT synchronised. evals_out (may be NULL) receives per-sim counts of evaluated
 * beam placements (value-model calls). Used for HBM-resident batches and CUDA
 * graph capture. With the widened network (num_params = TA3B_NUM_PARAMS_WIDE)
 * the call first repacks the weights into the kernel's layout (16-byte aligned,
 * layers 1 and 2 transposed, a per-model flag) in a copy owned by the context;
 * that copy is allocated by the first widened call of a larger size, so make
 * such a call once before capturing it. The call returns before the kernel
 * runs, so a device-side error is read afterwards with ta3b_device_status.
 * At most 2^32 - 1 sims per call (as for every context entry point). No
 * reference counterpart (the reference stages host buffers). */
int ta3b_eval_device(ta3b_ctx* ctx, const float* d_weights, uint32_t num_islands, uint32_t models_per_island,
                     uint32_t num_params, const uint64_t* d_seeds, uint32_t num_games, uint32_t max_moves,
                     float* d_score, uint32_t* d_pieces, uint32_t* d_lines, uint32_t* d_evals, void* stream);

/* Allocation-free variant of ta3b_eval_device, for callers that must not call
 * cudaMalloc where they evaluate (a host framework whose pooling allocator owns
 * all device memory; a scheduler thread that cannot afford cudaMalloc's implicit
 * device synchronisation). No context: pass device inputs and outputs and a
 * stream (NULL = legacy default stream); nothing is allocated. The kernel's only
 * scratch -- its 64-bit work-queue ticket and error status word -- is a
 * 256-byte static device array that every GPU loading this library keeps
 * until exit. The first
 * call on each device sets that device up (resolves the array's address,
 * configures the kernel) with the device current; make that first call before
 * any stream capture. Every call shares the one array and clears it on entry,
 * so calls whose kernels overlap on the GPU race: run them on one stream or
 * serialise them. A call may cover at most 2^32 - 1 sims; larger batches,
 * num_params != 97 and null pointers are rejected with TA3B_ERR_ARG and, when
 * error_out is not NULL, a static message in *error_out. Enqueued, not
 * synchronised; ta3b_noalloc_status reads the kernel's status word afterwards.
 * No counterpart in the reference. */
int ta3b_eval_device_noalloc(const float* d_weights, uint32_t num_islands, uint32_t models_per_island,
                             uint32_t num_params, const uint64_t* d_seeds, uint32_t num_games, uint32_t max_moves,
                             float* d_score, uint32_t* d_pieces, uint32_t* d_lines, uint32_t* d_evals,
                             void* stream, const char** error_out);

/* The status word of the most recent ta3b_eval_device_noalloc call on the
 * current device (0 = no error; any set bit is a device error, bit 0 = a
 * search found no move although a root placement was legal), copied on
 * `stream` (NULL = legacy default stream) after the work already queued there,
 * then that stream is synchronised. Allocates nothing. Returns TA3B_OK for
 * status 0, TA3B_ERR_DEVICE otherwise, TA3B_ERR_ARG before the first
 * allocation-free call on the device. Like the evaluation it shares the static
 * array with every call, so read it before the next call's kernel starts. No
 * counterpart in the reference. */
int ta3b_noalloc_status(void* stream, uint32_t* status_out, const char** error_out);

/* Status word of the context's most recent launch (any entry point; after
 * ta3b_eval_device, once the stream it ran on has finished): 0 = no error,
 * bit 1 = the time budget ran out, any other bit = a device error (bit 0: a
 * search found no move although a root placement was legal). Synchronises the
 * context's stream. Returns TA3B_OK, TA3B_ERR_TIMEOUT or TA3B_ERR_DEVICE
 * accordingly; status_out may be NULL. The host-buffer entry points check this
 * word themselves. No reference counterpart (the reference's kernel reports
 * no device status). */
int ta3b_device_status(ta3b_ctx* ctx, uint32_t* status_out);

/* Per-move trace of every sim (debug / parity tooling): trace_out receives
 * 3 bytes per move (hold, orientation, x + 2), max_moves moves per sim,
 * model-major; n_moves_out the number of searched moves per sim;
 * board_out the final 10 bit-columns per sim. keys_out (may be NULL; 2 x
 * max_moves per sim) receives, per searched move, the two largest keys of the
 * final argmax (leaf keys and dead-end fallbacks; ta3_ai/incl/ta3/ai/search/
 * beam.hpp:204-224,407-443): (ordered value bits << 32) | (2192 - order), so
 * key1 decodes to the chosen move's value and key1 - key2's values is the
 * decision's top-two margin. With keys_out the launch runs a tracing flavour
 * of the kernel, which ignores the time budget. Host buffers. */
int ta3b_eval_trace(ta3b_ctx* ctx, const float* weights, uint32_t num_models, uint32_t num_params,
                    const uint64_t* seeds, uint32_t num_games, uint32_t max_moves,
                    float* score_out, uint32_t* pieces_out, uint32_t* lines_out, uint32_t* evals_out,
                    uint8_t* trace_out, uint32_t* n_moves_out, uint32_t* board_out, uint64_t* keys_out);

/* Scheduling profile of one island-batched evaluation (tooling): like
 * ta3b_eval_islands plus, per sim, the number of evaluated placements and the
 * device global-timer (ns) at which a warp started and finished it
 * (timing_out: 2 values per sim). No reference counterpart. */
int ta3b_eval_timed(ta3b_ctx* ctx, const float* weights, uint32_t num_islands, uint32_t models_per_island,
                    uint32_t num_params, const uint64_t* seeds, uint32_t num_games, uint32_t max_moves,
                    float* score_out, uint32_t* pieces_out, uint32_t* evals_out, uint64_t* timing_out);

/* The seeds ta3::gpu::simulate derives for `games` games from one seed
 * (xoshiro256** draws), ta3_gpu/incl/ta3/gpu/model_eval.hpp:84-103. Host only. */
int ta3b_simulate_seeds(uint64_t seed, uint32_t games, uint64_t* seeds_out);

/* Kernel launch-shape variants (warps per block x register cap expressed as
 * minimum resident blocks per SM): the autotuner's search space. No reference
 * counterpart (the reference has one fixed launch, model_eval.cu:143).
 * ta3b_variant_warps_per_game: 1 for the single-warp kernels, 2 for the paired
 * kernels (two warps share every game's candidate passes; same results bit for
 * bit), -1 for a variant out of range. ta3b_config's warps_per_block /
 * blocks_per_sm select among the single-warp variants only.
 * Launch shape: a context created with the tuned default runs a batch of at most
 * 2 games per SM (v11 network, no time budget, no key tracing) on teams of four
 * warps, one of at most 4 games per SM on the paired kernel, and every other
 * batch on the default variant; a batch smaller than one
 * block per SM can hold is spread over all SMs. ta3b_select_variant (or a shape
 * in ta3b_config) fixes the variant for every batch. */
int ta3b_num_variants(void);
int ta3b_variant_info(int variant, uint32_t* warps_per_block, uint32_t* min_blocks_per_sm);
/* Tail hand-off (on by default): a full batch on the default variant hands the
 * games still playing when at most 4 per SM are left to the paired kernel, which
 * finishes them two warps each (checkpointed at a move boundary; same results bit
 * for bit). ta3b_set_tail_handoff(ctx, 0) keeps every game on one warp;
 * ta3b_handoff_info reports how many games the context's last launch handed over
 * (synchronises the context's stream). */
int ta3b_set_tail_handoff(ta3b_ctx* ctx, int on);
/* Tests of the team kernels' bounded waits (no GPU fault involved): with flag 1
 * the partner warps of every team leave at launch start, so each leader's first
 * team wait runs out after 1 s; the launch ends, the call returns
 * TA3B_ERR_DEVICE ("kernel reported status 4") and the context stays usable.
 * 0 (the default) turns it off. Affects launches that run a team kernel. */
int ta3b_set_test_flags(ta3b_ctx* ctx, uint32_t flags);
int ta3b_handoff_info(ta3b_ctx* ctx, uint32_t* games_out);
int ta3b_variant_warps_per_game(int variant);
int ta3b_select_variant(ta3b_ctx* ctx, int variant);

/* Device self-test of the per-candidate evaluation (tests and tooling): one
 * thread per candidate runs the incremental fast path and the full reference
 * path on caller-built parent records (68 words each, the layout of
 * tetris_ai3_b200/csrc/eval_core.h). cand[t] = piece | placement << 8 |
 * held-is-I << 16 | record index << 17. Outputs per candidate: fast status
 * (0 evaluated, 1 deferred) and value, full-path legality and value; dbg32
 * (may be NULL) receives 32 diagnostic floats per candidate from the fast path.
 * No reference counterpart. */
int ta3b_core_selftest(const uint32_t* recs, uint32_t num_recs, const uint32_t* cand, uint32_t n, const float* w97,
                       float* fast_v, int* fast_st, float* full_v, int* full_legal, float* dbg32);

/* Launch shape of the context's most recent evaluation (before the first one:
 * the selected variant's full grid): grid blocks and warps per block of its
 * first kernel, the device's SM count, and how many kernels the evaluation
 * launched (2 with the tail hand-off's paired kernel, else 1; 0 before the
 * first). Any output may be NULL. For tooling and the autotuner. */
int ta3b_launch_info(const ta3b_ctx* ctx, uint32_t* grid, uint32_t* warps_per_block, uint32_t* sms,
                     uint32_t* kernels);

#ifdef __cplusplus
}
#endif

#endif /* TA3B_H */
