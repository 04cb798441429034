"""B200-native (sm_100a) re-implementation of codethinki/tetris_ai3's hot path:
the batched model x game Tetris beam-search evaluation behind
ta3::gpu::ModelEvaluator. The CUDA kernel and its C ABI live in csrc/ and
include/ta3b.h; this package is the Python host side over that ABI."""
from .evaluator import EvaluatorError, ModelEvaluator, library, simulate, simulate_seeds  # noqa: F401
from .workload import NUM_PARAMS  # noqa: F401
