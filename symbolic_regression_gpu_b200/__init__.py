"""B200-native population evaluator for GP symbolic regression.

Drop-in for the fitness-evaluation hot path of phi-jkim/symbolic_regression_gpu
(evaluate_gpu_mse_wrapper, src/cleaned/cl_gpu_eval.cu:578-592): every
prefix-encoded expression of a population is evaluated on every datapoint of
a shared dataset and reduced to its MSE by hand-written sm_100a CUDA
(libsr_eval.so).  Importing the package loads the library and raises if it is
missing: there is no CPU fallback.
"""
from . import opcodes
from ._lib import SrError
from .evaluator import (Evaluator, detect_subtrees, mark_cached, subtree_hashes, subtree_key,
                        validate)
from .population import Population, concat

__all__ = ["Evaluator", "Population", "SrError", "concat", "detect_subtrees", "mark_cached",
           "opcodes", "subtree_hashes", "subtree_key", "validate"]
