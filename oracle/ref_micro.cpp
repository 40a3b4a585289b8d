// Thin C wrapper around the reference's CPU POTRF (src/micro_chol.hpp:14-44),
// compiled from the reference source tree by oracle/Makefile (target `ref`)
// into oracle/_ref/.  TEST/BASELINE INFRASTRUCTURE ONLY: it is the timed
// reference CPU path and a cross-check of the oracle's restatement.
#include "micro_chol.hpp"

extern "C" int ref_micro_cholesky(float* A, int n, int ld) { return micro_cholesky(A, n, ld); }
