// Generated by eri_flops_count.cu from eri_sq.cuh: arithmetic of one primitive quartet of the
// float32 ERI kernels per class combination g = (lI + 2 lJ) * 4 + (lK + 2 lL) (flops: +, -, *, /;
// special: sqrt, exp, reciprocal square root), constants folded as the compiler folds them.
#pragma once
static const int B2_ERI_FLOPS[16] = {23, 52, 52, 160, 52, 114, 114, 476, 52, 114, 114, 476, 183, 449, 449, 1708};
static const int B2_ERI_SPECIAL[16] = {3, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2, 2};
