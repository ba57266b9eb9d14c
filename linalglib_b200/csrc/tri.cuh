// Triangular path (tri.cu): one-launch triangular solves over a level order
// (per-row solved flags) and in-place ILU(0) / IC(0), bit-identical to the
// reference's sequential loops.
#pragma once

#include "internal.cuh"

namespace lab
{
    // Levels of the lower and upper dependency of A's pattern and the diagonal
    // positions (device analysis, cached on A until it is released).
    lab_status tri_analyse(lab_csr_impl* A, cudaStream_t s);

    // x = T^-1 b on the lower (columns < i) or upper (columns > i) part of A.
    // dscale != 0 scales the diagonal (SOR); skip: early-exit flag (graphs).
    lab_status tri_solve(lab_csr_impl* A, bool lower, bool unit, double dscale, const double* b,
                         double* x, cudaStream_t s, const int* skip);

    // The two triangles of the reference's SSOR preconditioner built from A
    // (new matrices owned by the caller).
    lab_status ssor_split(lab_csr_impl* A, double omega, lab_csr_impl** L, lab_csr_impl** U,
                          cudaStream_t s);

    // Reads (and clears) the error flag of A's solves: LAB_TIMEOUT if a solve
    // gave up waiting (synchronises the stream).
    lab_status tri_check(lab_csr_impl* A, cudaStream_t s);

    // In-place ILU(0) (ic = false) or IC(0); the smallest column of a missing /
    // zero pivot goes to *structural_zero / *numeric_zero (-1: none).
    lab_status tri_factor(lab_csr_impl* A, bool ic, int* structural_zero, int* numeric_zero,
                          cudaStream_t s);
}
