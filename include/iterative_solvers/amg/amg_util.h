// Galerkin product (library/include/iterative_solvers/amg/amg_util.h).
#ifndef LINALG_B200_AMG_UTIL_H
#define LINALG_B200_AMG_UTIL_H

#include "../../csr_matrix.h"

namespace linalg
{
    // A_coarse = R * (A * P)  (amg_util.cpp:31-46)
    void galarkin_triple_product(const csr_matrix<double>& R, const csr_matrix<double>& A,
                                 const csr_matrix<double>& P, csr_matrix<double>& A_coarse);
}

#endif
