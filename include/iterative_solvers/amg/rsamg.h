// rsamg_setup (library/include/iterative_solvers/amg/rsamg.h), built on the GPU.
#ifndef LINALG_B200_RSAMG_H
#define LINALG_B200_RSAMG_H

#include "../../csr_matrix.h"
#include "amg.h"

namespace linalg
{
    void rsamg_setup(const csr_matrix<double>& mat_A, int max_level, hierarchy& hierarchy);
}

#endif
