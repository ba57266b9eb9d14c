// uaamg_setup (library/include/iterative_solvers/amg/uaamg.h), built on the GPU.
#ifndef LINALG_B200_UAAMG_H
#define LINALG_B200_UAAMG_H

#include "../../csr_matrix.h"
#include "amg.h"

namespace linalg
{
    void uaamg_setup(const csr_matrix<double>& mat_A, int max_level, hierarchy& hierarchy);
}

#endif
