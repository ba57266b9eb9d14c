// saamg_setup (library/include/iterative_solvers/amg/saamg.h), built on the GPU.
#ifndef LINALG_B200_SAAMG_H
#define LINALG_B200_SAAMG_H

#include "../../csr_matrix.h"
#include "amg.h"

namespace linalg
{
    void saamg_setup(const csr_matrix<double>& mat_A, int max_level, hierarchy& hierarchy);
}

#endif
