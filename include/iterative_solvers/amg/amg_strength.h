// Strength of connection (library/include/iterative_solvers/amg/amg_strength.h:59-80).
#ifndef LINALG_B200_AMG_STRENGTH_H
#define LINALG_B200_AMG_STRENGTH_H

#include "../../csr_matrix.h"

namespace linalg
{
    void compute_strong_connections(const csr_matrix<double>& A, double eps,
                                    vector<int>& connections);
    void compute_classical_strong_connections(const csr_matrix<double>& A, double theta,
                                              csr_matrix<double>& S, vector<int>& connections);
}

#endif
