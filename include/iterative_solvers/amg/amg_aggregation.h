// Aggregation and C/F splitting (library/include/iterative_solvers/amg/amg_aggregation.h:66-104).
#ifndef LINALG_B200_AMG_AGGREGATION_H
#define LINALG_B200_AMG_AGGREGATION_H

#include <cstdint>

#include "../../csr_matrix.h"

namespace linalg
{
    bool compute_aggregates_using_pmis(const csr_matrix<double>& A,
                                       const vector<int>&        connections,
                                       vector<int64_t>&          aggregates,
                                       vector<int64_t>&          aggregate_root_nodes);
    void compute_cfpoint_first_pass(const csr_matrix<double>& S, const csr_matrix<double>& ST,
                                    vector<uint32_t>& cfpoints);
    void compute_cfpoint_second_pass(const csr_matrix<double>& S, vector<uint32_t>& cfpoints);
}

#endif
