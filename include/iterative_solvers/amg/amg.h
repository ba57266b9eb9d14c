// AMG hierarchy and stationary solve (library/include/iterative_solvers/amg/amg.h:65-418).
// The level operators are built and kept on the GPU; the std::array members
// expose them as csr_matrix objects borrowing the device levels.
#ifndef LINALG_B200_AMG_H
#define LINALG_B200_AMG_H

#include <array>
#include <memory>

#include "../../csr_matrix.h"
#include "../../vector.h"
#include "../iter_control.h"
#include "lab.h"

namespace linalg
{
    struct hierarchy
    {
        std::array<csr_matrix<double>, 20> prolongations;
        std::array<csr_matrix<double>, 20> restrictions;
        std::array<csr_matrix<double>, 21> A_cs;
        int                                total_levels = 0;
        bool                               on_host;

        hierarchy();
        bool is_on_host() const;
        void move_to_device();
        void move_to_host();

        // -- library access: the device hierarchy (null before a setup) --
        std::shared_ptr<lab_hier_s> device;
        void                        adopt(lab_hierarchy h);
    };

    enum class cycle
    {
        vcycle,
        wcycle,
        fcycle
    };

    enum class smoother
    {
        jacobi,
        gauss_seidel,
        symmetric_gauss_seidel,
        SOR,
        SSOR
    };

    // Write the levels of a built hierarchy to a file / load them back onto the
    // device (bit-identical), so a rerun on the same operator skips the setup.
    // No counterpart in the reference.  Return false on failure (the reason is
    // printed, as the reference reports its errors).
    bool save_hierarchy(const hierarchy& h, const char* path);
    bool load_hierarchy(const char* path, hierarchy& h);

    // amg.h:411-418.  Returns the number of cycles (amg.cpp:570).
    int amg_solve(const hierarchy&      hierarchy,
                  vector<double>&       x,
                  const vector<double>& b,
                  int                   n1,
                  int                   n2,
                  cycle                 cycle,
                  smoother              smoother,
                  iter_control          control);
}

#endif
