// iter_control (library/include/iterative_solvers/iter_control.h:43-108), same
// defaults and the same stopping test (iter_control.cpp:38-91).
#ifndef LINALG_B200_ITER_CONTROL_H
#define LINALG_B200_ITER_CONTROL_H

namespace linalg
{
    struct iter_control
    {
        double rel_tol   = 1e-06;
        double abs_tol   = 1e-06;
        int    max_iter  = 1000;
        int    max_cycle = 200;

        bool residual_converges(double residual_norm, double initial_residual_norm) const;
        bool exceed_max_iter(int iter) const;
        bool exceed_max_cycle(int cycle) const;
    };
}

#endif
