// cg_solver (library/include/iterative_solvers/krylov/cg.h:193-327).
#ifndef LINALG_B200_CG_H
#define LINALG_B200_CG_H

#include "../../csr_matrix.h"
#include "../../vector.h"
#include "../iter_control.h"
#include "../preconditioner/preconditioner.h"

namespace linalg
{
    class cg_solver
    {
    private:
        vector<double> z;
        vector<double> p;
        vector<double> res;
        int            restart_iter;
        bool           on_host;

    public:
        cg_solver();
        ~cg_solver();

        cg_solver(const cg_solver&)            = delete;
        cg_solver& operator=(const cg_solver&) = delete;

        void build(const csr_matrix<double>& A);
        int  solve_nonprecond(const csr_matrix<double>& A, vector<double>& x,
                              const vector<double>& b, iter_control control);
        int  solve_precond(const csr_matrix<double>& A, vector<double>& x, const vector<double>& b,
                           const preconditioner* precond, iter_control control);
        int  solve(const csr_matrix<double>& A, vector<double>& x, const vector<double>& b,
                   const preconditioner* precond, iter_control control);
        void move_to_host();
        void move_to_device();
        bool is_on_host() const;

        // Status and residuals of the last solve (not in the reference interface).
        lab_solve_info last_info() const
        {
            return info;
        }

    private:
        lab_solve_info info = {};
    };
}

#endif
