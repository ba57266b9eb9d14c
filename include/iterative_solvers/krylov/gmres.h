// gmres_solver (library/include/iterative_solvers/krylov/gmres.h:228-346).
#ifndef LINALG_B200_GMRES_H
#define LINALG_B200_GMRES_H

#include "../../csr_matrix.h"
#include "../../vector.h"
#include "../iter_control.h"
#include "../preconditioner/preconditioner.h"

namespace linalg
{
    class gmres_solver
    {
    private:
        int            restart;
        lab_solve_info info = {};

    public:
        gmres_solver();
        ~gmres_solver();

        gmres_solver(const gmres_solver&)            = delete;
        gmres_solver& operator=(const gmres_solver&) = delete;

        void build(const csr_matrix<double>& A, int restart);
        int  solve_nonprecond(const csr_matrix<double>& A, vector<double>& x,
                              const vector<double>& b, iter_control control);
        int  solve_precond(const csr_matrix<double>& A, vector<double>& x, const vector<double>& b,
                           const preconditioner* precond, iter_control control);
        int  solve(const csr_matrix<double>& A, vector<double>& x, const vector<double>& b,
                   const preconditioner* precond, iter_control control);

        lab_solve_info last_info() const
        {
            return info;
        }
    };
}

#endif
