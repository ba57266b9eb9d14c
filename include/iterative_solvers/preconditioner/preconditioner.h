// Preconditioner plug-in point (library/include/iterative_solvers/preconditioner/preconditioner.h:59-99)
// with the reference's Jacobi, Gauss-Seidel, SOR, SSOR, ILU(0) and IC(0)
// preconditioners (preconditioner.cpp:33-545) and the AMG preconditioner the
// reference lacks: one multigrid cycle from a zero guess per application.
#ifndef LINALG_B200_PRECONDITIONER_H
#define LINALG_B200_PRECONDITIONER_H

#include "../../csr_matrix.h"
#include "../amg/amg.h"
#include "lab.h"

namespace linalg
{
    class preconditioner
    {
    public:
        preconditioner() {}
        virtual ~preconditioner() {}
        virtual void build(const csr_matrix<double>& A)                          = 0;
        virtual void solve(const vector<double>& rhs, vector<double>& x) const = 0;
        virtual void move_to_device()                                            = 0;
        virtual void move_to_host()                                              = 0;
        virtual bool is_on_host() const                                          = 0;

        // Device preconditioner handle for the fused GPU solvers (null for a
        // user-defined subclass, which the solvers call through solve()).
        virtual lab_precond device_handle() const
        {
            return nullptr;
        }
    };

    class jacobi_precond : public preconditioner
    {
    private:
        lab_precond M       = nullptr;
        bool        on_host = true;

    public:
        jacobi_precond();
        ~jacobi_precond();
        void        build(const csr_matrix<double>& A) override;
        void        solve(const vector<double>& rhs, vector<double>& x) const override;
        void        move_to_device() override;
        void        move_to_host() override;
        bool        is_on_host() const override;
        lab_precond device_handle() const override
        {
            return M;
        }
    };

    // The triangular-solve preconditioners share one device implementation: build()
    // copies A (and factors the copy for ILU(0) / IC(0)); solve() runs the
    // level-scheduled triangular solves in the reference's arithmetic order.
    class tri_precond_base : public preconditioner
    {
    protected:
        lab_precond M       = nullptr;
        bool        on_host = true;
        void        rebuild(lab_precond created);

    public:
        ~tri_precond_base();
        void        solve(const vector<double>& rhs, vector<double>& x) const override;
        void        move_to_device() override;
        void        move_to_host() override;
        bool        is_on_host() const override;
        lab_precond device_handle() const override
        {
            return M;
        }
    };

    // x = (D + L)^-1 rhs (preconditioner.cpp:80-105)
    class gauss_seidel_precond : public tri_precond_base
    {
    public:
        gauss_seidel_precond() {}
        void build(const csr_matrix<double>& A) override;
    };

    // x = (D / omega + L)^-1 rhs (preconditioner.cpp:121-156)
    class SOR_precond : public tri_precond_base
    {
    private:
        double omega;

    public:
        SOR_precond(double omega)
            : omega(omega)
        {
        }
        void build(const csr_matrix<double>& A) override;
    };

    // x = U^-1 L^-1 rhs with L = (beta D - E) D^-1, U = beta D - F built from A
    // (preconditioner.cpp:270-395)
    class SSOR_precond : public tri_precond_base
    {
    private:
        double omega;

    public:
        SSOR_precond(double omega)
            : omega(omega)
        {
        }
        void build(const csr_matrix<double>& A) override;
    };

    // x = U^-1 L^-1 rhs with the in-place ILU(0) of a copy of A (preconditioner.cpp:418-467)
    class ilu_precond : public tri_precond_base
    {
    public:
        ilu_precond() {}
        void build(const csr_matrix<double>& A) override;
    };

    // the IC(0) of a copy of A, then a lower and an upper solve on it
    // (preconditioner.cpp:492-542)
    class ic_precond : public tri_precond_base
    {
    public:
        ic_precond() {}
        void build(const csr_matrix<double>& A) override;
    };

    // AMG preconditioner: z = cycle(0; r).  build() runs the setup of `kind`
    // on A; alternatively attach an existing hierarchy (not owned).
    class amg_precond : public preconditioner
    {
    private:
        hierarchy        own;
        const hierarchy* h       = nullptr;
        lab_precond      M       = nullptr;
        lab_amg_options  opts;
        int              kind      = LAB_AMG_SA;
        int              max_level = 20;
        bool             on_host   = true;

    public:
        // Reference defaults for the composition: V-cycle, 1+1 Jacobi sweeps.
        explicit amg_precond(int presmoothing = 1, int postsmoothing = 1,
                             cycle cyc = cycle::vcycle, smoother sm = smoother::jacobi,
                             double jacobi_omega = 1.0);
        ~amg_precond();
        void set_setup(lab_amg_kind kind, int max_level);
        void set_precision(lab_precision p);
        void set_coarse_solver(lab_coarse c);
        void attach(const hierarchy& hier);
        void build(const csr_matrix<double>& A) override;
        void solve(const vector<double>& rhs, vector<double>& x) const override;
        void move_to_device() override;
        void move_to_host() override;
        bool is_on_host() const override;
        lab_precond device_handle() const override
        {
            return M;
        }
        const hierarchy& get_hierarchy() const
        {
            return *h;
        }
    };
}

#endif
