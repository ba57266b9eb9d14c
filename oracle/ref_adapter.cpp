// Test infrastructure only: a C-ABI shim around the reference LinAlgLib host
// library, compiled together with the reference's own sources (oracle/Makefile)
// into oracle/_ref/liblinalg_ref.so.  Nothing in the product links it; the tests,
// __graft_entry__.smoke() and bench.py's CPU-baseline arm load it with ctypes.
//
// Each entry point drives the reference's public C++ API (namespace linalg) on
// host-resident objects exactly as the reference's own clients do
// (clients/testing/test_functions_amg.cpp:35-139, clients/examples/pcg_example.cpp).
// The one composition the reference lacks, AMG as a CG preconditioner, is the
// adapter class below: one V-cycle from a zero guess through amg_solve with
// max_cycle = 0 (library/src/iterative_solvers/amg/amg.cpp:516-571 runs exactly
// one cycle in that case, plus two fine-level residual evaluations).
#include "linalg.h"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fcntl.h>
#include <unistd.h>
#include <vector>

using namespace linalg;

namespace
{
    // The reference prints progress (and, without CUDA, a device warning per
    // vector) to stdout.  Route fd 1 to /dev/null while a reference call runs.
    int g_quiet = 1;

    struct quiet_scope
    {
        int saved = -1;
        quiet_scope()
        {
            if(!g_quiet)
                return;
            fflush(stdout);
            saved  = dup(1);
            int nf = open("/dev/null", O_WRONLY);
            dup2(nf, 1);
            close(nf);
        }
        ~quiet_scope()
        {
            if(saved < 0)
                return;
            fflush(stdout);
            dup2(saved, 1);
            close(saved);
        }
    };

    void to_csr(csr_matrix<double>& A, int m, int n, int nnz, const int* rp, const int* ci,
                const double* v)
    {
        std::vector<int>    r(rp, rp + m + 1);
        std::vector<int>    c(ci, ci + nnz);
        std::vector<double> x(v, v + nnz);
        A.resize(m, n, nnz);
        std::memcpy(A.get_row_ptr(), r.data(), sizeof(int) * (m + 1));
        if(nnz > 0)
        {
            std::memcpy(A.get_col_ind(), c.data(), sizeof(int) * nnz);
            std::memcpy(A.get_val(), x.data(), sizeof(double) * nnz);
        }
    }

    void copy_out(const csr_matrix<double>& A, int* rp, int* ci, double* v)
    {
        if(rp)
            std::memcpy(rp, A.get_row_ptr(), sizeof(int) * (A.get_m() + 1));
        if(ci && A.get_nnz() > 0)
            std::memcpy(ci, A.get_col_ind(), sizeof(int) * A.get_nnz());
        if(v && A.get_nnz() > 0)
            std::memcpy(v, A.get_val(), sizeof(double) * A.get_nnz());
    }

    // AMG V-cycle as a preconditioner: z = V(0; r).
    class amg_vcycle_precond : public preconditioner
    {
        const hierarchy* h;
        int              n1, n2;
        smoother         sm;

    public:
        amg_vcycle_precond(const hierarchy* h_, int n1_, int n2_, smoother sm_)
            : h(h_)
            , n1(n1_)
            , n2(n2_)
            , sm(sm_)
        {
        }
        void build(const csr_matrix<double>&) override {}
        void solve(const vector<double>& rhs, vector<double>& x) const override
        {
            x.zeros();
            iter_control c;
            c.max_cycle = 0;
            amg_solve(*h, x, rhs, n1, n2, cycle::vcycle, sm, c);
        }
        void move_to_device() override {}
        void move_to_host() override {}
        bool is_on_host() const override
        {
            return true;
        }
    };

    smoother to_smoother(int s)
    {
        switch(s)
        {
        case 1:
            return smoother::gauss_seidel;
        case 2:
            return smoother::symmetric_gauss_seidel;
        case 3:
            return smoother::SOR;
        case 4:
            return smoother::SSOR;
        default:
            return smoother::jacobi;
        }
    }
}

extern "C" {

void ref_set_quiet(int q)
{
    g_quiet = q;
}

// ---------------------------------------------------------------- hierarchy
// kind: 0 = SA (saamg.cpp:210), 1 = UA (uaamg.cpp:131), 2 = RS (rsamg.cpp:869)
void* ref_amg_setup(int kind, int m, int n, int nnz, const int* rp, const int* ci,
                    const double* v, int max_level)
{
    quiet_scope        q;
    csr_matrix<double> A;
    to_csr(A, m, n, nnz, rp, ci, v);
    hierarchy* h = new hierarchy();
    if(kind == 0)
        saamg_setup(A, max_level, *h);
    else if(kind == 1)
        uaamg_setup(A, max_level, *h);
    else
        rsamg_setup(A, max_level, *h);
    return h;
}

void ref_hier_free(void* h)
{
    quiet_scope q;
    delete static_cast<hierarchy*>(h);
}

int ref_hier_levels(void* h)
{
    return static_cast<hierarchy*>(h)->total_levels;
}

// which: 0 = A_l, 1 = P_l, 2 = R_l
static const csr_matrix<double>& hier_mat(void* hp, int l, int which)
{
    hierarchy* h = static_cast<hierarchy*>(hp);
    if(which == 1)
        return h->prolongations[l];
    if(which == 2)
        return h->restrictions[l];
    return h->A_cs[l];
}

void ref_hier_dims(void* h, int l, int which, int* m, int* n, int* nnz)
{
    const csr_matrix<double>& M = hier_mat(h, l, which);
    *m                          = M.get_m();
    *n                          = M.get_n();
    *nnz                        = M.get_nnz();
}

void ref_hier_copy(void* h, int l, int which, int* rp, int* ci, double* v)
{
    copy_out(hier_mat(h, l, which), rp, ci, v);
}

// PCG (cg.cpp:136-223) preconditioned by one AMG V-cycle per application.
// Returns the reference's iteration count.
int ref_amg_pcg(void* h, const double* b, double* x, int n1, int n2, int smoother_kind,
                double rel_tol, double abs_tol, int max_iter)
{
    quiet_scope               q;
    hierarchy*                hh = static_cast<hierarchy*>(h);
    const csr_matrix<double>& A  = hh->A_cs[0];
    int                       m  = A.get_m();
    vector<double>            vb(std::vector<double>(b, b + m));
    vector<double>            vx(std::vector<double>(x, x + m));
    amg_vcycle_precond        P(hh, n1, n2, to_smoother(smoother_kind));
    cg_solver                 cg;
    cg.build(A);
    iter_control c;
    c.rel_tol  = rel_tol;
    c.abs_tol  = abs_tol;
    c.max_iter = max_iter;
    int it     = cg.solve(A, vx, vb, &P, c);
    std::memcpy(x, vx.get_vec(), sizeof(double) * m);
    return it;
}

// Stationary AMG (amg.cpp:516-571). cycle: 0 = V, 1 = W, 2 = F.
int ref_amg_solve(void* h, const double* b, double* x, int n1, int n2, int cyc,
                  int smoother_kind, double rel_tol, double abs_tol, int max_cycle)
{
    quiet_scope               q;
    hierarchy*                hh = static_cast<hierarchy*>(h);
    const csr_matrix<double>& A  = hh->A_cs[0];
    int                       m  = A.get_m();
    vector<double>            vb(std::vector<double>(b, b + m));
    vector<double>            vx(std::vector<double>(x, x + m));
    iter_control              c;
    c.rel_tol   = rel_tol;
    c.abs_tol   = abs_tol;
    c.max_cycle = max_cycle;
    cycle cy    = cyc == 1 ? cycle::wcycle : (cyc == 2 ? cycle::fcycle : cycle::vcycle);
    int   it    = amg_solve(*hh, vx, vb, n1, n2, cy, to_smoother(smoother_kind), c);
    std::memcpy(x, vx.get_vec(), sizeof(double) * m);
    return it;
}

// One preconditioner application z = V(0; r), for V-cycle parity.
void ref_amg_vcycle(void* h, const double* r, double* z, int n1, int n2, int smoother_kind)
{
    quiet_scope        q;
    hierarchy*         hh = static_cast<hierarchy*>(h);
    int                m  = hh->A_cs[0].get_m();
    vector<double>     vr(std::vector<double>(r, r + m));
    vector<double>     vz(m);
    amg_vcycle_precond P(hh, n1, n2, to_smoother(smoother_kind));
    P.solve(vr, vz);
    std::memcpy(z, vz.get_vec(), sizeof(double) * m);
}

// Unpreconditioned / Jacobi-preconditioned CG and GMRES on the reference.
// precond: 0 = none, 1 = jacobi_precond (preconditioner.cpp:41-78)
int ref_cg(int m, int nnz, const int* rp, const int* ci, const double* v, const double* b,
           double* x, int precond, double rel_tol, double abs_tol, int max_iter)
{
    quiet_scope        q;
    csr_matrix<double> A;
    to_csr(A, m, m, nnz, rp, ci, v);
    vector<double> vb(std::vector<double>(b, b + m));
    vector<double> vx(std::vector<double>(x, x + m));
    cg_solver      cg;
    cg.build(A);
    iter_control c;
    c.rel_tol  = rel_tol;
    c.abs_tol  = abs_tol;
    c.max_iter = max_iter;
    jacobi_precond J;
    int            it;
    if(precond == 1)
    {
        J.build(A);
        it = cg.solve(A, vx, vb, &J, c);
    }
    else
        it = cg.solve(A, vx, vb, nullptr, c);
    std::memcpy(x, vx.get_vec(), sizeof(double) * m);
    return it;
}

int ref_gmres(int m, int nnz, const int* rp, const int* ci, const double* v, const double* b,
              double* x, int restart, void* amg_h, int n1, int n2, double rel_tol,
              double abs_tol, int max_iter)
{
    quiet_scope        q;
    csr_matrix<double> A;
    to_csr(A, m, m, nnz, rp, ci, v);
    vector<double> vb(std::vector<double>(b, b + m));
    vector<double> vx(std::vector<double>(x, x + m));
    gmres_solver   g;
    g.build(A, restart);
    iter_control c;
    c.rel_tol  = rel_tol;
    c.abs_tol  = abs_tol;
    c.max_iter = max_iter;
    int it;
    if(amg_h)
    {
        amg_vcycle_precond P(static_cast<hierarchy*>(amg_h), n1, n2, smoother::jacobi);
        it = g.solve(A, vx, vb, &P, c);
    }
    else
        it = g.solve(A, vx, vb, nullptr, c);
    std::memcpy(x, vx.get_vec(), sizeof(double) * m);
    return it;
}

// ---------------------------------------------------------------- kernels
void ref_spmv(int m, int n, int nnz, const int* rp, const int* ci, const double* v, double alpha,
              const double* x, double beta, double* y)
{
    quiet_scope        q;
    csr_matrix<double> A;
    to_csr(A, m, n, nnz, rp, ci, v);
    vector<double> vx(std::vector<double>(x, x + n));
    vector<double> vy(std::vector<double>(y, y + m));
    csrmv_descr*   d = nullptr;
    create_csrmv_descr(&d);
    csrmv_analysis(A, csrmv_algorithm::default_algorithm, d);
    csrmv_solve(alpha, A, vx, beta, vy, csrmv_algorithm::default_algorithm, d);
    destroy_csrmv_descr(d);
    std::memcpy(y, vy.get_vec(), sizeof(double) * m);
}

void ref_residual(int m, int n, int nnz, const int* rp, const int* ci, const double* v,
                  const double* x, const double* b, double* r)
{
    quiet_scope        q;
    csr_matrix<double> A;
    to_csr(A, m, n, nnz, rp, ci, v);
    vector<double> vx(std::vector<double>(x, x + n));
    vector<double> vb(std::vector<double>(b, b + m));
    vector<double> vr(m);
    compute_residual(A, vx, vb, vr);
    std::memcpy(r, vr.get_vec(), sizeof(double) * m);
}

// C = A * B through csr_matrix::multiply_by_matrix (csr_matrix.cpp:333-353).
// Returns an opaque matrix; read it with ref_mat_dims / ref_mat_copy.
void* ref_spgemm(int ma, int na, int nnza, const int* rpa, const int* cia, const double* va,
                 int mb, int nb, int nnzb, const int* rpb, const int* cib, const double* vb)
{
    quiet_scope        q;
    csr_matrix<double> A, B;
    to_csr(A, ma, na, nnza, rpa, cia, va);
    to_csr(B, mb, nb, nnzb, rpb, cib, vb);
    csr_matrix<double>* C = new csr_matrix<double>();
    A.multiply_by_matrix(*C, B);
    return C;
}

// C = alpha * A * B through the descriptor form csrgemm_nnz + csrgemm_solve
// (linalg_math.cpp:330-357, host_csrgemm.cpp:195-245) with beta = 0 and an empty D,
// the form the reference's host path runs.
void* ref_csrgemm(double alpha, int ma, int na, int nnza, const int* rpa, const int* cia,
                  const double* va, int mb, int nb, int nnzb, const int* rpb, const int* cib,
                  const double* vb)
{
    quiet_scope        q;
    csr_matrix<double> A, B, D;
    to_csr(A, ma, na, nnza, rpa, cia, va);
    to_csr(B, mb, nb, nnzb, rpb, cib, vb);
    csr_matrix<double>* C = new csr_matrix<double>();
    csrgemm_descr*      d = nullptr;
    create_csrgemm_descr(&d);
    csrgemm_nnz(A, B, D, *C, csrgemm_algorithm::default_algorithm, d);
    csrgemm_solve(alpha, A, B, 0.0, D, *C, csrgemm_algorithm::default_algorithm, d);
    destroy_csrgemm_descr(d);
    return C;
}

// C = alpha*A + beta*B through csrgeam (linalg_math.cpp:275-307).
void* ref_spgeam(double alpha, int m, int n, int nnza, const int* rpa, const int* cia,
                 const double* va, double beta, int nnzb, const int* rpb, const int* cib,
                 const double* vb)
{
    quiet_scope        q;
    csr_matrix<double> A, B;
    to_csr(A, m, n, nnza, rpa, cia, va);
    to_csr(B, m, n, nnzb, rpb, cib, vb);
    csr_matrix<double>* C = new csr_matrix<double>();
    csrgeam_descr*      d = nullptr;
    create_csrgeam_descr(&d);
    csrgeam_nnz(A, B, *C, csrgeam_algorithm::default_algorithm, d);
    csrgeam_solve(alpha, A, beta, B, *C, csrgeam_algorithm::default_algorithm, d);
    destroy_csrgeam_descr(d);
    return C;
}

void* ref_transpose(int m, int n, int nnz, const int* rp, const int* ci, const double* v)
{
    quiet_scope        q;
    csr_matrix<double> A;
    to_csr(A, m, n, nnz, rp, ci, v);
    csr_matrix<double>* T = new csr_matrix<double>();
    A.transpose(*T);
    return T;
}

void ref_mat_dims(void* M, int* m, int* n, int* nnz)
{
    csr_matrix<double>* A = static_cast<csr_matrix<double>*>(M);
    *m                    = A->get_m();
    *n                    = A->get_n();
    *nnz                  = A->get_nnz();
}

void ref_mat_copy(void* M, int* rp, int* ci, double* v)
{
    copy_out(*static_cast<csr_matrix<double>*>(M), rp, ci, v);
}

void ref_mat_free(void* M)
{
    quiet_scope q;
    delete static_cast<csr_matrix<double>*>(M);
}

// ---------------------------------------------------------------- AMG pieces
void ref_strength(int m, int nnz, const int* rp, const int* ci, const double* v, double eps,
                  int* conn)
{
    quiet_scope        q;
    csr_matrix<double> A;
    to_csr(A, m, m, nnz, rp, ci, v);
    vector<int> c(nnz, 0);
    compute_strong_connections(A, eps, c);
    std::memcpy(conn, c.get_vec(), sizeof(int) * nnz);
}

// PMIS aggregation (amg_aggregation.cpp:106-215) on a given connection array.
void ref_pmis(int m, int nnz, const int* rp, const int* ci, const double* v, const int* conn,
              int64_t* aggregates)
{
    quiet_scope        q;
    csr_matrix<double> A;
    to_csr(A, m, m, nnz, rp, ci, v);
    vector<int>     c(std::vector<int>(conn, conn + nnz));
    vector<int64_t> agg(m, 0);
    vector<int64_t> roots;
    agg.zeros();
    compute_aggregates_using_pmis(A, c, agg, roots);
    std::memcpy(aggregates, agg.get_vec(), sizeof(int64_t) * m);
}

// Classical (RS) strength: connections plus the S matrix (host_amg_strength.cpp:72-156).
void* ref_classical_strength(int m, int nnz, const int* rp, const int* ci, const double* v,
                             double theta, int* conn)
{
    quiet_scope        q;
    csr_matrix<double> A;
    to_csr(A, m, m, nnz, rp, ci, v);
    vector<int> c(nnz, 0);
    c.zeros();
    csr_matrix<double>* S = new csr_matrix<double>();
    compute_classical_strong_connections(A, theta, *S, c);
    std::memcpy(conn, c.get_vec(), sizeof(int) * nnz);
    return S;
}

// C/F splitting, both passes (amg_aggregation.cpp:225-251).
void ref_cfpoints(int m, int nnz, const int* rp, const int* ci, const double* v, uint32_t* cf)
{
    quiet_scope        q;
    csr_matrix<double> S, ST;
    to_csr(S, m, m, nnz, rp, ci, v);
    S.transpose(ST);
    vector<uint32_t> c(m, 0);
    compute_cfpoint_first_pass(S, ST, c);
    compute_cfpoint_second_pass(S, c);
    std::memcpy(cf, c.get_vec(), sizeof(uint32_t) * m);
}

void ref_exclusive_scan_i64(int64_t* x, int n)
{
    vector<int64_t> v(std::vector<int64_t>(x, x + n));
    exclusive_scan(v);
    std::memcpy(x, v.get_vec(), sizeof(int64_t) * n);
}

// In-place incomplete factorizations (linalg_math.h:95-109 -> host_csrilu0.cpp,
// host_csric0.cpp); the factored values overwrite v.
void ref_csrilu0(int m, int nnz, const int* rp, const int* ci, double* v, int* structural_zero,
                 int* numeric_zero)
{
    quiet_scope        q;
    csr_matrix<double> A;
    to_csr(A, m, m, nnz, rp, ci, v);
    csrilu0(A, structural_zero, numeric_zero);
    std::memcpy(v, A.get_val(), sizeof(double) * nnz);
}

void ref_csric0(int m, int nnz, const int* rp, const int* ci, double* v, int* structural_zero,
                int* numeric_zero)
{
    quiet_scope        q;
    csr_matrix<double> A;
    to_csr(A, m, m, nnz, rp, ci, v);
    csric0(A, structural_zero, numeric_zero);
    std::memcpy(v, A.get_val(), sizeof(double) * nnz);
}

// Triangular solve on the lower or upper part of A (csrtrsv_analysis/_solve,
// linalg_math.h:229-254 -> host_csrtrsv.cpp).
void ref_trsv(int m, int nnz, const int* rp, const int* ci, const double* v, int lower,
              int unit_diag, const double* b, double* x)
{
    quiet_scope        q;
    csr_matrix<double> A;
    to_csr(A, m, m, nnz, rp, ci, v);
    vector<double> vb(std::vector<double>(b, b + m));
    vector<double> vx(m);
    csrtrsv_descr* d = nullptr;
    create_csrtrsv_descr(&d);
    const triangular_type t = lower ? triangular_type::lower : triangular_type::upper;
    const diagonal_type   g = unit_diag ? diagonal_type::unit : diagonal_type::non_unit;
    csrtrsv_analysis(A, t, g, d);
    csrtrsv_solve(A, vb, vx, 1.0, t, g, d);
    destroy_csrtrsv_descr(d);
    std::memcpy(x, vx.get_vec(), sizeof(double) * m);
}

// One application x = M^-1 rhs of the reference's triangular-solve
// preconditioners (preconditioner.cpp): kind 0 ILU(0), 1 IC(0), 2 Gauss-Seidel,
// 3 SOR(omega), 4 SSOR(omega).
void ref_precond_apply(int kind, double omega, int m, int nnz, const int* rp, const int* ci,
                       const double* v, const double* rhs, double* x)
{
    quiet_scope        q;
    csr_matrix<double> A;
    to_csr(A, m, m, nnz, rp, ci, v);
    preconditioner* P = nullptr;
    if(kind == 0)
        P = new ilu_precond();
    else if(kind == 1)
        P = new ic_precond();
    else if(kind == 2)
        P = new gauss_seidel_precond();
    else if(kind == 3)
        P = new SOR_precond(omega);
    else
        P = new SSOR_precond(omega);
    P->build(A);
    vector<double> vr(std::vector<double>(rhs, rhs + m));
    vector<double> vx(m);
    P->solve(vr, vx);
    std::memcpy(x, vx.get_vec(), sizeof(double) * m);
    delete P;
}

// CG with one of the preconditioners above; returns the iteration count.
int ref_precond_cg(int kind, double omega, int m, int nnz, const int* rp, const int* ci,
                   const double* v, const double* b, double* x, double rel_tol, double abs_tol,
                   int max_iter)
{
    quiet_scope        q;
    csr_matrix<double> A;
    to_csr(A, m, m, nnz, rp, ci, v);
    preconditioner* P = nullptr;
    if(kind == 0)
        P = new ilu_precond();
    else if(kind == 1)
        P = new ic_precond();
    else if(kind == 2)
        P = new gauss_seidel_precond();
    else if(kind == 3)
        P = new SOR_precond(omega);
    else
        P = new SSOR_precond(omega);
    P->build(A);
    vector<double> vb(std::vector<double>(b, b + m));
    vector<double> vx(std::vector<double>(x, x + m));
    iter_control   c;
    c.rel_tol  = rel_tol;
    c.abs_tol  = abs_tol;
    c.max_iter = max_iter;
    cg_solver cg;
    cg.build(A);
    int it = cg.solve(A, vx, vb, P, c);
    std::memcpy(x, vx.get_vec(), sizeof(double) * m);
    delete P;
    return it;
}

// ---------------------------------------------------------------- Matrix Market
// csr_matrix::read_mtx (csr_matrix.cpp:523-729).  Returns a matrix to read with
// ref_mat_dims / ref_mat_copy, or null when read_mtx returned false.
void* ref_read_mtx(const char* path)
{
    quiet_scope         q;
    csr_matrix<double>* A = new csr_matrix<double>();
    if(!A->read_mtx(path))
    {
        delete A;
        return nullptr;
    }
    return A;
}

// csr_matrix::write_mtx (csr_matrix.cpp:731-795); returns its bool.
int ref_write_mtx(const char* path, int m, int n, int nnz, const int* rp, const int* ci,
                  const double* v)
{
    quiet_scope        q;
    csr_matrix<double> A;
    to_csr(A, m, n, nnz, rp, ci, v);
    return A.write_mtx(path) ? 1 : 0;
}

// ---------------------------------------------------------------- csr_matrix members
// copy_lower_triangular_from / copy_upper_triangular_from (csr_matrix.cpp:170-225)
void* ref_triangle(int m, int n, int nnz, const int* rp, const int* ci, const double* v,
                   int upper)
{
    quiet_scope         q;
    csr_matrix<double>  A;
    to_csr(A, m, n, nnz, rp, ci, v);
    csr_matrix<double>* T = new csr_matrix<double>();
    if(upper)
        T->copy_upper_triangular_from(A, false);
    else
        T->copy_lower_triangular_from(A, false);
    return T;
}

// scale_diagonal_by (kind 0) / scale_by_inverse_diagonal (kind 1), values out
void ref_scale(int m, int n, int nnz, const int* rp, const int* ci, const double* v, int kind,
               double scalar, double* out)
{
    quiet_scope        q;
    csr_matrix<double> A;
    to_csr(A, m, n, nnz, rp, ci, v);
    if(kind == 0)
        A.scale_diagonal_by(scalar);
    else
        A.scale_by_inverse_diagonal();
    std::memcpy(out, A.get_val(), sizeof(double) * nnz);
}

} // extern "C"
