// Triangular path: level-scheduled sparse triangular solves, in-place ILU(0) and
// IC(0), behind the reference's csrtrsv / csrilu0 / csric0 and its ILU(0),
// IC(0), Gauss-Seidel and SOR preconditioners.
//
// Rows are grouped into dependency levels once per matrix pattern (on the host:
// a row's level is one more than the deepest row it reads); a level's rows are
// independent, so each level is one launch with a thread per row.  Every row is
// computed by one thread in exactly the reference's operation order
// (host_csrtrsv.cpp, host_csrilu0.cpp, host_csric0.cpp), so the results are
// bit-identical to the reference's sequential loops.
#include "internal.cuh"
#include "tri.cuh"

#include <algorithm>
#include <climits>
#include <vector>

namespace lab
{
    struct tri_sched
    {
        std::vector<int> ptr;          // level k: rows[ptr[k] .. ptr[k+1])
        int32_t*         rows = nullptr; // device, rows ordered by level
    };

    struct tri_plan
    {
        tri_sched lower, upper;
        int32_t*  diag     = nullptr; // device: position of a_ii in row i, -1 if absent
        bool      all_diag = true;
    };

    void tri_release(lab_csr_impl* A)
    {
        if(!A->tri)
            return;
        if(A->tri->lower.rows)
            cudaFree(A->tri->lower.rows);
        if(A->tri->upper.rows)
            cudaFree(A->tri->upper.rows);
        if(A->tri->diag)
            cudaFree(A->tri->diag);
        delete A->tri;
        A->tri = nullptr;
    }

    // Levels of the lower (reads columns < i) or upper (columns > i) dependency.
    static void level_sched(const std::vector<int32_t>& rp, const std::vector<int32_t>& ci,
                            int m, bool lower, std::vector<int>& order, std::vector<int>& ptr)
    {
        std::vector<int> lev(m, 0);
        int              nlev = 0;
        for(int t = 0; t < m; t++)
        {
            const int i = lower ? t : m - 1 - t;
            int       l = 0;
            for(int j = rp[i]; j < rp[i + 1]; j++)
            {
                const int c = ci[j];
                if(lower ? c < i : c > i)
                    l = std::max(l, lev[c] + 1);
            }
            lev[i] = l;
            nlev   = std::max(nlev, l + 1);
        }
        ptr.assign(nlev + 1, 0);
        for(int i = 0; i < m; i++)
            ptr[lev[i] + 1]++;
        for(int k = 0; k < nlev; k++)
            ptr[k + 1] += ptr[k];
        order.assign(m, 0);
        std::vector<int> cur(ptr.begin(), ptr.end() - 1);
        for(int i = 0; i < m; i++) // ascending rows within a level
            order[cur[lev[i]]++] = i;
    }

    lab_status tri_analyse(lab_csr_impl* A, cudaStream_t s)
    {
        if(A->tri)
            return LAB_OK;
        const int            m = (int)A->m;
        std::vector<int32_t> rp((size_t)m + 1), ci((size_t)std::max<int64_t>(A->nnz, 1));
        LAB_TRY(copy_d2h_sync(rp.data(), A->row_ptr, sizeof(int32_t) * rp.size(), s));
        if(A->nnz)
            LAB_TRY(copy_d2h_sync(ci.data(), A->col_ind, sizeof(int32_t) * A->nnz, s));
        tri_plan* p = new(std::nothrow) tri_plan();
        if(!p)
            return LAB_OOM;
        std::vector<int> dpos(m, -1), order;
        for(int i = 0; i < m; i++)
        {
            for(int j = rp[i]; j < rp[i + 1]; j++)
                if(ci[j] == i)
                {
                    dpos[i] = j;
                    break;
                }
            if(dpos[i] < 0)
                p->all_diag = false;
        }
        lab_status st = LAB_OK;
        auto       up = [&](int32_t** dst, const std::vector<int>& src) {
            if(st != LAB_OK)
                return;
            st = dalloc(dst, std::max<size_t>(src.size(), 1), s);
            if(st == LAB_OK && !src.empty() &&
               cudaMemcpyAsync(*dst, src.data(), sizeof(int32_t) * src.size(),
                               cudaMemcpyHostToDevice, s) != cudaSuccess)
                st = LAB_CUDA_ERROR;
        };
        level_sched(rp, ci, m, true, order, p->lower.ptr);
        up(&p->lower.rows, order);
        level_sched(rp, ci, m, false, order, p->upper.ptr);
        up(&p->upper.rows, order);
        up(&p->diag, dpos);
        if(st == LAB_OK && cudaStreamSynchronize(s) != cudaSuccess) // host vectors go out of scope
            st = LAB_CUDA_ERROR;
        A->tri = p;
        if(st != LAB_OK)
            tri_release(A);
        return st;
    }

    // ------------------------------------------------------------ solves
    // host_forward_solve_impl (host_csrtrsv.cpp:36-64): fma over the entries left of
    // the diagonal in CSR order, (b - sum) / d.  dscale != 0: d = a_ii * dscale (the
    // diagonal of SOR_precond's M, preconditioner.cpp:137-147).
    __global__ void k_trsv_lower(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                 const double* __restrict__ v, const int32_t* __restrict__ rows,
                                 int n, int unit, double dscale, const double* __restrict__ b,
                                 double* __restrict__ x, const int* skip)
    {
        if(skip && *skip)
            return;
        const int t = blockIdx.x * blockDim.x + threadIdx.x;
        if(t >= n)
            return;
        const int i   = rows[t];
        double    d   = 1.0;
        double    sum = 0.0;
        for(int j = rp[i]; j < rp[i + 1]; j++)
        {
            const int c = ci[j];
            if(c < i)
                sum = fma(v[j], x[c], sum);
            else if(!unit && c == i)
                d = dscale != 0.0 ? __dmul_rn(v[j], dscale) : v[j];
            else
                break;
        }
        x[i] = __ddiv_rn(__dsub_rn(b[i], sum), d);
    }

    // host_backward_solve_impl (host_csrtrsv.cpp:66-90): x = b, subtract a_ij x_j
    // walking the row right to left (multiply, then subtract), divide by d.
    __global__ void k_trsv_upper(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                 const double* __restrict__ v, const int32_t* __restrict__ rows,
                                 int n, int unit, const double* __restrict__ b,
                                 double* __restrict__ x, const int* skip)
    {
        if(skip && *skip)
            return;
        const int t = blockIdx.x * blockDim.x + threadIdx.x;
        if(t >= n)
            return;
        const int i  = rows[t];
        double    d  = 1.0;
        double    xi = b[i];
        for(int j = rp[i + 1] - 1; j >= rp[i]; j--)
        {
            const int c = ci[j];
            if(c > i)
                xi = __dsub_rn(xi, __dmul_rn(v[j], x[c]));
            else if(!unit && c == i)
                d = v[j];
        }
        x[i] = __ddiv_rn(xi, d);
    }

    lab_status tri_solve(lab_csr_impl* A, bool lower, bool unit, double dscale, const double* b,
                         double* x, cudaStream_t s, const int* skip)
    {
        if(A->m == 0)
            return LAB_OK;
        LAB_TRY(tri_analyse(A, s));
        const tri_sched& sc = lower ? A->tri->lower : A->tri->upper;
        for(size_t k = 0; k + 1 < sc.ptr.size(); k++)
        {
            const int      r0 = sc.ptr[k], n = sc.ptr[k + 1] - r0;
            const unsigned g  = (unsigned)ceil_div(n, 128);
            if(lower)
                LAB_LAUNCH(k_trsv_lower, g, 128, 0, s, A->row_ptr, A->col_ind, (const double*)A->val,
                           (const int32_t*)(sc.rows + r0), n, (int)unit, dscale, b, x, skip);
            else
                LAB_LAUNCH(k_trsv_upper, g, 128, 0, s, A->row_ptr, A->col_ind, (const double*)A->val,
                           (const int32_t*)(sc.rows + r0), n, (int)unit, b, x, skip);
        }
        return LAB_OK;
    }

    // ------------------------------------------------------------ factorizations
    // get_diagonal_value_local (host_csrilu0.cpp:35-54): the pivot of column col,
    // 1.0 (recorded) when it is missing or zero.
    __device__ __forceinline__ double tri_pivot(int col, int di, const double* v, int* sz, int* nz)
    {
        if(di == -1)
        {
            atomicMin(sz, col);
            return 1.0;
        }
        const double d = v[di];
        if(d == 0.0)
        {
            atomicMin(nz, col);
            return 1.0;
        }
        return d;
    }

    // One row of host_csrilu0_impl (host_csrilu0.cpp:66-100).  The reference looks
    // entries of the row up through a column->position map; both rows are sorted
    // by column, so a forward walk finds the same positions.  A missing pivot
    // (di = -1) keeps the reference's k loop from position 0 of the whole array and
    // searches the row for each column.
    __device__ void ilu0_row(int row, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                             double* v, const int32_t* __restrict__ diag, int* sz, int* nz)
    {
        const int a = rp[row], b = rp[row + 1];
        for(int j = a; j < b; j++)
        {
            const int cj = ci[j];
            if(cj > row)
                break;
            if(cj == row)
                break;
            const int    di  = diag[cj];
            const double piv = tri_pivot(cj, di, v, sz, nz);
            const int    end = rp[cj + 1];
            v[j]             = __ddiv_rn(v[j], piv);
            int          p   = a;
            for(int k = di + 1; k < end; k++)
            {
                const int ck = ci[k];
                int       t  = -1;
                if(di >= 0)
                {
                    while(p < b && ci[p] < ck)
                        p++;
                    if(p < b && ci[p] == ck)
                        t = p;
                }
                else
                {
                    for(int q = b - 1; q >= a; q--) // the map keeps the last position
                        if(ci[q] == ck)
                        {
                            t = q;
                            break;
                        }
                }
                // v[j] is re-read: with a missing pivot t can be j itself
                if(t != -1)
                    v[t] = __dsub_rn(v[t], __dmul_rn(v[j], v[k]));
            }
        }
    }

    // One row of host_csric0_impl (host_csric0.cpp:68-106).
    __device__ void ic0_row(int row, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                            double* v, const int32_t* __restrict__ diag, int* sz, int* nz)
    {
        const int a = rp[row], b = rp[row + 1];
        double    sum = 0.0;
        for(int j = a; j < b; j++)
        {
            const int cj = ci[j];
            if(cj < row)
            {
                const int di = diag[cj];
                double    s  = 0.0;
                int       p  = a;
                for(int k = rp[cj]; k < di; k++)
                {
                    const int ck = ci[k];
                    while(p < b && ci[p] < ck)
                        p++;
                    if(p < b && ci[p] == ck)
                        s = fma(v[p], v[k], s);
                }
                const double piv = tri_pivot(cj, di, v, sz, nz);
                const double val = __ddiv_rn(__dsub_rn(v[j], s), piv);
                sum              = fma(val, val, sum);
                v[j]             = val;
            }
            else if(cj == row)
            {
                v[j] = __dsqrt_rn(fabs(__dsub_rn(v[j], sum)));
                break;
            }
            else
                break;
        }
    }

    template <int IC>
    __global__ void k_factor_level(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                   double* v, const int32_t* __restrict__ diag,
                                   const int32_t* __restrict__ rows, int n, int* flags)
    {
        const int t = blockIdx.x * blockDim.x + threadIdx.x;
        if(t >= n)
            return;
        if(IC)
            ic0_row(rows[t], rp, ci, v, diag, flags, flags + 1);
        else
            ilu0_row(rows[t], rp, ci, v, diag, flags, flags + 1);
    }

    // Rows in order on one thread: ILU(0) with a missing pivot reads rows of any
    // level (the reference's k loop from position 0).
    __global__ void k_ilu0_sequential(const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                      double* v, const int32_t* __restrict__ diag, int m, int* flags)
    {
        for(int row = 0; row < m; row++)
            ilu0_row(row, rp, ci, v, diag, flags, flags + 1);
    }

    lab_status tri_factor(lab_csr_impl* A, bool ic, int* structural_zero, int* numeric_zero,
                          cudaStream_t s)
    {
        LAB_TRY(tri_analyse(A, s));
        dbuf<int> flags;
        LAB_TRY(flags.alloc(2, s));
        const int init[2] = {INT_MAX, INT_MAX};
        LAB_CUDA(cudaMemcpyAsync(flags.get(), init, sizeof(init), cudaMemcpyHostToDevice, s));
        const tri_plan& p = *A->tri;
        if(A->m > 0)
        {
            if(!ic && !p.all_diag)
                LAB_LAUNCH(k_ilu0_sequential, 1, 1, 0, s, A->row_ptr, A->col_ind, A->val,
                           (const int32_t*)p.diag, (int)A->m, flags.get());
            else
                for(size_t k = 0; k + 1 < p.lower.ptr.size(); k++)
                {
                    const int      r0 = p.lower.ptr[k], n = p.lower.ptr[k + 1] - r0;
                    const unsigned g  = (unsigned)ceil_div(n, 128);
                    if(ic)
                        LAB_LAUNCH(k_factor_level<1>, g, 128, 0, s, A->row_ptr, A->col_ind, A->val,
                                   (const int32_t*)p.diag, (const int32_t*)(p.lower.rows + r0), n,
                                   flags.get());
                    else
                        LAB_LAUNCH(k_factor_level<0>, g, 128, 0, s, A->row_ptr, A->col_ind, A->val,
                                   (const int32_t*)p.diag, (const int32_t*)(p.lower.rows + r0), n,
                                   flags.get());
                }
        }
        int h[2];
        LAB_TRY(copy_d2h_sync(h, flags.get(), sizeof(h), s));
        if(structural_zero)
            *structural_zero = h[0] == INT_MAX ? -1 : h[0];
        if(numeric_zero)
            *numeric_zero = h[1] == INT_MAX ? -1 : h[1];
        return LAB_OK;
    }
}

using namespace lab;

extern "C" {

LAB_API lab_status lab_csrtrsv(lab_csr A, int lower, int unit_diag, const double* b, double* x,
                               lab_stream s)
{
    LAB_ARG(A && (A->m == 0 || (b && x)), "null argument");
    LAB_ARG(A->m == A->n, "triangular solve needs a square matrix");
    LAB_TRY(ensure_init());
    return tri_solve(A, lower != 0, unit_diag != 0, 0.0, b, x, to_stream(s), nullptr);
}

LAB_API lab_status lab_csrilu0(lab_csr A, int* structural_zero, int* numeric_zero, lab_stream s)
{
    LAB_ARG(A, "null matrix");
    LAB_ARG(A->m == A->n, "ILU(0) needs a square matrix");
    LAB_TRY(ensure_init());
    LAB_TRY(tri_factor(A, false, structural_zero, numeric_zero, to_stream(s)));
    return lab_csr_values_changed(A);
}

LAB_API lab_status lab_csric0(lab_csr A, int* structural_zero, int* numeric_zero, lab_stream s)
{
    LAB_ARG(A, "null matrix");
    LAB_ARG(A->m == A->n, "IC(0) needs a square matrix");
    LAB_TRY(ensure_init());
    LAB_TRY(tri_factor(A, true, structural_zero, numeric_zero, to_stream(s)));
    return lab_csr_values_changed(A);
}

} // extern "C"
