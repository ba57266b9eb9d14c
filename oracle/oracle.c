/* Test infrastructure only: CPU restatement of the reference AMG-PCG path.
 * See oracle.h for the contract.  Reference citations are paths inside the
 * LinAlgLib tree (library/src/...).  Compiled with -ffp-contract=off. */
#include "oracle.h"

#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ CSR utils */
void orc_csr_free(orc_csr* A)
{
    if(!A)
        return;
    free(A->rp);
    free(A->ci);
    free(A->v);
    A->rp = NULL;
    A->ci = NULL;
    A->v  = NULL;
    A->m = A->n = A->nnz = 0;
}

int orc_csr_alloc(orc_csr* A, int m, int n, int nnz)
{
    A->m   = m;
    A->n   = n;
    A->nnz = nnz;
    A->rp  = (int*)calloc((size_t)m + 1, sizeof(int));
    A->ci  = (int*)calloc(nnz > 0 ? (size_t)nnz : 1, sizeof(int));
    A->v   = (double*)calloc(nnz > 0 ? (size_t)nnz : 1, sizeof(double));
    return (A->rp && A->ci && A->v) ? 0 : -1;
}

/* ------------------------------------------------------------------ BLAS-like */
/* library/src/backend/host/host_extract.cpp:34-52: first diagonal entry, 0 if none */
void orc_diag(const orc_csr* A, double* d)
{
    for(int i = 0; i < A->m; i++)
    {
        d[i] = 0.0;
        for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
            if(A->ci[j] == i)
            {
                d[i] = A->v[j];
                break;
            }
    }
}

/* library/src/backend/host/host_matrix_vector.cpp:60-84: fma accumulation in CSR order */
void orc_spmv(const orc_csr* A, double alpha, const double* x, double beta, double* y)
{
    for(int i = 0; i < A->m; i++)
    {
        double s = 0.0;
        for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
            s = fma(A->v[j], x[A->ci[j]], s);
        y[i] = beta == 0.0 ? alpha * s : fma(alpha, s, beta * y[i]);
    }
}

/* library/src/backend/host/host_matrix_vector.cpp:36-57: plain multiply-add */
void orc_residual(const orc_csr* A, const double* x, const double* b, double* r)
{
    for(int i = 0; i < A->m; i++)
    {
        double s = 0.0;
        for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
            s += A->v[j] * x[A->ci[j]];
        r[i] = b[i] - s;
    }
}

/* library/src/backend/host/host_axpy.cpp:85-97 (sequential order) */
double orc_dot(const double* x, const double* y, int n)
{
    double s = 0.0;
    for(int i = 0; i < n; i++)
        s += x[i] * y[i];
    return s;
}

/* library/src/backend/host/host_math.cpp:36-50 */
double orc_norm_inf(const double* x, int n)
{
    double s = 0.0;
    for(int i = 0; i < n; i++)
    {
        double a = fabs(x[i]);
        s        = (s < a) ? a : s;
    }
    return s;
}

/* library/src/backend/host/host_primitives.cpp:76-91 */
void orc_exclusive_scan_i64(int64_t* x, int n)
{
    int64_t sum = 0;
    for(int i = 0; i < n; i++)
    {
        int64_t t = x[i];
        x[i]      = sum;
        sum += t;
    }
}

/* library/src/backend/host/host_csr2csc.cpp:30-75: stable (source rows ascending) */
int orc_transpose(const orc_csr* A, orc_csr* T)
{
    if(orc_csr_alloc(T, A->n, A->m, A->nnz))
        return -1;
    for(int j = 0; j < A->nnz; j++)
        T->rp[A->ci[j] + 1]++;
    for(int i = 0; i < A->n; i++)
        T->rp[i + 1] += T->rp[i];
    int* next = (int*)malloc(sizeof(int) * ((size_t)A->n + 1));
    memcpy(next, T->rp, sizeof(int) * ((size_t)A->n + 1));
    for(int i = 0; i < A->m; i++)
        for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
        {
            int p    = next[A->ci[j]]++;
            T->ci[p] = i;
            T->v[p]  = A->v[j];
        }
    free(next);
    return 0;
}

/* sort (col, val) pairs of one row by column; columns are unique */
static void sort_row(int* c, double* v, int n)
{
    for(int a = 1; a < n; a++)
    {
        int    kc = c[a];
        double kv = v[a];
        int    b  = a - 1;
        while(b >= 0 && c[b] > kc)
        {
            c[b + 1] = c[b];
            v[b + 1] = v[b];
            b--;
        }
        c[b + 1] = kc;
        v[b + 1] = kv;
    }
}

/* library/src/backend/host/host_csrgemm.cpp:37-183 (alpha = 1, no D):
 * Gustavson; the first product of a column sets the entry, later ones add, in
 * A-row order then B-row order; each output row is then sorted by column. */
int orc_spgemm(const orc_csr* A, const orc_csr* B, orc_csr* C)
{
    int  m    = A->m, n = B->n;
    int* mark = (int*)malloc(sizeof(int) * (n > 0 ? (size_t)n : 1));
    int* rp   = (int*)calloc((size_t)m + 1, sizeof(int));
    for(int c = 0; c < n; c++)
        mark[c] = -1;
    for(int i = 0; i < m; i++)
    {
        for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
        {
            int k = A->ci[j];
            for(int p = B->rp[k]; p < B->rp[k + 1]; p++)
            {
                int c = B->ci[p];
                if(mark[c] != i)
                {
                    mark[c] = i;
                    rp[i + 1]++;
                }
            }
        }
    }
    for(int i = 0; i < m; i++)
        rp[i + 1] += rp[i];
    if(orc_csr_alloc(C, m, n, rp[m]))
        return -1;
    memcpy(C->rp, rp, sizeof(int) * ((size_t)m + 1));
    free(rp);
    for(int c = 0; c < n; c++)
        mark[c] = -1;
    for(int i = 0; i < m; i++)
    {
        int begin = C->rp[i], end = begin;
        for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
        {
            int    k  = A->ci[j];
            double va = 1.0 * A->v[j];
            for(int p = B->rp[k]; p < B->rp[k + 1]; p++)
            {
                int c = B->ci[p];
                if(mark[c] < begin)
                {
                    mark[c]    = end;
                    C->ci[end] = c;
                    C->v[end]  = va * B->v[p];
                    end++;
                }
                else
                    C->v[mark[c]] += va * B->v[p];
            }
        }
        sort_row(C->ci + begin, C->v + begin, end - begin);
    }
    free(mark);
    return 0;
}

/* library/src/backend/host/host_csrgeam.cpp: C = alpha*A + beta*B; A's entries
 * first, then B's (added to an existing column or appended), rows sorted. */
int orc_spgeam(double alpha, const orc_csr* A, double beta, const orc_csr* B, orc_csr* C)
{
    int  m = A->m, n = A->n;
    int* mark = (int*)malloc(sizeof(int) * (n > 0 ? (size_t)n : 1));
    int* rp   = (int*)calloc((size_t)m + 1, sizeof(int));
    for(int c = 0; c < n; c++)
        mark[c] = -1;
    for(int i = 0; i < m; i++)
    {
        int cnt = 0;
        for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
            if(mark[A->ci[j]] != i)
            {
                mark[A->ci[j]] = i;
                cnt++;
            }
        for(int j = B->rp[i]; j < B->rp[i + 1]; j++)
            if(mark[B->ci[j]] != i)
            {
                mark[B->ci[j]] = i;
                cnt++;
            }
        rp[i + 1] = cnt;
    }
    for(int i = 0; i < m; i++)
        rp[i + 1] += rp[i];
    if(orc_csr_alloc(C, m, n, rp[m]))
        return -1;
    memcpy(C->rp, rp, sizeof(int) * ((size_t)m + 1));
    free(rp);
    for(int c = 0; c < n; c++)
        mark[c] = -1;
    for(int i = 0; i < m; i++)
    {
        int begin = C->rp[i], end = begin;
        for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
        {
            C->ci[end]     = A->ci[j];
            C->v[end]      = alpha * A->v[j];
            mark[A->ci[j]] = end++;
        }
        for(int j = B->rp[i]; j < B->rp[i + 1]; j++)
        {
            int c = B->ci[j];
            if(mark[c] >= begin)
                C->v[mark[c]] += beta * B->v[j];
            else
            {
                C->ci[end] = c;
                C->v[end]  = beta * B->v[j];
                mark[c]    = end++;
            }
        }
        sort_row(C->ci + begin, C->v + begin, end - begin);
    }
    free(mark);
    return 0;
}

/* ------------------------------------------------------------------ strength */
/* library/src/backend/host/host_amg_strength.cpp:33-70 */
void orc_strength(const orc_csr* A, double eps, int* conn)
{
    double* d = (double*)malloc(sizeof(double) * ((size_t)A->m + 1));
    orc_diag(A, d);
    for(int i = 0; i < A->m; i++)
        for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
        {
            int    c = A->ci[j];
            double v = A->v[j];
            conn[j]  = (c != i) && (fabs(v) >= eps * sqrt(fabs(d[i]) * fabs(d[c])));
        }
    free(d);
}

/* library/src/backend/host/host_amg_strength.cpp:72-156 */
int orc_classical_strength(const orc_csr* A, double theta, int* conn, orc_csr* S)
{
    int* cnt = (int*)calloc((size_t)A->m + 1, sizeof(int));
    for(int i = 0; i < A->m; i++)
    {
        double mx = -DBL_MAX;
        for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
            if(A->ci[j] != i)
                mx = (mx < -A->v[j]) ? -A->v[j] : mx;
        for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
            if(-A->v[j] >= theta * mx && A->ci[j] != i)
            {
                conn[j] = 1;
                cnt[i + 1]++;
            }
    }
    for(int i = 0; i < A->m; i++)
        cnt[i + 1] += cnt[i];
    if(orc_csr_alloc(S, A->m, A->n, cnt[A->m]))
        return -1;
    memcpy(S->rp, cnt, sizeof(int) * ((size_t)A->m + 1));
    free(cnt);
    for(int i = 0; i < A->m; i++)
    {
        int p = S->rp[i];
        for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
            if(conn[j] == 1)
            {
                S->ci[p] = A->ci[j];
                S->v[p]  = A->v[j];
                p++;
            }
    }
    return 0;
}

/* ------------------------------------------------------------------ PMIS */
/* library/src/backend/host/host_amg_aggregation.cpp:32-38 */
static unsigned int orc_hash1(unsigned int x)
{
    x = ((x >> 16) ^ x) * 0x45d9f3bu;
    x = ((x >> 16) ^ x) * 0x45d9f3bu;
    x = (x >> 16) ^ x;
    return x / 2u;
}

typedef struct
{
    int state, hash, row;
} orc_node;

/* host_amg_aggregation.cpp:77-93: the candidate wins only if strictly larger */
static orc_node lexmax(orc_node a, orc_node b)
{
    if(b.state > a.state)
        return b;
    if(b.state == a.state && b.hash > a.hash)
        return b;
    return a;
}

/* library/src/iterative_solvers/amg/amg_aggregation.cpp:106-215 with the host
 * kernels of library/src/backend/host/host_amg_aggregation.cpp:40-221.
 * aggregates is overwritten (the reference callers zero it first,
 * saamg.cpp:241-245). */
void orc_pmis(const orc_csr* A, const int* conn, int64_t* agg, int* rounds_out)
{
    int  m     = A->m;
    int* hash  = (int*)malloc(sizeof(int) * ((size_t)m + 1));
    int* state = (int*)malloc(sizeof(int) * ((size_t)m + 1));
    int* mx    = (int*)malloc(sizeof(int) * ((size_t)m + 1));
    for(int i = 0; i < m; i++)
    {
        int s = -2;
        for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
            if(conn[j] == 1)
            {
                s = 0;
                break;
            }
        mx[i]   = s;
        hash[i] = (int)orc_hash1((unsigned int)i);
        agg[i]  = 0;
    }
    int iter = 0;
    while(iter < 20)
    {
        memcpy(state, mx, sizeof(int) * (size_t)m);
        int complete = 1;
        for(int i = 0; i < m; i++)
        {
            orc_node best = {state[i], hash[i], i};
            for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
                if(conn[j] == 1)
                {
                    int      c = A->ci[j];
                    orc_node nd = {state[c], hash[c], c};
                    best        = lexmax(best, nd);
                }
            int r = best.row;
            for(int j = A->rp[r]; j < A->rp[r + 1]; j++)
                if(conn[j] == 1)
                {
                    int      c = A->ci[j];
                    orc_node nd = {state[c], hash[c], c};
                    best        = lexmax(best, nd);
                }
            if(state[i] == 0)
            {
                if(best.row == i)
                {
                    mx[i]  = 1;
                    agg[i] = 1;
                }
                else if(best.state == 1)
                {
                    mx[i]  = -1;
                    agg[i] = 0;
                }
                else
                    complete = 0;
            }
        }
        if(complete)
            break;
        iter++;
    }
    if(rounds_out)
        *rounds_out = iter;
    orc_exclusive_scan_i64(agg, m);
    for(int k = 0; k < 2; k++)
    {
        memcpy(state, mx, sizeof(int) * (size_t)m);
        for(int i = 0; i < m; i++)
        {
            if(state[i] == -1)
            {
                for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
                    if(conn[j] == 1 && state[A->ci[j]] == 1)
                    {
                        agg[i] = agg[A->ci[j]];
                        mx[i]  = 1;
                        break;
                    }
            }
            else if(state[i] == -2)
                agg[i] = -2;
        }
    }
    free(hash);
    free(state);
    free(mx);
}

/* ------------------------------------------------------------------ prolongation */
/* (key, value) pairs of one row, stably sorted by key, equal keys summed in order */
typedef struct
{
    int64_t key;
    double  val;
} orc_kv;

static int sort_reduce(orc_kv* kv, int n)
{
    for(int a = 1; a < n; a++)
    {
        orc_kv t = kv[a];
        int    b = a - 1;
        while(b >= 0 && kv[b].key > t.key)
        {
            kv[b + 1] = kv[b];
            b--;
        }
        kv[b + 1] = t;
    }
    int out = 0;
    for(int a = 0; a < n; a++)
    {
        if(out > 0 && kv[out - 1].key == kv[a].key)
            kv[out - 1].val += kv[a].val;
        else
            kv[out++] = kv[a];
    }
    return out;
}

/* library/src/iterative_solvers/amg/saamg.cpp:51-207 */
int orc_sa_prolongation(const orc_csr* A, const int* conn, const int64_t* agg, double relax,
                        orc_csr* P)
{
    int64_t nc = -1;
    for(int i = 0; i < A->m; i++)
        if(nc < agg[i])
            nc = agg[i];
    nc++;
    int maxrow = 0;
    for(int i = 0; i < A->m; i++)
        if(A->rp[i + 1] - A->rp[i] > maxrow)
            maxrow = A->rp[i + 1] - A->rp[i];
    orc_kv* kv = (orc_kv*)malloc(sizeof(orc_kv) * ((size_t)maxrow + 1));
    int*    rp = (int*)calloc((size_t)A->m + 1, sizeof(int));
    for(int i = 0; i < A->m; i++)
    {
        int n = 0;
        for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
        {
            int c = A->ci[j];
            if((c == i || conn[j] == 1) && agg[c] >= 0)
            {
                kv[n].key = agg[c];
                kv[n].val = 0.0;
                n++;
            }
        }
        rp[i + 1] = sort_reduce(kv, n);
    }
    for(int i = 0; i < A->m; i++)
        rp[i + 1] += rp[i];
    if(orc_csr_alloc(P, A->m, (int)nc, rp[A->m]))
        return -1;
    memcpy(P->rp, rp, sizeof(int) * ((size_t)A->m + 1));
    free(rp);
    for(int i = 0; i < A->m; i++)
    {
        double dg = 0.0;
        for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
        {
            if(A->ci[j] == i)
                dg += A->v[j];
            else if(conn[j] == 0)
                dg -= A->v[j];
        }
        double inv = 1.0 / dg;
        int    n   = 0;
        for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
        {
            int c = A->ci[j];
            if((c == i || conn[j] == 1) && agg[c] >= 0)
            {
                kv[n].key = agg[c];
                kv[n].val = (c == i) ? 1.0 - relax : -relax * inv * A->v[j];
                n++;
            }
        }
        n = sort_reduce(kv, n);
        for(int k = 0; k < n; k++)
        {
            P->ci[P->rp[i] + k] = (int)kv[k].key;
            P->v[P->rp[i] + k]  = kv[k].val;
        }
    }
    free(kv);
    return 0;
}

/* library/src/iterative_solvers/amg/uaamg.cpp:49-128 */
int orc_ua_prolongation(const orc_csr* A, const int64_t* agg, orc_csr* P)
{
    int64_t nc = -1;
    for(int i = 0; i < A->m; i++)
        if(nc < agg[i])
            nc = agg[i];
    nc++;
    int nnz = 0;
    for(int i = 0; i < A->m; i++)
        nnz += agg[i] >= 0;
    if(orc_csr_alloc(P, A->m, (int)nc, nnz))
        return -1;
    for(int i = 0; i < A->m; i++)
        P->rp[i + 1] = P->rp[i] + (agg[i] >= 0);
    for(int i = 0; i < A->m; i++)
        if(agg[i] >= 0)
        {
            P->ci[P->rp[i]] = (int)agg[i];
            P->v[P->rp[i]]  = 1.0;
        }
    return 0;
}

/* ------------------------------------------------------------------ RS C/F split */
#define ORC_F 0u
#define ORC_C 1u
#define ORC_U 2u
#define ORC_FF 3u

/* library/src/backend/host/host_amg_aggregation.cpp:228-439 (first pass: bucket
 * list of nodes ordered by lambda = |S^T row|, greedy from the largest) and
 * 441-519 (second pass: F-F pairs without a common C point). */
void orc_cfpoints(const orc_csr* S, const orc_csr* ST, uint32_t* cf)
{
    int  m      = S->m;
    int* lambda = (int*)calloc((size_t)m + 1, sizeof(int));
    int* ptr    = (int*)calloc((size_t)m + 2, sizeof(int));
    int* count  = (int*)calloc((size_t)m + 1, sizeof(int));
    int* i2n    = (int*)calloc((size_t)m + 1, sizeof(int));
    int* n2i    = (int*)calloc((size_t)m + 1, sizeof(int));
    for(int i = 0; i < m; i++)
    {
        cf[i]     = ORC_U;
        lambda[i] = ST->rp[i + 1] - ST->rp[i];
    }
    for(int i = 0; i < m; i++)
        ptr[lambda[i] + 1]++;
    for(int i = 0; i < m; i++)
        ptr[i + 1] += ptr[i];
    for(int i = 0; i < m; i++)
    {
        int lam    = lambda[i];
        int idx    = ptr[lam] + count[lam];
        i2n[idx]   = i;
        n2i[i]     = idx;
        count[lam] = count[lam] + 1;
    }
    for(int i = m - 1; i >= 0; i--)
    {
        int node = i2n[i];
        if(lambda[node] <= 0)
            break;
        if(cf[node] != ORC_U)
            continue;
        cf[node] = ORC_C;
        for(int j = ST->rp[node]; j < ST->rp[node + 1]; j++)
            if(cf[ST->ci[j]] == ORC_U)
                cf[ST->ci[j]] = ORC_FF;
        for(int j = ST->rp[node]; j < ST->rp[node + 1]; j++)
        {
            int f = ST->ci[j];
            if(cf[f] != ORC_FF)
                continue;
            cf[f] = ORC_F;
            for(int k = S->rp[f]; k < S->rp[f + 1]; k++)
            {
                int u = S->ci[k];
                if(cf[u] != ORC_U)
                    continue;
                /* move u to the top of its lambda bucket, then grow lambda */
                int lu      = lambda[u];
                int old_pos = n2i[u];
                int new_pos = ptr[lu] + count[lu] - 1;
                n2i[i2n[old_pos]] = new_pos;
                n2i[i2n[new_pos]] = old_pos;
                int t             = i2n[old_pos];
                i2n[old_pos]      = i2n[new_pos];
                i2n[new_pos]      = t;
                count[lu]--;
                count[lu + 1]++;
                ptr[lu + 1] = ptr[lu] + count[lu];
                lambda[u]++;
            }
        }
        for(int j = S->rp[node]; j < S->rp[node + 1]; j++)
        {
            int u = S->ci[j];
            if(cf[u] != ORC_U || lambda[u] <= 0)
                continue;
            /* move u to the bottom of its lambda bucket, then shrink lambda */
            int lu      = lambda[u];
            int old_pos = n2i[u];
            int new_pos = ptr[lu];
            n2i[i2n[old_pos]] = new_pos;
            n2i[i2n[new_pos]] = old_pos;
            int t             = i2n[old_pos];
            i2n[old_pos]      = i2n[new_pos];
            i2n[new_pos]      = t;
            count[lu]--;
            count[lu - 1]++;
            ptr[lu]++;
            lambda[u]--;
        }
    }
    for(int i = 0; i < m; i++)
        if(cf[i] == ORC_U)
            cf[i] = ORC_F;
    free(lambda);
    free(ptr);
    free(count);
    free(i2n);
    free(n2i);

    /* second pass */
    for(int i = 0; i < m; i++)
    {
        if(cf[i] != ORC_F)
            continue;
        int s0 = S->rp[i], s1 = S->rp[i + 1];
        int cand = -1;
        for(int j = s0; j < s1; j++)
        {
            int c = S->ci[j];
            if(cf[c] != ORC_F)
                continue;
            int a = s0, b = S->rp[c], be = S->rp[c + 1];
            int found = 0;
            while(a < s1 && b < be)
            {
                int c1 = S->ci[a], c2 = S->ci[b];
                if(c1 < c2)
                    a++;
                else if(c2 < c1)
                    b++;
                else
                {
                    a++;
                    b++;
                    if(cf[c1] == ORC_C)
                    {
                        found = 1;
                        break;
                    }
                }
            }
            if(!found)
            {
                if(cand >= 0)
                    cf[cand] = ORC_F;
                cand  = c;
                cf[c] = ORC_C;
            }
        }
    }
}

/* library/src/iterative_solvers/amg/rsamg.cpp:672-866, including the index
 * quirk at line 818 (A's column array read with an S position). */
int orc_direct_interpolation(const orc_csr* A, const orc_csr* S, const uint32_t* cf, orc_csr* P)
{
    int m  = A->m;
    int nc = 0;
    for(int i = 0; i < m; i++)
        nc += cf[i] == ORC_C;
    int* rp = (int*)calloc((size_t)m + 1, sizeof(int));
    for(int i = 0; i < m; i++)
    {
        if(cf[i] == ORC_C)
            rp[i + 1] = 1;
        else
            for(int j = S->rp[i]; j < S->rp[i + 1]; j++)
                rp[i + 1] += cf[S->ci[j]] == ORC_C;
    }
    for(int i = 0; i < m; i++)
        rp[i + 1] += rp[i];
    if(orc_csr_alloc(P, m, nc, rp[m]))
        return -1;
    memcpy(P->rp, rp, sizeof(int) * ((size_t)m + 1));
    free(rp);
    uint32_t* cidx = (uint32_t*)calloc((size_t)m + 1, sizeof(uint32_t));
    for(int i = 0; i < m; i++)
        cidx[i + 1] = cidx[i] + cf[i];
    for(int i = 0; i < m; i++)
    {
        int p = P->rp[i];
        if(cf[i] == ORC_C)
        {
            P->ci[p] = (int)cidx[i];
            P->v[p]  = 1.0;
            continue;
        }
        double dg = 0.0, pos = 0.0, neg = 0.0;
        for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
        {
            if(A->ci[j] == i)
                dg = A->v[j];
            else if(A->v[j] < 0.0)
                neg += A->v[j];
            else
                pos += A->v[j];
        }
        double spos = 0.0, sneg = 0.0;
        for(int j = S->rp[i]; j < S->rp[i + 1]; j++)
        {
            if(cf[A->ci[j]] == ORC_C)
            {
                if(S->v[j] < 0.0)
                    sneg += S->v[j];
                else
                    spos += S->v[j];
            }
        }
        double alpha = neg / sneg;
        double beta  = pos / spos;
        for(int j = S->rp[i]; j < S->rp[i + 1]; j++)
        {
            int c = S->ci[j];
            if(cf[c] != ORC_C)
                continue;
            P->ci[p] = (int)cidx[c];
            P->v[p]  = (S->v[j] < 0.0) ? -alpha * S->v[j] / dg : -beta * S->v[j] / dg;
            p++;
        }
    }
    free(cidx);
    return 0;
}

/* ------------------------------------------------------------------ setup */
static int csr_copy(orc_csr* dst, const orc_csr* src)
{
    if(orc_csr_alloc(dst, src->m, src->n, src->nnz))
        return -1;
    memcpy(dst->rp, src->rp, sizeof(int) * ((size_t)src->m + 1));
    if(src->nnz)
    {
        memcpy(dst->ci, src->ci, sizeof(int) * (size_t)src->nnz);
        memcpy(dst->v, src->v, sizeof(double) * (size_t)src->nnz);
    }
    return 0;
}

/* library/src/iterative_solvers/amg/saamg.cpp:210-282, uaamg.cpp:131-224,
 * rsamg.cpp:869-947 */
orc_hier* orc_amg_setup(int kind, const orc_csr* A0, int max_level)
{
    orc_hier* h = (orc_hier*)calloc(1, sizeof(orc_hier));
    if(max_level > 20)
        max_level = 20;
    csr_copy(&h->A[0], A0);
    double eps   = kind == ORC_UA ? 0.001 : 0.08;
    double relax = 2.0 / 3.0;
    double theta = 0.2;
    int    level = 0;
    while(level < max_level)
    {
        orc_csr* Af = &h->A[level];
        orc_csr* P  = &h->P[level];
        int*     conn = (int*)calloc(Af->nnz > 0 ? (size_t)Af->nnz : 1, sizeof(int));
        if(kind == ORC_RS)
        {
            orc_csr   S, ST;
            uint32_t* cf = (uint32_t*)calloc((size_t)Af->m + 1, sizeof(uint32_t));
            orc_classical_strength(Af, theta, conn, &S);
            orc_transpose(&S, &ST);
            orc_cfpoints(&S, &ST, cf);
            orc_direct_interpolation(Af, &S, cf, P);
            orc_csr_free(&S);
            orc_csr_free(&ST);
            free(cf);
        }
        else
        {
            int64_t* agg = (int64_t*)calloc((size_t)Af->m + 1, sizeof(int64_t));
            orc_strength(Af, eps, conn);
            orc_pmis(Af, conn, agg, NULL);
            if(kind == ORC_SA)
                orc_sa_prolongation(Af, conn, agg, relax, P);
            else
                orc_ua_prolongation(Af, agg, P);
            free(agg);
        }
        free(conn);
        if(P->n == 0)
        {
            orc_csr_free(P);
            break;
        }
        orc_transpose(P, &h->R[level]);
        orc_csr AP;
        orc_spgemm(Af, P, &AP);
        orc_spgemm(&h->R[level], &AP, &h->A[level + 1]);
        orc_csr_free(&AP);
        level++;
        eps *= 0.5;
    }
    h->levels = level;
    return h;
}

void orc_hier_free(orc_hier* h)
{
    if(!h)
        return;
    for(int l = 0; l < 21; l++)
        orc_csr_free(&h->A[l]);
    for(int l = 0; l < 20; l++)
    {
        orc_csr_free(&h->P[l]);
        orc_csr_free(&h->R[l]);
    }
    free(h->coarse_inv);
    for(int l = 0; l < 21; l++)
    {
        free(h->mc_order[l]);
        free(h->mc_ptr[l]);
    }
    free(h);
}

/* ------------------------------------------------------------------ solve */
/* library/src/iterative_solvers/classic/jacobi.cpp:43-75, with an optional weight:
 * x = xold + omega*(x_J - xold); omega == 1 is the reference's unweighted sweep. */
static void jacobi_sweep(const orc_csr* A, double* x, const double* b, double omega, double* xo)
{
    memcpy(xo, x, sizeof(double) * (size_t)A->m);
    for(int j = 0; j < A->m; j++)
    {
        double sigma = 0.0, ajj = 0.0;
        for(int k = A->rp[j]; k < A->rp[j + 1]; k++)
        {
            if(A->ci[k] != j)
                sigma = sigma + A->v[k] * xo[A->ci[k]];
            else
                ajj = A->v[k];
        }
        double xj = (b[j] - sigma) / ajj;
        x[j]      = omega == 1.0 ? xj : xo[j] + omega * (xj - xo[j]);
    }
}

/* library/src/iterative_solvers/classic/gauss_seidel.cpp:50-87 */
static void gs_sweep(const orc_csr* A, double* x, const double* b)
{
    for(int j = 0; j < A->m; j++)
    {
        double sigma = 0.0, ajj = 0.0;
        for(int k = A->rp[j]; k < A->rp[j + 1]; k++)
        {
            if(A->ci[k] != j)
                sigma = sigma + A->v[k] * x[A->ci[k]];
            else
                ajj = A->v[k];
        }
        x[j] = (b[j] - sigma) / ajj;
    }
}

/* ------------------------------------------------------------------ multicolour GS
 * No reference counterpart (the reference's Gauss-Seidel visits rows in order,
 * gauss_seidel.cpp:50-87).  This restates the device smoother, so its GS / SGS /
 * SOR / SSOR V-cycles are checked against something: a Jones-Plassmann-Luby
 * colouring of the pattern of A + A^T in which a row takes colour c when its
 * priority (hash(i), i) beats every neighbour still uncoloured at the start of
 * round c; a sweep visits the colours in order (SSOR: forward, then backward)
 * and sets x_i <- x_i + omega * ((1 / a_ii) * (b_i - sum_j a_ij x_j)), the sum in
 * CSR order over the whole row (a_ii included) with the current x. */
static unsigned mc_hash(unsigned x)
{
    x ^= 0x9e3779b9u;
    x = ((x >> 16) ^ x) * 0x45d9f3bu;
    x = ((x >> 16) ^ x) * 0x45d9f3bu;
    return (x >> 16) ^ x;
}

int orc_mc_colouring(const orc_csr* A, int* colour)
{
    const int m = A->m;
    orc_csr   T = {0}, G = {0};
    orc_transpose(A, &T);
    orc_spgeam(1.0, A, 1.0, &T, &G);
    orc_csr_free(&T);
    for(int i = 0; i < m; i++)
        colour[i] = -1;
    int left = m, c = 0;
    /* a row coloured earlier in this round still counts as uncoloured: the round
     * reads the state at its start, so colour c is a neighbour that competed */
    for(; left > 0; c++)
        for(int i = 0; i < m; i++)
        {
            if(colour[i] >= 0)
                continue;
            const unsigned hi = mc_hash((unsigned)i);
            int            win = 1;
            for(int j = G.rp[i]; j < G.rp[i + 1] && win; j++)
            {
                const int k = G.ci[j];
                if(k == i || (colour[k] >= 0 && colour[k] != c))
                    continue;
                const unsigned hk = mc_hash((unsigned)k);
                if(hk > hi || (hk == hi && k > i))
                    win = 0;
            }
            if(win)
            {
                colour[i] = c;
                left--;
            }
        }
    orc_csr_free(&G);
    return c;
}

static void mc_prepare(orc_hier* h, int level)
{
    if(h->mc_order[level])
        return;
    const orc_csr* A   = &h->A[level];
    int*           col = (int*)malloc(sizeof(int) * ((size_t)A->m + 1));
    int            nc  = orc_mc_colouring(A, col);
    int*           ptr = (int*)calloc((size_t)nc + 2, sizeof(int));
    int*           ord = (int*)malloc(sizeof(int) * ((size_t)A->m + 1));
    for(int i = 0; i < A->m; i++)
        ptr[col[i] + 1]++;
    for(int c = 0; c < nc; c++)
        ptr[c + 1] += ptr[c];
    int* cur = (int*)malloc(sizeof(int) * ((size_t)nc + 1));
    memcpy(cur, ptr, sizeof(int) * (size_t)nc);
    for(int i = 0; i < A->m; i++)
        ord[cur[col[i]]++] = i;
    free(cur);
    free(col);
    h->mc_order[level] = ord;
    h->mc_ptr[level]   = ptr;
    h->mc_ncol[level]  = nc;
}

static void mc_colour_pass(const orc_csr* A, const int* rows, int nr, const double* invd,
                           double* x, const double* b, double omega)
{
    for(int q = 0; q < nr; q++)
    {
        const int i = rows[q];
        double    s = 0.0;
        for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
            s = fma(A->v[j], x[A->ci[j]], s);
        x[i] = x[i] + omega * (invd[i] * (b[i] - s));
    }
}

static void mc_sweep(orc_hier* h, int level, double* x, const double* b, double omega, int sym)
{
    mc_prepare(h, level);
    const orc_csr* A    = &h->A[level];
    double*        invd = (double*)malloc(sizeof(double) * ((size_t)A->m + 1));
    orc_diag(A, invd);
    for(int i = 0; i < A->m; i++)
        invd[i] = 1.0 / invd[i];
    const int* ptr = h->mc_ptr[level];
    for(int c = 0; c < h->mc_ncol[level]; c++)
        mc_colour_pass(A, h->mc_order[level] + ptr[c], ptr[c + 1] - ptr[c], invd, x, b, omega);
    if(sym)
        for(int c = h->mc_ncol[level] - 1; c >= 0; c--)
            mc_colour_pass(A, h->mc_order[level] + ptr[c], ptr[c + 1] - ptr[c], invd, x, b,
                           omega);
    free(invd);
}

static void smooth_sweep(orc_hier* h, int level, double* x, const double* b, int smoother,
                         double omega, double* tmp)
{
    const orc_csr* A = &h->A[level];
    if(smoother == ORC_SMOOTH_GS)
        gs_sweep(A, x, b);
    else if(smoother == ORC_SMOOTH_MC_GS || smoother == ORC_SMOOTH_MC_SSOR)
        mc_sweep(h, level, x, b, omega, smoother == ORC_SMOOTH_MC_SSOR);
    else
        jacobi_sweep(A, x, b, omega, tmp);
}

/* dense inverse of the coarsest operator by Gauss-Jordan with partial pivoting */
static void build_coarse_inverse(orc_hier* h)
{
    const orc_csr* A = &h->A[h->levels];
    int            n = A->m;
    double*        M = (double*)calloc((size_t)n * n, sizeof(double));
    double*        I = (double*)calloc((size_t)n * n, sizeof(double));
    for(int i = 0; i < n; i++)
    {
        I[(size_t)i * n + i] = 1.0;
        for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
            M[(size_t)i * n + A->ci[j]] += A->v[j];
    }
    for(int c = 0; c < n; c++)
    {
        int p = c;
        for(int r = c + 1; r < n; r++)
            if(fabs(M[(size_t)r * n + c]) > fabs(M[(size_t)p * n + c]))
                p = r;
        if(p != c)
            for(int k = 0; k < n; k++)
            {
                double t              = M[(size_t)c * n + k];
                M[(size_t)c * n + k]  = M[(size_t)p * n + k];
                M[(size_t)p * n + k]  = t;
                t                     = I[(size_t)c * n + k];
                I[(size_t)c * n + k]  = I[(size_t)p * n + k];
                I[(size_t)p * n + k]  = t;
            }
        double piv = M[(size_t)c * n + c];
        for(int k = 0; k < n; k++)
        {
            M[(size_t)c * n + k] /= piv;
            I[(size_t)c * n + k] /= piv;
        }
        for(int r = 0; r < n; r++)
        {
            if(r == c)
                continue;
            double f = M[(size_t)r * n + c];
            if(f == 0.0)
                continue;
            for(int k = 0; k < n; k++)
            {
                M[(size_t)r * n + k] -= f * M[(size_t)c * n + k];
                I[(size_t)r * n + k] -= f * I[(size_t)c * n + k];
            }
        }
    }
    free(M);
    h->coarse_inv = I;
}

/* library/src/iterative_solvers/amg/amg.cpp:144-267 */
void orc_vcycle(orc_hier* h, int level, double* x, const double* b, int n1, int n2,
                int smoother, double omega, int coarse)
{
    const orc_csr* A = &h->A[level];
    int            N = A->m;
    if(level < h->levels)
    {
        const orc_csr* R  = &h->R[level];
        const orc_csr* P  = &h->P[level];
        int            Nc = h->A[level + 1].m;
        double*        tmp = (double*)malloc(sizeof(double) * ((size_t)N + 1));
        for(int i = 0; i < n1; i++)
            smooth_sweep(h, level, x, b, smoother, omega, tmp);
        double* r  = (double*)malloc(sizeof(double) * ((size_t)N + 1));
        double* wr = (double*)calloc((size_t)Nc + 1, sizeof(double));
        double* ec = (double*)calloc((size_t)Nc + 1, sizeof(double));
        orc_residual(A, x, b, r);
        orc_spmv(R, 1.0, r, 0.0, wr);
        orc_vcycle(h, level + 1, ec, wr, n1, n2, smoother, omega, coarse);
        orc_spmv(P, 1.0, ec, 1.0, x);
        for(int i = 0; i < n2; i++)
            smooth_sweep(h, level, x, b, smoother, omega, tmp);
        free(tmp);
        free(r);
        free(wr);
        free(ec);
        return;
    }
    if(N == 1)
    {
        x[0] = b[0] / A->v[0];
        return;
    }
    if(coarse == ORC_COARSE_DIRECT)
    {
        if(!h->coarse_inv)
            build_coarse_inverse(h);
        for(int i = 0; i < N; i++)
        {
            double s = 0.0;
            for(int k = 0; k < N; k++)
                s += h->coarse_inv[(size_t)i * N + k] * b[k];
            x[i] = s;
        }
        return;
    }
    for(int it = 0; it < 1000; it++)
        gs_sweep(A, x, b);
}

/* library/src/iterative_solvers/iter_control.cpp:38-78 */
static int converges(double rn, double r0, double rel_tol, double abs_tol)
{
    if(isnan(rn) || isnan(r0))
        return 0;
    if(rn <= abs_tol)
        return 1;
    if(rn / r0 <= rel_tol)
        return 1;
    return 0;
}

/* library/src/iterative_solvers/krylov/cg.cpp:136-223 with M^{-1} = one V-cycle
 * from a zero guess.  Returns the reference's iteration count. */
int orc_amg_pcg(orc_hier* h, const double* b, double* x, int n1, int n2, int smoother,
                double omega, int coarse, double rel_tol, double abs_tol, int max_iter,
                double* final_rel)
{
    const orc_csr* A = &h->A[0];
    int            m = A->m;
    double*        r = (double*)malloc(sizeof(double) * ((size_t)m + 1));
    double*        z = (double*)malloc(sizeof(double) * ((size_t)m + 1));
    double*        p = (double*)malloc(sizeof(double) * ((size_t)m + 1));
    orc_residual(A, x, b, r);
    double r0 = orc_norm_inf(r, m);
    memset(z, 0, sizeof(double) * (size_t)m);
    orc_vcycle(h, 0, z, r, n1, n2, smoother, omega, coarse);
    memcpy(p, z, sizeof(double) * (size_t)m);
    double gamma = orc_dot(z, r, m);
    int    iter  = 0;
    double rn    = r0;
    while(!(iter > max_iter))
    {
        orc_spmv(A, 1.0, p, 0.0, z);
        double alpha = gamma / orc_dot(z, p, m);
        for(int i = 0; i < m; i++)
            x[i] = alpha == 1.0 ? p[i] + x[i] : alpha * p[i] + x[i];
        double na = -1.0 * alpha;
        for(int i = 0; i < m; i++)
            r[i] = na == 1.0 ? z[i] + r[i] : na * z[i] + r[i];
        rn = orc_norm_inf(r, m);
        if(converges(rn, r0, rel_tol, abs_tol))
            break;
        memset(z, 0, sizeof(double) * (size_t)m);
        orc_vcycle(h, 0, z, r, n1, n2, smoother, omega, coarse);
        double old = gamma;
        gamma      = orc_dot(z, r, m);
        double beta = gamma / old;
        for(int i = 0; i < m; i++)
            p[i] = beta == 0.0 ? 1.0 * z[i] : 1.0 * z[i] + beta * p[i];
        iter++;
    }
    if(final_rel)
        *final_rel = rn / r0;
    free(r);
    free(z);
    free(p);
    return iter;
}

/* cg.cpp:60-134 (precond none; note the reference restarts every iteration
 * there because restart_iter = -1, cg.cpp:89) and cg.cpp:136-223 with
 * jacobi_precond (preconditioner.cpp:41-78, host_math.cpp:52-64) */
int orc_cg(const orc_csr* A, const double* b, double* x, int jacobi, double rel_tol,
           double abs_tol, int max_iter)
{
    int     m = A->m;
    double* r = (double*)malloc(sizeof(double) * ((size_t)m + 1));
    double* z = (double*)malloc(sizeof(double) * ((size_t)m + 1));
    double* p = (double*)malloc(sizeof(double) * ((size_t)m + 1));
    double* d = (double*)malloc(sizeof(double) * ((size_t)m + 1));
    orc_diag(A, d);
    orc_residual(A, x, b, r);
    double r0 = orc_norm_inf(r, m);
    double gamma;
    if(jacobi)
    {
        for(int i = 0; i < m; i++)
            z[i] = r[i] / d[i];
        memcpy(p, z, sizeof(double) * (size_t)m);
        gamma = orc_dot(z, r, m);
    }
    else
    {
        memcpy(p, r, sizeof(double) * (size_t)m);
        gamma = orc_dot(r, r, m);
    }
    int iter = 0;
    while(!(iter > max_iter))
    {
        if(!jacobi && iter > 0)
        {
            orc_residual(A, x, b, r);
            memcpy(p, r, sizeof(double) * (size_t)m);
            gamma = orc_dot(r, r, m);
        }
        orc_spmv(A, 1.0, p, 0.0, z);
        double alpha = gamma / orc_dot(z, p, m);
        for(int i = 0; i < m; i++)
            x[i] = alpha == 1.0 ? p[i] + x[i] : alpha * p[i] + x[i];
        double na = -1.0 * alpha;
        for(int i = 0; i < m; i++)
            r[i] = na == 1.0 ? z[i] + r[i] : na * z[i] + r[i];
        double rn = orc_norm_inf(r, m);
        if(converges(rn, r0, rel_tol, abs_tol))
            break;
        double old = gamma;
        if(jacobi)
        {
            for(int i = 0; i < m; i++)
                z[i] = r[i] / d[i];
            gamma = orc_dot(z, r, m);
        }
        else
            gamma = orc_dot(r, r, m);
        double beta = gamma / old;
        const double* src = jacobi ? z : r;
        for(int i = 0; i < m; i++)
            p[i] = beta == 0.0 ? 1.0 * src[i] : 1.0 * src[i] + beta * p[i];
        iter++;
    }
    free(r);
    free(z);
    free(p);
    free(d);
    return iter;
}

/* library/src/iterative_solvers/amg/amg.cpp:516-571 (V-cycle) */
int orc_amg_solve(orc_hier* h, const double* b, double* x, int n1, int n2, int smoother,
                  double omega, int coarse, double rel_tol, double abs_tol, int max_cycle)
{
    const orc_csr* A = &h->A[0];
    int            m = A->m;
    double*        r = (double*)malloc(sizeof(double) * ((size_t)m + 1));
    orc_residual(A, x, b, r);
    double r0    = orc_norm_inf(r, m);
    int    cycle = 0;
    while(!(cycle > max_cycle))
    {
        orc_vcycle(h, 0, x, b, n1, n2, smoother, omega, coarse);
        orc_residual(A, x, b, r);
        double rn = orc_norm_inf(r, m);
        if(converges(rn, r0, rel_tol, abs_tol))
            break;
        cycle++;
    }
    free(r);
    return cycle;
}

/* ======================================================================
 * Triangular path
 * ==================================================================== */

/* get_diagonal_value_local (host_csrilu0.cpp:35-54, host_csric0.cpp:35-54): the
 * pivot of column `col`, 1.0 for a missing or zero one (recorded). */
static double tri_pivot(int col, int diag_index, const double* v, int* sz, int* nz)
{
    if(diag_index == -1)
    {
        if(sz && col < *sz)
            *sz = col;
        return 1.0;
    }
    double d = v[diag_index];
    if(d == 0.0)
    {
        if(nz && col < *nz)
            *nz = col;
        return 1.0;
    }
    return d;
}

/* host_csrilu0_impl (host_csrilu0.cpp:57-102): row by row, every lower entry
 * (CSR order, up to the diagonal) is divided by its column's pivot and then
 * eliminates the matching entries of the row with the pivot row's part right of
 * its diagonal (k from diag_index + 1, as the reference writes it). */
void orc_csrilu0(orc_csr* A, int* structural_zero, int* numeric_zero)
{
    const int m = A->m;
    int*      dp  = (int*)malloc(sizeof(int) * (m > 0 ? m : 1));
    int*      map = (int*)malloc(sizeof(int) * (A->n > 0 ? A->n : 1));
    if(structural_zero)
        *structural_zero = INT_MAX;
    if(numeric_zero)
        *numeric_zero = INT_MAX;
    for(int i = 0; i < m; i++)
        dp[i] = -1;
    for(int c = 0; c < A->n; c++)
        map[c] = -1;
    double* v = A->v;
    for(int row = 0; row < m; row++)
    {
        const int a = A->rp[row], b = A->rp[row + 1];
        for(int j = a; j < b; j++)
            map[A->ci[j]] = j;
        for(int j = a; j < b; j++)
        {
            const int cj = A->ci[j];
            if(cj < row)
            {
                const int    di  = dp[cj];
                const double piv = tri_pivot(cj, di, v, structural_zero, numeric_zero);
                const int    end = A->rp[cj + 1];
                v[j]             = v[j] / piv;
                for(int k = di + 1; k < end; k++)
                {
                    const int t = map[A->ci[k]];
                    if(t != -1)
                        v[t] = v[t] - v[j] * v[k];
                }
            }
            else if(cj == row)
            {
                dp[row] = j;
                break;
            }
            else
                break;
        }
        for(int j = a; j < b; j++)
            map[A->ci[j]] = -1;
    }
    free(map);
    free(dp);
}

/* host_csric0_impl (host_csric0.cpp:57-110): lower entries in CSR order become
 * (a_ij - sum_k l_ik l_jk) / l_jj (fma-accumulated over the pivot row's part left
 * of its diagonal), the diagonal sqrt(|a_ii - sum_j l_ij^2|); the upper part is
 * left as it was. */
void orc_csric0(orc_csr* A, int* structural_zero, int* numeric_zero)
{
    const int m = A->m;
    int*      dp  = (int*)malloc(sizeof(int) * (m > 0 ? m : 1));
    int*      map = (int*)malloc(sizeof(int) * (A->n > 0 ? A->n : 1));
    if(structural_zero)
        *structural_zero = INT_MAX;
    if(numeric_zero)
        *numeric_zero = INT_MAX;
    for(int i = 0; i < m; i++)
        dp[i] = -1;
    for(int c = 0; c < A->n; c++)
        map[c] = -1;
    double* v = A->v;
    for(int row = 0; row < m; row++)
    {
        const int a = A->rp[row], b = A->rp[row + 1];
        for(int j = a; j < b; j++)
            map[A->ci[j]] = j;
        double sum = 0.0;
        for(int j = a; j < b; j++)
        {
            const int cj = A->ci[j];
            if(cj < row)
            {
                const int di = dp[cj];
                double    s  = 0.0;
                for(int k = A->rp[cj]; k < di; k++)
                {
                    const int t = map[A->ci[k]];
                    if(t != -1)
                        s = fma(v[t], v[k], s);
                }
                const double piv = tri_pivot(cj, di, v, structural_zero, numeric_zero);
                const double val = (v[j] - s) / piv;
                sum              = fma(val, val, sum);
                v[j]             = val;
            }
            else if(cj == row)
            {
                dp[row] = j;
                v[j]    = sqrt(fabs(v[j] - sum));
                break;
            }
            else
                break;
        }
        for(int j = a; j < b; j++)
            map[A->ci[j]] = -1;
    }
    free(map);
    free(dp);
}

/* host_forward_solve_impl / host_backward_solve_impl (host_csrtrsv.cpp:36-90):
 * forward: fma over the entries left of the diagonal in CSR order, then
 * (b - sum) / d; backward: x = b, subtract a_ij x_j walking the row right to
 * left, then divide by the diagonal. unit_diag: d = 1. */
void orc_trsv(const orc_csr* A, int lower, int unit_diag, const double* b, double* x)
{
    const int n = A->m;
    if(lower)
    {
        for(int i = 0; i < n; i++)
        {
            double d = 1.0, sum = 0.0;
            for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
            {
                const int c = A->ci[j];
                if(c < i)
                    sum = fma(A->v[j], x[c], sum);
                else if(!unit_diag && c == i)
                    d = A->v[j];
                else
                    break;
            }
            x[i] = (b[i] - sum) / d;
        }
    }
    else
    {
        for(int i = n - 1; i >= 0; i--)
        {
            double d  = 1.0;
            double xi = b[i];
            for(int j = A->rp[i + 1] - 1; j >= A->rp[i]; j--)
            {
                const int c = A->ci[j];
                if(c > i)
                    xi = xi - A->v[j] * x[c];
                else if(!unit_diag && c == i)
                    d = A->v[j];
            }
            x[i] = xi / d;
        }
    }
}

/* preconditioner.cpp: ilu_precond (432-468), ic_precond (506-543): factor a copy,
 * lower solve (unit / non-unit), upper solve of the same matrix (non-unit; for
 * IC(0) its upper part is A's, unchanged by the factorization);
 * gauss_seidel_precond (90-105): lower non-unit solve on A's lower part;
 * SOR_precond (137-156): the same with the diagonal scaled by 1 / omega;
 * SSOR_precond (kind 4, below).  tri_prepare is the build() (F gets its own
 * values), tri_apply the solve(). */
/* SSOR_precond::build (preconditioner.cpp:283-353) with host_ssor_fill_lower_precond
 * / host_ssor_fill_upper_precond (host_ssor.cpp:52-142): L holds a_ij / d_j left of
 * the diagonal and "beta" on it, U holds a_ij right of it and beta * a_ii on it, d
 * the first stored diagonal entry (0 if none).  build() passes 1 / omega as the
 * fill routines' omega, which compute beta = 1 / omega again, so beta is
 * 1 / (1 / omega) (rounded twice), not 1 / omega. */
static void ssor_split(double omega, const orc_csr* A, orc_csr* L, orc_csr* U)
{
    const int m     = A->m;
    double*   d     = (double*)calloc((size_t)(m > 0 ? m : 1), sizeof(double));
    const double b1 = 1.0 / omega;
    const double beta = 1.0 / b1;
    for(int i = 0; i < m; i++)
        for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
            if(A->ci[j] == i)
            {
                d[i] = A->v[j];
                break;
            }
    orc_csr* T[2] = {L, U};
    for(int t = 0; t < 2; t++)
    {
        orc_csr* X = T[t];
        X->m       = m;
        X->n       = A->n;
        X->rp      = (int*)malloc(sizeof(int) * ((size_t)m + 1));
        X->rp[0]   = 0;
        for(int i = 0; i < m; i++)
        {
            int c = 0;
            for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
                if(t == 0 ? A->ci[j] <= i : A->ci[j] >= i)
                    c++;
            X->rp[i + 1] = X->rp[i] + c;
        }
        const int nz = X->rp[m];
        X->nnz       = nz;
        X->ci        = (int*)malloc(sizeof(int) * (size_t)(nz > 0 ? nz : 1));
        X->v         = (double*)malloc(sizeof(double) * (size_t)(nz > 0 ? nz : 1));
        for(int i = 0; i < m; i++)
        {
            int k = X->rp[i];
            for(int j = A->rp[i]; j < A->rp[i + 1]; j++)
            {
                const int c = A->ci[j];
                if(t == 0 && c < i)
                    X->ci[k] = c, X->v[k++] = A->v[j] / d[c];
                else if(t == 1 && c > i)
                    X->ci[k] = c, X->v[k++] = A->v[j];
                else if(c == i)
                    X->ci[k] = c, X->v[k++] = t == 0 ? beta : beta * A->v[j];
            }
        }
    }
    free(d);
}

static void csr_free_all(orc_csr* X)
{
    free(X->rp);
    free(X->ci);
    free(X->v);
}

static void tri_prepare(int kind, double omega, const orc_csr* A, orc_csr* F, orc_csr* G)
{
    if(kind == 4)
    {
        ssor_split(omega, A, F, G);
        return;
    }
    const int nnz = A->rp[A->m];
    *F            = *A;
    F->v          = (double*)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
    memcpy(F->v, A->v, sizeof(double) * nnz);
    int sz, nz;
    if(kind == 0)
        orc_csrilu0(F, &sz, &nz);
    else if(kind == 1)
        orc_csric0(F, &sz, &nz);
    else if(kind == 3)
    {
        const double s = 1.0 / omega;
        for(int i = 0; i < F->m; i++)
            for(int j = F->rp[i]; j < F->rp[i + 1]; j++)
                if(F->ci[j] == i)
                    F->v[j] = F->v[j] * s;
    }
}

static void tri_release_pc(int kind, orc_csr* F, orc_csr* G)
{
    if(kind == 4)
    {
        csr_free_all(F);
        csr_free_all(G);
    }
    else
        free(F->v);
}

/* SSOR_precond::solve (preconditioner.cpp:355-395): lower solve with L (the host
 * csrtrsv_solve ignores its alpha argument), upper solve with U. */
static void tri_apply(int kind, const orc_csr* F, const orc_csr* G, const double* rhs, double* x,
                      double* y)
{
    if(kind == 0 || kind == 1)
    {
        orc_trsv(F, 1, kind == 0, rhs, y);
        orc_trsv(F, 0, 0, y, x);
    }
    else if(kind == 4)
    {
        orc_trsv(F, 1, 0, rhs, y);
        orc_trsv(G, 0, 0, y, x);
    }
    else
        orc_trsv(F, 1, 0, rhs, x);
}

void orc_precond_apply(int kind, double omega, const orc_csr* A, const double* rhs, double* x)
{
    orc_csr F, G;
    tri_prepare(kind, omega, A, &F, &G);
    double* y = (double*)malloc(sizeof(double) * (A->m > 0 ? A->m : 1));
    tri_apply(kind, &F, &G, rhs, x, y);
    free(y);
    tri_release_pc(kind, &F, &G);
}

/* cg_solver::solve_precond (cg.cpp:136-223) with one of the triangular
 * preconditioners above (built once, as the reference's build()). */
int orc_precond_cg(int kind, double omega, const orc_csr* A, const double* b, double* x,
                   double rel_tol, double abs_tol, int max_iter)
{
    const int m = A->m;
    orc_csr   F, G;
    tri_prepare(kind, omega, A, &F, &G);
    double* r = (double*)malloc(sizeof(double) * ((size_t)m + 1));
    double* z = (double*)malloc(sizeof(double) * ((size_t)m + 1));
    double* p = (double*)malloc(sizeof(double) * ((size_t)m + 1));
    double* y = (double*)malloc(sizeof(double) * ((size_t)m + 1));
    orc_residual(A, x, b, r);
    double r0 = orc_norm_inf(r, m);
    tri_apply(kind, &F, &G, r, z, y);
    memcpy(p, z, sizeof(double) * (size_t)m);
    double gamma = orc_dot(z, r, m);
    int    iter  = 0;
    while(!(iter > max_iter))
    {
        orc_spmv(A, 1.0, p, 0.0, z);
        double alpha = gamma / orc_dot(z, p, m);
        for(int i = 0; i < m; i++)
            x[i] = alpha == 1.0 ? p[i] + x[i] : alpha * p[i] + x[i];
        double na = -1.0 * alpha;
        for(int i = 0; i < m; i++)
            r[i] = na == 1.0 ? z[i] + r[i] : na * z[i] + r[i];
        if(converges(orc_norm_inf(r, m), r0, rel_tol, abs_tol))
            break;
        tri_apply(kind, &F, &G, r, z, y);
        double old  = gamma;
        gamma       = orc_dot(z, r, m);
        double beta = gamma / old;
        for(int i = 0; i < m; i++)
            p[i] = beta == 0.0 ? 1.0 * z[i] : 1.0 * z[i] + beta * p[i];
        iter++;
    }
    free(r);
    free(z);
    free(p);
    free(y);
    tri_release_pc(kind, &F, &G);
    return iter;
}
