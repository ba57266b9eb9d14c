// linalg::csr_matrix<T> -- the reference CSR container (library/include/csr_matrix.h:48-449),
// same public interface for the AMG-PCG path, backed by a device matrix of the
// C ABI (lab_csr) that is built on first use and cached.  Products, transposes
// and AMG levels produced on the GPU stay on the GPU; the host arrays are
// filled only when the caller reads them.
#ifndef LINALG_B200_CSR_MATRIX_H
#define LINALG_B200_CSR_MATRIX_H

#include <memory>
#include <string>
#include <vector>

#include "lab.h"
#include "vector.h"

namespace linalg
{
    template <typename T>
    class csr_matrix
    {
    private:
        int  m;
        int  n;
        int  nnz;
        bool on_host;

        mutable vector<int> csr_row_ptr;
        mutable vector<int> csr_col_ind;
        mutable vector<T>   csr_val;
        mutable bool        host_valid = true; // arrays above hold the current matrix

        // device representation (shared: a hierarchy level is borrowed, not owned)
        mutable std::shared_ptr<lab_csr_s> dev;

        void sync_host() const;

    public:
        csr_matrix();
        csr_matrix(const std::vector<int>& csr_row_ptr,
                   const std::vector<int>& csr_col_ind,
                   const std::vector<T>&   csr_val,
                   int                     m,
                   int                     n,
                   int                     nnz);
        ~csr_matrix();

        csr_matrix(const csr_matrix<T>&)               = delete;
        csr_matrix<T>& operator=(const csr_matrix<T>&) = delete;

        bool       is_on_host() const;
        int        get_m() const;
        int        get_n() const;
        int        get_nnz() const;
        const int* get_row_ptr() const;
        const int* get_col_ind() const;
        const T*   get_val() const;
        int*       get_row_ptr();
        int*       get_col_ind();
        T*         get_val();

        void resize(int m, int n, int nnz);
        void copy_from(const csr_matrix<T>& A);
        // csr_matrix.h:215-227: the triangle with columns <= i (>= i), diagonal
        // included; unit_diag is accepted and, as in the reference, not used
        void copy_lower_triangular_from(const csr_matrix<T>& A, bool unit_diag);
        void copy_upper_triangular_from(const csr_matrix<T>& A, bool unit_diag);
        void move_to_device();
        void move_to_host();
        void extract_diagonal(vector<T>& diag) const;
        // csr_matrix.h:254-262: a_ii *= scalar; a_ij *= 1 / a_jj (by column, as the
        // reference's host_scale.cpp computes it)
        void scale_diagonal_by(T scalar);
        void scale_by_inverse_diagonal();
        void multiply_by_vector(vector<T>& y, const vector<T>& x) const;
        void multiply_by_vector_and_add(vector<T>& y, const vector<T>& x) const;
        void multiply_by_matrix(csr_matrix<T>& C, const csr_matrix<T>& B) const;
        // csr_matrix.h:298-357: triangular solves on the lower / upper part and the
        // in-place IC(0) / ILU(0), bit-identical to the reference's host loops
        void triangular_solve_lower(vector<T>& x, const vector<T>& y, bool unit_diag) const;
        void triangular_solve_upper(vector<T>& x, const vector<T>& y, bool unit_diag) const;
        void compute_incomplete_cholesky_factorization();
        void compute_incomplete_LU_factorization();
        void transpose(csr_matrix<T>& Trans) const;
        bool read_mtx(const std::string& filename);
        bool write_mtx(const std::string& filename);
        void print_matrix(const std::string name) const;

        // -- library access (not in the reference interface) --------------
        // The device matrix (built from the host arrays on first use).
        lab_csr device() const;
        // Adopt a device matrix produced by the library (owned or borrowed).
        void adopt(lab_csr A, bool owned);
        // The library changed the device matrix's values in place: the host
        // arrays are refreshed on their next read.
        void device_changed();
        // Back to an empty 0 x 0 host matrix, dropping any device matrix.
        void reset();
    };
}

#endif
