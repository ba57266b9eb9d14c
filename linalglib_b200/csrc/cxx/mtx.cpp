// Matrix Market I/O on the host, with the reference's observable behaviour
// (csr_matrix::read_mtx / write_mtx, library/src/csr_matrix.cpp:523-795):
//
// read: the banner's second to fifth words must be "matrix", "coordinate",
//   "real" or "integer", and "general" or "symmetric" (array, complex, pattern,
//   hermitian and skew-symmetric files are refused); lines starting with '%'
//   after the banner are comments; then "m n entries"; each entry line is split
//   at its first and second space into row, column and value, parsed as
//   std::stoi / std::stoi / std::stod would; a symmetric file adds the mirrored
//   entry of every off-diagonal one; entries are put in (row, column) order by
//   std::sort and repeated positions are summed in that order; the rows become
//   CSR.  The same sort over the same sequence with an equivalent comparison
//   gives the same order of repeated entries, so the sums are bit-identical.
//   Where the reference would throw from std::stoi / std::stod (a missing or
//   unparsable field, a value outside the double range) or write outside its
//   arrays (a row or column outside 1..m, 1..n), this reader refuses the file.
//
// write: "%%MatrixMarket matrix coordinate real general", one comment line,
//   "m n nnz", then "row col value" per entry in CSR order with the value in
//   fixed notation with 10 decimals (std::fixed << std::setprecision(10), the
//   same text as printf's "%.10f").
#include "lab.h"

#include <algorithm>
#include <cerrno>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace lab
{
    void set_error(const char* fmt, ...);
}

namespace
{
    struct mtx_entry
    {
        uint64_t key; // row << 32 | column, both zero-based and in range
        double   v;
    };

    // std::stoi on s: leading blanks, sign, digits; no digits or an int overflow
    // is a failure (where std::stoi throws)
    bool int_field(const std::string& s, int& out)
    {
        const char* p   = s.c_str();
        char*       end = nullptr;
        errno           = 0;
        long v          = std::strtol(p, &end, 10);
        if(end == p || errno == ERANGE || v < INT_MIN || v > INT_MAX)
            return false;
        out = (int)v;
        return true;
    }

    // std::stod on s (strtod; no conversion or ERANGE is a failure)
    bool real_field(const std::string& s, double& out)
    {
        const char* p   = s.c_str();
        char*       end = nullptr;
        errno           = 0;
        double v        = std::strtod(p, &end);
        if(end == p || errno == ERANGE)
            return false;
        out = v;
        return true;
    }

    lab_status refuse(const char* why, const char* path)
    {
        lab::set_error("read_mtx %s: %s", path, why);
        return LAB_BAD_ARG;
    }
}

extern "C" {

LAB_API lab_status lab_mtx_read(const char* path, int64_t* m_out, int64_t* n_out,
                                int64_t* nnz_out, int32_t** row_ptr, int32_t** col_ind,
                                double** val)
{
    if(!path || !m_out || !n_out || !nnz_out || !row_ptr || !col_ind || !val)
    {
        lab::set_error("lab_mtx_read: null argument");
        return LAB_BAD_ARG;
    }
    *row_ptr = nullptr;
    *col_ind = nullptr;
    *val     = nullptr;
    std::ifstream f(path, std::ios::binary);
    if(!f)
        return refuse("could not open the file", path);
    std::stringstream whole;
    whole << f.rdbuf();
    std::istringstream in(whole.str());

    std::string line;
    std::getline(in, line);
    std::istringstream banner(line);
    std::string        word[5];
    for(int k = 0; k < 5; k++)
        if(!(banner >> word[k]) && k > 0)
            word[k] = word[k - 1]; // a missing word reads as the last one read
    if(word[1] != "matrix")
        return refuse("not a Matrix Market matrix", path);
    if(word[2] != "coordinate")
        return refuse("only the coordinate format is supported", path);
    if(word[3] != "real" && word[3] != "integer")
        return refuse("only real and integer values are supported", path);
    bool symmetric = false;
    if(word[4] == "symmetric")
        symmetric = true;
    else if(word[4] != "general")
        return refuse("only general and symmetric matrices are supported", path);

    bool more = false;
    while((more = (bool)std::getline(in, line)) && !line.empty() && line[0] == '%')
    {
    }
    std::istringstream dims(line);
    int                m = 0, n = 0;
    long long          count = 0;
    if(!more || !(dims >> m >> n >> count) || m < 0 || n < 0 || count < 0)
        return refuse("bad size line", path);

    std::vector<mtx_entry> e;
    e.reserve(symmetric ? 2 * (size_t)count : (size_t)count);
    for(long long k = 0; k < count; k++)
    {
        if(!std::getline(in, line))
            return refuse("fewer entries than the size line states", path);
        // the fields between the first and second space; a missing space makes
        // std::string::find return npos, whose successor is position 0
        const size_t s1 = line.find(' ');
        const size_t s2 = line.find(' ', s1 + 1);
        if(s1 + 1 > line.size() || s2 + 1 > line.size())
            return refuse("malformed entry line", path);
        int    r = 0, c = 0;
        double v = 0.0;
        if(!int_field(line.substr(0, s1), r) ||
           !int_field(line.substr(s1 + 1, s2 - (s1 + 1)), c) ||
           !real_field(line.substr(s2 + 1), v))
            return refuse("malformed entry line", path);
        if(r < 1 || r > m || c < 1 || c > n || (symmetric && r != c && (c > m || r > n)))
            return refuse("entry outside the matrix", path);
        e.push_back({((uint64_t)(r - 1) << 32) | (uint32_t)(c - 1), v});
        if(symmetric && r != c)
            e.push_back({((uint64_t)(c - 1) << 32) | (uint32_t)(r - 1), v});
    }
    std::sort(e.begin(), e.end(),
              [](const mtx_entry& a, const mtx_entry& b) { return a.key < b.key; });

    size_t distinct = 0;
    for(size_t k = 0; k < e.size(); k++)
        if(k == 0 || e[k].key != e[distinct - 1].key)
            e[distinct++] = e[k];
        else
            e[distinct - 1].v += e[k].v;
    e.resize(distinct);

    int32_t* rp = (int32_t*)std::calloc((size_t)m + 1, sizeof(int32_t));
    int32_t* ci = (int32_t*)std::malloc(sizeof(int32_t) * (distinct ? distinct : 1));
    double*  v  = (double*)std::malloc(sizeof(double) * (distinct ? distinct : 1));
    if(!rp || !ci || !v)
    {
        std::free(rp);
        std::free(ci);
        std::free(v);
        lab::set_error("lab_mtx_read: out of host memory");
        return LAB_OOM;
    }
    for(size_t k = 0; k < distinct; k++)
    {
        rp[(e[k].key >> 32) + 1]++;
        ci[k] = (int32_t)(e[k].key & 0xffffffffu);
        v[k]  = e[k].v;
    }
    for(int i = 0; i < m; i++)
        rp[i + 1] += rp[i];
    *m_out   = m;
    *n_out   = n;
    *nnz_out = (int64_t)distinct;
    *row_ptr = rp;
    *col_ind = ci;
    *val     = v;
    return LAB_OK;
}

LAB_API void lab_mtx_free(void* p)
{
    std::free(p);
}

LAB_API lab_status lab_mtx_write(const char* path, int64_t m, int64_t n, int64_t nnz,
                                 const int32_t* row_ptr, const int32_t* col_ind,
                                 const double* val)
{
    if(!path || m < 0 || n < 0 || nnz < 0 || (!row_ptr && m > 0) ||
       (nnz > 0 && (!col_ind || !val)))
    {
        lab::set_error("lab_mtx_write: bad argument");
        return LAB_BAD_ARG;
    }
    FILE* f = std::fopen(path, "wb");
    if(!f)
    {
        lab::set_error("write_mtx %s: could not open the file for writing", path);
        return LAB_BAD_ARG;
    }
    std::fprintf(f, "%%%%MatrixMarket matrix coordinate real general\n");
    std::fprintf(f, "%% Created by C++ CSR to Matrix Market writer\n");
    std::fprintf(f, "%lld %lld %lld\n", (long long)m, (long long)n, (long long)nnz);
    for(int64_t i = 0; i < m; i++)
        for(int32_t j = row_ptr[i]; j < row_ptr[i + 1]; j++)
            std::fprintf(f, "%lld %d %.10f\n", (long long)(i + 1), col_ind[j] + 1, val[j]);
    const bool ok = std::ferror(f) == 0;
    if(std::fclose(f) != 0 || !ok)
    {
        lab::set_error("write_mtx %s: write failed", path);
        return LAB_BAD_ARG;
    }
    return LAB_OK;
}

} // extern "C"
