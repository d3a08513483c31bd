// lablas::Matrix<T>: owns one gbk_matrix handle (device CSR, CSC built on
// first use, optional SELL-C / segmented / LAV format for both
// orientations), like backend::Matrix owns csr_data / csc_data / data /
// transposed_data (src/backend/matrix/matrix.h:34-207).  A host copy of the
// CSR is kept for the host-side queries the reference offers (degrees,
// symmetry).
#pragma once

#include <algorithm>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "core.hpp"
#include "gbk_ingest.h"

namespace lablas {

template <typename T>
class Matrix;

namespace backend {

// Host view of a matrix's CSR, the accessors of the reference's
// backend::MatrixCSR (src/backend/matrix/csr/csr_matrix.h) that its
// sequential checkers read (algorithms/*/ *_traditional.hpp reach it through
// get_matrix()->get_csr()).  64-bit row pointers and column ids as there;
// built from the matrix's host copy on first use.
template <typename T>
class MatrixCSR {
public:
    Index* get_row_ptr() { return row_ptr_.data(); }
    const Index* get_row_ptr() const { return row_ptr_.data(); }
    Index* get_col_ids() { return col_ids_.data(); }
    const Index* get_col_ids() const { return col_ids_.data(); }
    T* get_vals() { return vals_.get(); }
    const T* get_vals() const { return vals_.get(); }
    Index get_num_rows() const { return (Index)row_ptr_.size() - 1; }
    Index get_nnz() const { return (Index)col_ids_.size(); }

private:
    friend class lablas::Matrix<T>;
    std::vector<Index> row_ptr_, col_ids_;
    std::unique_ptr<T[]> vals_;
};

}  // namespace backend

template <typename T>
class Matrix {
public:
    static_assert(std::is_same<T, float>::value || std::is_same<T, int>::value,
                  "lablas::Matrix<T> stores float or int values on the device");
    static constexpr gbk_dtype dtype = dtype_of<T>::value;

    Matrix() = default;
    Matrix(Index nrows, Index ncols) : nrows_(nrows), ncols_(ncols) {}
    Matrix(const Matrix&) = delete;
    Matrix& operator=(const Matrix&) = delete;
    ~Matrix() { release(); }

    LA_Info set_preferred_matrix_format(const MatrixStorageFormat f) {
        format_ = f;
        if (h_) return apply_format();
        return GrB_SUCCESS;
    }
    LA_Info get_nrows(Index* n) const {
        *n = nrows_;
        return GrB_SUCCESS;
    }
    LA_Info get_ncols(Index* n) const {
        *n = ncols_;
        return GrB_SUCCESS;
    }
    LA_Info get_nvals(Index* n) const {
        *n = nnz_;
        return GrB_SUCCESS;
    }
    Index nrows() const { return nrows_; }
    Index ncols() const { return ncols_; }
    Index get_nnz() const { return nnz_; }
    LA_Info get_storage(Storage* s) const {
        *s = GrB_SPARSE;
        return GrB_SUCCESS;
    }
    LA_Info get_format(MatrixStorageFormat* f) const {
        *f = format_;
        return GrB_SUCCESS;
    }

    // Matrix::build from a COO list (build.hpp:122-166): square n = max id + 1,
    // duplicates kept, rows sorted by column (stable).
    template <typename BinaryOpT>
    LA_Info build(const std::vector<Index>* row_indices, const std::vector<Index>* col_indices,
                  const std::vector<T>* values, Index nvals, BinaryOpT dup, char* dat_name = nullptr) {
        (void)dup;
        (void)dat_name;
        (void)nvals;
        if (row_indices == nullptr || col_indices == nullptr || values == nullptr) return GrB_NULL_POINTER;
        if (row_indices->empty() && col_indices->empty() && values->empty()) return GrB_NO_VALUE;
        if (row_indices->size() != col_indices->size()) return GrB_DIMENSION_MISMATCH;
        const size_t m = row_indices->size();
        Index dim = 0;
        for (size_t k = 0; k < m; k++) dim = std::max(dim, std::max((*row_indices)[k], (*col_indices)[k]) + 1);
        std::vector<size_t> order(m);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
            Index ra = (*row_indices)[a], rb = (*row_indices)[b];
            return ra != rb ? ra < rb : (*col_indices)[a] < (*col_indices)[b];
        });
        rp_.assign(dim + 1, 0);
        col_.resize(m);
        val_.resize(m);
        for (size_t k = 0; k < m; k++) {
            size_t e = order[k];
            rp_[(*row_indices)[e] + 1]++;
            col_[k] = (int32_t)(*col_indices)[e];
            val_[k] = (*values)[e];
        }
        for (Index i = 0; i < dim; i++) rp_[i + 1] += rp_[i];
        return upload(dim, dim);
    }

    // build_from_csr_arrays (matrix.hpp:93-105, build.hpp:170-210): n is the
    // larger of nrows and the largest column id + 1.
    LA_Info build_from_csr_arrays(const Index* row_ptrs, const Index* col_ids, const T* values, Index nrows,
                                  Index nvals) {
        if (row_ptrs == nullptr || col_ids == nullptr || values == nullptr) return GrB_NULL_POINTER;
        Index maxc = 0;
        for (Index k = 0; k < nvals; k++) maxc = std::max(maxc, col_ids[k] + 1);
        Index dim = std::max(nrows, maxc);
        rp_.assign(dim + 1, (int32_t)nvals);
        for (Index i = 0; i <= nrows; i++) rp_[i] = (int32_t)row_ptrs[i];
        col_.assign(col_ids, col_ids + nvals);
        val_.assign(values, values + nvals);
        sort_rows();
        return upload(dim, dim);
    }

    // Same, from int32 arrays (no widening copy).
    LA_Info build_from_csr_arrays32(const int32_t* row_ptrs, const int32_t* col_ids, const T* values, Index nrows,
                                    Index nvals) {
        rp_.assign(row_ptrs, row_ptrs + nrows + 1);
        col_.assign(col_ids, col_ids + nvals);
        val_.assign(values, values + nvals);
        sort_rows();
        return upload(nrows, nrows);
    }

    // init_from_mtx (src/cpp_graphblas/matrix.hpp:107-110 ->
    // src/backend/matrix/read_file.hpp:565-617): a .mtx / .mtxbin file (or a
    // .gbkcsr CSR cache) parsed on the device; rows keep the file's order and
    // every value is 1.  Throws on a missing or malformed file.
    void init_from_mtx(const std::string& name) {
        release();
        gbk_matrix h = nullptr;
        int rc = gbk_matrix_create_from_file(&h, name.c_str(), dtype, stream());
        throw_if(rc, "init_from_mtx");
        adopt_handle(h);
    }

    // Take over a device matrix made by the library (SpGEMM, select, a file)
    // and download its host copy; rows keep the device's order.
    LA_Info adopt_handle(gbk_matrix h) {
        release();
        h_ = h;
        gbk_matrix_info inf;
        gbk_matrix_get_info(h_, &inf);
        nrows_ = (Index)inf.nrows;
        ncols_ = (Index)inf.ncols;
        nnz_ = (Index)inf.nnz;
        rp_.resize(nrows_ + 1);
        col_.resize(nnz_);
        val_.resize(nnz_);
        int rc = gbk_matrix_download_csr(h_, rp_.data(), col_.data(), val_.data(), stream());
        throw_if(rc, "adopt a device matrix");
        rowdeg_.clear();
        coldeg_.clear();
        return apply_format();
    }

    Index* get_rowdegrees() {
        degrees();
        return rowdeg_.data();
    }
    Index* get_coldegrees() {
        degrees();
        return coldeg_.data();
    }
    const Index* get_rowdegrees() const { return const_cast<Matrix*>(this)->get_rowdegrees(); }
    const Index* get_coldegrees() const { return const_cast<Matrix*>(this)->get_coldegrees(); }

    bool is_symmetric() const {
        std::vector<std::pair<int32_t, int32_t>> e, t;
        for (Index i = 0; i < nrows_; i++)
            for (int32_t k = rp_[i]; k < rp_[i + 1]; k++) {
                e.emplace_back((int32_t)i, col_[k]);
                t.emplace_back(col_[k], (int32_t)i);
            }
        std::sort(e.begin(), e.end());
        std::sort(t.begin(), t.end());
        return e == t;
    }
    // to_symmetric (symmetric.hpp): union of A and A^T, duplicates merged.
    void to_symmetric() {
        std::vector<std::tuple<int32_t, int32_t, T>> e;
        for (Index i = 0; i < nrows_; i++)
            for (int32_t k = rp_[i]; k < rp_[i + 1]; k++) {
                e.emplace_back((int32_t)i, col_[k], val_[k]);
                e.emplace_back(col_[k], (int32_t)i, val_[k]);
            }
        std::sort(e.begin(), e.end(), [](auto& a, auto& b) {
            return std::get<0>(a) != std::get<0>(b) ? std::get<0>(a) < std::get<0>(b) : std::get<1>(a) < std::get<1>(b);
        });
        e.erase(std::unique(e.begin(), e.end(),
                            [](auto& a, auto& b) { return std::get<0>(a) == std::get<0>(b) && std::get<1>(a) == std::get<1>(b); }),
                e.end());
        rp_.assign(nrows_ + 1, 0);
        col_.resize(e.size());
        val_.resize(e.size());
        for (size_t k = 0; k < e.size(); k++) {
            rp_[std::get<0>(e[k]) + 1]++;
            col_[k] = std::get<1>(e[k]);
            val_[k] = std::get<2>(e[k]);
        }
        for (Index i = 0; i < nrows_; i++) rp_[i + 1] += rp_[i];
        upload(nrows_, ncols_);
    }
    // Rows built from arrays are kept column-sorted; rows read from a file keep
    // the file's order until this sorts them (matrix.hpp:66-127).
    void sort_csr_columns(const std::string&) {
        if (rows_sorted()) return;
        sort_rows();
        upload(nrows_, ncols_);
    }
    void sort_csc_rows(const std::string&) {}     // the device CSC is built row-sorted
    void print() const {
        for (Index i = 0; i < nrows_; i++) {
            std::cout << i << ":";
            for (int32_t k = rp_[i]; k < rp_[i + 1]; k++) std::cout << " " << col_[k] << "(" << val_[k] << ")";
            std::cout << std::endl;
        }
    }

    // ---- device handle for the operations ----
    gbk_matrix handle() const { return h_; }
    const std::vector<int32_t>& host_row_ptr() const { return rp_; }
    const std::vector<int32_t>& host_col() const { return col_; }
    const std::vector<T>& host_val() const { return val_; }
    Matrix* get_matrix() { return this; }
    const Matrix* get_matrix() const { return this; }
    // get_matrix()->get_csr() (src/backend/matrix/matrix.h): the host CSR view
    const backend::MatrixCSR<T>* get_csr() const {
        if (!csr_view_) {
            auto* v = new backend::MatrixCSR<T>();
            v->row_ptr_.assign(rp_.begin(), rp_.end());
            if (v->row_ptr_.empty()) v->row_ptr_.push_back(0);
            v->col_ids_.assign(col_.begin(), col_.end());
            v->vals_.reset(new T[col_.size() > 0 ? col_.size() : 1]);
            std::copy(val_.begin(), val_.end(), v->vals_.get());
            csr_view_.reset(v);
        }
        return csr_view_.get();
    }

    // Adopt a result computed on the device with the structure of `pattern`
    // (masked SpGEMM output, backend mxm).
    LA_Info adopt(gbk_matrix h, const std::vector<int32_t>& rp, const std::vector<int32_t>& col,
                  std::vector<T>&& val) {
        release();
        h_ = h;
        rp_ = rp;
        col_ = col;
        val_ = std::move(val);
        nrows_ = (Index)rp_.size() - 1;
        ncols_ = nrows_;
        nnz_ = (Index)col_.size();
        rowdeg_.clear();
        coldeg_.clear();
        return GrB_SUCCESS;
    }

private:
    bool rows_sorted() const {
        for (size_t i = 0; i + 1 < rp_.size(); i++)
            if (!std::is_sorted(col_.begin() + rp_[i], col_.begin() + rp_[i + 1])) return false;
        return true;
    }
    void sort_rows() {
        for (size_t i = 0; i + 1 < rp_.size(); i++) {
            int32_t a = rp_[i], b = rp_[i + 1];
            if (std::is_sorted(col_.begin() + a, col_.begin() + b)) continue;
            std::vector<std::pair<int32_t, T>> tmp;
            for (int32_t k = a; k < b; k++) tmp.emplace_back(col_[k], val_[k]);
            std::stable_sort(tmp.begin(), tmp.end(), [](auto& x, auto& y) { return x.first < y.first; });
            for (int32_t k = a; k < b; k++) {
                col_[k] = tmp[k - a].first;
                val_[k] = tmp[k - a].second;
            }
        }
    }
    LA_Info upload(Index nrows, Index ncols) {
        release();
        nrows_ = nrows;
        ncols_ = ncols;
        nnz_ = (Index)col_.size();
        int rc = gbk_matrix_create_csr(&h_, nrows_, ncols_, nnz_, rp_.data(), col_.data(), val_.data(), dtype, 0,
                                       stream());
        throw_if(rc, "Matrix build");
        rowdeg_.clear();
        coldeg_.clear();
        return apply_format();
    }
    LA_Info apply_format() {
        gbk_format f = GBK_FMT_CSR;
        switch (format_) {
            case CSR: f = GBK_FMT_CSR; break;
            // COO (spmv_coo.h) holds the same entries in row order: stored as CSR, the
            // SpMV gives its results without its unsynchronised updates of shared rows
            case COO: f = GBK_FMT_CSR; break;
            case CSR_SEG: f = GBK_FMT_CSR_SEG; break;
            case LAV: f = GBK_FMT_LAV; break;
            case SELL_C: f = GBK_FMT_SELL_C; break;
            default: throw "Error: unsupported format in Matrix<T>::build";
        }
        int rc = gbk_matrix_set_format(h_, f, nullptr, stream());
        throw_if(rc, "set_preferred_matrix_format");
        return GrB_SUCCESS;
    }
    void degrees() {
        if (!rowdeg_.empty() || nrows_ == 0) return;
        rowdeg_.assign(nrows_, 0);
        coldeg_.assign(ncols_, 0);
        for (Index i = 0; i < nrows_; i++) {
            rowdeg_[i] = rp_[i + 1] - rp_[i];
            for (int32_t k = rp_[i]; k < rp_[i + 1]; k++) coldeg_[col_[k]]++;
        }
    }
    void release() {
        if (h_) gbk_matrix_destroy(h_);
        h_ = nullptr;
        csr_view_.reset();
    }

    gbk_matrix h_ = nullptr;
    Index nrows_ = 0, ncols_ = 0, nnz_ = 0;
    MatrixStorageFormat format_ = CSR;
    std::vector<int32_t> rp_, col_;
    std::vector<T> val_;
    std::vector<Index> rowdeg_, coldeg_;
    mutable std::unique_ptr<backend::MatrixCSR<T>> csr_view_;
};

}  // namespace lablas
