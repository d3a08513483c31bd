// lablas::Vector<T>: a device vector that, like backend::Vector
// (src/backend/vector/vector.h:22-276), is held either dense (n values) or
// sparse (ascending ids + values, zeros dropped) and switches between the
// two by density (convert_if_required: dense above 0.3 n non-zeros).
// Storage is device memory; host access (get_at, getDense()->get_vals())
// downloads a host copy on demand.
#pragma once

#include <algorithm>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

#include "core.hpp"

namespace lablas {

template <typename T>
class Vector;

// Host view returned by get_vector()->getDense(): a host copy of the dense
// form.  Through the non-const getDense() the caller may also write it (the
// reference's sequential checkers fill their result vectors this way); the
// vector then treats the host copy as the newer one and uploads it before
// its next device operation.  Plain array storage, so Vector<bool> has a
// bool* like every other element type.
template <typename T>
class HostDenseView {
public:
    const T* get_vals() const { return vals_.get(); }
    T* get_vals() { return vals_.get(); }
    Index get_size() const { return n_; }
    Index get_nvals() const {
        Index c = 0;
        for (Index i = 0; i < n_; i++) c += (vals_[i] != T(0));
        return c;
    }

private:
    template <typename U>
    friend class Vector;
    void resize(Index n) {
        if (n == n_ && vals_) return;
        vals_.reset(new T[n > 0 ? n : 1]);
        n_ = n;
    }
    void swap(HostDenseView& o) {
        std::swap(vals_, o.vals_);
        std::swap(n_, o.n_);
    }
    std::unique_ptr<T[]> vals_;
    Index n_ = 0;
};

template <typename T>
class Vector {
public:
    using ValueType = T;
    static constexpr gbk_dtype dtype = dtype_of<T>::value;

    Vector() = default;
    explicit Vector(Index nsize) : n_(nsize) {}
    Vector(const Vector&) = delete;
    Vector& operator=(const Vector&) = delete;

    // ---- reference API (src/cpp_graphblas/vector.hpp:11-123) ----

    LA_Info build(const std::vector<Index>* indices, const std::vector<T>* values, Index nvals) {
        if (indices == nullptr || values == nullptr) return GrB_NULL_POINTER;
        if (nvals == 0) return GrB_INVALID_VALUE;
        return build_sparse(indices->data(), values->data(), nvals);
    }
    LA_Info build(const std::vector<T>* values, Index nvals) {
        if (values == nullptr) return GrB_NULL_POINTER;
        if (nvals == 0) return GrB_INVALID_VALUE;
        return build(values->data(), nvals);
    }
    LA_Info build(const T* values, Index nvals) {
        touch();
        if (values == nullptr) return GrB_NULL_POINTER;
        if (nvals == 0) return GrB_INVALID_VALUE;
        ensure_dense_buf();
        const Index m = std::min<Index>(nvals, n_);
        if (m > 0) dense_.upload(values, m);
        dense_mode_ = true;
        return GrB_SUCCESS;
    }
    // set_constant (vector.h:38-56): zero empties the current form.
    LA_Info fill(T val) {
        touch();
        if (val == T(0)) {
            if (dense_mode_) {
                ensure_dense_buf();
                throw_if(gbk_vec_fill(dense_.p, dtype, n_, 0.0, stream()), "fill");
            } else {
                nvals_ = 0;
            }
        } else {
            ensure_dense_buf();
            dense_mode_ = true;
            throw_if(gbk_vec_fill(dense_.p, dtype, n_, (double)val, stream()), "fill");
        }
        return GrB_SUCCESS;
    }
    LA_Info clear() {
        touch();
        dense_mode_ = false;
        nvals_ = 0;
        return GrB_SUCCESS;
    }
    // set_element (dense_vector.hpp:58, sparse_vector.hpp:5-20)
    LA_Info set_element(T val, VNT pos) {
        touch();
        if (pos < 0 || pos >= n_) return GrB_INVALID_INDEX;
        if (dense_mode_) {
            ensure_dense_buf();
            cuda_check(cudaMemcpyAsync(dense_.p + pos, &val, sizeof(T), cudaMemcpyHostToDevice, current_stream()),
                       "set_element");
            cuda_check(cudaStreamSynchronize(current_stream()), "set_element");
            return GrB_SUCCESS;
        }
        ensure_sparse_buf();
        std::vector<int32_t> ids(nvals_);
        if (nvals_) ids_.download(ids.data(), nvals_);
        auto it = std::find(ids.begin(), ids.end(), (int32_t)pos);
        Index k = (it == ids.end()) ? nvals_ : (Index)(it - ids.begin());
        int32_t p32 = (int32_t)pos;
        cuda_check(cudaMemcpyAsync(ids_.p + k, &p32, sizeof(int32_t), cudaMemcpyHostToDevice, current_stream()),
                   "set_element");
        cuda_check(cudaMemcpyAsync(vals_.p + k, &val, sizeof(T), cudaMemcpyHostToDevice, current_stream()),
                   "set_element");
        cuda_check(cudaStreamSynchronize(current_stream()), "set_element");
        if (k == nvals_) nvals_++;
        return GrB_SUCCESS;
    }
    LA_Info get_nvals(Index* nv) const {
        *nv = nvals();
        return GrB_SUCCESS;
    }
    Index nvals() const {
        sync_host();
        if (!dense_mode_) return nvals_;
        if (n_ == 0) return 0;
        int64_t c = 0;
        throw_if(gbk_vec_nvals(dense_.p, dtype, n_, &c, stream()), "nvals");
        return c;
    }
    Index size() const { return n_; }
    Index get_size() const { return n_; }
    void swap(Vector* o) {
        std::swap(n_, o->n_);
        std::swap(dense_mode_, o->dense_mode_);
        std::swap(nvals_, o->nvals_);
        std::swap(host_valid_, o->host_valid_);
        std::swap(host_newer_, o->host_newer_);
        view_.swap(o->view_);
        dense_.swap(o->dense_);
        ids_.swap(o->ids_);
        vals_.swap(o->vals_);
    }
    // fillAscending (dense_vector.h): v[i] = i
    LA_Info fillAscending(Index) {
        touch();
        ensure_dense_buf();
        dense_mode_ = true;
        throw_if(gbk_vec_iota(dense_.p, dtype, n_, stream()), "fillAscending");
        return GrB_SUCCESS;
    }
    LA_Info dup(const Vector<T>* rhs) {
        touch();
        rhs->sync_host();
        if (rhs->n_ != n_) return GrB_DIMENSION_MISMATCH;
        dense_mode_ = rhs->dense_mode_;
        if (dense_mode_) {
            ensure_dense_buf();
            dense_.copy_from(rhs->dense_, n_);
        } else {
            ensure_sparse_buf();
            nvals_ = rhs->nvals_;
            if (nvals_) {
                ids_.copy_from(rhs->ids_, nvals_);
                vals_.copy_from(rhs->vals_, nvals_);
            }
        }
        return GrB_SUCCESS;
    }
    T const& get_at(Index i) const {
        const T* h = const_cast<Vector*>(this)->host_dense();
        if (i >= 0 && i < n_) return h[i];
        throw "Error: out of range in backend::vector";
    }
    void set_name(const std::string& nm) { name_ = nm; }
    const std::string& get_name() const { return name_; }
    void print() const {
        const T* h = const_cast<Vector*>(this)->host_dense();
        for (Index i = 0; i < n_; i++) std::cout << "[" << i << "]:" << h[i] << " ";
        std::cout << std::endl;
    }
    void print_storage_type() const { std::cout << (dense_mode_ ? "dense" : "sparse") << std::endl; }

    // ---- backend-style access (reference drivers and checkers read and write
    // host arrays this way) ----
    Vector* get_vector() { return this; }
    const Vector* get_vector() const { return this; }
    // Writable host copy: the caller may change it, so it becomes the newer
    // copy and is uploaded before the next device operation on this vector.
    HostDenseView<T>* getDense() {
        host_dense();
        host_newer_ = true;
        return &view_;
    }
    const HostDenseView<T>* getDense() const {
        const_cast<Vector*>(this)->host_dense();
        return &view_;
    }

    // ---- device form, used by the operations ----
    bool is_dense() const { return dense_mode_; }
    bool is_sparse() const { return !dense_mode_; }
    Storage get_storage() const { return dense_mode_ ? GrB_DENSE : GrB_SPARSE; }

    void force_to_dense() {
        sync_host();
        ensure_dense_buf();
        if (dense_mode_) return;
        ensure_sparse_buf();
        throw_if(gbk_vec_to_dense(ids_.p, vals_.p, nvals_, dtype, dense_.p, n_, stream()), "to_dense");
        dense_mode_ = true;
    }
    void force_to_sparse() {
        sync_host();
        ensure_sparse_buf();
        if (!dense_mode_) return;
        ensure_dense_buf();
        int64_t nv = 0;
        throw_if(gbk_vec_to_sparse(dense_.p, dtype, n_, ids_.p, vals_.p, &nv, stream()), "to_sparse");
        nvals_ = nv;
        dense_mode_ = false;
    }
    // vector.h:117-129
    void convert_if_required() {
        Index nv = nvals();
        if (nv > (Index)(n_ * SPARSE_VECTOR_THRESHOLD))
            force_to_dense();
        else
            force_to_sparse();
    }
    T* dense_ptr() {
        force_to_dense();
        touch();
        return dense_.p;
    }
    const T* dense_ptr() const { return const_cast<Vector*>(this)->dense_ptr(); }
    int32_t* ids_ptr() {
        force_to_sparse();
        touch();
        return ids_.p;
    }
    T* vals_ptr() {
        force_to_sparse();
        touch();
        return vals_.p;
    }
    Index sparse_nvals() {
        force_to_sparse();
        return nvals_;
    }
    // mask argument in its current form
    gbk_mask as_mask(Desc_value mode) const {
        sync_host();
        gbk_mask m{};
        m.mode = (int32_t)mode;
        if (dense_mode_) {
            m.dense = dense_.p;
            m.dtype = dtype;
        } else {
            m.dense = nullptr;
            m.ids = ids_.p;
            m.nvals = nvals_;
        }
        return m;
    }
    // host copy of the dense form (forces the dense form, as getDense() does)
    const T* host_dense() {
        if (host_newer_) return view_.get_vals();
        force_to_dense();
        if (!host_valid_) {
            view_.resize(n_);
            if (n_) dense_.download(view_.vals_.get(), n_);
            host_valid_ = true;
        }
        return view_.get_vals();
    }
    // Sparse form with the ids of another device list (copied) and values
    // written by fill_vals into this vector's value buffer.
    template <typename F>
    void adopt_sparse(const int32_t* ids, Index nv, F&& fill_vals) {
        touch();
        ensure_sparse_buf();
        if (nv) {
            cuda_check(cudaMemcpyAsync(ids_.p, ids, sizeof(int32_t) * nv, cudaMemcpyDeviceToDevice,
                                       current_stream()), "adopt_sparse");
            fill_vals(vals_.p);
        }
        nvals_ = nv;
        dense_mode_ = false;
    }
    // A host copy handed out writable goes back to the device first.
    void sync_host() const {
        auto* self = const_cast<Vector*>(this);
        if (!self->host_newer_) return;
        self->host_newer_ = false;
        self->ensure_dense_buf();
        if (n_) self->dense_.upload(self->view_.vals_.get(), n_);
        self->dense_mode_ = true;
        self->host_valid_ = true;
    }
    // every device-side change drops the host copy
    void touch() {
        sync_host();
        host_valid_ = false;
    }

private:
    LA_Info build_sparse(const Index* ids, const T* vals, Index nvals) {
        touch();
        ensure_sparse_buf();
        std::vector<int32_t> i32(ids, ids + nvals);
        ids_.upload(i32.data(), nvals);
        vals_.upload(vals, nvals);
        nvals_ = nvals;
        dense_mode_ = false;
        return GrB_SUCCESS;
    }
    void ensure_dense_buf() {
        if (!dense_.p) {
            dense_.alloc(n_);
            cuda_check(cudaMemsetAsync(dense_.p, 0, sizeof(T) * (n_ ? n_ : 1), current_stream()), "memset");
        }
    }
    void ensure_sparse_buf() {
        if (!ids_.p) {
            ids_.alloc(n_);
            vals_.alloc(n_);
        }
    }

    Index n_ = 0;
    bool dense_mode_ = false;
    Index nvals_ = 0;
    DeviceBuffer<T> dense_;
    DeviceBuffer<int32_t> ids_;
    DeviceBuffer<T> vals_;
    HostDenseView<T> view_;
    bool host_valid_ = false;
    bool host_newer_ = false;
    std::string name_;

    template <typename Y>
    friend bool operator==(Vector<Y>& lhs, Vector<Y>& rhs);
};

// Vector equality with absolute tolerance 1e-3 (dense_vector.h:101-116).
template <typename T>
bool operator==(Vector<T>& lhs, Vector<T>& rhs) {
    if (lhs.size() != rhs.size()) return false;
    const T* a = lhs.host_dense();
    std::vector<T> acopy(a, a + lhs.size());
    const T* b = rhs.host_dense();
    for (Index i = 0; i < lhs.size(); i++)
        if (std::fabs((double)acopy[i] - (double)b[i]) > 0.001) return false;
    return true;
}
template <typename T>
bool operator!=(Vector<T>& lhs, Vector<T>& rhs) {
    return !(lhs == rhs);
}
template <typename T>
void print_diff(Vector<T>& lhs, Vector<T>& rhs) {
    const T* a = lhs.host_dense();
    std::vector<T> acopy(a, a + lhs.size());
    const T* b = rhs.host_dense();
    Index shown = 0;
    for (Index i = 0; i < lhs.size() && shown < 16; i++)
        if (std::fabs((double)acopy[i] - (double)b[i]) > 0.001) {
            std::cout << "Error in " << i << " : " << acopy[i] << " " << b[i] << std::endl;
            shown++;
        }
}

// Range-for over host values (vector.hpp:128-199).
template <typename V>
class VectorIteratorType {
public:
    using ValueType = typename V::ValueType;
    VectorIteratorType(V& c, Index i) : index(i), collection(c) {}
    bool operator!=(VectorIteratorType const& o) const { return index != o.index; }
    ValueType const& operator*() const { return collection.get_at(index); }
    VectorIteratorType const& operator++() {
        ++index;
        return *this;
    }

private:
    Index index;
    V& collection;
};
template <typename T>
inline VectorIteratorType<Vector<T>> begin(Vector<T>& c) {
    return VectorIteratorType<Vector<T>>(c, 0);
}
template <typename T>
inline VectorIteratorType<Vector<T>> end(Vector<T>& c) {
    return VectorIteratorType<Vector<T>>(c, c.size());
}

}  // namespace lablas
