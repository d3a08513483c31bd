// lablas::Descriptor: per-field settings, presets and toggle() exactly as
// src/backend/descriptor/descriptor.h:10-54 and
// src/cpp_graphblas/descriptor.hpp:12-65.
#pragma once

#include <utility>
#include <vector>

#include "types.hpp"

namespace lablas {
namespace backend {

class Descriptor {
public:
    Descriptor() {
        for (auto& v : desc_) v = GrB_DEFAULT;
    }
    LA_Info set(Desc_field f, Desc_value v) {
        desc_[f] = v;
        return GrB_SUCCESS;
    }
    LA_Info get(Desc_field f, Desc_value* v) const {
        *v = desc_[f];
        return GrB_SUCCESS;
    }
    // Fields below GrB_MODE flip between their default and a set value:
    // GrB_MASK -> GrB_SCMP (0), GrB_OUTPUT -> GrB_REPLACE, GrB_INP0/1 -> GrB_TRAN.
    LA_Info toggle(Desc_field f) {
        int field = static_cast<int>(f);
        if (field < 4) {
            if (desc_[f] != GrB_DEFAULT)
                desc_[f] = GrB_DEFAULT;
            else
                desc_[f] = field > 2 ? GrB_TRAN : static_cast<Desc_value>(field);
        }
        return GrB_SUCCESS;
    }
    bool debug() const { return false; }

private:
    Desc_value desc_[GrB_NDESCFIELD]{};
};

}  // namespace backend

typedef std::pair<Desc_field, Desc_value> desc_pair;

class Descriptor {
public:
    Descriptor() = default;
    explicit Descriptor(const std::vector<desc_pair>& init) {
        for (auto& p : init) d_.set(p.first, p.second);
    }
    LA_Info set(Desc_field f, Desc_value v) { return d_.set(f, v); }
    LA_Info get(Desc_field f, Desc_value* v) { return d_.get(f, v); }
    LA_Info toggle(Desc_field f) { return d_.toggle(f); }
    Desc_value get(Desc_field f) {
        Desc_value v;
        d_.get(f, &v);
        return v;
    }
    backend::Descriptor* get_descriptor() { return &d_; }
    const backend::Descriptor* get_descriptor() const { return &d_; }

private:
    backend::Descriptor d_;
};

inline Descriptor GrB_DESC_RSC({{GrB_OUTPUT, GrB_REPLACE}, {GrB_MASK, GrB_STR_COMP}});
inline Descriptor GrB_DESC_C({{GrB_MASK, GrB_COMP}});
inline Descriptor GrB_DESC_S({{GrB_MASK, GrB_STRUCTURE}});
inline Descriptor GrB_DESC_SC({{GrB_MASK, GrB_STR_COMP}});
inline Descriptor GrB_DESC_IKJ({{GrB_MXMMODE, GrB_IKJ}});
inline Descriptor GrB_DESC_IKJ_MASKED({{GrB_MXMMODE, GrB_IKJ_MASKED}});
inline Descriptor GrB_DESC_IJK({{GrB_MXMMODE, GrB_IJK}});
inline Descriptor GrB_DESC_IJK_DOUBLE_SORT({{GrB_MXMMODE, GrB_IJK_DOUBLE_SORT}});

inline Desc_value mask_mode(const Descriptor* d) {
    if (!d) return GrB_DEFAULT;
    Desc_value v;
    d->get_descriptor()->get(GrB_MASK, &v);
    return v;
}

}  // namespace lablas
