// C entry point over the reference's own aggregation builder
// (NP/src/solver/amg_builder.cpp:9 buildAMG, compiled from its source by
// ref.mk into _ref/libpfsf_ref_amg.so).  Test infrastructure only: the
// oracle's restatement (o_amg_build) is checked against it bit for bit.
#include <cstring>

#include "amg_builder.h"

extern "C" long long ref_build_amg(const float* sigma, const unsigned char* vtype, int lx, int ly, int lz, int* agg,
                                   float* w, float* dc) {
    const pfsf::AMGData d = pfsf::buildAMG(sigma, vtype, lx, ly, lz);
    if (!d.aggregation.empty()) {
        std::memcpy(agg, d.aggregation.data(), d.aggregation.size() * sizeof(int));
        std::memcpy(w, d.weights.data(), d.weights.size() * sizeof(float));
    }
    if (!d.diag_c.empty()) std::memcpy(dc, d.diag_c.data(), d.diag_c.size() * sizeof(float));
    return d.n_coarse;
}
