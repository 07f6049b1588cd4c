// filter.h -- device non-maximal removal (filter.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace qcb {

// Device scratch owned by a context, grown on demand.
struct FilterScratch {
    void *sorted = nullptr, *sig = nullptr, *poff = nullptr, *post = nullptr, *ctr = nullptr, *ents = nullptr, *bents = nullptr,
         *temp = nullptr, *ikey = nullptr, *ikey2 = nullptr, *ival = nullptr, *rsig = nullptr,
         *hsh = nullptr, *table = nullptr, *dead = nullptr, *rstarts = nullptr, *ikey3 = nullptr,
         *bents2 = nullptr, *rsz = nullptr;
    size_t sorted_n = 0, sig_n = 0, poff_n = 0, post_n = 0, ctr_n = 0, ents_n = 0, bents_n = 0,
           temp_n = 0, ikey_n = 0, ikey2_n = 0, ival_n = 0, rsig_n = 0, hsh_n = 0, table_n = 0,
           dead_n = 0, rstarts_n = 0, ikey3_n = 0, bents2_n = 0, rsz_n = 0;
    // page-locked host buffer the survivors are read back into (grown on demand)
    int32_t* host = nullptr;
    size_t host_n = 0;
    std::string ensure(void** p, size_t* have, size_t need);
    void release();
};

// Maximal sets of the emitted family (d_res with set starts d_starts) in
// lexicographic order, flat [k, ids..] on the host.  Returns "" or an error.
std::string filter_maximal(FilterScratch& F, const int32_t* d_res, int64_t nints,
                           const unsigned long long* d_starts, int64_t nsets, int32_t n_vertices,
                           cudaStream_t s, int sms, std::vector<int32_t>& host_out,
                           int64_t& host_nsets, int64_t* launches);

} // namespace qcb
