// schedule.cu -- the balanced kernel scheduler stored in ptiSparseTensorHiCOO
// (kschr_balanced, kschr_balanced_pos, nkpars, kschr_rest), restating
// src/sptensor/hicoo/convert.c:475-571 on the host.  It is an O(#kernels)
// pass over the per-mode kernel lists and only fills struct fields that the
// reference's scheduled OpenMP kernels read.
#include "common.cuh"

namespace pti {

int assign_index_vector(ptiIndexVector *v, const uint32_t *src, uint64_t len);

int balanced_schedule(ptiSparseTensorHiCOO *h, uint64_t nnz)
{
    (void)nnz;
    const uint32_t N = h->nmodes;
    const uint64_t nk = h->kptr.len ? h->kptr.len - 1 : 0;
    uint64_t max_nnzk = 0;
    for (uint64_t k = 0; k < nk; ++k) max_nnzk = std::max<uint64_t>(max_nnzk, h->knnzs.data[k]);
    // par_nnzk_th = 5 * max_nnzk (convert.c:481-483)
    const uint64_t par_nnzk_th = 5 * max_nnzk;
    const uint64_t sk = (uint64_t)1 << h->sk_bits;
    for (uint32_t m = 0; m < N; ++m) {
        const uint64_t rows = ((uint64_t)h->ndims[m] + sk - 1) / sk;
        std::vector<std::vector<uint32_t>> bal(rows), pos(rows);
        std::vector<uint32_t> rest;
        for (uint64_t i = 0; i < rows; ++i) pos[i].push_back(0);
        const ptiIndexVector *kschr = h->kschr[m];
        uint32_t npars = 0;
        bool tag_rest = false;
        uint64_t count_nk = 0;
        const uint64_t empty_th = rows > 1 ? rows : 1;
        while (!tag_rest && count_nk < nk) {
            uint32_t max_per_col = 0;  // ptiIndex in the reference
            uint64_t empty = 0;
            for (uint64_t i = 0; i < rows; ++i) {
                if (empty > empty_th) {
                    tag_rest = true;
                    break;
                }
                if (npars >= pos[i].size()) {
                    ++empty;
                    continue;
                }
                uint32_t j = pos[i][npars];
                if (j >= kschr[i].len) {
                    ++empty;
                    continue;
                }
                uint64_t knz = h->knnzs.data[kschr[i].data[j]];
                if (max_per_col < knz) max_per_col = (uint32_t)knz;
            }
            if (tag_rest) {
                for (uint64_t i = 0; i < rows; ++i) {
                    if (npars >= pos[i].size()) continue;
                    for (uint64_t j2 = pos[i][npars]; j2 < kschr[i].len; ++j2) {
                        rest.push_back(kschr[i].data[j2]);
                        ++count_nk;
                    }
                }
            } else {
                const uint32_t par_nnzk = max_per_col > par_nnzk_th ? max_per_col : (uint32_t)par_nnzk_th;
                for (uint64_t i = 0; i < rows; ++i) {
                    if (npars >= pos[i].size()) continue;
                    uint32_t tmp_j = pos[i][npars];
                    if (tmp_j >= kschr[i].len) continue;
                    uint32_t kernel_num = kschr[i].data[tmp_j];
                    uint64_t sum = h->knnzs.data[kernel_num];
                    while (sum <= par_nnzk) {
                        bal[i].push_back(kernel_num);
                        ++count_nk;
                        ++tmp_j;
                        if (tmp_j < kschr[i].len) {
                            kernel_num = kschr[i].data[tmp_j];
                            sum += h->knnzs.data[kernel_num];
                        } else {
                            break;
                        }
                    }
                    pos[i].push_back(tmp_j);
                }
                ++npars;
            }
        }
        h->nkpars[m] = npars;
        for (uint64_t i = 0; i < rows; ++i) {
            PTI_TRY(assign_index_vector(&h->kschr_balanced[m][i], bal[i].data(), bal[i].size()));
            PTI_TRY(assign_index_vector(&h->kschr_balanced_pos[m][i], pos[i].data(), pos[i].size()));
        }
        PTI_TRY(assign_index_vector(&h->kschr_rest[m], rest.data(), rest.size()));
    }
    return 0;
}

}  // namespace pti
