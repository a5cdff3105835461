// psr_candidates.cpp -- host-side candidate lists of the periodicity search
// (aa_periodicity_candidates / aa_periodicity_candidates_data,
// include/aa_periodicity_candidates.hpp:14-202): records of 4 floats
// (DM trial, bin, power, harmonic count) from peak finding, converted to
// (DM, frequency, S/N, harmonic count) per range and accumulated in order.
#include "aa_b200.h"

#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace {

thread_local std::string g_cand_error;

struct PsrCandidateList {
    struct Part {
        std::vector<float> records;
        int range_id;
    };
    std::vector<Part> parts;
};

// include/aa_periodicity_candidates.hpp:81-105: per record, the harmonic
// count (greedy lists carry a bin offset in its hundreds, which becomes a
// frequency correction of offset / harmonics bin widths); DM =
// trial * dm_step + dm_low; frequency = bin / (tsamp * nTimesamples * mod)
// (+ correction); S/N = (power - mean_h) / sd_h; each in the reference's
// mixed float/double expressions.
void process(float *all, size_t n, const float *msd, double dm_low, double dm_step, double sampling_time,
             size_t nTimesamples, float mod, int greedy)
{
    for (size_t c = 0; c < n; ++c) {
        float *r = all + 4 * c;
        int harmonics = static_cast<int>(r[3]);
        float freq_correction = 0;
        if (greedy) {
            const int datashift = static_cast<int>(r[3] / 100.0);
            harmonics = harmonics - datashift * 100;
            if (harmonics > 0) {
                const float bin_width = (1.0 / sampling_time) / (nTimesamples * mod);
                const float fraction = static_cast<double>(datashift) / static_cast<double>(harmonics);
                freq_correction = bin_width * fraction;
            }
        }
        r[0] = r[0] * dm_step + dm_low;
        r[1] = r[1] * (1.0 / (sampling_time * nTimesamples * mod)) + freq_correction;
        r[2] = (r[2] - msd[2 * harmonics]) / (msd[2 * harmonics + 1]);
        r[3] = harmonics;
    }
}

PsrCandidateList *as_list(void *obj) { return static_cast<PsrCandidateList *>(obj); }

} // namespace

extern "C" {

int aa_b200_psr_candidates_process(float *records, size_t n, const float *msd, double dm_low, double dm_step,
                                   double sampling_time, size_t nTimesamples, float mod, int greedy)
{
    if (n > 0 && (!records || !msd)) {
        g_cand_error = "periodicity candidates: null argument";
        return 1;
    }
    process(records, n, msd, dm_low, dm_step, sampling_time, nTimesamples, mod, greedy);
    return 0;
}

void *aa_b200_psr_candidates_create(void) { return new (std::nothrow) PsrCandidateList(); }

void aa_b200_psr_candidates_destroy(void *obj) { delete as_list(obj); }

int aa_b200_psr_candidates_add(void *obj, const float *records, size_t n, int on_device, int range_id,
                               const float *msd, double dm_low, double dm_step, double sampling_time,
                               size_t nTimesamples, float mod, int greedy)
{
    PsrCandidateList *L = as_list(obj);
    if (!L || (n > 0 && (!records || !msd))) {
        g_cand_error = "periodicity candidates: null argument";
        return 1;
    }
    PsrCandidateList::Part part;
    part.range_id = range_id;
    try {
        part.records.resize(4 * n);
    } catch (const std::bad_alloc &) {
        g_cand_error = "periodicity candidates: out of host memory";
        return 1;
    }
    if (n > 0) {
        if (on_device) {
            const cudaError_t e =
                cudaMemcpy(part.records.data(), records, 4 * n * sizeof(float), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) {
                g_cand_error = std::string("periodicity candidates: ") + cudaGetErrorString(e);
                return 1;
            }
        } else {
            std::memcpy(part.records.data(), records, 4 * n * sizeof(float));
        }
    }
    process(part.records.data(), n, msd, dm_low, dm_step, sampling_time, nTimesamples, mod, greedy);
    L->parts.push_back(std::move(part));
    return 0;
}

size_t aa_b200_psr_candidates_count(const void *obj)
{
    const PsrCandidateList *L = static_cast<const PsrCandidateList *>(obj);
    size_t n = 0;
    if (L)
        for (const auto &p : L->parts)
            n += p.records.size() / 4;
    return n;
}

int aa_b200_psr_candidates_copy(const void *obj, float *list)
{
    const PsrCandidateList *L = static_cast<const PsrCandidateList *>(obj);
    if (!L || !list) {
        g_cand_error = "periodicity candidates: null argument";
        return 1;
    }
    size_t pos = 0;
    for (const auto &p : L->parts) {
        std::memcpy(list + pos, p.records.data(), p.records.size() * sizeof(float));
        pos += p.records.size();
    }
    return 0;
}

// include/aa_periodicity_candidates.hpp:170-182: the lists one after the
// other as raw float records
int aa_b200_psr_candidates_export(const void *obj, const char *filename)
{
    const PsrCandidateList *L = static_cast<const PsrCandidateList *>(obj);
    if (!L || !filename) {
        g_cand_error = "periodicity candidates: null argument";
        return 1;
    }
    FILE *fp = std::fopen(filename, "wb");
    if (!fp) {
        g_cand_error = std::string("periodicity candidates: cannot open ") + filename;
        return 1;
    }
    int rc = 0;
    for (const auto &p : L->parts)
        if (!p.records.empty() && std::fwrite(p.records.data(), 4 * sizeof(float), p.records.size() / 4, fp) !=
                                      p.records.size() / 4)
            rc = 1;
    std::fclose(fp);
    if (rc)
        g_cand_error = std::string("periodicity candidates: cannot write ") + filename;
    return rc;
}

const char *aa_b200_psr_candidates_last_error(void) { return g_cand_error.c_str(); }

} // extern "C"
