/* TEST INFRASTRUCTURE ONLY -- runs the reference's own host-side candidate
 * conversion of the periodicity search (aa_periodicity_candidates_data::
 * Process, include/aa_periodicity_candidates.hpp:81-105) on given host
 * records, for tests/golden/make_psr_candidates_golden.py.  The class keeps
 * its records private and fills them only by a device copy, so its members
 * are opened here to set them from the host; Process itself is the
 * reference's, compiled from its header where it lies. */
#include <cstdlib>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "aa_log.hpp"
#define private public
#include "aa_periodicity_candidates.hpp"
#undef private

extern "C" int aaref_psr_candidates_process(float *records, size_t n, float *msd, double dm_low, double dm_step,
                                            double sampling_time, size_t nTimesamples, float mod, int greedy)
{
    astroaccelerate::aa_periodicity_candidates_data d;
    d.c_nCandidates = n;
    d.c_nElements = 4;
    d.Allocate();
    if (!d.all)
        return -1;
    memcpy(d.all, records, n * 4 * sizeof(float));
    d.Process(msd, dm_low, dm_step, sampling_time, nTimesamples, mod, greedy);
    memcpy(records, d.all, n * 4 * sizeof(float));
    return 0;
}
