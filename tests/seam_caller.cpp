// seam_caller.cpp -- a caller written against AstroAccelerate's own seam
// (namespace astroaccelerate: load_chunk_data, corner_turn_SM_inplace,
// bin_gpu, set_dedispersion_constants, dedisperse, save_data_offset_stream),
// driving them in the order of the reference runner's DDTR loop
// (include/aa_permitted_pipelines_generic.hpp:693-900).  tests/test_seam.py
// compiles it against aa_b200_seam.hpp and links it with libaa_b200.so only,
// so it checks that such a caller links unchanged and gets the oracle's
// output.
//
//   seam_caller <plan file> <input [t][c] uint16> <output float32>
//
// plan file (text): nchans nsamp nbits tsamp maxshift nranges nchunks, then
// per range: low step inBin ndms, then per range the nchunks t_processed
// values, then nchans dmshifts.  Output: every range's [ndms][sum of
// t_processed] rows, ranges one after the other.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include <cuda_runtime.h>

#include "aa_b200_seam.hpp"

int main(int argc, char **argv)
{
    if (argc != 4)
        return 2;
    FILE *pf = std::fopen(argv[1], "r");
    if (!pf)
        return 2;
    int nchans, nsamp, nbits, maxshift, nranges, nchunks;
    double tsamp_d;
    if (std::fscanf(pf, "%d %d %d %lf %d %d %d", &nchans, &nsamp, &nbits, &tsamp_d, &maxshift, &nranges, &nchunks) != 7)
        return 2;
    std::vector<float> dm_low(nranges), dm_step(nranges);
    std::vector<int> inBin(nranges), ndms(nranges);
    for (int r = 0; r < nranges; ++r)
        if (std::fscanf(pf, "%f %f %d %d", &dm_low[r], &dm_step[r], &inBin[r], &ndms[r]) != 4)
            return 2;
    std::vector<std::vector<int>> tp(nranges, std::vector<int>(nchunks));
    std::vector<int *> tp_rows(nranges);
    for (int r = 0; r < nranges; ++r) {
        for (int k = 0; k < nchunks; ++k)
            if (std::fscanf(pf, "%d", &tp[r][k]) != 1)
                return 2;
        tp_rows[r] = tp[r].data();
    }
    std::vector<float> dmshifts(nchans);
    for (int c = 0; c < nchans; ++c)
        if (std::fscanf(pf, "%f", &dmshifts[c]) != 1)
            return 2;
    std::fclose(pf);

    std::vector<unsigned short> input(static_cast<size_t>(nsamp) * nchans);
    FILE *fi = std::fopen(argv[2], "rb");
    if (!fi || std::fread(input.data(), 2, input.size(), fi) != input.size())
        return 2;
    std::fclose(fi);

    // host output rows, as the runner allocates them (float***)
    std::vector<size_t> total(nranges, 0);
    for (int r = 0; r < nranges; ++r)
        for (int k = 0; k < nchunks; ++k)
            total[r] += tp[r][k];
    float ***out = new float **[nranges];
    for (int r = 0; r < nranges; ++r) {
        out[r] = new float *[ndms[r]];
        for (int d = 0; d < ndms[r]; ++d)
            out[r][d] = new float[total[r]];
    }

    // device buffers sized for the first (largest) chunk
    size_t in_elems = static_cast<size_t>(nchans) * (tp[0][0] + maxshift);
    size_t out_elems = 0;
    for (int r = 0; r < nranges; ++r)
        out_elems = std::max(out_elems, static_cast<size_t>(ndms[r]) * tp[r][0]);
    out_elems = std::max(out_elems, in_elems);
    unsigned short *d_input = nullptr;
    float *d_output = nullptr;
    if (cudaMalloc(&d_input, in_elems * 2) != cudaSuccess || cudaMalloc(&d_output, out_elems * 4) != cudaSuccess)
        return 3;

    long inc = 0;
    for (int k = 0; k < nchunks; ++k) {
        astroaccelerate::load_chunk_data(d_input, input.data() + static_cast<size_t>(inc) * nchans, tp[0][k],
                                         maxshift, nchans, dmshifts.data(), nullptr, nbits);
        astroaccelerate::corner_turn_SM_inplace(d_input, reinterpret_cast<unsigned short *>(d_output), nchans,
                                                tp[0][k] + maxshift);
        int oldBin = 1;
        for (int r = 0; r < nranges; ++r) {
            float tsamp = static_cast<float>(tsamp_d) * inBin[r];
            const int ms_r = maxshift / inBin[r];
            if (inBin[r] > oldBin)
                astroaccelerate::bin_gpu(d_input, d_output, nchans, tp[r - 1][k] + ms_r * inBin[r]);
            astroaccelerate::set_dedispersion_constants(tp[r][k], ms_r);
            if (astroaccelerate::dedisperse(r, tp[r][k], inBin.data(), dmshifts.data(), d_input, d_output, nullptr,
                                            nchans, &tsamp, dm_low.data(), dm_step.data(), ndms.data(), nbits,
                                            0) != 0)
                return 4;
            astroaccelerate::save_data_offset_stream(r, k, tp_rows.data(), inc, inBin.data(), ndms.data(), d_output,
                                                     out);
            oldBin = inBin[r];
        }
        inc += tp[0][k];
    }

    FILE *fo = std::fopen(argv[3], "wb");
    if (!fo)
        return 2;
    for (int r = 0; r < nranges; ++r)
        for (int d = 0; d < ndms[r]; ++d)
            std::fwrite(out[r][d], 4, total[r], fo);
    std::fclose(fo);
    cudaFree(d_input);
    cudaFree(d_output);
    return 0;
}
