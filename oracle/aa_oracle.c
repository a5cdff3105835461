/*
 * aa_oracle.c -- CPU restatement of AstroAccelerate's brute-force dedispersion
 * (DDTR) path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: tests/, the
 * smoke() check in __graft_entry__.py and the cpu_baseline leg of bench.py may
 * load it, nothing else may.  The product library never links it and never
 * falls back to it.
 *
 * Every function restates one piece of the reference (AstroAccelerate v1.3.1)
 * and cites the file:line it follows.  Float expressions are written in the
 * same evaluation order as the reference and the file is compiled with
 * -ffp-contract=off so that host-side arithmetic rounds exactly like the
 * reference's host code (x86-64 SSE, no FMA).  Device-side arithmetic of the
 * reference kernels (CUDA, built with --use_fast_math => --fmad=true) is
 * restated with an explicit switch between the fused (fmaf) and the unfused
 * form of each contractible expression; which one the reference GPU build
 * produces is pinned by the golden vectors generated from the reference's own
 * kernels (tests/golden/).
 *
 * Accumulation semantics restated:
 *   shared 8-bit kernel  : exact integer sums (src/aa_device_dedispersion_kernel.cu:176-241)
 *   shared 4-bit kernel  : exact integer sums, (x & 0xFF), /nchans only (:105-174, :16-103)
 *   shared 16-bit kernel : fp32 sequential sum in ascending channel order (:303-362)
 *   cache kernel         : fp32 sequential sum in ascending channel order (:422-477)
 * Output scaling (float)S / nchans / bin is evaluated here with IEEE division;
 * the reference GPU build uses the fast-math division, which is identical
 * whenever nchans*bin is a power of two.  aao_dedisperse() therefore also
 * returns the raw sums so that tests can compare the integer work exactly.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "aa_oracle.h"

/* Tuning constants the strategy and the kernels are built around
 * (include/aa_params.hpp:95-99). */
#define O_SDIVINT 8
#define O_SDIVINDM 64
#define O_SNUMREG 14
#define O_MAX_OUTPUT_SIZE 17179869184ULL /* src/aa_ddtr_strategy.cpp:7 */

/* ------------------------------------------------------------------------ */
/* Strategy: src/aa_ddtr_strategy.cpp:27-428                                 */
/* ------------------------------------------------------------------------ */

static int request_memory(size_t *available, size_t bytes)
{
    /* include/aa_device_info.hpp request_memory(): strictly greater. */
    if (*available > bytes) {
        *available -= bytes;
        return 1;
    }
    return 0;
}

int aao_strategy(const aao_dm *plan, int nranges, float power, int nchans,
                 int nsamp, double fch1_d, double foff_d, double tsamp_d,
                 int nbits, size_t free_memory, int enable_analysis,
                 int max_chunks, float *dmshifts, int *ndms, aao_dm *str_dm,
                 int *maxshift_out, int *max_ndms_out, int *num_tchunks_out,
                 int *t_processed)
{
    /* :42-46 -- metadata narrowed to float */
    const float fch1 = (float)fch1_d;
    const float foff = (float)foff_d;
    const float tsamp = (float)tsamp_d;
    const int range = nranges;
    const int unit = O_SDIVINT * 2 * O_SNUMREG; /* 224 */
    const int unit4 = O_SDIVINT * 4 * O_SNUMREG; /* 448 */
    int c, i, j;
    int max_ndms = 0;
    int maxshift = 0, maxshift_high = 0;
    int num_tchunks = 0;
    unsigned int max_tsamps;
    size_t available = free_memory;

    if (range <= 0)
        return AAO_ERR_NO_RANGES; /* :63-66 */

    /* :81-92 dmshifts.  power != 2 takes the float pow overload that the
     * unqualified C++ call resolves to; power == 2 promotes to double. */
    if (power != 2.0) {
        for (c = 0; c < nchans; c++) {
            float fc = fch1 + (foff * (float)c);
            dmshifts[c] = (float)(4148.741601f *
                                  ((1.0 / (double)powf(fc, power)) -
                                   (1.0 / (double)powf(fch1, power))));
        }
    } else {
        for (c = 0; c < nchans; c++) {
            float fc = fch1 + (foff * (float)c);
            dmshifts[c] = (float)(4148.741601f *
                                  ((1.0 / pow((double)fc, (double)power)) -
                                   (1.0 / pow((double)fch1, (double)power))));
        }
    }

    /* :94-101 number of DM trials per range, a multiple of SDIVINDM */
    for (i = 0; i < range; i++) {
        float span = (plan[i].high - plan[i].low) / plan[i].step;
        int nblk = ((int)span + O_SDIVINDM) / O_SDIVINDM;
        ndms[i] = nblk * O_SDIVINDM;
        if (max_ndms < ndms[i])
            max_ndms = ndms[i];
    }

    /* :104-135 contiguous DM grid and the binned-range maxshift */
    str_dm[0].low = plan[0].low;
    str_dm[0].high = str_dm[0].low + ((float)ndms[0] * plan[0].step);
    str_dm[0].step = plan[0].step;
    for (i = 1; i < range; i++) {
        str_dm[i].low = str_dm[i - 1].high;
        str_dm[i].high = str_dm[i].low + (float)ndms[i] * plan[i].step;
        str_dm[i].step = plan[i].step;
        if (plan[i - 1].inBin > 1) {
            float top = str_dm[i - 1].low + str_dm[i - 1].step * (float)ndms[i - 1];
            float modulo = (float)unit;
            maxshift = (int)ceil((double)((top * dmshifts[nchans - 1]) / tsamp));
            maxshift = (int)(((float)maxshift / (float)plan[i - 1].inBin + modulo) / modulo);
            maxshift = maxshift * unit * plan[i - 1].inBin;
            if (maxshift > maxshift_high)
                maxshift_high = maxshift;
        }
    }
    if (plan[range - 1].inBin > 1) {
        float top = str_dm[range - 1].low + str_dm[range - 1].step * (float)ndms[range - 1];
        float modulo = (float)unit;
        maxshift = (int)ceil((double)((top * dmshifts[nchans - 1]) / tsamp));
        maxshift = (int)(((float)maxshift / (float)plan[range - 1].inBin + modulo) / modulo);
        maxshift = maxshift * unit * plan[range - 1].inBin;
        if (maxshift > maxshift_high)
            maxshift_high = maxshift;
    }
    /* :137-139 */
    if (maxshift_high == 0) {
        float top = str_dm[range - 1].low + str_dm[range - 1].step * (float)ndms[range - 1];
        maxshift_high = (int)ceil((double)((top * dmshifts[nchans - 1]) / tsamp));
    }
    maxshift = maxshift_high + O_SNUMREG * 2 * O_SDIVINT; /* :142 */

    if (maxshift >= nsamp)
        return AAO_ERR_MAXSHIFT; /* :146-149 */

    /* :156-389 time chunking (four memory cases) */
    {
        const size_t gpu_memory = free_memory - 104857600;
        const double SPDT_fraction = 3.0 / 4.0;
        const int bin_last = plan[range - 1].inBin;
        const int u = (nbits == 4) ? unit4 : unit;
        size_t spdt = enable_analysis ? (size_t)((double)(sizeof(float) * (size_t)max_ndms) * SPDT_fraction) : 0;
        int local_t = 0;
        int nblocks = 0, rem_block = 0, remainder = 0;
        int single = 0;

        if (nchans < max_ndms) {
            max_tsamps = (unsigned int)((gpu_memory) / (sizeof(unsigned short) * (size_t)nchans +
                                                         sizeof(float) * (size_t)max_ndms + spdt));
            {
                size_t out_per_chunk = ((size_t)max_tsamps) * sizeof(float) * ((size_t)max_ndms);
                if (out_per_chunk > O_MAX_OUTPUT_SIZE)
                    max_tsamps = (unsigned int)((O_MAX_OUTPUT_SIZE) / (sizeof(float) * (size_t)max_ndms));
            }
            if ((unsigned int)maxshift > max_tsamps)
                return AAO_ERR_MEMORY;
            if ((unsigned int)nsamp < max_tsamps) {
                /* case 1 (:186-207): double precision for the common length */
                unsigned long lt = (unsigned long)floor(((double)(nsamp - maxshift) / (double)bin_last) / (double)u);
                lt = lt * (unsigned long)u * (unsigned long)bin_last;
                if (1 > max_chunks)
                    return AAO_ERR_TOO_MANY_CHUNKS;
                for (i = 0; i < range; i++) {
                    int tp = (int)floor((double)(((float)(lt) / (float)plan[i].inBin) / (float)u));
                    t_processed[i * max_chunks + 0] = tp * u;
                }
                single = 1;
            } else {
                /* case 3 (:209-274) */
                int samp_block_size = (int)max_tsamps - maxshift;
                local_t = (int)floor((double)(((float)(samp_block_size) / (float)bin_last) / (float)u));
                local_t = local_t * u * bin_last;
            }
        } else {
            max_tsamps = (unsigned int)((gpu_memory) / ((size_t)nchans * (sizeof(float) + sizeof(unsigned short)) + spdt));
            {
                size_t out_per_chunk = ((size_t)max_tsamps) * sizeof(float) * ((size_t)nchans);
                if (out_per_chunk > O_MAX_OUTPUT_SIZE)
                    max_tsamps = (unsigned int)((O_MAX_OUTPUT_SIZE) / (sizeof(float) * (size_t)nchans));
            }
            if ((maxshift) > (int)max_tsamps)
                return AAO_ERR_MEMORY;
            if ((unsigned int)nsamp < max_tsamps) {
                /* case 2 (:300-322): float precision for the common length */
                int lt = (int)floor((double)(((float)(nsamp - (maxshift)) / (float)bin_last) / (float)u));
                lt = lt * u * bin_last;
                if (1 > max_chunks)
                    return AAO_ERR_TOO_MANY_CHUNKS;
                for (i = 0; i < range; i++) {
                    int tp = (int)floor((double)(((float)(lt) / (float)plan[i].inBin) / (float)u));
                    t_processed[i * max_chunks + 0] = tp * u;
                }
                single = 1;
            } else {
                /* case 4 (:324-388) */
                int samp_block_size = (int)max_tsamps - maxshift;
                local_t = (int)floor((double)(((float)(samp_block_size) / (float)bin_last) / (float)u));
                local_t = local_t * u * bin_last;
            }
        }

        if (single) {
            num_tchunks = 1;
        } else {
            /* shared tail of cases 3 and 4.  A chunk length of zero (device
             * memory below one chunk unit) divides by zero in the reference;
             * it is refused here. */
            if (local_t <= 0)
                return AAO_ERR_MEMORY;
            nblocks = (int)(((float)(nsamp - maxshift)) / ((float)local_t));
            remainder = nsamp - (nblocks * local_t) - (maxshift);
            /* (int)floor(x) / (float)u, truncated back to int on assignment */
            remainder = (int)((float)(int)floor((double)((float)remainder / (float)bin_last)) / (float)u);
            remainder = remainder * u * bin_last;
            rem_block = (remainder > 0) ? 1 : 0;
            if (nblocks + rem_block > max_chunks)
                return AAO_ERR_TOO_MANY_CHUNKS;
            for (i = 0; i < range; i++) {
                for (j = 0; j < nblocks; j++) {
                    int tp = (int)floor((double)(((float)(local_t) / (float)plan[i].inBin) / (float)u));
                    t_processed[i * max_chunks + j] = tp * u;
                }
                if (rem_block == 1) {
                    int tp = (int)floor((double)(((float)(remainder) / (float)plan[i].inBin) / (float)u));
                    t_processed[i * max_chunks + nblocks] = tp * u;
                }
            }
            num_tchunks = nblocks + rem_block;
        }
    }

    /* :401-415 device-memory reservation */
    {
        int time_samps = t_processed[0] + maxshift;
        request_memory(&available, (size_t)time_samps * (size_t)nchans * sizeof(unsigned short));
        if (nchans < max_ndms) {
            if (!request_memory(&available, (size_t)time_samps * (size_t)max_ndms * sizeof(float)))
                return AAO_ERR_REQUEST;
        } else {
            if (!request_memory(&available, (size_t)time_samps * (size_t)nchans * sizeof(float)))
                return AAO_ERR_REQUEST;
        }
    }

    /* :420-423 inBin/outBin are copied back from the plan */
    for (i = 0; i < range; i++) {
        str_dm[i].inBin = plan[i].inBin;
        str_dm[i].outBin = plan[i].outBin;
    }
    *maxshift_out = maxshift;
    *max_ndms_out = max_ndms;
    *num_tchunks_out = num_tchunks;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Kernel selection: src/aa_dedisperse.cpp:5-163                             */
/* ------------------------------------------------------------------------ */

int aao_select_kernel(int nbits, float dm_step, float tsamp_r,
                      float dmshift_last, int failsafe)
{
    const int limit = (O_SDIVINT - 1) + ((O_SDIVINDM - 1) * O_SDIVINT) - 1; /* 510 */
    if (failsafe != 0)
        return AAO_K_CACHE;
    if (nbits == 16 || nbits == 32) {
        /* :8-11, :20 */
        float shift_one = (float)(O_SDIVINDM - 1) * (dm_step / tsamp_r);
        int shifta = (int)floorf(shift_one * dmshift_last) + (O_SDIVINT - 1) * 2;
        int lineshift = shifta + ((O_SNUMREG - 1) * 2 * O_SDIVINT);
        return (limit > lineshift) ? AAO_K_SHARED16 : AAO_K_CACHE;
    } else if (nbits == 4) {
        /* :48-51, :62 */
        float shift_one = (float)(O_SDIVINDM - 1) * (dm_step / tsamp_r);
        int shifta = (int)floorf(shift_one * dmshift_last) + (O_SDIVINT - 1) * 4;
        int lineshift = shifta + ((O_SNUMREG - 1) * 4 * O_SDIVINT);
        return (limit > lineshift) ? AAO_K_SHARED4 : AAO_K_CACHE;
    } else {
        /* :88-92, :101 (8-bit and unpacked 1/2-bit data) */
        float shift_one = (float)(O_SDIVINDM - 1) * (dm_step / tsamp_r);
        int shifta = (int)floorf(shift_one * dmshift_last) + (O_SDIVINT - 1) * 2;
        int lineshift = shifta + ((O_SNUMREG - 1) * 2 * O_SDIVINT);
        return (limit > lineshift) ? AAO_K_SHARED8 : AAO_K_CACHE;
    }
}

/* ------------------------------------------------------------------------ */
/* Per-(channel, DM trial, time) delay of each reference kernel              */
/* ------------------------------------------------------------------------ */

/* Class of an output sample inside the thread tile of a shared kernel: the
 * index tx of the thread that produced it.  8/16-bit: t = bx*224 + 16*i +
 * 2*tx + {0,1}; 4-bit: t = bx*448 + 32*i + 4*tx + {0..3}. */
static inline int class_of(int kernel, int t)
{
    if (kernel == AAO_K_SHARED4)
        return (t & 31) >> 2;
    return (t & 15) >> 1;
}

/* findex of a class: 2tx+1 (8-bit, :185), 2tx (16-bit, :310), 4tx+3 (4-bit, :115) */
static inline int findex_of(int kernel, int tx)
{
    if (kernel == AAO_K_SHARED8)
        return 2 * tx + 1;
    if (kernel == AAO_K_SHARED16)
        return 2 * tx;
    return 4 * tx + 3;
}

int aao_delay(int kernel, int fma_mode, float dms, int dm, int tx,
              float mstartdm, float mdmstep)
{
    if (kernel == AAO_K_CACHE) {
        /* :430 shift_temp = mstartdm + (dm * mdmstep); :440 trunc(dms * shift_temp) */
        float dmf = (float)dm;
        float shift_temp = (fma_mode & AAO_FMA_CACHE) ? fmaf(dmf, mdmstep, mstartdm)
                                                       : mstartdm + (dmf * mdmstep);
        return (int)(dms * shift_temp);
    } else {
        /* :196-197 shift_two / shift_one, :206 base, :211 per-thread shift */
        float byf = (float)(dm / O_SDIVINDM);
        float tyf = (float)(dm % O_SDIVINDM);
        float two = byf * 64.0f;
        float shift_two = (fma_mode & AAO_FMA_TWO) ? fmaf(two, mdmstep, mstartdm)
                                                    : mstartdm + (two * mdmstep);
        float shift_one = tyf * mdmstep;
        int findex = findex_of(kernel, tx);
        int base = (int)(dms * shift_two);
        float s = (fma_mode & AAO_FMA_ONE) ? fmaf(shift_one, dms, (float)findex)
                                           : (shift_one * dms) + (float)findex;
        return base + (int)s - findex;
    }
}

/* ------------------------------------------------------------------------ */
/* Dedispersion of one (chunk, range): the kernels of                        */
/* src/aa_device_dedispersion_kernel.cu restated on a flat buffer.           */
/* ------------------------------------------------------------------------ */

int aao_dedisperse(int kernel, int fma_mode, const uint16_t *in, size_t in_len,
                   int i_nsamp, int nchans, int t_processed, int ndms,
                   const float *dmshifts, float mstartdm, float mdmstep,
                   int bin, float *out, double *sums)
{
    return aao_dedisperse_window(kernel, fma_mode, in, in_len, i_nsamp, nchans, 0, ndms, 0,
                                 t_processed, 0, dmshifts, mstartdm, mdmstep, bin, out, sums);
}

/* The same kernels for DM trials dm_first .. dm_first+ndm-1 of the range
 * (delays from the absolute trial index, so the block decomposition of
 * :196-197 is kept) and outputs t_first .. t_first+nt-1; output t reads
 * in[c*i_nsamp + t - t_shift + delay], so a caller may pass a buffer that
 * starts t_shift samples into the channel rows.  out/sums are [ndm][nt]. */
int aao_dedisperse_window(int kernel, int fma_mode, const uint16_t *in, size_t in_len,
                          int i_nsamp, int nchans, int dm_first, int ndm, long long t_first,
                          int nt, long long t_shift, const float *dmshifts, float mstartdm,
                          float mdmstep, int bin, float *out, double *sums)
{
    int j;
    int err = 0;
    /* 4-bit wide-band kernel drops the channels beyond 4096*floor(nchans/4096)
     * (call wrapper :520 uses integer division inside ceil). */
    int nch_used = nchans;
    if (kernel == AAO_K_SHARED4 && nchans > 4096)
        nch_used = 4096 * (nchans / 4096);
    if (nt <= 0 || ndm <= 0)
        return 0;

#pragma omp parallel for schedule(dynamic, 1) reduction(| : err)
    for (j = 0; j < ndm; j++) {
        int t, c, k;
        const int dm = dm_first + j;
        int *dl = (int *)malloc(sizeof(int) * 8 * (size_t)nchans);
        int64_t *isum = NULL;
        float *fsum = NULL;
        int integer = (kernel == AAO_K_SHARED8 || kernel == AAO_K_SHARED4);
        if (integer)
            isum = (int64_t *)calloc((size_t)nt, sizeof(int64_t));
        else
            fsum = (float *)calloc((size_t)nt, sizeof(float));
        for (c = 0; c < nchans; c++)
            for (k = 0; k < 8; k++)
                dl[c * 8 + k] = aao_delay(kernel, fma_mode, dmshifts[c], dm, k, mstartdm, mdmstep);
        for (c = 0; c < nch_used; c++) {
            const long long row = (long long)c * (long long)i_nsamp - t_shift;
            const int *d = dl + c * 8;
            for (t = 0; t < nt; t++) {
                const long long ta = t_first + t;
                int delay = (kernel == AAO_K_CACHE) ? d[0] : d[class_of(kernel, (int)(ta & 31))];
                long long idx = row + ta + delay;
                unsigned v;
                if (idx < 0 || (size_t)idx >= in_len) {
                    err |= 1;
                    continue;
                }
                v = in[idx];
                if (kernel == AAO_K_SHARED4)
                    v &= 0xFFu; /* :135 (unsigned char) cast */
                if (integer)
                    isum[t] += v;
                else
                    fsum[t] = fsum[t] + (float)v;
            }
        }
        for (t = 0; t < nt; t++) {
            float o;
            size_t oi = (size_t)j * (size_t)nt + t;
            if (integer) {
                float s = (float)isum[t];
                if (kernel == AAO_K_SHARED4)
                    o = s / (float)nchans; /* :169-172 no /bin */
                else
                    o = (s / (float)nchans) / (float)bin; /* :239 */
                if (sums)
                    sums[oi] = (double)isum[t];
            } else {
                o = (fsum[t] / (float)nchans) / (float)bin; /* :360, :448 */
                if (sums)
                    sums[oi] = (double)fsum[t];
            }
            out[oi] = o;
        }
        free(dl);
        free(isum);
        free(fsum);
    }
    return err ? AAO_ERR_BOUNDS : 0;
}

/* ------------------------------------------------------------------------ */
/* Corner turn and binning on the flat device buffer                         */
/* ------------------------------------------------------------------------ */

/* src/aa_corner_turn.cpp:118-121 + src/aa_device_corner_turn_kernel.cu:10-70:
 * [t][c] -> [c][t] (length nsamp per channel row). */
void aao_corner_turn(const uint16_t *in_tc, uint16_t *out_ct, int nchans, int nsamp)
{
    int c;
#pragma omp parallel for schedule(static)
    for (c = 0; c < nchans; c++) {
        int t;
        for (t = 0; t < nsamp; t++)
            out_ct[(size_t)c * nsamp + t] = in_tc[(size_t)t * nchans + c];
    }
}

/* src/aa_bin_gpu.cpp:8-44: memset(tmp), bin kernel
 * (src/aa_device_binning_kernel.cu:33-45), swap kernel
 * (src/aa_device_corner_turn_kernel.cu:91-98), i.e. on the flat buffer:
 *   tmp[c*(nsamp/2)+t] = (a+b)/2.0f for c < 32*(nchans/32), t < 8*((nsamp+1)/16)
 *   buf[c*nsamp+t]     = (ushort)tmp[c*nsamp+t] for c < 8*(nchans/8), t < 32*(nsamp/32)
 * Requires nchans*nsamp <= buf_len. */
int aao_bin_flat(uint16_t *buf, size_t buf_len, int nchans, int nsamp)
{
    size_t n = (size_t)nchans * (size_t)nsamp;
    float *tmp;
    int c;
    int cb = 32 * (nchans / 32), tb = 8 * ((nsamp + 1) / 16);
    int cs = 8 * (nchans / 8), ts = 32 * (nsamp / 32);
    int out_nsamp = nsamp / 2;
    if (n > buf_len)
        return AAO_ERR_BOUNDS;
    tmp = (float *)calloc(n, sizeof(float));
    if (!tmp)
        return AAO_ERR_ALLOC;
    /* sequential over c so that overlapping writes (odd nsamp) resolve in a
     * fixed order; the strategy only produces even nsamp. */
    for (c = 0; c < cb; c++) {
        int t;
        for (t = 0; t < tb; t++) {
            size_t s = (size_t)c * nsamp + 2 * (size_t)t;
            size_t d = (size_t)c * out_nsamp + t;
            if (s + 1 >= n || d >= n)
                continue;
            tmp[d] = (float)((float)(buf[s] + buf[s + 1]) / 2.0f);
        }
    }
#pragma omp parallel for schedule(static)
    for (c = 0; c < cs; c++) {
        int t;
        for (t = 0; t < ts; t++) {
            size_t i = (size_t)c * nsamp + t;
            buf[i] = (uint16_t)tmp[i];
        }
    }
    free(tmp);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Whole DDTR replay: include/aa_permitted_pipelines_generic.hpp:606-914     */
/* ------------------------------------------------------------------------ */

int aao_run_ddtr(const uint16_t *input_tc, int nchans, int nsamp,
                 double tsamp_d, int nbits, const float *dmshifts,
                 const aao_dm *str_dm, const int *ndms, int nranges,
                 int maxshift, int num_tchunks, const int *t_processed,
                 int max_chunks, int fma_mode, int stride_mode, int failsafe,
                 float *out, int *kernels_used)
{
    const float tsamp_original = (float)tsamp_d;
    size_t L0 = (size_t)t_processed[0] + (size_t)maxshift; /* chunk 0 is the largest */
    size_t buf_len = (size_t)nchans * L0;
    uint16_t *buf = (uint16_t *)malloc(buf_len * sizeof(uint16_t));
    float *tmp_out = NULL;
    size_t *row_len = (size_t *)calloc((size_t)nranges, sizeof(size_t));
    size_t *range_off = (size_t *)calloc((size_t)nranges, sizeof(size_t));
    long inc = 0;
    int k, r, err = 0;
    size_t max_tile = 0;

    if (!buf || !row_len || !range_off) {
        free(buf);
        free(row_len);
        free(range_off);
        return AAO_ERR_ALLOC;
    }
    /* output layout: per range [ndms][sum_k t_processed[r][k]] (the rows of
     * the host float*** buffer, :418-445), ranges concatenated */
    {
        size_t off = 0;
        for (r = 0; r < nranges; r++) {
            size_t tot = 0;
            for (k = 0; k < num_tchunks; k++) {
                size_t tile = (size_t)ndms[r] * (size_t)t_processed[r * max_chunks + k];
                tot += (size_t)t_processed[r * max_chunks + k];
                if (tile > max_tile)
                    max_tile = tile;
            }
            row_len[r] = tot;
            range_off[r] = off;
            off += tot * (size_t)ndms[r];
        }
    }
    tmp_out = (float *)malloc((max_tile ? max_tile : 1) * sizeof(float));
    if (!tmp_out) {
        free(buf);
        free(row_len);
        free(range_off);
        return AAO_ERR_ALLOC;
    }

    for (k = 0; k < num_tchunks && !err; k++) {
        int t0 = t_processed[0 * max_chunks + k];
        int L = t0 + maxshift;
        int oldBin = 1;
        size_t cur_stride = (size_t)L; /* row stride the data really has */
        int cur_bin = 1;                /* binning the data really has */
        if ((size_t)inc + (size_t)L > (size_t)nsamp) {
            err = AAO_ERR_BOUNDS;
            break;
        }
        /* :693 load + :741 corner turn */
        aao_corner_turn(input_tc + (size_t)inc * nchans, buf, nchans, L);

        for (r = 0; r < nranges && !err; r++) {
            int tp = t_processed[r * max_chunks + k];
            float tsamp = tsamp_original * ((float)str_dm[r].inBin); /* :778 */
            int ms_r = maxshift / str_dm[r].inBin;                   /* :782 */
            int i_nsamp;
            int kernel;
            float mstartdm, mdmstep;
            if (stride_mode == AAO_STRIDE_REFERENCE) {
                if (str_dm[r].inBin > oldBin) {
                    /* :797-798: one x2 binning with the runner's length */
                    int nsb = t_processed[(r - 1) * max_chunks + k] + ms_r * str_dm[r].inBin;
                    err = aao_bin_flat(buf, buf_len, nchans, nsb);
                    if (err)
                        break;
                }
                i_nsamp = tp + ms_r; /* :786 set_dedispersion_constants */
            } else {
                /* mathematically intended binning: the true row stride and as
                 * many x2 steps as the binning factor needs */
                while (cur_bin < str_dm[r].inBin) {
                    err = aao_bin_flat(buf, buf_len, nchans, (int)cur_stride);
                    if (err)
                        break;
                    cur_stride /= 2;
                    cur_bin *= 2;
                }
                if (err)
                    break;
                i_nsamp = (int)cur_stride;
            }
            mstartdm = (float)(str_dm[r].low / tsamp); /* :18-30 of aa_dedisperse.cpp */
            mdmstep = (float)(str_dm[r].step / tsamp);
            kernel = aao_select_kernel(nbits, str_dm[r].step, tsamp, dmshifts[nchans - 1], failsafe);
            if (kernels_used)
                kernels_used[r * max_chunks + k] = kernel;
            err = aao_dedisperse(kernel, fma_mode, buf, buf_len, i_nsamp, nchans, tp,
                                 ndms[r], dmshifts, mstartdm, mdmstep, str_dm[r].inBin,
                                 tmp_out, NULL);
            if (err)
                break;
            /* :835-840 -> src/aa_device_save_data.cu:19-62: each DM row lands at
             * output_buffer[r][dm] + inc/inBin */
            {
                int dm;
                size_t host_off = (size_t)(inc / str_dm[r].inBin);
                for (dm = 0; dm < ndms[r]; dm++)
                    memcpy(out + range_off[r] + (size_t)dm * row_len[r] + host_off,
                           tmp_out + (size_t)dm * tp, (size_t)tp * sizeof(float));
            }
            oldBin = str_dm[r].inBin;
        }
        inc += t0; /* :898 */
    }
    free(buf);
    free(tmp_out);
    free(row_len);
    free(range_off);
    return err;
}

/* ------------------------------------------------------------------------ */
/* Fake signal: src/aa_host_fake_signal_generator.cpp:13-116                 */
/* ------------------------------------------------------------------------ */

int aao_fake_signal(uint16_t *out_tc, int nchans, int nsamples, double tsamp,
                    const float *dmshifts, int maxshift, double dm_pos,
                    int width, int signal_start, float sigma, int period_ms,
                    int *maximum_pos_out)
{
    const double PI = 3.14159265359;
    const int MAX_VALUE = 255;
    float *mask = (float *)malloc(sizeof(float) * (size_t)(width > 0 ? width : 1));
    int *shift_index = (int *)malloc(sizeof(int) * (size_t)nchans);
    float maximum = 0.0f;
    float g_mean = 1.0f;
    int maximum_pos = 0;
    int i, j, r;
    int repeats = 1, period = 0;
    float temp;
    if (!mask || !shift_index) {
        free(mask);
        free(shift_index);
        return AAO_ERR_ALLOC;
    }
    /* produce_mask :13-32 */
    {
        float wid = (float)(2 * sigma * pow(3 * log(30), 0.5));
        float step = wid * sigma / (float)(width);
        for (i = 0; i < width; i++) {
            float x = (float)(i + 1) * step;
            mask[i] = (float)(sqrt((double)sigma / (2 * PI * pow((double)x, 3))) *
                              exp((-(double)sigma * pow((double)(x - g_mean), 2)) /
                                  (2 * pow((double)g_mean, 2) * (double)x)));
            if (maximum <= mask[i]) {
                maximum = mask[i];
                maximum_pos = i;
            }
        }
        for (i = 0; i < width; i++)
            mask[i] = mask[i] / maximum;
    }
    if (signal_start + maxshift > nsamples) {
        free(mask);
        free(shift_index);
        return AAO_ERR_BOUNDS; /* :53-60 */
    }
    if (signal_start == 0)
        signal_start = -maximum_pos - 2 * maxshift;
    temp = (float)(dm_pos / tsamp);
    for (i = 0; i < nchans; i++)
        shift_index[i] = (int)floor((double)(dmshifts[i] * temp));
    if (period_ms > 0) {
        period = (int)(period_ms / 1000.0 / tsamp);
        repeats = (nsamples + 2 * maxshift) / (period) + 1;
    }
    for (r = 0; r < repeats; r++) {
        for (i = 0; i < width; i++) {
            const int time_pos = (i - maximum_pos + signal_start + period * r) * nchans;
            for (j = 0; j < nchans; j++) {
                const int gi = j + nchans * shift_index[j] + time_pos;
                if ((gi < nsamples * nchans) && (gi > 0))
                    out_tc[gi] = (uint16_t)((float)MAX_VALUE * mask[i]);
            }
        }
    }
    if (maximum_pos_out)
        *maximum_pos_out = maximum_pos;
    free(mask);
    free(shift_index);
    return 0;
}

int aao_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void aao_set_num_threads(int n)
{
#ifdef _OPENMP
    if (n > 0)
        omp_set_num_threads(n);
#else
    (void)n;
#endif
}
