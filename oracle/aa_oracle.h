/*
 * aa_oracle.h -- CPU restatement of AstroAccelerate's DDTR path.
 * TEST INFRASTRUCTURE ONLY (see aa_oracle.c).  Loaded by tests/, by smoke()
 * and by bench.py's cpu_baseline leg; never by the product library.
 */
#ifndef AA_ORACLE_H
#define AA_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* include/aa_ddtr_plan.hpp:28-34 struct dm */
typedef struct {
    float low;
    float high;
    float step;
    int inBin;
    int outBin;
} aao_dm;

enum {
    AAO_K_SHARED8 = 0,  /* shared_dedisperse_kernel (8-bit, 1/2-bit unpacked) */
    AAO_K_SHARED16 = 1, /* shared_dedisperse_kernel_16 (16/32-bit) */
    AAO_K_SHARED4 = 2,  /* shared_dedisperse_kernel_4bit[_4096p] */
    AAO_K_CACHE = 3     /* cache_dedisperse_kernel ("failsafe") */
};

/* Which contractible device expressions are evaluated fused. */
enum {
    AAO_FMA_TWO = 1,   /* shift_two = mstartdm + (by*64)*mdmstep          (:196) */
    AAO_FMA_ONE = 2,   /* shift_one*dm_shifts[c] + findex                  (:211) */
    AAO_FMA_CACHE = 4, /* shift_temp = mstartdm + dm*mdmstep               (:430) */
    AAO_FMA_ALL = 7
};

enum {
    AAO_STRIDE_REFERENCE = 0, /* binning length exactly as the reference runner passes it */
    AAO_STRIDE_TRUE = 1       /* binning on the true row stride, repeated to reach inBin */
};

enum {
    AAO_OK = 0,
    AAO_ERR_NO_RANGES = -1,
    AAO_ERR_MAXSHIFT = -2,
    AAO_ERR_MEMORY = -3,
    AAO_ERR_REQUEST = -4,
    AAO_ERR_TOO_MANY_CHUNKS = -5,
    AAO_ERR_BOUNDS = -6,
    AAO_ERR_ALLOC = -7
};

int aao_strategy(const aao_dm *plan, int nranges, float power, int nchans,
                 int nsamp, double fch1, double foff, double tsamp, int nbits,
                 size_t free_memory, int enable_analysis, int max_chunks,
                 float *dmshifts, int *ndms, aao_dm *str_dm, int *maxshift_out,
                 int *max_ndms_out, int *num_tchunks_out, int *t_processed);

int aao_select_kernel(int nbits, float dm_step, float tsamp_r,
                      float dmshift_last, int failsafe);

int aao_delay(int kernel, int fma_mode, float dms, int dm, int tx,
              float mstartdm, float mdmstep);

int aao_dedisperse(int kernel, int fma_mode, const uint16_t *in, size_t in_len,
                   int i_nsamp, int nchans, int t_processed, int ndms,
                   const float *dmshifts, float mstartdm, float mdmstep,
                   int bin, float *out, double *sums);

int aao_dedisperse_window(int kernel, int fma_mode, const uint16_t *in, size_t in_len,
                          int i_nsamp, int nchans, int dm_first, int ndm, long long t_first,
                          int nt, long long t_shift, const float *dmshifts, float mstartdm,
                          float mdmstep, int bin, float *out, double *sums);

void aao_corner_turn(const uint16_t *in_tc, uint16_t *out_ct, int nchans, int nsamp);

int aao_bin_flat(uint16_t *buf, size_t buf_len, int nchans, int nsamp);

int aao_run_ddtr(const uint16_t *input_tc, int nchans, int nsamp,
                 double tsamp, int nbits, const float *dmshifts,
                 const aao_dm *str_dm, const int *ndms, int nranges,
                 int maxshift, int num_tchunks, const int *t_processed,
                 int max_chunks, int fma_mode, int stride_mode, int failsafe,
                 float *out, int *kernels_used);

int aao_fake_signal(uint16_t *out_tc, int nchans, int nsamples, double tsamp,
                    const float *dmshifts, int maxshift, double dm_pos,
                    int width, int signal_start, float sigma, int period_ms,
                    int *maximum_pos_out);

int aao_num_threads(void);
void aao_set_num_threads(int n);

#ifdef __cplusplus
}
#endif

#endif
