/*
 * aa_b200.h -- C ABI of the B200-native dedispersion (DDTR) and
 * single-pulse detection library
 * (libaa_b200.so, built from astro-accelerate_b200/csrc/).
 *
 * Two layers:
 *
 *  1. aa_py_* : the entry points of the reference's own C ABI for the DDTR
 *     path (AstroAccelerate v1.3.1, src/aa_py_*.cpp, bound by ctypes in
 *     cmake/py_astro_accelerate.py.in).  Same names, argument meaning, return
 *     values and status codes, so the reference's Python wrapper binds this
 *     library by changing the library path.  The dedispersion, analysis
 *     (single-pulse detection) and periodicity components are implemented;
 *     FDAS plans are refused (return false).
 *
 *  2. aa_b200_* : the seam the reference's runner calls internally
 *     (load/corner turn/binning/dedisperse, include/aa_permitted_pipelines_generic.hpp),
 *     made stateless (explicit strides and streams instead of __constant__
 *     state), plus the pipeline extensions this library adds (whole-job run,
 *     rewind, device-resident input/output, options).
 *
 * All pointers are plain; "stream" is a cudaStream_t passed as void*.
 * Functions returning int return 0 on success unless stated otherwise;
 * aa_b200_last_error() gives the message of the last failure of this thread.
 */
#ifndef AA_B200_H
#define AA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
#include <cstdbool>
extern "C" {
#else
#include <stdbool.h>
#endif

/* ------------------------------------------------------------------------ */
/* 1. Reference C ABI (aa_py_*)                                              */
/* ------------------------------------------------------------------------ */

/* include/aa_py_filterbank_metadata.hpp:15-25 */
typedef struct {
    double m_tstart;
    double m_tsamp;
    double m_fch1;
    double m_foff;
    int m_nbits;
    int m_nsamples;
    int m_nchans;
    double m_src_raj;
} aa_py_filterbank_metadata_struct;

/* include/aa_py_pipeline_api.hpp:20-25 */
typedef struct {
    bool dedispersion;
    bool analysis;
    bool periodicity;
    bool fdas;
} pipeline_components_struct;

/* include/aa_py_pipeline_api.hpp:32-48 */
typedef struct {
    bool zero_dm;
    bool zero_dm_with_outliers;
    bool input_DDTR_normalization;
    bool output_DDTR_normalization;
    bool set_bandpass_average;
    bool old_rfi;
    bool copy_ddtr_data_to_host;
    bool msd_baseline_noise;
    bool output_dmt;
    bool output_ffdot_plan;
    bool output_fdas_list;
    bool candidate_algorithm;
    bool fdas_custom_fft;
    bool fdas_inbin;
    bool fdas_norm;
} pipeline_component_option_struct;

/* src/aa_py_filterbank_metadata.cpp:7-28, :30-32, :34-36 */
aa_py_filterbank_metadata_struct *aa_py_filterbank_metadata(double tstart, double tsamp, int nbits, int nsamples,
                                                            double fch1, double foff, int nchans, double src_raj);
void aa_py_filterbank_metadata_delete(const aa_py_filterbank_metadata_struct *obj);
double aa_py_filterbank_metadata_tstart(const aa_py_filterbank_metadata_struct *obj);

/* src/aa_py_ddtr_plan.cpp:7-46 (aa_ddtr_plan*, opaque) */
void *aa_py_ddtr_plan(void);
void aa_py_ddtr_plan_delete(const void *obj);
bool aa_py_ddtr_plan_add_dm(void *obj, float low, float high, float step, int inBin, int outBin);
size_t aa_py_ddtr_plan_range(const void *obj);
bool aa_py_ddtr_plan_set_power(void *obj, float power);
float aa_py_ddtr_plan_power(const void *obj);
bool aa_py_ddtr_plan_set_enable_msd_baseline(void *obj, bool flag);
bool aa_py_ddtr_plan_enable_msd_baseline_noise(const void *obj);
bool aa_py_ddtr_plan_bind_bandpass_normalization(void *obj, const float *data, int data_size);

/* src/aa_py_pipeline_api.cpp:9-40 (aa_pipeline_api<unsigned short>*, opaque).
 * input_data: host [nsamples][nchans] unsigned short, one value per sample. */
void *aa_py_pipeline_api(pipeline_components_struct pipeline, pipeline_component_option_struct options,
                         aa_py_filterbank_metadata_struct metadata, const unsigned short *input_data,
                         int card_number);
/* :42-44 */
void aa_py_pipeline_api_delete(const void *obj);
/* :46-48 */
bool aa_py_pipeline_api_bind_ddtr_plan(void *obj, const void *plan);
/* :50-52: a new strategy object; free with aa_py_ddtr_strategy_delete */
void *aa_py_pipeline_api_ddtr_strategy(void *obj);
/* src/aa_py_ddtr_strategy.cpp:6-8 */
void aa_py_ddtr_strategy_delete(const void *obj);
/* :54-56 */
size_t aa_py_get_ddtr_nRanges(void *obj);
/* :58-60 */
const int *aa_py_get_ndms_array(void *obj);
/* :62-64 t_processed[i][j] */
int aa_py_get_t_proc(void *obj, int i, int j);
/* :66-68 (the reference truncates the float DM to int) */
int aa_py_dm_low(void *obj, int range);
/* :70-72 */
int aa_py_total_computed_samples(void *obj);
/* src/aa_py_analysis_plan.cpp:6-44 (aa_analysis_plan*, opaque): the
 * single-pulse detection settings; ddtr_strategy from
 * aa_py_pipeline_api_ddtr_strategy.  candidate_algorithm 0 peak finding,
 * 1 thresholding, 2 peak filtering (7 x 7 stencil peaks, then the
 * suppression of weaker peaks within 15 ms). */
void *aa_py_analysis_plan(const void *ddtr_strategy, float sigma_cutoff, float sigma_constant,
                          float max_boxcar_width_in_sec, int candidate_algorithm, bool enable_msd_baseline_noise);
void aa_analysis_plan_delete(const void *obj);
float aa_py_analysis_plan_sigma_cutoff(const void *obj);
float aa_py_analysis_plan_sigma_constant(const void *obj);
float aa_py_analysis_plan_max_boxcar_width_in_sec(const void *obj);
bool aa_py_analysis_plan_enable_msd_baseline_noise(const void *obj);
/* src/aa_py_pipeline_api.cpp:74-76 (include/aa_pipeline_api.hpp:182-219):
 * needs the analysis component requested, the DDTR plan bound (its strategy
 * is then computed for analysis) and sigma_cutoff, sigma_constant and
 * max_boxcar_width_in_sec above 0.  With it bound, every
 * aa_py_pipeline_api_run step that dedisperses also runs analysis_GPU on the
 * step's rows (include/aa_permitted_pipelines_generic.hpp:848-889) and writes
 * the reference's candidate file (aa_b200_pipeline_set_candidate_output). */
bool aa_py_pipeline_api_bind_analysis_plan(void *obj, const void *plan);
/* :109-127: the candidates of the last step (DM trial index in the range,
 * sample, S/N, boxcar width in samples of the range); the arrays stay valid
 * until the next step (NULL when there are none). */
size_t aa_py_spd_nCandidates(void *obj);
/* :78-80: the bound analysis settings as a new object (NULL when none is
 * bound); free with aa_analysis_plan_delete. */
void *aa_py_pipeline_api_analysis_strategy(void *obj);
/* :129-141: periodicity candidates after the search ran (Get_PSR_candidates,
 * Get_PSR_interbin_candidates, Write_to_disk_PSR_candidates of
 * include/aa_permitted_pipelines_generic.hpp:1173-1193): records of 4 floats
 * (DM, frequency, S/N, harmonics), every batch's in order, in a copy the
 * pipeline object owns (valid until the next call of the same getter; the
 * count is aa_b200_pipeline_psr_count).  NULL (write: nothing) with an
 * error message before the search has run. */
float *aa_py_get_psr_nCandidates(void *obj);
float *aa_py_get_psr_interbin_nCandidates(void *obj);
void aa_py_write_to_disk_psr_candidates(void *obj, const char *filename);
unsigned int *aa_py_h_dm(void *obj);
unsigned int *aa_py_h_ts(void *obj);
float *aa_py_h_snr(void *obj);
unsigned int *aa_py_h_width(void *obj);
/* :82-85: the periodicity plan (aa_periodicity_plan's six-argument
 * constructor, include/aa_periodicity_plan.hpp:39-60: greedy harmonic sum,
 * scalloping-loss mitigation and whitening on) built from the bound DDTR
 * strategy, and its strategy for the device's free memory
 * (include/aa_periodicity_strategy.hpp:178-355).  The pipeline must have
 * been created with the periodicity component and the DDTR plan bound; the
 * search then runs on the run() call after the dedispersion component
 * finished (status finished_component), over the host rows or, when they
 * are kept on the device, the device rows.  :87-90: FDAS is out of scope
 * and refused (false). */
bool aa_py_pipeline_api_bind_periodicity_plan(void *obj, float sigma_cutoff, bool enable_outlier_rejection,
                                              float sigma_outlier_rejection_threshold, int nHarmonics,
                                              int candidate_selection_algorithm);
bool aa_py_pipeline_api_bind_fdas_plan(void *obj, float sigma_cutoff, float sigma_constant,
                                       bool enable_msd_baseline_noise);
/* aa_periodicity_plan's ten-argument constructor
 * (include/aa_periodicity_plan.hpp:62-89): harmonic_sum_algorithm 0 simple
 * (on corner-turned spectra), 1 greedy, 2 PRESTO plus, 3 PRESTO;
 * candidate_selection_algorithm 0 peak finding, 1 thresholding.  The
 * interbinning and whitening switches are carried as the reference carries
 * them (its search computes both either way). */
bool aa_b200_pipeline_bind_periodicity_plan(void *obj, float sigma_cutoff, int enable_outlier_rejection,
                                            float sigma_outlier_rejection_threshold, int nHarmonics,
                                            int harmonic_sum_algorithm, int candidate_selection_algorithm,
                                            int enable_scalloping_loss_mitigation, int enable_interbinning,
                                            int enable_spectrum_whitening);
/* on != 0: keep every range's whole output on the device as well
 * ([ndms][total samples] per range, aa_b200_pipeline_device_output), also
 * for pipelines made by aa_py_pipeline_api; before the DDTR plan is bound.
 * The periodicity search then reads these rows instead of the host rows. */
bool aa_b200_pipeline_set_device_output(void *obj, int on);
/* Bytes the periodicity strategy plans its batches for, instead of the
 * device's free memory at bind time (before binding the plan). */
bool aa_b200_pipeline_set_periodicity_memory(void *obj, size_t bytes);
/* Candidates of the power (interbin = 0) or interbin (1) spectra. */
size_t aa_b200_pipeline_psr_count(void *obj, int interbin);
/* Write_to_disk_PSR_interbin_candidates (include/aa_pipeline_api.hpp:1142-1144). */
bool aa_b200_pipeline_write_psr_interbin_candidates(void *obj, const char *filename);
/* The bound periodicity strategy: FFT length of unbinned ranges, DM trials
 * per batch, batches over all ranges; compute_ms: device time of the last
 * search's stages (after each batch's input copy).  Returns 0, or 1 when no
 * periodicity plan is bound. */
int aa_b200_pipeline_psr_info(void *obj, size_t *fft_length, size_t *dms_per_batch, int *batches, double *compute_ms);
/* :92-103: one (time chunk, DM range) step; *status_code receives
 * aa_pipeline_runner::status (-1 error, 0 finished, 1 has_more,
 * 2 finished_component, include/aa_pipeline_runner.hpp:25-30). */
bool aa_py_pipeline_api_run(void *obj, int *status_code);
/* :105-107 float*** [range][dm][sum_k t_processed[range][k]] */
float ***aa_py_buffer(void *obj);
/* :143-157 */
int aa_py_current_range(void *obj);
int aa_py_current_time_chunk(void *obj);
long aa_py_current_inc(void *obj);
bool aa_py_cleanup(void *obj);

/* ------------------------------------------------------------------------ */
/* 2. Seam and extensions (aa_b200_*)                                        */
/* ------------------------------------------------------------------------ */

/* aa_ddtr_plan::dm, include/aa_ddtr_plan.hpp:28-34 */
typedef struct {
    float low;
    float high;
    float step;
    int inBin;
    int outBin;
} aa_b200_dm;

/* The strategy of src/aa_ddtr_strategy.cpp:27-428 on the host (no GPU
 * needed).  t_processed is [nranges][max_chunks].  Returns 0, or the
 * strategy's refusal code (<0). */
int aa_b200_strategy(const aa_b200_dm *plan, int nranges, float power, int nchans, int nsamp, double fch1,
                     double foff, double tsamp, int nbits, size_t free_memory, int enable_analysis,
                     int max_chunks, float *dmshifts, int *ndms, aa_b200_dm *str_dm, int *maxshift,
                     int *max_ndms, int *num_tchunks, int *t_processed);
/* The periodicity strategy (include/aa_periodicity_strategy.hpp:178-355)
 * for the DDTR strategy of a plan (ddtr_memory bytes) and memory_available
 * bytes, host only: info[0..6] = FFT length of unbinned ranges, samples
 * copied per row, DM trials of the first batch per unit of binning, input
 * plane size, cuFFT work area, largest MSD block count, ready flag; per
 * range (max_ranges) its FFT length and batch count; per batch
 * (max_batches, ranges in order) range, DM trials, first DM trial, FFT
 * length, samples copied.  Returns the number of batches, or < 0. */
int aa_b200_psr_strategy(const aa_b200_dm *plan, int nranges, int nchans, int nsamp, double tsamp, double fch1,
                         double foff, int nbits, size_t ddtr_memory, size_t memory_available, float sigma_cutoff,
                         int nHarmonics, int harmonic_sum_algorithm, long long *info, long long *range_info,
                         int max_ranges, long long *batches, int max_batches);

/* Kernel choice of src/aa_dedisperse.cpp:8-11,20,48-51,62,88-92,101,133:
 * 0 shared 8-bit, 1 shared 16-bit, 2 shared 4-bit, 3 cache ("failsafe"). */
int aa_b200_select_kernel(int nbits, float dm_step, float tsamp, float dmshift_last, int failsafe);

/* corner_turn_SM_inplace (src/aa_corner_turn.cpp:118-121) fused with the
 * chunk narrowing: d_in_tc [nsamp][nchans] uint16 -> d_out [nchans][out_stride]
 * uint8 (nbits <= 8) or uint16 (nbits 16/32).  Samples above the bit depth's
 * range are reported as an error. */
int aa_b200_corner_turn(const unsigned short *d_in_tc, void *d_out, int nbits, int nchans, long long nsamp,
                        long long out_stride, void *stream);

/* bin_gpu (src/aa_bin_gpu.cpp:8-44) as it acts on the flat buffer: d_dst
 * [0, nchans*nsamp/2) = (a+b)>>1 of [c][nsamp] pairs, [.., nchans*nsamp) = 0.
 * Element type as for aa_b200_corner_turn.  nsamp must be even. */
int aa_b200_bin_gpu(const void *d_src, void *d_dst, int nbits, int nchans, long long nsamp, void *stream);

/* dedisperse() (src/aa_dedisperse.cpp:5) for DM range i: reads d_input
 * [nchans][i_nsamp] (the reference's i_nsamp constant, set by
 * set_dedispersion_constants, src/aa_device_load_data.cu:58-61) and writes
 * d_output [ndms[i]][out_pitch] (the reference uses out_pitch = t_processed).
 * tsamp points at the range's sampling time (tsamp_original * inBin[i]),
 * dmshifts is the host delay table.  d_input_elems is the number of elements
 * the caller allocated at d_input: the staged windows read up to a few KB
 * past the last sample a valid output uses, and a call whose reads would
 * leave the allocation is refused with the padding it needs.  Allocates its
 * own device scratch (delay, window and offset tables) for the call.
 * Returns 0 or 1 like the reference; the device work is complete when it
 * returns. */
int aa_b200_dedisperse(int i, int t_processed, const int *inBin, const float *dmshifts, const void *d_input,
                       long long i_nsamp, size_t d_input_elems, float *d_output, long long out_pitch, int nchans,
                       const float *tsamp, const float *dm_low, const float *dm_step, const int *ndms, int nbits,
                       int failsafe, void *stream);

/* aa_b200_dedisperse without device allocation.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc/cudaFree --
 * code running inside a memory pool or arena that owns the GPU's memory,
 * real-time loops that must not synchronise with the allocator, hosts that
 * reserve all device memory at start-up.  Same arguments, results and return
 * values as aa_b200_dedisperse; the delay, window and offset tables live in
 * one fixed array of AA_B200_NOALLOC_SCRATCH_BYTES in the library's device
 * image, which every GPU that loads the library holds until the process
 * exits.  Limits: nchans <= AA_B200_NOALLOC_MAX_CHANS and
 * nchans * ndms[i] <= AA_B200_NOALLOC_MAX_ENTRIES; larger calls are refused
 * (return 1, message in aa_b200_noalloc_last_error).  It runs the generic
 * one-byte kernel (k_ddtr_u8) or the two-byte gather kernel (k_ddtr_u16), not
 * the faster channel-quad kernel, whose pattern tables would not fit the
 * array.  Each call waits on `stream` (cudaStreamSynchronize) to read the
 * device's error flags back, so it blocks the calling thread until its work
 * is done.  The first call on each device looks up the array's device
 * address (cudaGetSymbolAddress), so make that first call before any stream
 * capture.  All calls share the array: calls that overlap on the GPU (other
 * threads, other streams) race and must be serialised by the caller.  Each
 * call clears what must start at zero. */
#define AA_B200_NOALLOC_SCRATCH_BYTES (16u << 20)
#define AA_B200_NOALLOC_MAX_CHANS 16384
#define AA_B200_NOALLOC_MAX_ENTRIES (1u << 20)
int aa_b200_dedisperse_noalloc(int i, int t_processed, const int *inBin, const float *dmshifts, const void *d_input,
                               long long i_nsamp, size_t d_input_elems, float *d_output, long long out_pitch,
                               int nchans, const float *tsamp, const float *dm_low, const float *dm_step,
                               const int *ndms, int nbits, int failsafe, void *stream);
/* Message of the last refusal or failure of aa_b200_dedisperse_noalloc in
 * this thread ("" if the last call succeeded). */
const char *aa_b200_noalloc_last_error(void);

/* ---------------------------------------------------------------------------
 * The reference's dedispersion seam with its own argument lists (C twins of
 * the C++ functions of namespace astroaccelerate declared in
 * aa_b200_seam.hpp, which link unchanged against code written for the
 * reference's runner).  Reference buffers: one unsigned short per sample,
 * [t][c] as loaded, [c][t] after the corner turn; float rows out.  All on
 * the legacy default stream.
 * ------------------------------------------------------------------------- */
/* load_chunk_data (src/aa_device_load_data.cu:39-56): H2D of
 * (t_processed + maxshift) * nchans samples, the delay table to d_dm_shifts
 * where the reference does that, and set_dedispersion_constants. */
void aa_b200_seam_load_chunk_data(unsigned short *device_pointer, const unsigned short *host_pointer, int t_processed,
                                  int maxshift, int nchans, float *dmshifts, float *d_dm_shifts, int nbits);
/* set_dedispersion_constants (src/aa_device_load_data.cu:58-61): row length
 * t_processed + maxshift and t_processed for the next aa_b200_seam_dedisperse
 * of this thread (per thread; the reference's are process-wide constants). */
void aa_b200_seam_set_dedispersion_constants(int t_processed, int maxshift);
/* corner_turn_SM_inplace (src/aa_corner_turn.cpp:118-121): [secondary][primary]
 * to [primary][secondary] in place, through d_temporary. */
void aa_b200_seam_corner_turn_SM_inplace(unsigned short *d_input, unsigned short *d_temporary, size_t primary_size,
                                         size_t secondary_size);
/* bin_gpu (src/aa_bin_gpu.cpp:8-44): the x2 binning of the flat buffer in
 * place, d_output as scratch. */
void aa_b200_seam_bin_gpu(unsigned short *d_input, float *d_output, int nchans, int nsamp);
/* dedisperse (src/aa_dedisperse.cpp:5-163): DM range i of d_input
 * [nchans][row length of set_dedispersion_constants] into d_output
 * [ndms[i]][t_processed].  Tables per range are built on the first call and
 * kept per thread; the rows are staged into a padded buffer of the library.
 * Returns 0, or 1 with the reason in aa_b200_last_error(); the device work
 * is complete when it returns. */
int aa_b200_seam_dedisperse(int i, int t_processed, int *inBin, float *dmshifts, unsigned short *d_input,
                            float *d_output, float *d_dm_shifts, int nchans, float *tsamp, float *dm_low,
                            float *dm_step, const int *ndms, int nbits, int failsafe);
/* save_data_offset_stream (src/aa_device_save_data.cu:19-62): the chunk's DM
 * rows of range dm_range to output_buffer[dm_range][dm] + inc/inBin. */
void aa_b200_seam_save_data_offset_stream(int dm_range, int current_time_chunk, int **t_processed, long inc,
                                          int *inBin, const int *ndms, float *d_DDTR_output, float ***output_buffer);

/* Message of the last failure of this thread ("" if none). */
const char *aa_b200_last_error(void);
/* Kernels this library has launched in this process. */
long long aa_b200_kernel_launches(void);
/* Library build identification. */
const char *aa_b200_version(void);

/* ---------------------------------------------------------------------------
 * Failure handling checks (no reference counterpart; they fault nothing).
 * ------------------------------------------------------------------------- */
/* Runs a kernel whose bounded mbarrier wait is made to run out (an expected
 * arrival never comes) after `limit` polls (1..2^22); *status receives the
 * device error flags (8 = the wait ran out, as the staged kernels report an
 * overdue copy).  Returns 0 when the kernel ran and the flags were read. */
int aa_b200_selftest_bounded_wait(int limit, int *status);
/* The compute capability the library's device code was compiled for, as the
 * CUDA runtime reports it for one of its kernels (major*10 + minor; 100 for
 * the sm_100a build).  Needs a GPU.  Returns 0 on success. */
int aa_b200_binary_version(int *version);
/* Host-side failure injection: the n-th CUDA result checked by any pipeline
 * or batch engine after this call reads as a failure ("injected failure" in
 * the error message); n <= 0 disarms.  For tests of the error paths. */
void aa_b200_debug_fail_after(long long n);
long long aa_b200_debug_fail_countdown(void);

/* ---------------------------------------------------------------------------
 * Measured roof (no reference counterpart): 32-bit shared-memory loads per
 * second over the whole GPU, from conflict-free warp-wide loads (two
 * 1024-thread CTAs per SM, iters x 16 loads per thread), timed with CUDA
 * events on `stream` (a cudaStream_t, NULL = legacy default stream).  The
 * channel-quad dedispersion kernel adds four channel samples per such load,
 * so 4 x *loads_per_s is its shared-memory bound in adds/s.  Returns 0 on
 * success; *ms_out (may be NULL) receives the timed kernel's duration.
 * ------------------------------------------------------------------------- */
int aa_b200_smem_load_rate(int iters, void *stream, double *loads_per_s, float *ms_out);

/* ---------------------------------------------------------------------------
 * SIGPROC filterbank input (src/aa_py_sigproc_input.cpp:7-33, reader
 * src/aa_sigproc_input.cpp:85-543): the reference's header keyword rules,
 * sample count from the file size and unpacking into one unsigned short per
 * sample ([t][c]; 4-bit high nibble first, 2-bit most significant pair first,
 * 1-bit least significant bit first; 32-bit rescaled by the file's min/max).
 * Files whose channels do not fill whole bytes, or with nifs != 1, are
 * refused (read_metadata returns nbits = 0; the reason is in
 * aa_b200_sigproc_last_error).
 * ------------------------------------------------------------------------- */
void *aa_py_sigproc_input(const char *path);
void aa_py_sigproc_input_del(const void *obj);
aa_py_filterbank_metadata_struct aa_py_sigproc_input_read_metadata(void *obj);
/* true once, after the samples were read and unpacked */
bool aa_py_sigproc_input_read_signal(void *obj);
/* [nsamples][nchans] unsigned short owned by obj; null before read_signal */
const unsigned short *aa_py_sigproc_input_input_buffer(const void *obj);

/* Extensions (no reference counterpart): the data section as stored, for
 * aa_b200_pipeline_set_packed_input; for 32-bit files the 16-bit rescaled
 * samples of read_signal.  True once, after a successful read. */
bool aa_b200_sigproc_read_packed(void *obj);
const void *aa_b200_sigproc_packed_buffer(const void *obj);
long long aa_b200_sigproc_packed_bytes(const void *obj);
typedef struct {
    int telescope_id, machine_id, data_type, barycentric, pulsarcentric;
    double az_start, za_start, src_raj, src_dej, tstart, tsamp;
    int nbits, nsamples_keyword, nchans, nifs;
    double fch1, foff, fchannel, refdm, period;
    long long data_start, data_bytes, nsamp; /* byte offset and size of the data; samples per channel */
} aa_b200_sigproc_header_struct;
/* every header value read (false before a successful read_metadata) */
bool aa_b200_sigproc_header(const void *obj, aa_b200_sigproc_header_struct *out);
const char *aa_b200_sigproc_last_error(const void *obj);

/* Pipeline extensions (obj from aa_py_pipeline_api or aa_b200_pipeline_create). */
/* Options, before bind: stride_mode 0 = the reference runner's binning length
 * (bit-exact with the reference), 1 = true row stride; fma_mode bit mask of
 * fused delay expressions (7 = all, the reference's --fmad=true build);
 * free_memory 0 = query the device; tile_words/group_dms 0 = autotune. */
bool aa_b200_pipeline_set_options(void *obj, int stride_mode, int fma_mode, int failsafe, size_t free_memory,
                                  int tile_words, int group_dms);
/* Dedispersion kernels, before bind: 0 chooses per range (for one-byte data
 * the faster, timed at setup, of the channel-quad and subband kernels where
 * they fit, else the byte-phase kernel; for two-byte data the staged fp32
 * kernel where it fits), 1 the generic kernels
 * (byte-phase for one-byte data, a global-memory gather for two-byte data),
 * 2 the channel-quad kernel for one-byte data, 3 the subband kernel for
 * one-byte data, 4 the warp-specialised channel-quad kernel for one-byte data
 * (never chosen by 0: its four row-building warps cannot keep up with the
 * sixteen summing warps) (2, 3 and 4 run the staged fp32 kernel on two-byte
 * data; refused where they do not fit).  All give identical results. */
/* Before bind: the pipeline reads `packed` (host memory, or device memory
 * for a pipeline created with device_input) instead of the unsigned-short
 * input: the SIGPROC data section as stored, [nsamples][nchans*nbits/8]
 * bytes for nbits 1, 2, 4, 8, [nsamples][nchans] uint16 for nbits 16, and for
 * nbits 32 the 16-bit rescaled samples (aa_b200_sigproc_read_packed).  Each
 * chunk crosses PCIe at nbits/16 of the unsigned-short size (1/2 for 8-bit)
 * and is unpacked on the GPU in the corner-turn kernel; outputs are
 * identical to the unsigned-short input of the same samples. */
bool aa_b200_pipeline_set_packed_input(void *obj, const void *packed);
/* Before bind: the kernel family per range.  0 chooses per range (the
 * autotuner times the candidates), 1 the generic kernels, 2 the channel-quad
 * kernel (one-byte data) / staged fp32 kernel (two-byte data), 3 the subband
 * kernel / fp32, 4 the warp-specialised channel-quad kernel / fp32, 5 the
 * split-phase channel-quad kernel / fp32, 6 the channel-quad kernel with its
 * register reuse chosen per warp by the pattern of equal offsets / fp32, 7
 * the channel-quad kernel on 256-sample tiles, two CTAs per SM / fp32.  A
 * forced family that cannot run a range makes the bind fail with the reason. */
bool aa_b200_pipeline_set_kernel_variant(void *obj, int variant);
/* Before bind: whether the set-up times the staged kernels' stage depth (and,
 * for variant 0, the candidate kernels) per range on a slice of the first
 * chunk (default 1).  0 keeps the largest stage that fits shared memory. */
bool aa_b200_pipeline_set_autotune(void *obj, int enable);
/* output_dmt (pipeline_component_option_struct): when the run finishes, the
 * DM-time output of every range is written in the reference's
 * Export_DD_data files (include/aa_pipeline_runner.hpp:165-216), DM rows per
 * file for 1000 MB files as include/aa_permitted_pipelines_1.hpp:312-323
 * computes them; needs copy_ddtr_data_to_host.  Base name "DD_data" in the
 * working directory, or this one: */
bool aa_b200_pipeline_set_export_base(void *obj, const char *base);
/* Analysis output: write_files != 0 writes the reference's candidate files
 * (the default) under dir (NULL or "" = the working directory, as the
 * reference). */
bool aa_b200_pipeline_set_candidate_output(void *obj, int write_files, const char *dir);
/* The analysis batch in elements (the reference's maxtimesamples); 0 (the
 * default) takes the reference's rule, 95% of the free device memory at 26
 * bytes per element, capped at the largest step's rows.  Set before the
 * first step. */
bool aa_b200_pipeline_set_analysis_batch(void *obj, long long max_time_samples);
/* include/aa_pipeline_runner.hpp:165-216 Export_DD_data: per range r with
 * ranges_to_export[r] != 0, <base>_<r>.txt (nTimesamples, nDMs,
 * DMs_per_file, number of files; one per line) and <base>_<r>_<i>.dat
 * (float32 [DMs][nTimesamples]), nTimesamples = max_nTimesamples/inBin[r];
 * DMs_per_file < 0: all of a range's DM trials in one file (the first
 * exported range's count, kept for later ranges as there).  Every row must
 * hold nTimesamples values.  0 on success, 1 on error (aa_b200_last_error). */
int aa_b200_export_dd_data(int range, float ***dedispersed_data, size_t max_nTimesamples, const int *ndms,
                           const int *inBin, const char *base_filename, const int *ranges_to_export, int DMs_per_file);
/* include/aa_pipeline_runner.hpp:219-223 Calculate_sd_per_file_from_file_size */
size_t aa_b200_sd_per_file_from_file_size(size_t size_in_MB, size_t primary_dimension, size_t floats_per_element);
/* A pipeline whose input (and optionally output) stay in device memory:
 * input [nsamples][nchans] uint16 on the device when device_input != 0;
 * device_output != 0 keeps [range][dm][t] on the device
 * (aa_b200_pipeline_device_output). */
void *aa_b200_pipeline_create(aa_py_filterbank_metadata_struct metadata, const unsigned short *input,
                              int device_input, int device_output, int copy_to_host, void *stream,
                              int card_number);
bool aa_b200_pipeline_run_all(void *obj);
/* The pipeline's set-up (device buffers, delay and pattern tables, the
 * autotuner) now instead of at the first run, so that it can happen before
 * the data arrives.  Idempotent; needs a bound DDTR plan. */
bool aa_b200_pipeline_setup(void *obj);
bool aa_b200_pipeline_rewind(void *obj);
bool aa_b200_pipeline_synchronize(void *obj);
float *aa_b200_pipeline_device_output(void *obj, int range);
/* kind (| 0x100 when the range runs the channel-quad kernel, | 0x200 for the
 * staged fp32 kernel, | 0x400 for the two-byte gather kernel, | 0x800 for the
 * subband kernel, | 0x1000 for the warp-specialised channel-quad kernel), DMs
 * per thread block, window span (samples), time words per lane */
int aa_b200_pipeline_range_info(void *obj, int range, int *kind, int *group_dms, int *span, int *tile_words);
/* channel quads (channel-quad kernel) or channels (fp32 kernel) per
 * shared-memory stage of a range, as the autotuner chose it; 0 for the
 * generic kernels */
int aa_b200_pipeline_stage_depth(void *obj, int range);
/* The autotuner's choices (kernel, tile shape, stage depth, flavour) are
 * kept for the life of the process, one entry per distinct range shape (the
 * device, channel delays, DM range, chunk length, row pitch and kernel
 * options): a later pipeline of the same shape takes them without timing
 * again.  No choice changes the output.  clear != 0 drops every entry first.
 * Returns the entries held; host only. */
long long aa_b200_tuned_ranges(int clear);
/* The kept choices written to a text file, and read back into this process
 * (added to the entries held): a tuning run's choices reused by later
 * processes on the same device.  Return the entries written or read, or -1
 * (message in aa_b200_tuned_ranges_last_error).  Host only. */
long long aa_b200_tuned_ranges_save(const char *path);
long long aa_b200_tuned_ranges_load(const char *path);
const char *aa_b200_tuned_ranges_last_error(void);
/* Ranges set up from a kept choice in this process, without timing.  A kept
 * choice that does not fit the range (a file from another build, an edited
 * file) is not taken: the range is timed again.  Host only. */
long long aa_b200_tuned_ranges_used(void);
/* The kernel shape a range runs (after set-up, which includes the
 * autotuner): the channel-quad flavour (-1 for other kernels; 0 with the
 * per-byte path, 1 with its warp switch, 4 loading every DM trial's word
 * before the sums, 6 the same without a per-byte path, 7 as 6 with 32-bit
 * shared addresses, 2 the 16-warp form of the 256-sample tile), the DM trials
 * and samples of one CTA's output tile and the DM trials one warp sums.
 * Returns 0, or 1 for an unknown range. */
int aa_b200_pipeline_range_kernel(void *obj, int range, int *flavour, int *tile_dms, int *tile_samples,
                                  int *dms_per_warp);
long long aa_b200_pipeline_kernel_launches(void *obj);
const char *aa_b200_pipeline_last_error(void *obj);
int aa_b200_pipeline_num_tchunks(void *obj);
int aa_b200_pipeline_maxshift(void *obj);
/* CUDA-event timing of every kernel launch (off by default).  family:
 * 0 dedispersion, 1 corner turn, 2 binning.  Times are collected when the
 * pipeline synchronises; reset clears them. */
bool aa_b200_pipeline_time_kernels(void *obj, int on);
int aa_b200_pipeline_kernel_time(void *obj, int family, double *ms, long long *count);
bool aa_b200_pipeline_reset_kernel_times(void *obj);

/* ---------------------------------------------------------------------------
 * Multi-beam dedispersion (no counterpart in the reference, which runs one
 * beam per aa_pipeline_api and one kernel launch per (chunk, range)).
 *
 * Beams of different channel counts, bit depths, lengths and DM plans are
 * added with their [nsamples][nchans] uint16 input already on the device;
 * setup computes each beam's strategy (as aa_ddtr_strategy would with
 * free_memory bytes free; 0 = the device's free memory at setup), its delay
 * tables and device outputs, gives every (beam, chunk, binning level) its own
 * filterbank buffer, and records the whole job as one CUDA graph: corner
 * turns and binning of all beams on parallel streams, then one persistent
 * dedispersion kernel over all (beam, chunk, range, DM group, time tile) work
 * items (persistent = 0: one launch per (beam, chunk, range) instead).
 * autotune != 0 times the shared-memory stage depth per range shape at setup,
 * and, for one-byte ranges that both kernels can run, the subband body
 * against the channel-quad body; the subband jobs run in a second
 * persistent launch right after the first.
 * Each beam's output [range][dm][t] is bit-identical to a plain pipeline's
 * (aa_b200_pipeline_create with device_output) for the same free_memory.
 * run is asynchronous on `stream` (a cudaStream_t as void*, 0 = a stream of
 * the batch's own); synchronize waits and checks every beam's device flags.
 * --------------------------------------------------------------------------- */
void *aa_b200_batch_create(int stride_mode, int fma_mode, size_t free_memory, int persistent, int use_graph,
                           int autotune, void *stream);
/* returns the beam index, or -1 (message in aa_b200_batch_last_error) */
int aa_b200_batch_add_beam(void *batch, aa_py_filterbank_metadata_struct metadata, void *ddtr_plan,
                           const unsigned short *d_input);
/* Before setup: which body runs the one-byte ranges that both can run:
 * 0 the faster on a timed slice (with autotune; else channel-quad), 1 the
 * channel-quad body, 2 the subband body.  Returns false for another value
 * or after setup. */
bool aa_b200_batch_set_kernel_choice(void *batch, int choice);
/* After setup: persistent jobs run by the subband body. */
int aa_b200_batch_sub_jobs(void *batch);
bool aa_b200_batch_setup(void *batch);
bool aa_b200_batch_run(void *batch);
bool aa_b200_batch_synchronize(void *batch);
/* [ndms][total_samps] float rows of one range of one beam (device memory) */
float *aa_b200_batch_device_output(void *batch, int beam, int range);
int aa_b200_batch_range_shape(void *batch, int beam, int range, int *ndms, long long *total_samps, int *inBin);
int aa_b200_batch_info(void *batch, long long *work_items, int *persistent_jobs, int *other_jobs, int *grid,
                       size_t *smem_bytes, size_t *level_bytes, long long *launches_per_run);
/* device time (ms) of the last run: which = 0 whole run, 1 dedispersion part
 * (measured only when the batch runs without a graph; -1 otherwise) */
double aa_b200_batch_last_ms(void *batch, int which);
/* device bytes a beam needs inside a batch (outputs, tables, filterbank
 * levels), to split a beam list into batches that fit */
int aa_b200_batch_estimate_bytes(aa_py_filterbank_metadata_struct metadata, void *ddtr_plan, size_t free_memory,
                                 size_t *bytes);
const char *aa_b200_batch_last_error(void *batch);
void aa_b200_batch_delete(void *batch);

/* ---------------------------------------------------------------------------
 * Differentiable candidate refinement (no counterpart in the reference, whose
 * dedispersion uses integer delays only).  Device pointers; return 0 or 1
 * (message in aa_b200_frac_last_error).
 *
 * Fractional-delay dedispersion of nsnip snippets x[nsnip][nchans][nsamp]
 * (float32) at a continuous DM per snippet dm[nsnip] (float32) into FP64
 * series y[nsnip][nsamp]: with
 * tau_c = dm * kc[c] (kc: FP64 delay in samples per unit DM),
 * n = floor(tau_c) - base[s][c], w = tau_c - floor(tau_c) (FP64; d_base, an
 * int array [nsnip][nchans] of row shifts for snippets cut per channel, may
 * be null),
 *   y[s][t] = sum_c x[s][c][t+n] + w (x[s][c][t+n+1] - x[s][c][t+n]),
 * samples outside [0, nsamp) read as 0.  The adjoint recomputes the delays and
 * writes, from gy = dL/dy (FP64), gx = dL/dx (float32, skipped when d_gx is
 * null) and gdm = dL/ddm (float32, skipped
 * when d_gdm is null; needs d_partial, nsnip*nchans doubles of scratch the
 * caller provides).
 * --------------------------------------------------------------------------- */
int aa_b200_frac_dedisperse_fwd(const float *d_x, const float *d_dm, const double *d_kc, const int *d_base, int nsnip,
                                int nchans, int nsamp, double *d_y, void *stream);
int aa_b200_frac_dedisperse_adj(const float *d_x, const float *d_dm, const double *d_kc, const int *d_base,
                                const double *d_gy, int nsnip, int nchans, int nsamp, float *d_gx, float *d_gdm,
                                double *d_partial, void *stream);
/* Boxcar S/N (FP64 in and out): snr[s][i][t] = (sum_{k<w_i} y'[s][t+k] - w_i mu[s]) /
 * (sigma[s] sqrt(w_i)), y' = y inside [0, nsamp) and mu beyond; widths (host
 * array) ascending in 1..1024, at most 16.  mu and sigma are constants of the
 * adjoint, which writes gy = dL/dy from gsnr. */
int aa_b200_boxcar_snr_fwd(const double *d_y, int nsnip, int nsamp, const int *widths, int nwidths, const float *d_mu,
                           const float *d_sigma, double *d_snr, void *stream);
int aa_b200_boxcar_snr_adj(const double *d_gsnr, int nsnip, int nsamp, const int *widths, int nwidths,
                           const float *d_sigma, double *d_gy, void *stream);
const char *aa_b200_frac_last_error(void);

/* Single-pulse search on a DM-time range (rows of nsamp floats, row pitch in
 * floats), a reduced form of the reference's analysis step
 * (src/aa_device_analysis.cu:130-510): row mean and standard deviation (FP64
 * sums), then per (row, block of aa_b200_sps_block_samples() samples) the
 * largest white-noise boxcar S/N (sum_{k<w} y[t+k] - w mean) / (std sqrt w)
 * over the block's start samples t and the widths (ascending, 1..1024, at
 * most 16), with its t and w.  Peak arrays hold nrows * nblocks entries. */
int aa_b200_sps_row_stats(const float *d_y, int nrows, long long pitch, long long nsamp, float *d_mean,
                          float *d_stdev, void *stream);
int aa_b200_sps_block_peaks(const float *d_y, int nrows, long long pitch, long long nsamp, const float *d_mean,
                            const float *d_stdev, const int *widths, int nwidths, float *d_peak_snr, int *d_peak_t,
                            int *d_peak_w, void *stream);
int aa_b200_sps_block_samples(void);

/* ---------------------------------------------------------------------------
 * Single-pulse detection with the reference's own rules: analysis_GPU
 * (src/aa_device_analysis.cu:130-345) on one DM-time plane [nDMs][nT] of
 * float32 in device memory, for candidate algorithms 0 (peak finding), 1
 * (thresholding) and 2 (peak filtering).  The MSD profile (src/aa_device_MSD_plane_profile.cu), the
 * boxcar S/N planes (src/aa_device_SPS_long.cu:32-80) and the candidate
 * lists are bit-identical to the reference's; the order of the candidates
 * inside one batch follows the GPU's atomics, as in the reference.
 *
 * create: buffers for planes of up to max_elems elements; the search takes
 * the DM trials in batches of floor(max_time_samples / nT), rounded down to
 * a multiple of 4 (the reference's maxTimeSamples of
 * include/aa_analysis_strategy.hpp:209-258; 0 = the whole plane).  The work
 * area starts zeroed; samples the reference's kernels read without writing
 * them first come from it.  clear zeroes it again.
 * run: tsamp is the range's sampling time (the data's tsamp times inBin, as
 * float), the settings those of aa_analysis_plan
 * (include/aa_analysis_plan.hpp:36-47).  The plane is overwritten (the
 * reference's search decimates into it).  Candidates -- DM trial index,
 * sample, S/N, boxcar width in samples of the range -- go to the host arrays
 * of max_candidates entries; a batch whose candidates would reach
 * max_candidates is dropped whole, as in the reference
 * (src/aa_device_analysis.cu:319-354).  Returns 0, or 1 with a message in
 * aa_b200_spd_last_error.  stream: cudaStream_t as void*, 0 = the legacy
 * stream; run returns after the candidates are on the host.
 * --------------------------------------------------------------------------- */
void *aa_b200_spd_create(long long max_elems, long long max_time_samples);
void aa_b200_spd_destroy(void *obj);
/* obj == NULL: the message of the last failed create or write */
const char *aa_b200_spd_last_error(const void *obj);
int aa_b200_spd_clear(void *obj, void *stream);
int aa_b200_spd_run(void *obj, float *d_plane, int nDMs, int nTimesamples, float tsamp, int inBin,
                    float sigma_cutoff, float sigma_constant, float max_boxcar_width_in_sec, int candidate_algorithm,
                    int enable_msd_baseline_noise, void *stream, size_t max_candidates, unsigned *h_dm,
                    unsigned *h_ts, float *h_snr, unsigned *h_bw, size_t *n_candidates);
/* The plan and the interpolated (mean, deviation) per boxcar width of the
 * last run: widths[msd_cap], msd[2 * msd_cap]; dropped_batches counts the
 * batches dropped for max_candidates. */
int aa_b200_spd_profile(const void *obj, float *msd, int msd_cap, int *widths, int *nwidths,
                        int *max_width_performed, int *max_iteration, int *dropped_batches);
/* on != 0: run keeps the S/N and width planes of its last batch (2 * batch
 * elements each, the reference's d_output_SNR and d_output_taps), which
 * aa_b200_spd_planes copies out when cap is large enough; returns their
 * length. */
int aa_b200_spd_keep_planes(void *obj, int on);
long long aa_b200_spd_planes(const void *obj, float *snr, unsigned short *taps, long long cap);
long long aa_b200_spd_kernel_launches(void);
/* The MSD plane profile alone (MSD_plane_profile of
 * src/aa_device_MSD_plane_profile.cu:564-604) on a device plane
 * [nDMs][nTimesamples] (not modified) for ascending widths[nwidths]:
 * h_msd[2 * nwidths] = (mean, deviation) per width.  high_memory != 0 takes
 * the width-2 decimation in one piece, as the periodicity search does
 * (src/aa_device_periods.cu:469, widths 1..nHarmonics); 0 splits it in two
 * halves of the DM trials, as the analysis does.  Uses obj's work area. */
int aa_b200_spd_msd_profile(void *obj, const float *d_input, int nDMs, int nTimesamples, const int *widths,
                            int nwidths, int high_memory, float sigma_constant, int outlier_rejection, float *h_msd,
                            void *stream);
/* The first boxcar S/N plane alone (call_kernel_SPDT_GPU_1st_plane of
 * src/aa_device_SPS_long_kernel.cu, as tests/test_single_pulse_search_scan_1.cpp
 * drives it): device input [nDMs][nTimesamples], outputs boxcar values and
 * decimated sums [nDMs][dtm] (dtm = nTimesamples/2 rounded down to even), S/N
 * and widths [nDMs][nTimesamples]; h_msd: host (mean, deviation) for widths
 * 1..nBoxcars (8, 16 or 32).  Asynchronous on stream. */
int aa_b200_spd_first_plane(const float *d_input, float *d_boxcar_values, float *d_decimated, float *d_snr,
                            unsigned short *d_taps, const float *h_msd, int nTimesamples, int nBoxcars, int nDMs,
                            void *stream);
/* on != 0: CUDA events around every launch of the following runs; family_time
 * gives the last run's device time (ms) and launches of a family: 0 MSD
 * statistics, 1 decimations and boxcars of the MSD profile, 2 the first
 * boxcar S/N plane, 3 the later S/N planes, 4 candidate selection. */
int aa_b200_spd_time_kernels(void *obj, int on);
int aa_b200_spd_family_time(const void *obj, int family, double *ms, long long *launches);
/* The plan analysis_GPU builds (src/aa_device_analysis.cu:24-121, :138-179)
 * for rows of nTimesamples at the range's tsamp (no GPU needed): the boxcar
 * widths (widths_cap), the widest width performed, the iterations run, and
 * per iteration (plan_cap) the ten fields of PulseDetection_plan
 * (include/aa_device_BC_plan.hpp:12-23) in the order decimated_timesamples,
 * dtm, iteration, nBoxcars, nBlocks, output_shift, shift, startTaps,
 * unprocessed_samples, total_ut. */
int aa_b200_spd_plan(int nTimesamples, float tsamp, int inBin, float max_boxcar_width_in_sec, int *widths,
                     int widths_cap, int *nwidths, int *max_width_performed, int *max_iteration, int *plan,
                     int plan_cap, int *nplan);
/* The candidate file of src/aa_device_analysis.cu:420-466 (float records
 * DM, time, S/N, width) under dir; returns 0 or 1. */
int aa_b200_spd_write_candidates(const char *dir, int candidate_algorithm, float tstart, float dm_low, float dm_high,
                                 float dm_step, float tsamp, int inBin, const unsigned *dm, const unsigned *ts,
                                 const float *snr, const unsigned *bw, size_t n);

/* ---------------------------------------------------------------------------
 * Periodicity building blocks: the stages of the reference's periodicity
 * search (src/aa_device_periods.cu:368-541) one at a time, each
 * bit-identical to the reference's kernel where the reference is
 * deterministic; the pipeline's periodicity component
 * (aa_py_pipeline_api_bind_periodicity_plan) runs them in the reference's
 * order.  Device pointers; return 0 or 1 (message in aa_b200_psr_last_error).
 *
 * power_interbin (src/aa_device_power.cu:34-52): d_spectra holds nDMs
 * spectra of nTimesamples/2+1 complex float bins (cufftExecR2C output);
 * power [nDMs][nTimesamples/2] and interbin [nDMs][nTimesamples] spectra
 * normalised by sqrt(nTimesamples).
 * harmonic_sum_simple (src/aa_device_harmonic_summing.cu:11-37): input
 * [nBins][nSpectra]; per bin and spectrum the best S/N of harmonic sums up to
 * nHarmonics (d_msd: device (mean, deviation) per harmonic count) and the
 * number of added harmonics.
 * --------------------------------------------------------------------------- */
int aa_b200_psr_power_interbin(const void *d_spectra, float *d_power, float *d_interbin, int nTimesamples, int nDMs,
                               void *stream);
int aa_b200_psr_harmonic_sum_simple(const float *d_input, float *d_snr, unsigned short *d_harmonics,
                                    const float *d_msd, int nBins, int nSpectra, int nHarmonics, void *stream);
/* Peak finding for the periodicity search (Peak_find_for_periodicity_search,
 * src/aa_device_peak_find.cu:53-131): values above threshold that are the
 * maximum of their clipped 3 x 3 neighbourhood, on a transposed
 * [nTimesamples][nDMs] or normal [nDMs][nTimesamples] S/N plane with its
 * harmonic counts; records (DM trial + dm_shift, bin / in_bin, power =
 * S/N * sd_h + mean_h, harmonic count) appended at *d_count (at most
 * max_peaks); greedy (normal planes) drops the hundreds of the harmonic count
 * for the power.  Planes of at least 2 x 2. */
int aa_b200_psr_peak_find(const float *d_snr, const unsigned short *d_harmonics, float *d_list, int nTimesamples,
                          int nDMs, float threshold, int max_peaks, int *d_count, const float *d_msd, int dm_shift,
                          int in_bin, int transposed, int greedy, void *stream);
/* Thresholding for the periodicity search (Threshold_for_periodicity_transposed
 * and _normal, src/aa_device_threshold.cu:56-163): every value above
 * threshold, recorded as aa_b200_psr_peak_find records peaks. */
int aa_b200_psr_threshold(const float *d_snr, const unsigned short *d_harmonics, float *d_list, int nTimesamples,
                          int nDMs, float threshold, int max_peaks, int *d_count, const float *d_msd, int dm_shift,
                          int in_bin, int transposed, int greedy, void *stream);
/* The other harmonic sums of the periodicity search on a normal plane
 * [nDMs][nTimesamples] (src/aa_device_harmonic_summing.cu:38-169): algorithm
 * 1 greedy (counts carry 100 x the bin offsets taken), 2 PRESTO plus, 3
 * PRESTO (sums of 1, 2, 4, ... harmonics, floor(log2 nHarmonics) + 1 of
 * them); nHarmonics 1..32; scalloping != 0 corrects each bin for the
 * scalloping loss.  d_msd: (mean, deviation) per harmonic count. */
int aa_b200_psr_harmonic_sum(int algorithm, const float *d_input, float *d_snr, unsigned short *d_harmonics,
                             const float *d_msd, int nTimesamples, int nDMs, int nHarmonics, int scalloping,
                             void *stream);
/* Spectral whitening of the periodicity search (spectrum_whitening_SGP2
 * with enable_median, src/aa_device_spectral_whitening.cu:60-118), in place
 * on nDMs spectra of nSamples complex float bins (nSamples >= 8): segment
 * medians of the power, a linear interpolation of median / ln 2 between
 * segment middles, every bin divided by its square root; bin 0 set to
 * (1, 0). */
int aa_b200_psr_whitening(void *d_spectra, size_t nSamples, int nDMs, void *stream);
/* The segment boundaries of the whitening
 * (create_dered_segment_sizes_prefix_sum, src/aa_device_spectral_whitening.cu:17-31,
 * lengths 6 .. 250): writes up to cap of them, returns their count. */
int aa_b200_psr_segment_sizes(size_t nSamples, int *out, int cap);
/* The whitening's segment medians alone (GPU_kernel_segmented_median,
 * src/aa_device_spectral_whitening_kernel.cu:338-376) over a caller's
 * boundary table segments[0..nSegments-1] (host memory; increasing, each
 * segment 1 to 256 bins, the last boundary at most nSamples): writes
 * d_medians[dm * nSegments + s] for s < nSegments - 1.  Synchronises the
 * stream; for checking median selection on segment lengths the whitening's
 * own table does not produce. */
int aa_b200_psr_segment_medians(const void *d_spectra, size_t nSamples, int nDMs, const int *segments,
                                int nSegments, float *d_medians, void *stream);
long long aa_b200_psr_kernel_launches(void);
const char *aa_b200_psr_last_error(void);

/* ---------------------------------------------------------------------------
 * Periodicity candidate lists (aa_periodicity_candidates,
 * include/aa_periodicity_candidates.hpp:14-202), host side.  Records of 4
 * floats (DM trial, bin, power, harmonic count) as the periodicity peak
 * finding writes them become (DM = trial * dm_step + dm_low, frequency =
 * bin / (sampling_time * nTimesamples * mod), S/N = (power - msd[2h]) /
 * msd[2h+1], h); with greedy the hundreds of the harmonic count are a bin
 * offset that adds offset / h bin widths to the frequency.  mod is 1 for
 * power lists and 2 for interbin lists (src/aa_device_periods.cu:655-660).
 * --------------------------------------------------------------------------- */
/* In place on host records */
int aa_b200_psr_candidates_process(float *records, size_t n, const float *msd, double dm_low, double dm_step,
                                   double sampling_time, size_t nTimesamples, float mod, int greedy);
void *aa_b200_psr_candidates_create(void);
void aa_b200_psr_candidates_destroy(void *list);
/* Add_Candidates: copies n records (from device memory when on_device) and
 * converts them; lists keep the order they were added in. */
int aa_b200_psr_candidates_add(void *list, const float *records, size_t n, int on_device, int range_id,
                               const float *msd, double dm_low, double dm_step, double sampling_time,
                               size_t nTimesamples, float mod, int greedy);
size_t aa_b200_psr_candidates_count(const void *list);
/* Copy_candidates: every record, list after list, into out (4 * count floats) */
int aa_b200_psr_candidates_copy(const void *list, float *out);
/* Export_candidates_to_file: the same records as raw floats */
int aa_b200_psr_candidates_export(const void *list, const char *filename);
const char *aa_b200_psr_candidates_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* AA_B200_H */
