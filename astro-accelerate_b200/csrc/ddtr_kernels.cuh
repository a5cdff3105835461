// ddtr_kernels.cuh -- launchers of the sm_100a DDTR kernels (ddtr_kernels.cu).
//
// Device data layout (row-major and flat, like the reference's device buffers,
// so that the reference runner's flat-buffer behaviour replays exactly):
//   raw chunk    : [t][c]  uint16  (host format, one value per sample)
//   filterbank   : [c][stride] uint8 (nbits <= 8) or uint16 (nbits 16/32)
//   delay table  : [c][ndms] int32 = smallest delay | (class mask << 24)
//   window table : [group][c4] int32 = smallest delay of the DM group
//   offset table : [c][ndms] int32 = word offset in the staged window or -1
//   output       : [dm][pitch] float32
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace aab200 {

// Delay semantics of the reference kernel a range is dispatched to
// (src/aa_dedisperse.cpp:5-163).
enum DelayKind : int {
    KIND_SHARED8 = 0,  // shared_dedisperse_kernel: findex = 2tx+1, classes (t%16)/2
    KIND_SHARED16 = 1, // shared_dedisperse_kernel_16: findex = 2tx, classes (t%16)/2
    KIND_SHARED4 = 2,  // shared_dedisperse_kernel_4bit: findex = 4tx+3, classes (t%32)/4
    KIND_CACHE = 3     // cache_dedisperse_kernel: one delay per (c, dm)
};

enum FmaBits : int { FMA_TWO = 1, FMA_ONE = 2, FMA_CACHE = 4, FMA_ALL = 7 };

// Device error flags (bitwise OR into one int).
enum DevErr : int {
    DERR_DELAY_RANGE = 1, // a delay outside [0, 2^24) or a class step > 1
    DERR_INPUT_RANGE = 2, // a sample above the bit depth's range
    DERR_WINDOW = 4,      // a delay outside the staged window
    DERR_TIMEOUT = 8,     // a staging copy did not complete within the wait limit
};

struct DdtrLaunch {
    const void *in;       // filterbank [c][stride]
    long long stride;     // elements per channel row
    int nchans;           // channels in the data
    int nch_used;         // channels summed (4-bit wide-band truncation)
    int tp;               // outputs per DM row (t_processed)
    int ndms;             // DM trials in the range
    const int32_t *table; // [c][ndms]
    const int32_t *wmin;  // [group][c4]
    int group_dms;        // DM trials per CTA
    int span;             // max window span of any (group, channel)
    int kind;             // DelayKind
    float nchans_f;       // divisor (reference i_nchans)
    float bin_f;          // divisor (reference bin)
    int divide_by_bin;    // 0 for the 4-bit kernel
    float *out;           // [dm][out_pitch]
    long long out_pitch;
    int *err;             // device error flags
};

cudaError_t launch_delay_table(const float *dmshifts, int nchans, int ndms, int kind, int fma_mode,
                               float mstartdm, float mdmstep, int32_t *table, int *err, cudaStream_t st);
cudaError_t launch_group_windows(const int32_t *table, int nchans, int ndms, int group_dms,
                                 int32_t *wmin, int *span_max, int *delay_max, cudaStream_t st);
cudaError_t launch_offset_table(const int32_t *table, const int32_t *wmin, int nchans, int ndms,
                                int group_dms, int rw, int span, int32_t *offtab, cudaStream_t st);

// [t][c] uint16 chunk -> [c][stride] storage type, rows of length nsamp.
cudaError_t launch_corner_turn(const uint16_t *in_tc, void *out_ct, int elem_bytes, int nchans,
                               long long nsamp, long long out_stride, int max_value, int *err,
                               cudaStream_t st);
// A chunk of the SIGPROC data section as stored, [t][nchans*nbits/8 bytes]
// (nbits 1, 2, 4, 8; 16 for 16-bit records, also used for the 16-bit
// rescaled samples of a 32-bit file) -> [c][stride], one byte per sample for
// nbits <= 8, uint16 otherwise.  Channels inside a byte in the reference
// reader's order (src/aa_sigproc_input.cpp:441-521).
cudaError_t launch_corner_turn_packed(const uint8_t *in_rec, int nbits, void *out_ct, int nchans, long long nsamp,
                                      long long out_stride, cudaStream_t st);

// Reference x2 binning on the flat buffer (src/aa_bin_gpu.cpp:8-44), out of
// place: for nchans and nsamp multiples of 32, dst[0, nchans*nsamp/2) = binned
// [c][nsamp/2] and dst[.., nchans*nsamp) = 0; otherwise the reference grids'
// partial coverage (channels beyond 32*floor(nchans/32) are not binned,
// positions its copy-back does not reach keep src).  nsamp must be even.
cudaError_t launch_bin_flat(const void *src, void *dst, int elem_bytes, int nchans, long long nsamp,
                            cudaStream_t st);

// Dedispersion of one (chunk, range).
cudaError_t launch_ddtr_u8(const DdtrLaunch &p, const int32_t *offtab, int tile_words, cudaStream_t st);
cudaError_t launch_ddtr_u16(const DdtrLaunch &p, cudaStream_t st);

size_t ddtr_u8_smem_bytes(int span, int group_dms, int tile_words, int nchans);
int ddtr_u8_rw(int span, int tile_words);

// Channel-quad kernel (ddtr_quad.cu).  Tables per range:
//   qpat [group][nquads][16] int32: skews (d1 | d2<<8 | d3<<16) in 0..14, count in 15
//   qwin [group][nq_pad] int32: smallest base-channel delay of the group
//   qtmp [nquads][ndms] int32: slot<<24 | tau (tau = delay - window start), -1 per-byte path
//   stats [4]: max tau, max skew, max patterns, entries on the per-byte path
//   qoff [nquads][ndms] int32: slot*W + tau, -1 per-byte path
struct QuadLaunch {
    const int32_t *qpat;
    const int32_t *qwin;
    const int32_t *qoff;
    int nquads, nq_pad;
    int W;     // words per pre-skewed row
    int raww;  // words per staged raw row
    int qs;    // channel quads per stage
    int npool; // pre-skewed rows per stage buffer
    int M;     // outputs per lane per DM trial (tile = 32*M)
    int maxpat;      // most patterns of one quad in a DM group
    int npool_qs[4]; // pre-skewed rows a stage of 1, 2, 4, 8 quads needs at most (0: qs x maxpat)
    int flavour; // 0: per-trial reuse test; 1: reuse by a switch over the warp's offset pattern
                 // (M = 16); 2: M = 8 with 16 warps and two CTAs per SM; 3: the pair body
                 // (rows summed over the quad, 16-bit pairs; pair-mode offsets; M = 16);
                 // 4: every DM trial loads its own words (M = 16); 5: no per-byte path
                 // (M = 16, ranges without per-byte entries); 6: 4 and 5
};

struct QuadGeometry {
    int M, W, raww, qs, npool, nq_pad;
    size_t smem_bytes;
};

QuadGeometry quad_geometry(int span, int dmax, int maxcnt, int group_dms, int nquads, int out_words, int qs,
                           int npool = 0);
// Rows a stage of qs quads needs: the table of the range when it has one,
// else qs x the most patterns of a quad.
inline int quad_npool(const QuadLaunch &q, int qs)
{
    const int k = (qs == 1) ? 0 : (qs == 2) ? 1 : (qs == 4) ? 2 : (qs == 8) ? 3 : -1;
    return (k >= 0 && q.npool_qs[k] > 0) ? q.npool_qs[k] : qs * (q.maxpat > 0 ? q.maxpat : 1);
}
cudaError_t launch_quad_patterns(const int32_t *table, int nch_used, int ndms, int group_dms, int nquads, int nq_pad,
                                 int32_t *qpat, int32_t *qwin, int32_t *qtmp, int *stats, cudaStream_t st);
cudaError_t launch_quad_offsets(const int32_t *qtmp, size_t n, int W, int32_t *qoff, cudaStream_t st,
                                int pairs = 0);
cudaError_t launch_ddtr_quad(const DdtrLaunch &p, const QuadLaunch &q, cudaStream_t st);
// Warp-specialised channel-quad kernel (M = 16 only): producer warps build the
// pre-skewed rows of the next stage while consumer warps sum the current one.
// Runs only ranges without per-byte entries (stats[3] of the pattern kernel = 0).
cudaError_t launch_ddtr_quadws(const DdtrLaunch &p, const QuadLaunch &q, cudaStream_t st);
size_t quadws_smem_bytes(const QuadLaunch &q);
// Split-phase channel-quad kernel (M = 16 only): the quad kernel's sums with
// mbarrier hand-offs between the row builds and the sums instead of a CTA
// barrier per stage.  Runs only ranges without per-byte entries.
cudaError_t launch_ddtr_quadsp(const DdtrLaunch &p, const QuadLaunch &q, cudaStream_t st);
size_t quadsp_smem_bytes(const QuadLaunch &q);

// Subband kernel (ddtr_sub.cu): 16-channel partial sums per skew pattern.
constexpr int SUB_BLK_WORDS = 128; // pattern block per (subband, DM group)
constexpr int SUB_MAX_PAT = 16;    // patterns per (subband, DM group)
constexpr int SUB_MAX_QPAT = 8;    // distinct skews per quad and group
constexpr int SUB_MAX_OFF = 1023;  // largest quad offset inside a subband

struct SubLaunch {
    const int32_t *sblk; // [group][nsub][SUB_BLK_WORDS]
    const int32_t *swin; // [group][nsub_pad]
    const int32_t *soff; // [nsub][ndms]
    int nsub, nsub_pad;
    int W;     // samples per partial-sum row (even)
    int wq;    // samples per quad-sum row (a multiple of 4; 16-bit sums, two per word)
    int raww;  // words per staged raw row
    int npat;  // partial-sum rows per buffer (max patterns)
    int nqrow; // quad rows per buffer (max distinct skews per subband)
};

struct SubGeometry {
    int W, wq, raww, npat, nqrow, nsub_pad;
    size_t smem_bytes;
};

SubGeometry sub_geometry(int maxtau, int maxoff, int maxd, int maxpat, int maxqrows, int nsub);
cudaError_t launch_sub_patterns(const int32_t *table, int nch_used, int ndms, int nsub, int nsub_pad, int32_t *sblk,
                                int32_t *swin, int32_t *stmp, int *stats, cudaStream_t st);
cudaError_t launch_sub_offsets(const int32_t *stmp, size_t n, int W, int32_t *soff, cudaStream_t st);
cudaError_t launch_ddtr_sub(const DdtrLaunch &p, const SubLaunch &s, cudaStream_t st);

// Dynamic shared memory the staged kernels may use per CTA (the sm_100a
// opt-in limit less 1 KB, which the persistent kernel keeps for its job
// descriptor).
constexpr size_t kStagedSmemLimit = 227 * 1024 - 1024;

// Staged fp32 kernel for two-byte samples (ddtr_f32.cu).
struct F32Launch {
    int cs;      // channels per stage (4, 8, 16 or 32)
    int W;       // floats per converted row (multiple of 4, >= span + 32*M)
    int rawh;    // samples per staged raw row (multiple of 8, >= W + 8)
    int nch_pad; // channels rounded up to 4 (row length of the window table)
};

struct F32Geometry {
    F32Launch f;
    size_t smem_bytes;
};

// Geometry for a delay span; cs = 0 picks the largest stage that fits the
// shared-memory limit.  smem_bytes = 0 when nothing fits.
F32Geometry f32_geometry(int span, int group_dms, int nchans, int cs);
cudaError_t launch_ddtr_f32(const DdtrLaunch &p, const F32Launch &f, cudaStream_t st);

// Persistent multi-beam dedispersion (ddtr_batch.cu).  One descriptor per
// (beam, chunk, range) job of the staged kernels; a job is groups x tiles
// work items (one 64-DM x 512-sample tile each, DM group fastest), numbered
// from item0 in the order of the table.
struct BatchJobDev {
    DdtrLaunch p;
    QuadLaunch q;
    F32Launch f;
    SubLaunch s;
    int variant; // 2 channel-quad, 3 staged fp32, 4 subband, 6 split-phase channel-quad
    int groups;
    long long item0;
};

// Body sets of the persistent kernel's instances: the channel-quad and fp32
// bodies (jobs of variants 2 and 3), those and the split-phase quad body
// (variant 6 too), the subband body alone (variant 4).
enum PersistentSet : int { PSET_QUAD = 0, PSET_SP = 1, PSET_SUB = 2 };

// Dynamic shared memory of one job in the persistent kernel.
size_t persistent_job_smem(const BatchJobDev &j);
// CTAs of the persistent kernel instance that fit one SM at this dynamic
// shared memory.
int persistent_blocks_per_sm(size_t smem_bytes, int set);
// counter: device work counter, zero before the launch; every job must have
// a body in the instance's set.
cudaError_t launch_ddtr_persistent(const BatchJobDev *jobs, int njobs, long long total_items,
                                   unsigned long long *counter, size_t smem_bytes, int grid, int set, cudaStream_t st);

} // namespace aab200
