// pipeline.hpp -- the DDTR runner behind the aa_pipeline_api surface.
//
// Mirrors the dedispersion part of the reference's generic runner
// (include/aa_permitted_pipelines_generic.hpp:606-914): one call of next()
// processes one (time chunk, DM range) step in the reference's order --
// chunk load and corner turn on the first range of a chunk, a single x2
// binning whenever inBin grows, dedispersion, copy into the host output
// rows at inc/inBin -- and reports has_more / finished_component / finished
// / error like aa_pipeline_runner::status (include/aa_pipeline_runner.hpp:25-30).
//
// B200 specifics: the input is corner-turned and narrowed to one byte per
// sample for nbits <= 8, every delay of a range is evaluated once into a
// device table when the pipeline is set up, host<->device copies run on their
// own streams against double buffers, and run_all() issues the whole job
// without host synchronisation between steps.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "ddtr_kernels.cuh"
#include "planner.hpp"

namespace aab200 {

struct StageTuneCache;
struct TunedRange;

enum class RunStatus : int { error = -1, finished = 0, has_more = 1, finished_component = 2 };

enum StrideMode : int {
    STRIDE_REFERENCE = 0, // binning length exactly as the reference runner passes it (:797-798)
    STRIDE_TRUE = 1       // binning on the true row stride, repeated to reach inBin
};

struct PipelineOptions {
    bool copy_to_host = true;   // aa_pipeline::component_option::copy_ddtr_data_to_host
    int stride_mode = STRIDE_REFERENCE;
    int fma_mode = 7;           // which contractible delay expressions are fused
    int failsafe = 0;           // force the cache-kernel delay semantics
    size_t free_memory = 0;     // 0: query the device like aa_device_info::free_memory()
    int tile_words = 0;         // 0: autotune
    int kernel_variant = 0;     // 0: choose per range, 1: generic kernels, 2: channel-quad / fp32 kernels,
                                // 3: subband / fp32 kernels, 4: warp-specialised channel-quad
                                // / fp32 kernels, 5: split-phase channel-quad / fp32 kernels
    int group_dms = 0;          // 0: autotune
    bool device_input = false;  // the input pointer is device memory ([t][c] uint16)
    // the input holds the SIGPROC data section as stored ([t][nchans*nbits/8]
    // bytes; 16-bit samples for nbits 16, and the reader's 16-bit rescaled
    // samples for nbits 32) instead of one uint16 per sample
    bool packed_input = false;
    bool device_output = false; // keep the whole output on the device ([range][dm][t])
    bool time_kernels = false;  // CUDA events around every kernel launch
    bool external_buffers = false; // no filterbank/raw/tile buffers: the caller runs the ops (batch engine)
    bool autotune = true;          // time stage depth, tile shape and kernel per range at setup
    // the reference runner's optional processing (aa_pipeline::component_option)
    bool zero_dm = false;          // zero_dm
    bool zero_dm_outliers = false; // zero_dm_with_outliers (zero_dm takes precedence)
    bool input_norm = false;       // input_DDTR_normalization
    bool output_norm = false;      // output_DDTR_normalization
    bool old_rfi = false;          // old_rfi
    bool bandpass_average = false; // set_bandpass_average
    // the analysis component is requested: the strategy keeps room for it
    // (include/aa_pipeline_api.hpp:142-154)
    bool enable_analysis = false;
    cudaStream_t stream = nullptr;
};

// The DM-time rows one dedispersion step wrote (device memory).
struct StepPlane {
    float *d = nullptr;
    long long pitch = 0; // floats between rows
    int ndms = 0, tp = 0, range = -1, chunk = -1;
    long long inc = 0;   // first input sample of the chunk
};

// One step of the reference runner's DDTR loop
// (include/aa_permitted_pipelines_generic.hpp:606-914), in order.  Filterbank
// "levels" name the copies a chunk goes through: level 0 is the corner-turned
// chunk, every x2 binning makes the next level from the current one.
struct DdtrOp {
    enum Kind : int { CORNER_TURN = 0, BIN = 1, DDTR = 2 };
    int kind = CORNER_TURN;
    int chunk = 0, range = 0;
    int src_level = 0, dst_level = 0;
    long long len = 0;     // CORNER_TURN: samples per channel row; BIN: the binning length
    long long inc = 0;     // first input sample of the chunk
    long long i_nsamp = 0; // DDTR: row stride of the level it reads
    int tp = 0;            // DDTR: outputs per DM row
    long long out_off = 0; // DDTR: first column of the chunk in the range's output rows (inc / inBin)
};

// A dedispersion launch, ready for a stream (launch_job) or a batch queue.
struct DdtrJob {
    int variant = 1; // 1 generic, 2 channel-quad, 3 staged fp32, 4 subband, 5 warp-specialised quad,
                     // 6 split-phase quad
    int elem_bytes = 1;
    int tile_words = 4;
    const int32_t *offtab = nullptr;
    DdtrLaunch p{};
    QuadLaunch q{};
    F32Launch f{};
    SubLaunch s{};
    int groups = 0;       // CTAs along DM
    long long tiles = 0;  // CTAs along time
    int tile_samples = 0; // samples per CTA tile
};

cudaError_t launch_job(const DdtrJob &job, cudaStream_t st);

// Kernel families timed when PipelineOptions::time_kernels is set.
enum KernelFamily : int { KF_DDTR = 0, KF_CORNER_TURN = 1, KF_BIN = 2, KF_COUNT = 3 };

struct RangeConfig {
    int kind = 0;
    int elem_bytes = 1;
    int group_dms = 64;
    int tile_words = 4;
    int span = 0;
    int delay_max = 0;
    int nch_used = 0;
    float mstartdm = 0.f;
    float mdmstep = 0.f;
    float tsamp = 0.f;
    int32_t *d_table = nullptr;
    int32_t *d_wmin = nullptr;
    int32_t *d_offtab = nullptr;
    // channel-quad kernel
    // 1: generic kernel (k_ddtr_u8 byte-phase / k_ddtr_u16 gather), 2: channel-quad
    // kernel (k_ddtr_quad, one-byte data), 3: staged fp32 kernel (k_ddtr_f32, two-byte data),
    // 4: subband kernel (k_ddtr_sub, one-byte data), 5: warp-specialised channel-quad
    // kernel (k_ddtr_quadws, one-byte data), 6: split-phase channel-quad kernel
    // (k_ddtr_quadsp, one-byte data)
    int variant = 1;
    QuadGeometry quad{};
    int quad_span = 0, quad_dmax = 0, quad_maxcnt = 0, nquads = 0;
    int quad_npool_qs[4] = {0, 0, 0, 0}; // rows a stage of 1, 2, 4, 8 quads needs (largest over groups and stages)
    int32_t *d_qpat = nullptr;
    int32_t *d_qwin = nullptr;
    int32_t *d_qoff = nullptr;
    // staged fp32 kernel
    F32Launch f32{};
    // subband kernel (variant 4); with the variant chosen per range both the
    // subband and the channel-quad tables may exist until the autotuner picks
    bool has_sub = false, has_quad = false;
    bool quad_ws_ok = false; // no per-byte entries: the warp-specialised quad kernel may run it
    bool quad_pairs = false; // the offset table is in pair mode (the pair body runs the range)
    int quad_flavour = -1;   // channel-quad kernel flavour the autotuner chose (-1: the default rule)
    int32_t *d_qtmp = nullptr; // (stage row, offset) of every (quad, DM trial) before the row pitch, kept
                               // while the autotuner tries tile shapes (their row pitches differ)
    SubGeometry sub{};
    int nsub = 0;
    int32_t *d_sblk = nullptr;
    int32_t *d_swin = nullptr;
    int32_t *d_soff = nullptr;
};

class DdtrPipeline {
public:
    // input: [t][c] uint16, or the stored records with opt.packed_input
    DdtrPipeline(const FilterbankMetadata &meta, const void *input, const PipelineOptions &opt);
    ~DdtrPipeline();
    DdtrPipeline(const DdtrPipeline &) = delete;
    DdtrPipeline &operator=(const DdtrPipeline &) = delete;

    bool bind(const DdtrPlan &plan);
    bool ready() const { return bound_; }
    bool setup();                       // allocates and builds the delay tables (idempotent)
    bool next(RunStatus &status);       // one (chunk, range) step
    bool run_all();                     // the whole job, no host sync between steps
    bool rewind();                      // start again from the first chunk, same buffers
    bool synchronize();

    const DdtrStrategy &strategy() const { return strategy_; }
    float ***output_buffer() { return host_rows_.empty() ? nullptr : host_rows_.data(); }
    float *device_output(int range) const
    {
        return (range >= 0 && range < static_cast<int>(d_out_full_.size())) ? d_out_full_[range] : nullptr;
    }
    int current_range() const { return cur_range_; }
    int current_tchunk() const { return cur_chunk_; }
    long long current_inc() const { return inc_; }
    const RangeConfig &range_config(int r) const { return ranges_[r]; }
    const std::string &last_error() const { return error_; }
    // The run as a list of steps (valid after setup()).
    const std::vector<DdtrOp> &ops() const { return ops_; }
    // Elements a filterbank level must hold past nchans x its row length for
    // the staged windows' over-read (valid after setup()).
    size_t pad_elems() const { return pad_elems_; }
    int elem_bytes() const { return elem_bytes_; }
    int *device_flags() const { return d_err_; }
    // The launch of a DDTR op reading level buffer `in` (in_elems elements)
    // and writing rows of `out` with pitch out_pitch.
    // as_variant 2 or 4: the job with the channel-quad or subband kernel
    // instead of the range's own (the range must have that kernel's tables)
    bool make_job(const DdtrOp &op, const void *in, size_t in_elems, float *out, long long out_pitch, DdtrJob &job,
                  int as_variant = 0);
    bool range_has_sub(int r) const { return ranges_[r].has_sub; }
    bool check_flags() { return check_device_flags(); }
    long long kernel_launches() const { return launches_; }
    // Device time (ms) and launch count of one kernel family since the last
    // reset, collected at synchronize().
    double kernel_ms(int family) const { return (family >= 0 && family < KF_COUNT) ? kernel_ms_[family] : 0.0; }
    long long kernel_count(int family) const { return (family >= 0 && family < KF_COUNT) ? kernel_n_[family] : 0; }
    void reset_kernel_times();
    bool set_time_kernels(bool on)
    {
        opt_.time_kernels = on;
        return true;
    }
    bool cleanup();
    // The rows of the last dedispersion step; in copy_to_host mode they sit
    // in a tile the next steps reuse, so they are valid until the next step.
    bool last_step_plane(StepPlane &p) const
    {
        p = last_plane_;
        return last_plane_.d != nullptr;
    }
    cudaStream_t stream() const { return st_; }
    // The channel-quad kernel flavour a range runs (make_job's choice).
    int quad_flavour_of(const RangeConfig &rc) const;

private:
    bool fail(const std::string &msg);
    bool check_cuda(cudaError_t e, const char *what);
    bool check_device_flags();
    bool build_range(int r);
    bool setup_processing(long long L0);
    bool quad_ws_fits(const RangeConfig &rc) const;
    int quad_sp_depth(const RangeConfig &rc) const;
    bool build_quad_tables(int r);
    QuadGeometry quad_fit(const RangeConfig &rc, int M) const;
    bool tune_quad_shape(int r, const DdtrOp &op, float *out, long long pitch, StageTuneCache &cache, DdtrJob &job);
    bool build_sub_tables(int r);
    bool tune_ranges();
    std::vector<long long> tune_key(int r, const DdtrOp &op, long long pitch) const;
    bool tuned_valid(const RangeConfig &rc, const TunedRange &t) const;
    bool step(bool allow_sync);
    bool enumerate_ops();
    bool exec_corner_turn(const DdtrOp &op);
    bool exec_bin(const DdtrOp &op);
    bool exec_ddtr(const DdtrOp &op);
    size_t buffer_elems() const { return flat_elems_; }
    bool timed_launch_begin(int family);
    bool timed_launch_end();
    bool collect_kernel_times();

    FilterbankMetadata meta_;
    const uint8_t *input_;
    long long in_rec_bytes_ = 0; // bytes of one input time sample (all channels)
    PipelineOptions opt_;
    DdtrPlan plan_;
    DdtrStrategy strategy_;
    bool bound_ = false;
    bool setup_done_ = false;
    bool finished_component_sent_ = false;
    std::string error_;

    // device state
    int device_ = 0;
    cudaStream_t st_ = nullptr;       // compute stream
    cudaStream_t st_h2d_ = nullptr;
    cudaStream_t st_d2h_ = nullptr;
    bool own_stream_ = false;
    int elem_bytes_ = 1;
    size_t flat_elems_ = 0;           // elements per flat buffer incl. padding
    void *d_flat_[2] = {nullptr, nullptr};
    uint8_t *d_raw_[2] = {nullptr, nullptr}; // staged H2D chunks, in_rec_bytes_ per time sample
    uint16_t *d_stage_ = nullptr;             // writable [t][c] chunk for input processing of device or packed input
    float *d_norm_ = nullptr;                 // bandpass normalisation [nchans] (zero DM)
    std::vector<float> bandpass_;             // its host copy
    float *d_dmshifts_ = nullptr;
    int *d_err_ = nullptr;
    int *h_err_ = nullptr;            // pinned
    std::vector<RangeConfig> ranges_;
    std::vector<float *> d_out_full_; // device_output mode: [range] -> [ndms][total]
    float *d_tile_[2] = {nullptr, nullptr}; // copy_to_host mode: per-(chunk,range) output
    size_t tile_elems_ = 0;
    cudaEvent_t ev_tile_free_[2] = {nullptr, nullptr};
    cudaEvent_t ev_tile_done_[2] = {nullptr, nullptr};
    cudaEvent_t ev_raw_ready_[2] = {nullptr, nullptr};
    cudaEvent_t ev_raw_free_[2] = {nullptr, nullptr};

    // host output: rows of one pinned block, like float*** [range][dm][t]
    float *h_block_ = nullptr;
    std::vector<float **> host_rows_;
    std::vector<std::vector<float *>> host_row_ptrs_;

    // iteration state (reference :1053-1054 current_time_chunk/current_range)
    std::vector<DdtrOp> ops_;
    size_t op_cursor_ = 0;
    size_t pad_elems_ = 0;
    int cur_chunk_ = 0;
    int cur_range_ = 0;
    long long inc_ = 0;
    int tile_slot_ = 0;
    StepPlane last_plane_;
    long long launches_ = 0;

    struct TimedLaunch {
        cudaEvent_t start = nullptr, stop = nullptr;
        int family = 0;
    };
    std::vector<TimedLaunch> kev_;
    size_t kev_used_ = 0;
    double kernel_ms_[KF_COUNT] = {0.0, 0.0, 0.0};
    long long kernel_n_[KF_COUNT] = {0, 0, 0};
};

} // namespace aab200
