// autotune.hpp -- stage depth of the staged dedispersion kernels, by
// measurement.
//
// The channel-quad kernel stages qs channel quads per shared-memory stage and
// the fp32 kernel cs channels; deeper stages mean fewer CTA barriers per
// channel but more shared memory (and, for the quad kernel, more pattern rows
// built per stage).  tune_stage_depth times every depth that fits (also
// inside the persistent kernel, which keeps 256 bytes for its job descriptor)
// on a slice of the job -- about two CTAs per SM -- with CUDA events, keeps
// the fastest, and caches it by the job's shape.  The slice writes into the
// job's own output rows, which the real run overwrites.
//
// The plain pipeline (DdtrPipeline::tune_ranges) searches further per range
// with the same slice timing: the channel-quad output tile (64 DM trials x
// 512 samples, or x 256 samples with 8 or 4 DM trials per warp), the sum-loop
// flavour, each at its own tuned depth; then the split-phase and subband
// kernels against the winner.  The DM-group size (64) is fixed by the staged
// kernels' tables; the generic kernels take tile words and group sizes from
// the options.
#pragma once
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include <cuda_runtime.h>

#include "pipeline.hpp"

namespace aab200 {

struct StageTuneCache {
    std::map<std::tuple<int, int, int, int, int, int, long long>, int> best;
};

bool tune_stage_depth(DdtrJob &job, cudaStream_t st, int device, StageTuneCache &cache, std::string &err);

// Device time (ms, best of two after a warm-up launch) of a slice of the job:
// about two CTAs per SM, or (samples > 0) that many output samples per DM
// trial rounded up to the job's tile, at most the job's; timed_samples
// receives the slice's samples.  Negative on a launch error (message in err).
float time_job_slice(const DdtrJob &job, cudaStream_t st, int device, std::string &err, long long samples = 0,
                     long long *timed_samples = nullptr);

// What the plain pipeline's autotuner chose for a range: the kernel variant,
// the channel-quad geometry (tile shape, stage depth) and flavour, and the
// fp32 kernel's stage depth.  The choices are kept for the life of the
// process under a key of everything the slice timings depend on (device,
// channel delays, the range, its delay-table summary, chunk length, row
// pitch and the kernel options), so that a later pipeline of the same shape
// -- the next beam or file of a survey -- takes them without timing again.
// No choice changes the output: every kernel gives the same bits.
struct TunedRange {
    int variant = 0;
    QuadGeometry quad{};
    int quad_flavour = -1;
    int f32_cs = 0;
};
bool tuned_range_find(const std::vector<long long> &key, TunedRange &out);
void tuned_range_keep(const std::vector<long long> &key, const TunedRange &t);
// Entries held; clear empties the store first.
size_t tuned_range_entries(bool clear);
// Ranges set up from a kept choice (counted by the pipeline that took it).
void tuned_range_note_use();
long long tuned_range_uses();
// The store as a text file (one entry per line), and back: a tuning run's
// choices reused by later processes (a profiling run, a production run).
// Loading adds to the entries held.  Return the entries written or read, -1
// if the file cannot be opened or a line is malformed (err says which).
long long tuned_ranges_save(const std::string &path, std::string &err);
long long tuned_ranges_load(const std::string &path, std::string &err);

} // namespace aab200
