// capi_batch.cpp -- extern "C" entry points of the multi-beam engine
// (aa_b200_batch_*, declared in include/aa_b200.h).
#include "aa_b200.h"

#include <string>

#include <cuda_runtime.h>

#include "batch.hpp"
#include "planner.hpp"

using namespace aab200;

namespace {

thread_local std::string g_batch_error;

FilterbankMetadata batch_meta(const aa_py_filterbank_metadata_struct &m)
{
    FilterbankMetadata f;
    f.tstart = m.m_tstart;
    f.tsamp = m.m_tsamp;
    f.fch1 = m.m_fch1;
    f.foff = m.m_foff;
    f.nbits = m.m_nbits;
    f.nsamples = m.m_nsamples;
    f.nchans = m.m_nchans;
    return f;
}

BatchDdtr *as_batch(void *p) { return static_cast<BatchDdtr *>(p); }

bool batch_ok(BatchDdtr *b, bool ok)
{
    if (!ok && b)
        g_batch_error = b->last_error();
    return ok;
}

} // namespace

extern "C" {

void *aa_b200_batch_create(int stride_mode, int fma_mode, size_t free_memory, int persistent, int use_graph,
                           int autotune, void *stream)
{
    if (stride_mode != 0 && stride_mode != 1) {
        g_batch_error = "stride_mode must be 0 (reference) or 1 (true stride)";
        return nullptr;
    }
    BatchOptions o;
    o.stride_mode = stride_mode;
    o.fma_mode = fma_mode;
    o.free_memory = free_memory;
    o.persistent = persistent != 0;
    o.use_graph = use_graph != 0;
    o.autotune = autotune != 0;
    o.stream = static_cast<cudaStream_t>(stream);
    return new BatchDdtr(o);
}

int aa_b200_batch_add_beam(void *batch, aa_py_filterbank_metadata_struct metadata, void *ddtr_plan,
                           const unsigned short *d_input)
{
    BatchDdtr *b = as_batch(batch);
    if (!b || !ddtr_plan) {
        g_batch_error = "null batch or plan";
        return -1;
    }
    const int i = b->add_beam(batch_meta(metadata), *static_cast<const DdtrPlan *>(ddtr_plan), d_input);
    if (i < 0)
        g_batch_error = b->last_error();
    return i;
}

bool aa_b200_batch_setup(void *batch) { return batch_ok(as_batch(batch), as_batch(batch) && as_batch(batch)->setup()); }

bool aa_b200_batch_run(void *batch) { return batch_ok(as_batch(batch), as_batch(batch) && as_batch(batch)->run()); }

bool aa_b200_batch_synchronize(void *batch)
{
    return batch_ok(as_batch(batch), as_batch(batch) && as_batch(batch)->synchronize());
}

float *aa_b200_batch_device_output(void *batch, int beam, int range)
{
    return as_batch(batch) ? as_batch(batch)->device_output(beam, range) : nullptr;
}

int aa_b200_batch_range_shape(void *batch, int beam, int range, int *ndms, long long *total_samps, int *inBin)
{
    BatchDdtr *b = as_batch(batch);
    DdtrPipeline *p = b ? b->beam(beam) : nullptr;
    if (!p || !p->ready() || range < 0 || range >= static_cast<int>(p->strategy().nranges())) {
        g_batch_error = "no such beam or range (or the batch is not set up)";
        return 1;
    }
    *ndms = p->strategy().ndms(range);
    *total_samps = p->strategy().total_samps(range);
    *inBin = p->strategy().dm(range).inBin;
    return 0;
}

bool aa_b200_batch_set_kernel_choice(void *batch, int choice)
{
    BatchDdtr *b = as_batch(batch);
    return b && b->set_kernel_choice(choice);
}

int aa_b200_batch_sub_jobs(void *batch)
{
    BatchDdtr *b = as_batch(batch);
    return b ? b->sub_jobs() : 0;
}

int aa_b200_batch_info(void *batch, long long *work_items, int *persistent_jobs, int *other_jobs, int *grid,
                       size_t *smem_bytes, size_t *level_bytes, long long *launches_per_run)
{
    BatchDdtr *b = as_batch(batch);
    if (!b)
        return 1;
    *work_items = b->work_items();
    *persistent_jobs = b->persistent_jobs();
    *other_jobs = b->other_jobs();
    *grid = b->grid();
    *smem_bytes = b->smem_bytes();
    *level_bytes = b->level_bytes();
    *launches_per_run = b->launches_per_run();
    return 0;
}

double aa_b200_batch_last_ms(void *batch, int which)
{
    BatchDdtr *b = as_batch(batch);
    if (!b)
        return -1.0;
    return which == 0 ? b->last_run_ms() : b->last_ddtr_ms();
}

int aa_b200_batch_estimate_bytes(aa_py_filterbank_metadata_struct metadata, void *ddtr_plan, size_t free_memory,
                                 size_t *bytes)
{
    std::string err;
    if (!ddtr_plan || !BatchDdtr::estimate_beam_bytes(batch_meta(metadata), *static_cast<const DdtrPlan *>(ddtr_plan),
                                                      free_memory, *bytes, err)) {
        g_batch_error = ddtr_plan ? err : "null plan";
        return 1;
    }
    return 0;
}

const char *aa_b200_batch_last_error(void *batch)
{
    if (batch && !as_batch(batch)->last_error().empty())
        return as_batch(batch)->last_error().c_str();
    return g_batch_error.c_str();
}

void aa_b200_batch_delete(void *batch) { delete as_batch(batch); }

} // extern "C"
