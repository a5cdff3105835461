// capi_sigproc.cpp -- the reference's SIGPROC reader entry points
// (src/aa_py_sigproc_input.cpp:7-33) and the packed-read extensions declared
// in include/aa_b200.h.
#include "aa_b200.h"

#include "sigproc.hpp"

using namespace aab200;

namespace {

SigprocInput *as_in(void *p) { return static_cast<SigprocInput *>(p); }
const SigprocInput *as_in(const void *p) { return static_cast<const SigprocInput *>(p); }

} // namespace

extern "C" {

void *aa_py_sigproc_input(const char *path) { return path ? new SigprocInput(path) : nullptr; }

void aa_py_sigproc_input_del(const void *obj) { delete as_in(obj); }

aa_py_filterbank_metadata_struct aa_py_sigproc_input_read_metadata(void *obj)
{
    aa_py_filterbank_metadata_struct m{};
    if (!obj)
        return m;
    const FilterbankMetadata f = as_in(obj)->read_metadata();
    m.m_tstart = f.tstart;
    m.m_tsamp = f.tsamp;
    m.m_fch1 = f.fch1;
    m.m_foff = f.foff;
    m.m_nbits = f.nbits;
    m.m_nsamples = f.nsamples;
    m.m_nchans = f.nchans;
    m.m_src_raj = as_in(obj)->header().src_raj;
    return m;
}

bool aa_py_sigproc_input_read_signal(void *obj) { return obj && as_in(obj)->read_signal(); }

const unsigned short *aa_py_sigproc_input_input_buffer(const void *obj)
{
    if (!obj || as_in(obj)->input_buffer().empty())
        return nullptr;
    return as_in(obj)->input_buffer().data();
}

bool aa_b200_sigproc_read_packed(void *obj) { return obj && as_in(obj)->read_packed(); }

const void *aa_b200_sigproc_packed_buffer(const void *obj)
{
    if (!obj || as_in(obj)->packed_buffer().empty())
        return nullptr;
    return as_in(obj)->packed_buffer().data();
}

long long aa_b200_sigproc_packed_bytes(const void *obj)
{
    return obj ? static_cast<long long>(as_in(obj)->packed_buffer().size()) : 0;
}

bool aa_b200_sigproc_header(const void *obj, aa_b200_sigproc_header_struct *out)
{
    if (!obj || !out || !as_in(obj)->header_ok())
        return false;
    const SigprocHeader &h = as_in(obj)->header();
    out->telescope_id = h.telescope_id;
    out->machine_id = h.machine_id;
    out->data_type = h.data_type;
    out->barycentric = h.barycentric;
    out->pulsarcentric = h.pulsarcentric;
    out->az_start = h.az_start;
    out->za_start = h.za_start;
    out->src_raj = h.src_raj;
    out->src_dej = h.src_dej;
    out->tstart = h.tstart;
    out->tsamp = h.tsamp;
    out->nbits = h.nbits;
    out->nsamples_keyword = h.nsamples_keyword;
    out->nchans = h.nchans;
    out->nifs = h.nifs;
    out->fch1 = h.fch1;
    out->foff = h.foff;
    out->fchannel = h.fchannel;
    out->refdm = h.refdm;
    out->period = h.period;
    out->data_start = h.data_start;
    out->data_bytes = h.data_bytes;
    out->nsamp = static_cast<long long>(h.nsamp);
    return true;
}

const char *aa_b200_sigproc_last_error(const void *obj) { return obj ? as_in(obj)->last_error().c_str() : ""; }

} // extern "C"
