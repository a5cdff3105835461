// sigproc.hpp -- SIGPROC filterbank reader with the reference reader's header
// rules and sample unpacking (src/aa_sigproc_input.cpp:85-543), plus a read
// of the data section as stored, for the pipeline's packed input (the
// unpacking then happens on the GPU, fused with the corner turn).
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "planner.hpp"

namespace aab200 {

// Header values the reference reads (src/aa_sigproc_input.cpp:85-269); every
// other keyword is skipped without consuming a value, as there.
struct SigprocHeader {
    int telescope_id = 0, machine_id = 0, data_type = 0, barycentric = 0, pulsarcentric = 0;
    double az_start = 0, za_start = 0, src_raj = 0, src_dej = 0, tstart = 0, tsamp = 0;
    int nbits = 0, nsamples_keyword = 0, nchans = 0, nifs = 0;
    double fch1 = 0, foff = 0, fchannel = 0, refdm = 0, period = 0;
    long long data_start = 0;     // byte offset of the first sample
    long long data_bytes = 0;     // bytes after the header
    unsigned long long nsamp = 0; // samples per channel, from the data size (:296-326)
};

// Bytes of one time sample (all channels) as stored, 0 when nchans does not
// fill whole bytes at this bit depth.
long long sigproc_record_bytes(int nbits, int nchans);

// Unpacks n records of the stored data section into one unsigned short per
// sample, [t][c], with the reference's channel order inside a byte
// (:441-521): 4-bit high nibble first, 2-bit most significant pair first,
// 1-bit least significant bit first.  nbits 1, 2, 4, 8 or 16.
void sigproc_unpack(const uint8_t *rec, int nbits, int nchans, long long n, uint16_t *out);

// 32-bit samples rescaled to unsigned short as the reference does (:361-386):
// bin = (max - min) / 65535, value = (unsigned short)((x - min) / bin).
void sigproc_rescale32(const float *x, long long n, float min, float max, uint16_t *out);

class SigprocInput {
  public:
    explicit SigprocInput(std::string path);
    ~SigprocInput();
    SigprocInput(const SigprocInput &) = delete;
    SigprocInput &operator=(const SigprocInput &) = delete;

    bool open();
    bool close();
    // aa_sigproc_input::read_metadata: opens the file if needed and parses the
    // header; a failed parse returns empty metadata (nbits 0, nchans 0).
    FilterbankMetadata read_metadata();
    // aa_sigproc_input::read_signal: one unsigned short per sample, [t][c];
    // true once, after a successful read.
    bool read_signal();
    // The data section as stored (nbits 1-16), or for 32-bit files the
    // reader's 16-bit rescaled samples; true once, after a successful read.
    bool read_packed();

    const SigprocHeader &header() const { return h_; }
    bool header_ok() const { return header_ok_; }
    const std::vector<uint16_t> &input_buffer() const { return buf_; }
    const std::vector<uint8_t> &packed_buffer() const { return packed_; }
    const std::string &last_error() const { return error_; }

  private:
    bool parse_header();
    bool read_data(std::vector<uint8_t> &raw);
    bool fail(const std::string &m);

    std::string path_;
    FILE *fp_ = nullptr;
    SigprocHeader h_;
    bool header_read_ = false, header_ok_ = false, data_read_ = false, packed_read_ = false;
    std::vector<uint16_t> buf_;
    std::vector<uint8_t> packed_;
    std::string error_;
};

} // namespace aab200
