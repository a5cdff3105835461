// sigproc.cpp -- SIGPROC filterbank reader (see sigproc.hpp).
#include "sigproc.hpp"

#include <climits>
#include <cstring>

namespace aab200 {

long long sigproc_record_bytes(int nbits, int nchans)
{
    if (nchans <= 0)
        return 0;
    switch (nbits) {
    case 32:
        return 4LL * nchans;
    case 16:
        return 2LL * nchans;
    case 8:
        return nchans;
    case 4:
    case 2:
    case 1:
        return (static_cast<long long>(nchans) * nbits % 8) ? 0 : static_cast<long long>(nchans) * nbits / 8;
    default:
        return 0;
    }
}

void sigproc_unpack(const uint8_t *rec, int nbits, int nchans, long long n, uint16_t *out)
{
    const long long rb = sigproc_record_bytes(nbits, nchans);
    for (long long t = 0; t < n; ++t) {
        const uint8_t *r = rec + t * rb;
        uint16_t *o = out + t * nchans;
        switch (nbits) {
        case 16:
            std::memcpy(o, r, static_cast<size_t>(nchans) * 2); // little-endian host, as the reference's fread
            break;
        case 8:
            for (int c = 0; c < nchans; ++c)
                o[c] = r[c];
            break;
        case 4:
            for (int b = 0; b < nchans / 2; ++b) {
                o[2 * b] = static_cast<uint16_t>((r[b] >> 4) & 0x0F);
                o[2 * b + 1] = static_cast<uint16_t>(r[b] & 0x0F);
            }
            break;
        case 2:
            for (int b = 0; b < nchans / 4; ++b)
                for (int k = 0; k < 4; ++k)
                    o[4 * b + k] = static_cast<uint16_t>((r[b] >> (6 - 2 * k)) & 0x03);
            break;
        case 1:
            for (int b = 0; b < nchans / 8; ++b)
                for (int i = 0; i < 8; ++i)
                    o[8 * b + i] = static_cast<uint16_t>((r[b] >> i) & 0x01);
            break;
        default:
            break;
        }
    }
}

void sigproc_rescale32(const float *x, long long n, float min, float max, uint16_t *out)
{
    const float bin = (max - min) / 65535.0f;
    for (long long i = 0; i < n; ++i) {
        const float q = (x[i] - min) / bin;
        // float -> unsigned short as x86-64 compiles it: a truncating
        // conversion to int32 (INT_MIN for NaN or out of range), low 16 bits
        int32_t v = INT_MIN;
        if (q == q && q < 2147483648.0f && q >= -2147483648.0f)
            v = static_cast<int32_t>(q);
        out[i] = static_cast<uint16_t>(static_cast<uint32_t>(v) & 0xFFFFu);
    }
}

SigprocInput::SigprocInput(std::string path) : path_(std::move(path)) {}

SigprocInput::~SigprocInput() { close(); }

bool SigprocInput::fail(const std::string &m)
{
    error_ = m;
    return false;
}

bool SigprocInput::open()
{
    if (fp_)
        return true;
    fp_ = std::fopen(path_.c_str(), "rb");
    return fp_ ? true : fail("cannot open " + path_);
}

bool SigprocInput::close()
{
    if (!fp_)
        return true;
    const bool ok = std::fclose(fp_) == 0;
    fp_ = nullptr;
    return ok;
}

// Keyword loop of src/aa_sigproc_input.cpp:110-269: a length-prefixed string,
// then for a known keyword its binary value; strings of length <= 1 or >= 80
// are passed over, unknown keywords consume nothing more.
bool SigprocInput::parse_header()
{
    h_ = SigprocHeader();
    struct Kw {
        const char *name;
        void *dst;
        size_t size;
    };
    const Kw kws[] = {
        {"telescope_id", &h_.telescope_id, sizeof(int)}, {"machine_id", &h_.machine_id, sizeof(int)},
        {"data_type", &h_.data_type, sizeof(int)},       {"barycentric", &h_.barycentric, sizeof(int)},
        {"pulsarcentric", &h_.pulsarcentric, sizeof(int)}, {"az_start", &h_.az_start, sizeof(double)},
        {"za_start", &h_.za_start, sizeof(double)},      {"src_raj", &h_.src_raj, sizeof(double)},
        {"src_dej", &h_.src_dej, sizeof(double)},        {"tstart", &h_.tstart, sizeof(double)},
        {"tsamp", &h_.tsamp, sizeof(double)},            {"nbits", &h_.nbits, sizeof(int)},
        {"nsamples", &h_.nsamples_keyword, sizeof(int)}, {"fch1", &h_.fch1, sizeof(double)},
        {"foff", &h_.foff, sizeof(double)},              {"fchannel", &h_.fchannel, sizeof(double)},
        {"nchans", &h_.nchans, sizeof(int)},             {"nifs", &h_.nifs, sizeof(int)},
        {"refdm", &h_.refdm, sizeof(double)},            {"period", &h_.period, sizeof(double)},
    };
    char s[81];
    for (;;) {
        int nchar = 0;
        if (std::fread(&nchar, sizeof(int), 1, fp_) != 1 || std::feof(fp_))
            return fail("error while reading the header (no HEADER_END)");
        if (nchar <= 1 || nchar >= 80)
            continue;
        if (std::fread(s, static_cast<size_t>(nchar), 1, fp_) != 1)
            return fail("error while reading the header");
        s[nchar] = '\0';
        if (std::strcmp(s, "HEADER_END") == 0)
            break;
        for (const Kw &k : kws)
            if (std::strcmp(s, k.name) == 0) {
                if (std::fread(k.dst, k.size, 1, fp_) != 1)
                    return fail(std::string("error while reading the value of ") + k.name);
                break;
            }
    }
    if (h_.nifs != 1)
        return fail("only one IF channel is supported (nifs must be 1)");
    h_.data_start = std::ftell(fp_);
    if (h_.data_start < 0 || std::fseek(fp_, 0, SEEK_END) != 0)
        return fail("cannot find the end of the data");
    const long end = std::ftell(fp_);
    if (end < 0 || std::fseek(fp_, static_cast<long>(h_.data_start), SEEK_SET) != 0)
        return fail("cannot find the end of the data");
    h_.data_bytes = end - h_.data_start;
    if (h_.nchans <= 0)
        return fail("nchans must be positive");
    // :296-326
    const long long T = h_.data_bytes, n = h_.nchans;
    switch (h_.nbits) {
    case 32:
        h_.nsamp = static_cast<unsigned long long>(T / (n * 4));
        break;
    case 16:
        h_.nsamp = static_cast<unsigned long long>(T / (n * 2));
        break;
    case 8:
        h_.nsamp = static_cast<unsigned long long>(T / n);
        break;
    case 4:
        h_.nsamp = static_cast<unsigned long long>(2 * T / n);
        break;
    case 2:
        h_.nsamp = static_cast<unsigned long long>(4 * T / n);
        break;
    case 1:
        h_.nsamp = static_cast<unsigned long long>(8 * T / n);
        break;
    default:
        return fail("only 1, 2, 4, 8, 16 and 32-bit data are supported");
    }
    // the reference reads nchans*nbits/8 bytes per record but sizes its buffer
    // by the count above; the two agree only when channels fill whole bytes
    if (sigproc_record_bytes(h_.nbits, h_.nchans) == 0)
        return fail("nchans * nbits must be a multiple of 8");
    if (h_.nsamp > static_cast<unsigned long long>(INT_MAX))
        return fail("more samples than the metadata's int holds");
    return true;
}

FilterbankMetadata SigprocInput::read_metadata()
{
    FilterbankMetadata m;
    m.nbits = 0;
    if (!open())
        return m;
    if (!header_read_) {
        header_ok_ = parse_header();
        header_read_ = true;
    }
    if (!header_ok_)
        return m;
    m.tstart = h_.tstart;
    m.tsamp = h_.tsamp;
    m.fch1 = h_.fch1;
    m.foff = h_.foff;
    m.nbits = h_.nbits;
    m.nsamples = static_cast<int>(h_.nsamp);
    m.nchans = h_.nchans;
    return m;
}

// The data section as stored: nsamp records of nchans*nbits/8 bytes.
bool SigprocInput::read_data(std::vector<uint8_t> &raw)
{
    const long long rb = sigproc_record_bytes(h_.nbits, h_.nchans);
    const size_t bytes = static_cast<size_t>(h_.nsamp) * static_cast<size_t>(rb);
    raw.resize(bytes);
    if (std::fseek(fp_, static_cast<long>(h_.data_start), SEEK_SET) != 0)
        return fail("cannot seek to the data");
    if (bytes && std::fread(raw.data(), 1, bytes, fp_) != bytes)
        return fail("short read of the data section");
    return true;
}

bool SigprocInput::read_signal()
{
    if (!fp_ || !header_read_ || data_read_)
        return false;
    if (!header_ok_)
        return fail("the header was not read successfully");
    std::vector<uint8_t> raw;
    if (!read_data(raw))
        return false;
    const long long n = static_cast<long long>(h_.nsamp) * h_.nchans;
    buf_.assign(static_cast<size_t>(n), 0);
    if (h_.nbits == 32) {
        // :344-359 min and max over the file, initial values as there
        const float *x = reinterpret_cast<const float *>(raw.data());
        float mx = -10000000000.0f, mn = 10000000000.0f;
        for (long long i = 0; i < n; ++i) {
            if (x[i] > mx)
                mx = x[i];
            if (x[i] < mn)
                mn = x[i];
        }
        sigproc_rescale32(x, n, mn, mx, buf_.data());
    } else {
        sigproc_unpack(raw.data(), h_.nbits, h_.nchans, static_cast<long long>(h_.nsamp), buf_.data());
    }
    data_read_ = true;
    return true;
}

bool SigprocInput::read_packed()
{
    if (!fp_ || !header_read_ || packed_read_)
        return false;
    if (!header_ok_)
        return fail("the header was not read successfully");
    if (!read_data(packed_))
        return false;
    if (h_.nbits == 32) {
        const long long n = static_cast<long long>(h_.nsamp) * h_.nchans;
        const float *x = reinterpret_cast<const float *>(packed_.data());
        float mx = -10000000000.0f, mn = 10000000000.0f;
        for (long long i = 0; i < n; ++i) {
            if (x[i] > mx)
                mx = x[i];
            if (x[i] < mn)
                mn = x[i];
        }
        std::vector<uint8_t> r16(static_cast<size_t>(n) * 2);
        sigproc_rescale32(x, n, mn, mx, reinterpret_cast<uint16_t *>(r16.data()));
        packed_.swap(r16);
    }
    packed_read_ = true;
    return true;
}

} // namespace aab200
