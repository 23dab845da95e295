// SIGPROC filterbank header reader: the input frost's `open_input` reads
// through psrio (lib/pipeline/input.cpp:32-69) for the file path of the
// per-gulp search. psrio is not available here, so this restates the
// published SIGPROC header layout: "HEADER_START", then keyword records
// until "HEADER_END", each keyword a 32-bit length and its characters
// followed by a value whose type the keyword fixes (32-bit int, 64-bit
// double, a length-prefixed string, or one byte for `signed`); a channel
// frequency table may sit between FREQUENCY_START and FREQUENCY_END as
// `fchannel` doubles. Packed sample rows follow the header.

#include "sigproc.hpp"

#include <algorithm>
#include <cstring>
#include <fstream>
#include <string>

namespace fb::io {

namespace {

enum class Kind { Int, Double, String, Byte, Marker };

Kind kind_of(const std::string& key) {
    static const char* const ints[] = {"telescope_id", "machine_id", "data_type", "barycentric",
                                       "pulsarcentric", "nbits",     "nsamples",  "nchans",
                                       "nifs",          "nbeams",    "ibeam"};
    static const char* const doubles[] = {"tstart",   "tsamp",   "fch1",    "foff",   "refdm",   "az_start",
                                          "za_start", "src_raj", "src_dej", "period", "fchannel"};
    for (const char* k : ints)
        if (key == k)
            return Kind::Int;
    for (const char* k : doubles)
        if (key == k)
            return Kind::Double;
    if (key == "source_name" || key == "rawdatafile")
        return Kind::String;
    if (key == "signed")
        return Kind::Byte;
    if (key == "FREQUENCY_START" || key == "FREQUENCY_END")
        return Kind::Marker;
    invalid("sigproc: unknown header keyword '" + key + "'");
}

class Reader {
public:
    explicit Reader(const std::string& path) : m_in(path, std::ios::binary), m_path(path) {
        if (!m_in)
            throw Error(FROST_ERR_IO, "sigproc: cannot open " + path);
    }
    template <class T> T value() {
        T v{};
        m_in.read(reinterpret_cast<char*>(&v), sizeof(T));
        if (!m_in)
            truncated();
        m_pos += sizeof(T);
        return v;
    }
    std::string string(int32_t max_len) {
        const auto len = value<int32_t>();
        if (len <= 0 || len > max_len)
            invalid("sigproc: " + m_path + " has a header string of length " + std::to_string(len) +
                    " at byte " + std::to_string(m_pos - 4) + " (not a SIGPROC header?)");
        std::string s(static_cast<size_t>(len), '\0');
        m_in.read(s.data(), len);
        if (!m_in)
            truncated();
        m_pos += static_cast<uint64_t>(len);
        return s;
    }
    uint64_t pos() const { return m_pos; }
    uint64_t file_size() {
        const auto here = m_in.tellg();
        m_in.seekg(0, std::ios::end);
        const auto end = m_in.tellg();
        m_in.seekg(here);
        return static_cast<uint64_t>(end);
    }

private:
    [[noreturn]] void truncated() { invalid("sigproc: " + m_path + " ends inside its header"); }
    std::ifstream m_in;
    std::string m_path;
    uint64_t m_pos = 0;
};

} // namespace

frost_sigproc_header read_sigproc_header(const std::string& path) {
    constexpr int32_t kMaxKey     = 64;
    constexpr int32_t kMaxValue   = 4096;
    constexpr uint64_t kMaxHeader = uint64_t{1} << 20;
    Reader r(path);
    if (r.string(kMaxKey) != "HEADER_START")
        invalid("sigproc: " + path + " does not start with HEADER_START");
    frost_sigproc_header h{};
    h.nifs           = 1;
    h.data_type      = 1;
    bool have_nchans = false, have_nbits = false, have_tsamp = false, have_fch1 = false, have_foff = false;
    while (true) {
        if (r.pos() > kMaxHeader)
            invalid("sigproc: " + path + " header is longer than 1 MiB");
        const std::string key = r.string(kMaxKey);
        if (key == "HEADER_END")
            break;
        switch (kind_of(key)) {
        case Kind::Int: {
            const int32_t v = r.value<int32_t>();
            if (key == "telescope_id")
                h.telescope_id = v;
            else if (key == "machine_id")
                h.machine_id = v;
            else if (key == "data_type")
                h.data_type = v;
            else if (key == "nbits") {
                h.nbits    = v;
                have_nbits = true;
            } else if (key == "nchans") {
                if (v <= 0)
                    invalid("sigproc: " + path + " has nchans " + std::to_string(v));
                h.nchans    = static_cast<uint64_t>(v);
                have_nchans = true;
            } else if (key == "nifs")
                h.nifs = v;
            else if (key == "nbeams")
                h.nbeams = v;
            else if (key == "ibeam")
                h.ibeam = v;
            else if (key == "nsamples")
                h.nsamples = static_cast<uint64_t>(v < 0 ? 0 : v);
            break;
        }
        case Kind::Double: {
            const double v = r.value<double>();
            if (key == "tstart")
                h.tstart = v;
            else if (key == "tsamp") {
                h.tsamp    = v;
                have_tsamp = true;
            } else if (key == "fch1") {
                h.fch1    = v;
                have_fch1 = true;
            } else if (key == "foff") {
                h.foff    = v;
                have_foff = true;
            } else if (key == "src_raj")
                h.src_raj = v;
            else if (key == "src_dej")
                h.src_dej = v;
            else if (key == "refdm")
                h.refdm = v;
            break;
        }
        case Kind::String: {
            const std::string v = r.string(kMaxValue);
            if (key == "source_name") {
                const size_t n = std::min(v.size(), sizeof(h.source_name) - 1);
                std::memcpy(h.source_name, v.data(), n);
                h.source_name[n] = '\0';
            }
            break;
        }
        case Kind::Byte:
            h.signed_samples = r.value<int8_t>() != 0 ? 1 : 0;
            break;
        case Kind::Marker:
            break;
        }
    }
    if (!have_nchans || !have_nbits || !have_tsamp || !have_fch1 || !have_foff)
        invalid("sigproc: " + path + " header lacks nchans, nbits, tsamp, fch1 or foff");
    if (h.nifs != 1)
        invalid("sigproc: " + path + " has nifs " + std::to_string(h.nifs) + "; only total intensity is searched");
    h.header_bytes     = r.pos();
    const uint64_t row = h.nchans * static_cast<uint64_t>(h.nbits > 0 ? h.nbits : 0);
    if (row == 0 || row % 8 != 0)
        invalid("sigproc: " + path + " rows are not whole bytes");
    const uint64_t size = r.file_size();
    h.row_bytes         = row / 8;
    h.data_rows         = size > h.header_bytes ? (size - h.header_bytes) / h.row_bytes : 0;
    return h;
}

frost_block_layout sigproc_layout(const frost_sigproc_header& h, uint64_t block_rows) {
    frost_block_layout l{};
    l.nchans     = h.nchans;
    l.max_nsamps = block_rows;
    switch (h.nbits) {
    case 1: l.dtype = FROST_UINT1; break;
    case 2: l.dtype = FROST_UINT2; break;
    case 4: l.dtype = FROST_UINT4; break;
    case 8: l.dtype = FROST_UINT8; break;
    case 16: l.dtype = FROST_UINT16; break;
    case 32: l.dtype = FROST_FLOAT32; break;
    default: invalid("sigproc: unsupported nbits " + std::to_string(h.nbits));
    }
    if (h.signed_samples != 0 && h.nbits != 32)
        invalid("sigproc: signed integer samples are not supported");
    l.tsamp = h.tsamp;
    l.f0    = h.fch1;
    l.df    = h.foff;
    return l;
}

} // namespace fb::io
