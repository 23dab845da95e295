// `.cand` writer (see cand_writer.hpp). Each value is printed the way
// frost's writer prints it (lib/output/cand_writer.cpp:40-71): floats as an
// ostream prints them (the shortest of %f / %e at 6 significant digits, i.e.
// "%g"), integers in decimal, the two time columns as doubles with 10
// significant digits ("%.10g").

#include "cand_writer.hpp"

#include <cerrno>
#include <cstring>
#include <filesystem>
#include <system_error>

namespace fb::output {

namespace {
void ensure_parent_dir(const std::string& path) {
    const auto parent = std::filesystem::path(path).parent_path();
    if (parent.empty())
        return;
    std::error_code ec;
    std::filesystem::create_directories(parent, ec);
    if (ec)
        throw Error(FROST_ERR_IO, "Cannot create output directory " + parent.string() + ": " + ec.message());
}

uint64_t box_width(const frost_giant& g) {
    if (g.filter_width > 0)
        return g.filter_width;
    return uint64_t{1} << (g.filter_idx < 63 ? g.filter_idx : 63);
}
} // namespace

CandWriter::CandWriter(const std::string& path, double dt, bool append) : m_dt(dt), m_path(path) {
    ensure_parent_dir(path);
    m_file = std::fopen(path.c_str(), append ? "a" : "w");
    if (m_file == nullptr)
        throw Error(FROST_ERR_IO, "Failed to open candidate file: " + path);
}

CandWriter::~CandWriter() {
    if (m_file != nullptr)
        std::fclose(m_file);
}

void CandWriter::write(const frost_giant* giants, size_t n, uint64_t first) {
    for (size_t i = 0; i < n; ++i) {
        const frost_giant& g = giants[i];
        const uint64_t samp  = first + g.samp_idx;
        const bool best_ext  = g.has_location_best != 0 || g.snr_best > g.snr;
        const float best_snr = g.snr_best > g.snr ? g.snr_best : g.snr;
        // strongest_location(): location_best, else the row's own
        const uint64_t loc_samp = g.has_location_best ? g.loc_samp_idx : g.samp_idx;
        const float loc_dm      = g.has_location_best ? g.loc_dm : g.dm;
        const uint64_t loc_w    = g.has_location_best ? g.loc_filter_width : box_width(g);
        const float loc_lo      = g.has_location_best ? g.loc_f_low : g.f_low;
        const float loc_hi      = g.has_location_best ? g.loc_f_high : g.f_high;
        const uint64_t best_sample = first + loc_samp;
        std::fprintf(m_file,
                     "%g\t%llu\t%.10g\t%llu\t%llu\t%g\t%llu\t%llu\t%llu\t%g\t%g\t%llu\t%llu\t%g\t%llu\t%llu\t%llu\t"
                     "%llu\t%.10g\t%g\t%llu\t%g\t%g\n",
                     static_cast<double>(g.snr), static_cast<unsigned long long>(samp),
                     static_cast<double>(samp) * m_dt, static_cast<unsigned long long>(g.filter_idx),
                     static_cast<unsigned long long>(g.dm_idx), static_cast<double>(g.dm),
                     static_cast<unsigned long long>(g.members), static_cast<unsigned long long>(first + g.begin),
                     static_cast<unsigned long long>(first + g.end), static_cast<double>(g.f_low),
                     static_cast<double>(g.f_high), static_cast<unsigned long long>(g.chan_begin),
                     static_cast<unsigned long long>(g.chan_end), static_cast<double>(best_snr),
                     static_cast<unsigned long long>(best_ext ? g.best_chan_begin : g.chan_begin),
                     static_cast<unsigned long long>(best_ext ? g.best_chan_end : g.chan_end),
                     static_cast<unsigned long long>(g.n_extents), static_cast<unsigned long long>(best_sample),
                     static_cast<double>(best_sample) * m_dt, static_cast<double>(loc_dm),
                     static_cast<unsigned long long>(loc_w), static_cast<double>(loc_lo),
                     static_cast<double>(loc_hi));
    }
    if (std::fflush(m_file) != 0 || std::ferror(m_file))
        throw Error(FROST_ERR_IO, "Failed writing candidate file (disk full?)");
}

std::string cand_filename(std::time_t utc, uint64_t beam) {
    std::tm tm{};
    if (gmtime_r(&utc, &tm) == nullptr)
        invalid("Candidate filename UTC is out of range");
    char buf[32];
    const size_t len = std::strftime(buf, sizeof(buf), "%Y-%m-%d-%H:%M:%S", &tm);
    if (len == 0)
        throw Error(FROST_ERR_INTERNAL, "Cannot format candidate filename UTC");
    char out[64];
    std::snprintf(out, sizeof(out), "%.*s_%02llu.cand", static_cast<int>(len), buf,
                  static_cast<unsigned long long>(beam));
    return out;
}

} // namespace fb::output
