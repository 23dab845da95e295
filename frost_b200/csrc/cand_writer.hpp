// The `.cand` candidate file: frost's 23 tab-separated columns per giant
// (include/frost/output/cand_writer.hpp:15-34), written from the giants the
// device post-processing returns.
#pragma once

#include <cstdint>
#include <cstdio>
#include <ctime>
#include <string>

#include "common.hpp"
#include "frost_b200.h"

namespace fb::output {

class CandWriter {
public:
    /** Creates missing parent directories; `dt` (seconds) turns sample
     * indices into the time columns. */
    CandWriter(const std::string& path, double dt, bool append);
    ~CandWriter();
    CandWriter(const CandWriter&)            = delete;
    CandWriter& operator=(const CandWriter&) = delete;

    /** One row per giant; sample-index columns offset by first_samp_idx. */
    void write(const frost_giant* giants, size_t n, uint64_t first_samp_idx);

private:
    std::FILE* m_file = nullptr;
    double m_dt;
    std::string m_path;
};

/** `YYYY-MM-DD-HH:MM:SS_BB.cand` (UTC; beam 1-based, at least 2 digits). */
std::string cand_filename(std::time_t utc, uint64_t beam);

} // namespace fb::output
