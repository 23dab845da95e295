// SIGPROC filterbank header reader (see sigproc.cpp).
#pragma once

#include <cstdint>
#include <string>

#include "common.hpp"

namespace fb::io {

/** Parses the header of the SIGPROC filterbank at `path`; FROST_ERR_IO if
 * the file cannot be opened, FROST_ERR_INVALID_ARGUMENT if the header is
 * malformed, names an unknown keyword, lacks nchans / nbits / tsamp / fch1
 * / foff, or has nifs != 1. */
frost_sigproc_header read_sigproc_header(const std::string& path);

/** The BlockLayout of the file's rows for gulps of `block_rows` samples
 * (channel 0 at fch1, spacing foff). */
frost_block_layout sigproc_layout(const frost_sigproc_header& h, uint64_t block_rows);

} // namespace fb::io
