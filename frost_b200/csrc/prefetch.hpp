// Input staging for one beam: the B200 form of frost's GulpPrefetch
// (lib/pipeline/pipeline.cpp:105-262). A reader thread fills pinned host
// slots from a block source, copies each filled slot to its device slot on
// its own stream, and hands gulps out in order: the caller's stream waits on
// the copy's event (no host synchronisation) and a slot is refilled only
// after the work the caller enqueued on it has run.
#pragma once

#include <condition_variable>
#include <cstdint>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime_api.h>

#include "common.hpp"
#include "frost_b200.h"

namespace fb::staging {

class Prefetch {
public:
    Prefetch(SizeType block_rows, SizeType row_bytes, int depth, int device, frost_read_fn read, void* ctx);
    ~Prefetch();
    Prefetch(const Prefetch&)            = delete;
    Prefetch& operator=(const Prefetch&) = delete;

    /** The next gulp on the device (valid until the next call); nread = 0 at
     * the end of the source. `stream` (the caller's) is made to wait for the
     * gulp's copy. */
    const uint8_t* next(SizeType* nread, cudaStream_t stream);
    frost_prefetch_stats stats() const;

private:
    struct Slot {
        uint8_t* host = nullptr;
        uint8_t* dev  = nullptr;
        cudaEvent_t copied   = nullptr; // H2D done (on the copy stream)
        cudaEvent_t consumed = nullptr; // the caller's work on it done
        bool consumed_recorded = false;
        SizeType nread         = 0;
        bool ready             = false;
    };
    void run();

    SizeType m_rows, m_row_bytes;
    int m_device;
    frost_read_fn m_read;
    void* m_ctx;
    cudaStream_t m_copy = nullptr;
    std::vector<Slot> m_slots;
    int m_next_fill = 0, m_next_out = 0, m_handed = -1;
    int m_free;              // slots the reader may fill
    bool m_stop = false, m_eof = false;
    std::string m_error_msg;
    int m_error_code = FROST_OK;
    mutable std::mutex m_mu;
    std::condition_variable m_cv;
    std::thread m_thread;
    double m_read_s = 0, m_wait_s = 0;
    uint64_t m_gulps = 0, m_bytes = 0;
};

} // namespace fb::staging
