// Batched multi-beam search: one gulp of every beam of the batch in one
// pass. Each beam keeps its own cleaner, engine, calibration and FDMT
// histories (as a served beam does); the RFI stages run concurrently on the
// beams' own streams, then the searches run as rounds (one tile and level
// step of every beam per round) in which the level steps of all beams are
// one launch and the searches of all beams one launch, over segment tables
// (fdmt_kernels.hpp LevelSeg, search_kernels.hpp SearchSeg), on the
// batch's stream; the rounds are captured once as a CUDA graph and replayed
// while the beams' waterfalls stay where they are. Beams may differ in
// channel count, sample type, gulp length, DM range and plane count; each
// beam's launch shape comes from the engine's autotuner (cached per
// geometry). frost runs one engine per pipeline and one beam per process
// (lib/pipeline/pipeline.cpp:346-367); a beam's candidates here equal those
// of the same beam run alone.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "common.hpp"
#include "server.hpp"

namespace fb::serve {

class Batch {
public:
    /** memory_budget 0 = 90 % of the device's free memory. */
    Batch(int device, SizeType memory_budget);
    ~Batch();
    Batch(const Batch&)            = delete;
    Batch& operator=(const Batch&) = delete;

    /** Admits a beam (its buffers allocated now, its launch shape tuned);
     * FROST_ERR_OUT_OF_MEMORY when it would exceed the budget. */
    uint32_t add_beam(const BeamSpec& spec);
    /** One gulp of every beam: blocks[i] is beam i's whole block of
     * max_nsamps rows (host, or device when on_device), nread[i] valid. */
    void execute(const uint8_t* const* blocks, const SizeType* nread, bool on_device);
    const std::vector<frost_candidate>& results(uint32_t beam) const;
    std::vector<frost_candidate> drain(uint32_t beam);
    void use_graph(bool on);
    frost_batch_stats stats() const;

private:
    void run_rounds(cudaStream_t s, frost_batch_stats& st);
    int m_device;
    SizeType m_budget;
    SizeType m_used = 0;
    cudaStream_t m_stream = nullptr;
    cudaEvent_t m_done    = nullptr;
    std::vector<cudaEvent_t> m_ready;
    std::vector<std::unique_ptr<Beam>> m_beams;
    std::vector<std::vector<frost_candidate>> m_results;
    bool m_graph_on         = true;
    cudaGraphExec_t m_graph = nullptr;
    std::vector<const float*> m_graph_wf;
    frost_batch_stats m_graph_counts{};
    frost_batch_stats m_stats{};
};

} // namespace fb::serve
