// Serving loop: many beams on one GPU, each with its RFI calibration and
// FDMT tails resident, gulps admitted as worker slots free up so one beam's
// host-side phases overlap other beams' kernels (continuous batching at the
// stream level), beams admitted by device memory, and per-gulp latency
// (arrival -> candidates ready) recorded for p50/p99.
#pragma once

#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "common.hpp"
#include "postprocess.hpp"
#include "rfi_cleaner.hpp"
#include "search_engine.hpp"

namespace fb::serve {

struct BeamSpec {
    frost_rfi_config rfi;
    std::vector<frost_channel_range> zap_chans;
    std::vector<frost_frequency_range> zap_freqs;
    frost_block_layout layout;
    float baseline_length;
    frost_dedisp_plan_config plan;
    frost_boxcar_config search;
};

/** One beam's resident state and its per-gulp body (Pipeline::execute_block's
 * hot path, lib/pipeline/pipeline.cpp:529-619). */
class Beam {
public:
    Beam(const BeamSpec& spec, int device);
    /** Allocates the beam's steady-state device buffers up front. */
    void preallocate() { m_cleaner->preallocate(); }
    /** Picks the engine's FDMT launch shape by measurement (cached per
     * geometry, so only the first beam of a shape pays). */
    void autotune() { m_engine->autotune(); }
    void set_residency(int32_t ctas_per_sm) { m_engine->set_residency(ctas_per_sm); }
    /** Cleans and searches one gulp (a block of max_nsamps rows, nread
     * valid, on the host or on the beam's device). */
    void process(const uint8_t* block, SizeType bytes, SizeType nread, bool on_device);
    /** The RFI half of process(): cleans and normalises the gulp on the
     * cleaner's stream and takes its channel mask into FDMT order; returns
     * the device waterfall. */
    const float* clean(const uint8_t* block, SizeType bytes, SizeType nread, bool on_device);
    /** The bookkeeping after a gulp's search: frost's searched-samples
     * accounting and the post-processing, if any. */
    void account(SizeType nread);
    fdmt::Engine& engine() { return *m_engine; }
    rfi::Cleaner& cleaner() { return *m_cleaner; }
    const std::vector<uint8_t>& fdmt_mask() const { return m_fdmt_mask; }
    SizeType gulp_nsamps() const { return m_spec.layout.max_nsamps; }
    std::vector<frost_candidate> results() const { return m_engine->results(); }
    std::vector<frost_candidate> drain();
    /** Adds CandidatePostprocessPlan after the search of every gulp
     * (Pipeline::publish, lib/pipeline/pipeline.cpp:478-493), on the device
     * over the engine's candidates. */
    void attach_postprocess(const frost_postprocess_config& cfg);
    bool has_postprocess() const { return m_post != nullptr; }
    const std::vector<frost_giant>& giants() const;
    uint64_t samples_searched() const { return m_searched; }
    /** Kernels launched by the last process() call. */
    uint64_t last_launches() const { return m_last_launches; }
    double tsamp() const { return m_spec.layout.tsamp; }
    SizeType device_bytes() const;
    SizeType block_bytes() const;

    /** Input staging (Server::set_staging): `slots` device blocks that host
     * gulps in pinned memory are copied into when they are submitted, on a
     * copy stream of their own, so that the copy of a queued gulp overlaps
     * the work on the gulp before it (0 releases them). */
    void set_staging(uint32_t slots);
    SizeType staging_bytes() const { return static_cast<SizeType>(m_stage.size()) * block_bytes(); }
    /** Starts the copy of a host gulp into a free slot; -1 when none is free
     * or the block is not in pinned memory (it is then copied when it is
     * processed). Called with the server's lock held. */
    int stage(const uint8_t* block, SizeType bytes);
    /** process() of a staged gulp: the beam's stream waits for its copy. */
    void process_staged(int slot, SizeType bytes, SizeType nread);
    /** Frees a slot after process_staged (server's lock held). */
    void unstage(int slot) { m_stage[static_cast<size_t>(slot)].busy = false; }
    ~Beam();

private:
    struct Stage {
        DeviceBuffer block;
        cudaEvent_t copied   = nullptr; // the host block is on the device
        cudaEvent_t consumed = nullptr; // the gulp that read it has run
        bool busy = false, used = false;
    };
    void release_staging();
    std::vector<Stage> m_stage;
    cudaStream_t m_copy = nullptr;
    BeamSpec m_spec;
    std::unique_ptr<rfi::Cleaner> m_cleaner;
    std::unique_ptr<fdmt::Engine> m_engine;
    std::unique_ptr<pp::PostprocessPlan> m_post;
    int m_device;
    bool m_descending;
    std::vector<uint8_t> m_fdmt_mask;
    uint64_t m_read = 0, m_searched = 0, m_max_delay = 0, m_last_launches = 0, m_last_nread = 0;
    void postprocess(bool final_call);
};

struct Request {
    uint64_t ticket;
    uint32_t beam;
    const uint8_t* block;
    SizeType bytes;
    SizeType nread;
    bool on_device;
    int slot = -1;   // staging slot holding the block, or -1
    double arrival;  // steady seconds
    double done = 0;
    bool finished = false;
    int status    = FROST_OK;
    std::string error;
    std::vector<frost_candidate> cands;
    std::vector<frost_giant> giants;
};

class Server {
public:
    Server(int device, SizeType memory_budget, uint32_t slots);
    ~Server();
    uint32_t add_beam(const BeamSpec& spec);
    void remove_beam(uint32_t beam);
    uint64_t submit(uint32_t beam, const uint8_t* block, SizeType bytes, SizeType nread,
                    bool on_device);
    /** Blocks until the ticket is done; moves its candidates out. */
    std::vector<frost_candidate> wait(uint64_t ticket, double* latency_s);
    /** As wait, moving out the gulp's post-processed giants instead. */
    std::vector<frost_giant> wait_giants(uint64_t ticket, double* latency_s);
    /** Caps the beam's level and search kernels at `ctas_per_sm` resident
     * CTAs per SM (fdmt::Engine::set_residency). */
    void set_residency(uint32_t beam, int32_t ctas_per_sm);
    /** Attaches a post-processor to an idle beam; its device memory is
     * charged against the server's budget. */
    void set_postprocess(uint32_t beam, const frost_postprocess_config& cfg);
    /** Gives an idle beam `slots` (0-4) input staging blocks
     * (Beam::set_staging), charged against the server's budget. */
    void set_staging(uint32_t beam, uint32_t slots);
    /** drain() of a beam with a post-processor: the final giants. */
    std::vector<frost_giant> drain_giants(uint32_t beam);
    frost_server_stats stats();
    void reset_stats();
    std::vector<frost_candidate> drain(uint32_t beam);

private:
    int m_device;
    SizeType m_budget, m_used = 0;
    std::mutex m_mu;
    std::condition_variable m_work_cv, m_done_cv;
    bool m_stop = false;
    uint64_t m_next_ticket = 1;
    uint32_t m_next_beam = 0;
    std::map<uint32_t, std::unique_ptr<Beam>> m_beams;
    std::map<uint32_t, std::deque<uint64_t>> m_queue; // per-beam FIFO of tickets
    std::map<uint32_t, bool> m_busy;
    std::map<uint32_t, bool> m_held; // a setter is reconfiguring the beam: submits do not stage
    std::map<uint32_t, SizeType> m_charge; // device bytes charged at admission
    std::map<uint64_t, std::shared_ptr<Request>> m_requests;
    std::vector<double> m_latencies;
    double m_beam_seconds = 0, m_first_arrival = -1, m_last_done = 0;
    uint64_t m_completed = 0, m_launches = 0;
    std::vector<std::thread> m_workers;

    void worker();
    bool pick(uint32_t& beam, std::shared_ptr<Request>& req);
    std::shared_ptr<Request> finish(uint64_t ticket, double* latency_s);
    Beam* hold(uint32_t beam, std::unique_lock<std::mutex>& lk);
    void release(uint32_t beam);
};

double now_seconds();

} // namespace fb::serve
