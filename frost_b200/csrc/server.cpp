// Serving loop (see server.hpp).

#include "server.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>

namespace fb::serve {

double now_seconds() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

Beam::Beam(const BeamSpec& spec, int device) : m_spec(spec), m_device(device) {
    frost_rfi_config c = spec.rfi;
    c.zap_chans        = spec.zap_chans.data();
    c.n_zap_chans      = spec.zap_chans.size();
    c.zap_freqs        = spec.zap_freqs.data();
    c.n_zap_freqs      = spec.zap_freqs.size();
    if (spec.plan.nchans != spec.layout.nchans || spec.plan.block_nsamps != spec.layout.max_nsamps)
        invalid("serve: plan and layout disagree on nchans or gulp length");
    m_cleaner    = std::make_unique<rfi::Cleaner>(c, spec.layout, spec.baseline_length, device);
    m_descending = spec.layout.df < 0.0;
    // Static zaps in FDMT order are the engine's constructor mask
    // (fdmt_kill_mask, lib/pipeline/pipeline.cpp:334-344).
    m_fdmt_mask = m_cleaner->channel_mask();
    if (m_descending)
        std::reverse(m_fdmt_mask.begin(), m_fdmt_mask.end());
    m_engine    = std::make_unique<fdmt::Engine>(spec.plan, spec.search, m_fdmt_mask.data(), 0, device);
    m_max_delay = static_cast<uint64_t>(m_engine->plan().dt_max());
}

SizeType Beam::block_bytes() const {
    return m_spec.layout.max_nsamps * m_spec.layout.nchans *
           static_cast<SizeType>(bits_of(m_spec.layout.dtype)) / 8;
}

SizeType Beam::device_bytes() const {
    return m_cleaner->memory_usage() + m_engine->device_bytes() + (m_post ? m_post->memory_usage() : 0) +
           staging_bytes();
}

Beam::~Beam() { release_staging(); }

void Beam::release_staging() {
    DeviceGuard g(m_device);
    if (m_copy != nullptr)
        cudaStreamSynchronize(m_copy);
    for (auto& st : m_stage) {
        if (st.consumed != nullptr) {
            cudaEventSynchronize(st.consumed);
            cudaEventDestroy(st.consumed);
        }
        if (st.copied != nullptr)
            cudaEventDestroy(st.copied);
    }
    m_stage.clear();
    if (m_copy != nullptr)
        cudaStreamDestroy(m_copy);
    m_copy = nullptr;
}

void Beam::set_staging(uint32_t slots) {
    if (slots > 4)
        invalid("serve: staging slots must be in [0, 4]");
    release_staging();
    if (slots == 0)
        return;
    DeviceGuard g(m_device);
    try {
        FB_CUDA(cudaStreamCreateWithFlags(&m_copy, cudaStreamNonBlocking));
        m_stage.resize(slots);
        for (auto& st : m_stage) {
            st.block.reserve(block_bytes());
            FB_CUDA(cudaEventCreateWithFlags(&st.copied, cudaEventDisableTiming));
            FB_CUDA(cudaEventCreateWithFlags(&st.consumed, cudaEventDisableTiming));
        }
    } catch (...) {
        release_staging();
        throw;
    }
}

int Beam::stage(const uint8_t* block, SizeType bytes) {
    if (m_stage.empty() || bytes != block_bytes())
        return -1;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, block) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    if (a.type != cudaMemoryTypeHost)
        return -1; // pageable: a copy from it would hold the caller
    for (size_t i = 0; i < m_stage.size(); ++i) {
        Stage& st = m_stage[i];
        if (st.busy)
            continue;
        DeviceGuard g(m_device);
        // the slot's last reader was queued before the slot was freed
        if (st.used)
            FB_CUDA(cudaStreamWaitEvent(m_copy, st.consumed, 0));
        FB_CUDA(cudaMemcpyAsync(st.block.get(), block, bytes, cudaMemcpyHostToDevice, m_copy));
        FB_CUDA(cudaEventRecord(st.copied, m_copy));
        st.busy = true;
        return static_cast<int>(i);
    }
    return -1;
}

void Beam::process_staged(int slot, SizeType bytes, SizeType nread) {
    Stage& st = m_stage[static_cast<size_t>(slot)];
    FB_CUDA(cudaStreamWaitEvent(m_cleaner->stream(), st.copied, 0));
    auto done = [&] {
        cudaEventRecord(st.consumed, m_cleaner->stream());
        st.used = true;
    };
    try {
        process(st.block.as<uint8_t>(), bytes, nread, true);
    } catch (...) {
        done();
        throw;
    }
    done();
}

void Beam::attach_postprocess(const frost_postprocess_config& cfg) {
    const frost_postprocess_layout lay{m_spec.layout.nchans, m_spec.layout.tsamp, m_spec.layout.df};
    m_post = std::make_unique<pp::PostprocessPlan>(cfg, lay, m_device);
}

const std::vector<frost_giant>& Beam::giants() const {
    static const std::vector<frost_giant> kNone;
    return m_post ? m_post->results() : kNone;
}

void Beam::postprocess(bool final_call) {
    if (!m_post)
        return;
    const uint64_t l0 = pp::launch_counter();
    m_post->execute(m_engine->device_results(), m_engine->results().size(), true, m_read, m_last_nread,
                    final_call, m_engine->frontier());
    m_last_launches += pp::launch_counter() - l0;
}

const float* Beam::clean(const uint8_t* block, SizeType bytes, SizeType nread, bool on_device) {
    if (bytes != block_bytes())
        invalid("serve: a gulp must be a whole block of max_nsamps rows");
    const float* wf = m_cleaner->execute_normalized(block, bytes, nread, on_device, nullptr);
    m_fdmt_mask     = m_cleaner->channel_mask();
    if (m_descending)
        std::reverse(m_fdmt_mask.begin(), m_fdmt_mask.end());
    return wf;
}

void Beam::account(SizeType nread) {
    // samples searched: frost's accounting, lib/pipeline/pipeline.cpp:610-614
    m_read += nread;
    m_last_nread            = nread;
    const uint64_t previous = m_read - nread;
    if (m_read > m_max_delay)
        m_searched += m_read - std::max(previous, m_max_delay);
    postprocess(false);
}

void Beam::process(const uint8_t* block, SizeType bytes, SizeType nread, bool on_device) {
    const uint64_t l0 = m_cleaner->launches();
    const float* wf   = clean(block, bytes, nread, on_device);
    m_engine->execute(wf, m_spec.layout.max_nsamps, true, m_fdmt_mask.data(), m_cleaner->stream());
    m_last_launches = (m_cleaner->launches() - l0) + m_engine->last_launches();
    account(nread);
}

std::vector<frost_candidate> Beam::drain() {
    m_engine->drain();
    postprocess(true);
    return m_engine->results();
}

Server::Server(int device, SizeType memory_budget, uint32_t slots)
    : m_device(device), m_budget(memory_budget) {
    if (slots == 0 || slots > 64)
        invalid("serve: slots must be in [1, 64]");
    int ndev = 0;
    FB_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev)
        invalid("serve: device " + std::to_string(device) + " does not exist");
    if (m_budget == 0) {
        DeviceGuard g(device);
        size_t free_b = 0, total_b = 0;
        FB_CUDA(cudaMemGetInfo(&free_b, &total_b));
        m_budget = static_cast<SizeType>(0.9 * static_cast<double>(free_b));
    }
    for (uint32_t i = 0; i < slots; ++i)
        m_workers.emplace_back([this] { worker(); });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lk(m_mu);
        m_stop = true;
    }
    m_work_cv.notify_all();
    for (auto& t : m_workers)
        t.join();
}

uint32_t Server::add_beam(const BeamSpec& spec) {
    // Admission by device memory: build the beam (its buffers are sized by
    // its plan), then keep it only if the server's budget still holds.
    DeviceGuard g(m_device);
    auto beam = std::make_unique<Beam>(spec, m_device);
    // every steady-state buffer is allocated now, so the charge is the
    // beam's footprint (plus a margin for small per-gulp transfers)
    beam->autotune();
    beam->preallocate();
    const SizeType need = beam->device_bytes() + (SizeType{16} << 20);
    std::lock_guard<std::mutex> lk(m_mu);
    if (m_used + need > m_budget)
        throw Error(FROST_ERR_OUT_OF_MEMORY,
                    "serve: beam needs " + std::to_string(need) + " device bytes; " +
                        std::to_string(m_budget - m_used) + " of the budget left");
    m_used += need;
    const uint32_t id = m_next_beam++;
    m_beams[id]       = std::move(beam);
    m_queue[id];
    m_busy[id]   = false;
    m_held[id]   = false;
    m_charge[id] = need;
    return id;
}

void Server::remove_beam(uint32_t beam) {
    std::unique_lock<std::mutex> lk(m_mu);
    auto it = m_beams.find(beam);
    if (it == m_beams.end())
        invalid("serve: unknown beam");
    m_done_cv.wait(lk, [&] { return !m_busy[beam] && m_queue[beam].empty(); });
    m_used -= std::min(m_used, m_charge[beam]);
    m_beams.erase(it);
    m_charge.erase(beam);
    m_queue.erase(beam);
    m_busy.erase(beam);
    m_held.erase(beam);
}

uint64_t Server::submit(uint32_t beam, const uint8_t* block, SizeType bytes, SizeType nread,
                        bool on_device) {
    if (block == nullptr)
        invalid("serve: null block");
    std::lock_guard<std::mutex> lk(m_mu);
    if (m_beams.find(beam) == m_beams.end())
        invalid("serve: unknown beam");
    auto req     = std::make_shared<Request>();
    req->ticket  = m_next_ticket++;
    req->beam    = beam;
    req->block   = block;
    req->bytes   = bytes;
    req->nread     = nread;
    req->on_device = on_device;
    // Staging touches the beam's slots and copy stream, which a setter
    // holding the beam may be replacing; such a gulp is uploaded when it is
    // processed instead.
    if (!on_device && !m_held[beam])
        req->slot = m_beams[beam]->stage(block, bytes);
    req->arrival = now_seconds();
    if (m_first_arrival < 0)
        m_first_arrival = req->arrival;
    m_requests[req->ticket] = req;
    m_queue[beam].push_back(req->ticket);
    m_work_cv.notify_one();
    return req->ticket;
}

// The oldest queued gulp of a beam that is not being processed (a beam's
// gulps run in order: its FDMT history carries from one to the next).
bool Server::pick(uint32_t& beam, std::shared_ptr<Request>& req) {
    double best = 0;
    bool found  = false;
    for (auto& [id, q] : m_queue) {
        if (q.empty() || m_busy[id])
            continue;
        const auto& r = m_requests[q.front()];
        if (!found || r->arrival < best) {
            best  = r->arrival;
            beam  = id;
            req   = r;
            found = true;
        }
    }
    if (found) {
        m_queue[beam].pop_front();
        m_busy[beam] = true;
    }
    return found;
}

void Server::worker() {
    cudaSetDevice(m_device);
    while (true) {
        uint32_t beam = 0;
        std::shared_ptr<Request> req;
        Beam* b = nullptr;
        {
            std::unique_lock<std::mutex> lk(m_mu);
            m_work_cv.wait(lk, [&] { return m_stop || pick(beam, req); });
            if (m_stop && !req)
                return;
            b = m_beams[beam].get();
        }
        int status = FROST_OK;
        std::string err;
        std::vector<frost_candidate> cands;
        std::vector<frost_giant> giants;
        uint64_t launches = 0;
        try {
            if (req->slot >= 0)
                b->process_staged(req->slot, req->bytes, req->nread);
            else
                b->process(req->block, req->bytes, req->nread, req->on_device);
            cands    = b->results();
            launches = b->last_launches();
            if (b->has_postprocess())
                giants = b->giants();
        } catch (const Error& e) {
            status = e.code();
            err    = e.what();
        } catch (const std::exception& e) {
            status = FROST_ERR_INTERNAL;
            err    = e.what();
        }
        {
            std::lock_guard<std::mutex> lk(m_mu);
            req->done     = now_seconds();
            req->status   = status;
            req->error    = err;
            req->cands    = std::move(cands);
            req->giants   = std::move(giants);
            req->finished = true;
            m_busy[beam]  = false;
            if (req->slot >= 0)
                b->unstage(req->slot);
            if (status == FROST_OK) {
                m_latencies.push_back(req->done - req->arrival);
                m_beam_seconds += static_cast<double>(req->nread) * b->tsamp();
                m_last_done = std::max(m_last_done, req->done);
                m_launches += launches;
                ++m_completed;
            }
        }
        m_done_cv.notify_all();
        m_work_cv.notify_all();
    }
}

std::shared_ptr<Request> Server::finish(uint64_t ticket, double* latency_s) {
    std::unique_lock<std::mutex> lk(m_mu);
    auto it = m_requests.find(ticket);
    if (it == m_requests.end())
        invalid("serve: unknown ticket");
    auto req = it->second;
    m_done_cv.wait(lk, [&] { return req->finished; });
    m_requests.erase(ticket);
    if (req->status != FROST_OK)
        throw Error(req->status, req->error);
    if (latency_s != nullptr)
        *latency_s = req->done - req->arrival;
    return req;
}

std::vector<frost_candidate> Server::wait(uint64_t ticket, double* latency_s) {
    return std::move(finish(ticket, latency_s)->cands);
}

std::vector<frost_giant> Server::wait_giants(uint64_t ticket, double* latency_s) {
    return std::move(finish(ticket, latency_s)->giants);
}

/** Waits until the beam is idle with nothing queued and marks it busy. */
Beam* Server::hold(uint32_t beam, std::unique_lock<std::mutex>& lk) {
    auto it = m_beams.find(beam);
    if (it == m_beams.end())
        invalid("serve: unknown beam");
    m_done_cv.wait(lk, [&] { return !m_busy[beam] && m_queue[beam].empty(); });
    m_busy[beam] = true;
    m_held[beam] = true;
    return it->second.get();
}

void Server::release(uint32_t beam) {
    {
        std::lock_guard<std::mutex> lk(m_mu);
        m_busy[beam] = false;
        m_held[beam] = false;
    }
    m_work_cv.notify_all();
}

std::vector<frost_candidate> Server::drain(uint32_t beam) {
    std::unique_lock<std::mutex> lk(m_mu);
    Beam* b = hold(beam, lk);
    lk.unlock();
    std::vector<frost_candidate> out;
    try {
        out = b->drain();
    } catch (...) {
        release(beam);
        throw;
    }
    release(beam);
    return out;
}

std::vector<frost_giant> Server::drain_giants(uint32_t beam) {
    std::unique_lock<std::mutex> lk(m_mu);
    Beam* b = hold(beam, lk);
    lk.unlock();
    std::vector<frost_giant> out;
    try {
        if (!b->has_postprocess())
            invalid("serve: beam has no post-processor");
        b->drain();
        out = b->giants();
    } catch (...) {
        release(beam);
        throw;
    }
    release(beam);
    return out;
}

void Server::set_residency(uint32_t beam, int32_t ctas_per_sm) {
    std::unique_lock<std::mutex> lk(m_mu);
    Beam* b = hold(beam, lk);
    lk.unlock();
    try {
        DeviceGuard g(m_device);
        b->set_residency(ctas_per_sm);
    } catch (...) {
        release(beam);
        throw;
    }
    release(beam);
}

void Server::set_postprocess(uint32_t beam, const frost_postprocess_config& cfg) {
    std::unique_lock<std::mutex> lk(m_mu);
    Beam* b = hold(beam, lk);
    lk.unlock();
    try {
        DeviceGuard g(m_device);
        if (b->has_postprocess())
            invalid("serve: beam already has a post-processor");
        const SizeType need = pp::PostprocessPlan::estimate_memory(cfg);
        {
            std::lock_guard<std::mutex> g2(m_mu);
            if (m_budget != 0 && m_used + need > m_budget)
                throw Error(FROST_ERR_OUT_OF_MEMORY, "serve: the post-processor does not fit the memory budget");
            m_used += need;
            m_charge[beam] += need;
        }
        try {
            b->attach_postprocess(cfg);
        } catch (...) {
            std::lock_guard<std::mutex> g2(m_mu);
            m_used -= need;
            m_charge[beam] -= need;
            throw;
        }
    } catch (...) {
        release(beam);
        throw;
    }
    release(beam);
}

void Server::set_staging(uint32_t beam, uint32_t slots) {
    std::unique_lock<std::mutex> lk(m_mu);
    Beam* b = hold(beam, lk);
    lk.unlock();
    try {
        if (slots > 4)
            invalid("serve: staging slots must be in [0, 4]");
        const SizeType had  = b->staging_bytes();
        const SizeType need = static_cast<SizeType>(slots) * b->block_bytes();
        {
            std::lock_guard<std::mutex> g2(m_mu);
            if (need > had && m_budget != 0 && m_used + (need - had) > m_budget)
                throw Error(FROST_ERR_OUT_OF_MEMORY, "serve: the staging blocks do not fit the memory budget");
            m_used = m_used - had + need;
            m_charge[beam] = m_charge[beam] - had + need;
        }
        try {
            b->set_staging(slots);
        } catch (...) {
            std::lock_guard<std::mutex> g2(m_mu);
            m_used = m_used - need + b->staging_bytes();
            m_charge[beam] = m_charge[beam] - need + b->staging_bytes();
            throw;
        }
    } catch (...) {
        release(beam);
        throw;
    }
    release(beam);
}

void Server::reset_stats() {
    std::lock_guard<std::mutex> lk(m_mu);
    m_latencies.clear();
    m_beam_seconds  = 0;
    m_first_arrival = -1;
    m_last_done     = 0;
    m_completed     = 0;
    m_launches      = 0;
}

frost_server_stats Server::stats() {
    std::lock_guard<std::mutex> lk(m_mu);
    frost_server_stats s{};
    s.completed    = m_completed;
    s.beams        = m_beams.size();
    s.device_bytes = m_used;
    s.beam_seconds = m_beam_seconds;
    s.wall_seconds = m_first_arrival >= 0 && m_completed > 0 ? m_last_done - m_first_arrival : 0.0;
    s.launches     = m_launches;
    if (!m_latencies.empty()) {
        std::vector<double> l = m_latencies;
        std::sort(l.begin(), l.end());
        auto q = [&](double f) {
            const double pos = f * static_cast<double>(l.size() - 1);
            return l[static_cast<size_t>(std::llround(pos))];
        };
        s.p50_latency_s = q(0.5);
        s.p99_latency_s = q(0.99);
        s.max_latency_s = l.back();
    }
    return s;
}

} // namespace fb::serve
