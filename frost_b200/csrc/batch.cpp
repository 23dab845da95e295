// Batched multi-beam search (see batch.hpp).

#include "batch.hpp"

#include <algorithm>
#include <exception>
#include <map>
#include <thread>
#include <tuple>

namespace fb::serve {

Batch::Batch(int device, SizeType memory_budget) : m_device(device), m_budget(memory_budget) {
    int ndev = 0;
    FB_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev)
        invalid("batch: device " + std::to_string(device) + " does not exist");
    DeviceGuard g(device);
    if (m_budget == 0) {
        size_t free_b = 0, total_b = 0;
        FB_CUDA(cudaMemGetInfo(&free_b, &total_b));
        m_budget = static_cast<SizeType>(0.9 * static_cast<double>(free_b));
    }
    FB_CUDA(cudaStreamCreateWithFlags(&m_stream, cudaStreamNonBlocking));
    FB_CUDA(cudaEventCreateWithFlags(&m_done, cudaEventDisableTiming));
}

Batch::~Batch() {
    cudaSetDevice(m_device);
    if (m_stream != nullptr)
        cudaStreamSynchronize(m_stream);
    if (m_graph != nullptr)
        cudaGraphExecDestroy(m_graph);
    for (auto e : m_ready)
        cudaEventDestroy(e);
    if (m_done != nullptr)
        cudaEventDestroy(m_done);
    m_beams.clear();
    if (m_stream != nullptr)
        cudaStreamDestroy(m_stream);
}

uint32_t Batch::add_beam(const BeamSpec& spec) {
    DeviceGuard g(m_device);
    auto beam = std::make_unique<Beam>(spec, m_device);
    beam->autotune();
    beam->preallocate();
    const SizeType need = beam->device_bytes() + (SizeType{16} << 20);
    if (m_used + need > m_budget)
        throw Error(FROST_ERR_OUT_OF_MEMORY, "batch: beam needs " + std::to_string(need) + " device bytes; " +
                                                 std::to_string(m_budget - m_used) + " of the budget left");
    cudaEvent_t ev = nullptr;
    FB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    m_used += need;
    m_ready.push_back(ev);
    m_beams.push_back(std::move(beam));
    m_results.emplace_back();
    if (m_graph != nullptr) {
        FB_CUDA(cudaGraphExecDestroy(m_graph));
        m_graph = nullptr;
    }
    m_stats.beams        = m_beams.size();
    m_stats.device_bytes = m_used;
    return static_cast<uint32_t>(m_beams.size() - 1);
}

void Batch::use_graph(bool on) {
    DeviceGuard g(m_device);
    if (!on && m_graph != nullptr) {
        FB_CUDA(cudaStreamSynchronize(m_stream));
        FB_CUDA(cudaGraphExecDestroy(m_graph));
        m_graph = nullptr;
    }
    m_graph_on = on;
}

// The rounds of one batched gulp: in round r every beam that still has one
// runs its r-th (tile, level step); the level steps of all those beams are
// one launch per (kind, element type, stages) and their searches one
// launch per search shape.
void Batch::run_rounds(cudaStream_t s, frost_batch_stats& st) {
    const size_t K = m_beams.size();
    std::vector<int64_t> rounds(K);
    int64_t R = 0;
    for (size_t k = 0; k < K; ++k) {
        rounds[k] = m_beams[k]->engine().batch_rounds();
        R         = std::max(R, rounds[k]);
    }
    std::vector<fdmt::Engine::RoundWork> w(K);
    using LevelKey  = std::tuple<bool, bool, int32_t>;
    using SearchKey = std::tuple<int32_t, int32_t, int32_t, int32_t, int32_t, int32_t, int32_t, int32_t, int32_t,
                                 int32_t>;
    for (int64_t r = 0; r < R; ++r) {
        std::map<LevelKey, std::vector<fdmt::LevelSeg>> levels;
        for (size_t k = 0; k < K; ++k) {
            if (r >= rounds[k])
                continue;
            st.beam_launches += static_cast<uint64_t>(m_beams[k]->engine().batch_pre(r, s, w[k]));
            if (w[k].has_level)
                levels[{w[k].fused, w[k].fp16, w[k].fused ? w[k].stages : 0}].push_back(w[k].level);
        }
        for (auto& [key, segs] : levels) {
            fdmt::launch_level_segs(segs.data(), static_cast<int>(segs.size()), std::get<0>(key), std::get<1>(key),
                                    std::get<2>(key), s);
            st.merged_level_launches += (segs.size() + fdmt::kMaxLevelSegs - 1) / fdmt::kMaxLevelSegs;
        }
        std::map<SearchKey, std::vector<fdmt::SearchSeg>> searches;
        for (size_t k = 0; k < K; ++k) {
            if (r >= rounds[k])
                continue;
            st.beam_launches += static_cast<uint64_t>(m_beams[k]->engine().batch_mid(r, s, w[k]));
            if (!w[k].has_search)
                continue;
            const auto& p = w[k].search.p;
            searches[{w[k].search.fp16, w[k].chunk, p.nwidths, p.wmax, p.halo, p.peak_mode, p.trapezoid,
                      p.skip_cold, p.pow2_widths, p.n_valid}]
                .push_back(w[k].search);
        }
        for (auto& [key, segs] : searches) {
            fdmt::launch_search_segs(segs.data(), static_cast<int>(segs.size()), s, std::get<1>(key));
            st.merged_search_launches += (segs.size() + fdmt::kMaxSearchSegs - 1) / fdmt::kMaxSearchSegs;
        }
        for (size_t k = 0; k < K; ++k)
            if (r < rounds[k])
                st.beam_launches += static_cast<uint64_t>(m_beams[k]->engine().batch_post(r, s));
    }
    st.rounds += static_cast<uint64_t>(R);
}

void Batch::execute(const uint8_t* const* blocks, const SizeType* nread, bool on_device) {
    const size_t K = m_beams.size();
    if (K == 0)
        fail_state("batch: no beams");
    if (blocks == nullptr || nread == nullptr)
        invalid("batch: null blocks or nread");
    for (size_t k = 0; k < K; ++k)
        if (blocks[k] == nullptr || nread[k] == 0 || nread[k] > m_beams[k]->gulp_nsamps())
            invalid("batch: beam " + std::to_string(k) + " has no block or an invalid nread");
    DeviceGuard g(m_device);
    // RFI excision and normalisation of every beam, concurrently on the
    // beams' own streams (each cleaner synchronises only its stream)
    std::vector<const float*> wf(K, nullptr);
    std::vector<std::exception_ptr> errs(K);
    {
        std::vector<std::thread> th;
        th.reserve(K);
        for (size_t k = 0; k < K; ++k)
            th.emplace_back([&, k] {
                try {
                    cudaSetDevice(m_device);
                    wf[k] = m_beams[k]->clean(blocks[k], m_beams[k]->block_bytes(), nread[k], on_device);
                } catch (...) {
                    errs[k] = std::current_exception();
                }
            });
        for (auto& t : th)
            t.join();
    }
    for (auto& e : errs)
        if (e)
            std::rethrow_exception(e);
    // every engine takes its gulp on its own stream; the batch's stream
    // waits for all of them
    for (size_t k = 0; k < K; ++k) {
        auto& eng = m_beams[k]->engine();
        eng.batch_begin(wf[k], m_beams[k]->gulp_nsamps(), m_beams[k]->fdmt_mask().data(),
                        m_beams[k]->cleaner().stream());
        FB_CUDA(cudaEventRecord(m_ready[k], eng.stream()));
        FB_CUDA(cudaStreamWaitEvent(m_stream, m_ready[k], 0));
    }
    frost_batch_stats st{};
    if (m_graph_on) {
        if (m_graph == nullptr || m_graph_wf != wf) {
            if (m_graph != nullptr) {
                FB_CUDA(cudaGraphExecDestroy(m_graph));
                m_graph = nullptr;
            }
            cudaGraph_t graph = nullptr;
            FB_CUDA(cudaStreamBeginCapture(m_stream, cudaStreamCaptureModeThreadLocal));
            try {
                run_rounds(m_stream, st);
            } catch (...) {
                cudaStreamEndCapture(m_stream, &graph);
                if (graph != nullptr)
                    cudaGraphDestroy(graph);
                throw;
            }
            FB_CUDA(cudaStreamEndCapture(m_stream, &graph));
            const cudaError_t e = cudaGraphInstantiate(&m_graph, graph, 0);
            cudaGraphDestroy(graph);
            FB_CUDA(e);
            m_graph_wf     = wf;
            m_graph_counts = st;
        } else {
            m_stats.graph_replays += 1;
        }
        st = m_graph_counts;
        FB_CUDA(cudaGraphLaunch(m_graph, m_stream));
    } else {
        run_rounds(m_stream, st);
    }
    FB_CUDA(cudaEventRecord(m_done, m_stream));
    // results on every engine's stream after the batch's work
    std::exception_ptr first;
    for (size_t k = 0; k < K; ++k) {
        try {
            auto& eng = m_beams[k]->engine();
            FB_CUDA(cudaStreamWaitEvent(eng.stream(), m_done, 0));
            eng.batch_finish();
            m_results[k] = eng.results();
            m_beams[k]->account(nread[k]);
        } catch (...) {
            if (!first)
                first = std::current_exception();
        }
    }
    m_stats.executes += 1;
    m_stats.rounds += st.rounds;
    m_stats.merged_level_launches += st.merged_level_launches;
    m_stats.merged_search_launches += st.merged_search_launches;
    m_stats.beam_launches += st.beam_launches;
    if (first)
        std::rethrow_exception(first);
}

const std::vector<frost_candidate>& Batch::results(uint32_t beam) const {
    if (beam >= m_beams.size())
        invalid("batch: unknown beam");
    return m_results[beam];
}

std::vector<frost_candidate> Batch::drain(uint32_t beam) {
    if (beam >= m_beams.size())
        invalid("batch: unknown beam");
    DeviceGuard g(m_device);
    return m_beams[beam]->drain();
}

frost_batch_stats Batch::stats() const { return m_stats; }

} // namespace fb::serve
