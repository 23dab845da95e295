// Input staging for one beam (see prefetch.hpp).

#include "prefetch.hpp"

#include <chrono>
#include <cstring>

namespace fb::staging {

namespace {
double since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}
} // namespace

Prefetch::Prefetch(SizeType block_rows, SizeType row_bytes, int depth, int device, frost_read_fn read,
                   void* ctx)
    : m_rows(block_rows), m_row_bytes(row_bytes), m_device(device), m_read(read), m_ctx(ctx), m_free(depth) {
    if (block_rows == 0 || row_bytes == 0)
        invalid("prefetch: block rows and row bytes must be positive");
    if (depth < 2 || depth > 8)
        invalid("prefetch: depth must be in [2, 8]");
    if (read == nullptr)
        invalid("prefetch: null block source");
    DeviceGuard g(device);
    FB_CUDA(cudaStreamCreateWithFlags(&m_copy, cudaStreamNonBlocking));
    m_slots.resize(static_cast<size_t>(depth));
    const SizeType bytes = block_rows * row_bytes;
    try {
        for (auto& s : m_slots) {
            FB_CUDA(cudaMallocHost(reinterpret_cast<void**>(&s.host), bytes));
            FB_CUDA(cudaMalloc(reinterpret_cast<void**>(&s.dev), bytes));
            FB_CUDA(cudaEventCreateWithFlags(&s.copied, cudaEventDisableTiming));
            FB_CUDA(cudaEventCreateWithFlags(&s.consumed, cudaEventDisableTiming));
        }
    } catch (...) {
        for (auto& s : m_slots) {
            if (s.host)
                cudaFreeHost(s.host);
            if (s.dev)
                cudaFree(s.dev);
            if (s.copied)
                cudaEventDestroy(s.copied);
            if (s.consumed)
                cudaEventDestroy(s.consumed);
        }
        cudaStreamDestroy(m_copy);
        throw;
    }
    m_thread = std::thread([this] { run(); });
}

Prefetch::~Prefetch() {
    {
        std::lock_guard<std::mutex> lk(m_mu);
        m_stop = true;
    }
    m_cv.notify_all();
    if (m_thread.joinable())
        m_thread.join();
    cudaSetDevice(m_device);
    cudaStreamSynchronize(m_copy);
    for (auto& s : m_slots) {
        cudaEventSynchronize(s.consumed);
        cudaFreeHost(s.host);
        cudaFree(s.dev);
        cudaEventDestroy(s.copied);
        cudaEventDestroy(s.consumed);
    }
    cudaStreamDestroy(m_copy);
}

void Prefetch::run() {
    cudaSetDevice(m_device);
    while (true) {
        int idx = -1;
        {
            std::unique_lock<std::mutex> lk(m_mu);
            m_cv.wait(lk, [&] { return m_stop || (m_free > 0 && !m_eof && m_error_code == FROST_OK); });
            if (m_stop)
                return;
            idx = m_next_fill;
            --m_free;
        }
        Slot& s = m_slots[static_cast<size_t>(idx)];
        long n  = 0;
        int code = FROST_OK;
        std::string msg;
        const auto t0 = std::chrono::steady_clock::now();
        try {
            // the slot's last copy out of its host buffer has finished, and
            // the device buffer is written only after the caller's work on it
            FB_CUDA(cudaEventSynchronize(s.copied));
            n = m_read(m_ctx, s.host, m_rows);
            if (n < 0 || static_cast<SizeType>(n) > m_rows) {
                code = FROST_ERR_IO;
                msg  = "prefetch: the block source returned " + std::to_string(n);
            } else {
                if (s.consumed_recorded)
                    FB_CUDA(cudaStreamWaitEvent(m_copy, s.consumed, 0));
                if (n > 0)
                    FB_CUDA(cudaMemcpyAsync(s.dev, s.host, static_cast<SizeType>(n) * m_row_bytes,
                                            cudaMemcpyHostToDevice, m_copy));
                FB_CUDA(cudaEventRecord(s.copied, m_copy));
            }
        } catch (const Error& e) {
            code = e.code();
            msg  = e.what();
        } catch (const std::exception& e) {
            code = FROST_ERR_IO;
            msg  = e.what();
        }
        const double dt = since(t0);
        {
            std::lock_guard<std::mutex> lk(m_mu);
            m_read_s += dt;
            if (code != FROST_OK) {
                m_error_code = code;
                m_error_msg  = msg;
            } else {
                s.nread     = static_cast<SizeType>(n);
                s.ready     = true;
                m_next_fill = (idx + 1) % static_cast<int>(m_slots.size());
                if (static_cast<SizeType>(n) < m_rows)
                    m_eof = true;
            }
        }
        m_cv.notify_all();
    }
}

const uint8_t* Prefetch::next(SizeType* nread, cudaStream_t stream) {
    DeviceGuard g(m_device);
    std::unique_lock<std::mutex> lk(m_mu);
    if (m_handed >= 0) {
        // the caller's work on the previous gulp: the slot is refilled after it
        Slot& prev = m_slots[static_cast<size_t>(m_handed)];
        if (stream != nullptr) {
            FB_CUDA(cudaEventRecord(prev.consumed, stream));
            prev.consumed_recorded = true;
        } else {
            prev.consumed_recorded = false;
        }
        m_handed = -1;
        ++m_free;
        m_cv.notify_all();
    }
    const auto t0 = std::chrono::steady_clock::now();
    Slot& s       = m_slots[static_cast<size_t>(m_next_out)];
    m_cv.wait(lk, [&] {
        return s.ready || m_error_code != FROST_OK || (m_eof && m_free == static_cast<int>(m_slots.size()));
    });
    m_wait_s += since(t0);
    if (!s.ready) {
        if (m_error_code != FROST_OK)
            throw Error(m_error_code, m_error_msg);
        *nread = 0; // the source has ended
        return nullptr;
    }
    if (s.nread == 0) {
        // the source ended on a whole gulp: the slot goes back unused
        s.ready = false;
        ++m_free;
        *nread = 0;
        return nullptr;
    }
    s.ready   = false;
    m_handed  = m_next_out;
    m_next_out = (m_next_out + 1) % static_cast<int>(m_slots.size());
    *nread    = s.nread;
    ++m_gulps;
    m_bytes += s.nread * m_row_bytes;
    lk.unlock();
    if (stream != nullptr)
        FB_CUDA(cudaStreamWaitEvent(stream, s.copied, 0));
    else
        FB_CUDA(cudaEventSynchronize(s.copied));
    return s.dev;
}

frost_prefetch_stats Prefetch::stats() const {
    std::lock_guard<std::mutex> lk(m_mu);
    return frost_prefetch_stats{m_gulps, m_bytes, m_read_s, m_wait_s};
}

} // namespace fb::staging
