// Device kernels of frost's candidate post-processing
// (lib/search/postprocess.cpp:67-241 and the plans it calls).
//
// Layout: giants are 160-byte frost_giant rows; the friends-of-friends
// sweep reads thirteen time-ordered columns instead (88 bytes a row,
// L2-resident at a few hundred thousand rows). Orderings the reference gets
// from std::sort / std::stable_sort come from one stable LSD radix sort of
// (64-bit key, 32-bit row) pairs, 8 bits a pass, keys packed from the
// fields' value ranges so a pass is spent only on bits that vary.
// Union-find links the larger root under the smaller with atomicCAS, so a
// component's root is its smallest row index whatever order the edges are
// found in: the labels equal the reference's sequential union-find.
//
// Built with --fmad=false: the predicates of pp_math.cuh must round like
// the reference's strict-IEEE host code.

#include <atomic>
#include <utility>

#include "common.hpp"
#include "postprocess_kernels.hpp"
#include "pp_math.cuh"

namespace fb::pp {

namespace {

std::atomic<u64> g_launches{0};

constexpr int kThreads = 256;
constexpr int kItems   = 8;
static_assert(kThreads * kItems == static_cast<int>(kTile), "tile");

inline unsigned blocks_for(size_t n, int per = kThreads) {
    return static_cast<unsigned>((n + per - 1) / per);
}

inline void count() { g_launches.fetch_add(1, std::memory_order_relaxed); }

__device__ __forceinline__ u32 lanemask_lt() {
    u32 m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

/** Order-preserving unsigned image of a float (NaN maps to 0, below all). */
__device__ __forceinline__ u32 ordered_bits(float x) {
    if (x != x)
        return 0u;
    const u32 b = __float_as_uint(x);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__device__ __forceinline__ u64 field_value(int kind, const frost_giant& g, u32 row, const u32* aux32,
                                           const u64* aux64) {
    switch (kind) {
    case kKeyPlane: return g.plane;
    case kKeyDmIdx: return g.dm_idx;
    case kKeyFilter: return g.filter_idx;
    case kKeySamp: return g.samp_idx;
    case kKeySnrDesc: return static_cast<u64>(0xFFFFFFFFu - ordered_bits(g.snr));
    case kKeySpanDesc: return ~span_of(g.chan_begin, g.chan_end);
    case kKeyAux32: return aux32[row];
    case kKeyAux64: return aux64[row];
    default: return 0;
    }
}

// ---- union-find ------------------------------------------------------------

/** Root of x with path halving; parent[x] <= x always holds. */
__device__ __forceinline__ u32 find_root(volatile u32* parent, u32 x) {
    while (true) {
        const u32 px = parent[x];
        if (px == x)
            return x;
        const u32 gp = parent[px];
        if (gp == px)
            return px;
        parent[x] = gp;
        x         = gp;
    }
}

/** Links the larger root under the smaller (retrying if a root was linked
 * meanwhile). */
__device__ __forceinline__ void unite(volatile u32* parent, u32 a, u32 b) {
    a = find_root(parent, a);
    b = find_root(parent, b);
    while (a != b) {
        if (a > b) {
            const u32 t = a;
            a           = b;
            b           = t;
        }
        const u32 old = atomicCAS(const_cast<u32*>(parent) + b, b, a);
        if (old == b)
            return;
        b = find_root(parent, old);
        a = find_root(parent, a);
    }
}

// ---- generic kernels --------------------------------------------------------

__global__ void k_iota(u32* v, size_t n) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n)
        v[i] = static_cast<u32>(i);
}

__global__ void k_rs_hist(const u64* __restrict__ keys, size_t n, int shift, u32* __restrict__ hist,
                          u32 nblk) {
    __shared__ u32 h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const size_t base = blockIdx.x * kTile;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        const size_t i = base + j * kThreads + threadIdx.x;
        if (i < n)
            atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[static_cast<size_t>(threadIdx.x) * nblk + blockIdx.x] = h[threadIdx.x];
}

/** In-place exclusive scan of a[0, total) by one block of 1024 threads;
 * *sum = the total when sum is given. */
__global__ void k_scan_single(u32* __restrict__ a, size_t total, u32* sum) {
    __shared__ u32 ws[32];
    const size_t per = (total + blockDim.x - 1) / blockDim.x;
    const size_t b   = threadIdx.x * per;
    const size_t e   = b + per < total ? b + per : total;
    u32 s            = 0;
    for (size_t i = b; i < e; ++i)
        s += a[i];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    u32 x          = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const u32 y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o)
            x += y;
    }
    if (lane == 31)
        ws[w] = x;
    __syncthreads();
    if (w == 0) {
        u32 v = lane < static_cast<int>(blockDim.x >> 5) ? ws[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const u32 y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o)
                v += y;
        }
        ws[lane] = v;
    }
    __syncthreads();
    u32 run = x - s + (w > 0 ? ws[w - 1] : 0u);
    for (size_t i = b; i < e; ++i) {
        const u32 v = a[i];
        a[i]        = run;
        run += v;
    }
    if (sum != nullptr && threadIdx.x == blockDim.x - 1)
        *sum = ws[(blockDim.x >> 5) - 1];
}

/** Stable scatter of one 8-bit digit: items of a tile keep their order
 * (round j holds tile rows j*256 .. j*256+255; ranks inside a warp come
 * from __match_any_sync, across warps from per-digit prefix counts). */
__global__ void k_rs_scatter(const u64* __restrict__ kin, const u32* __restrict__ vin, u64* __restrict__ kout,
                             u32* __restrict__ vout, size_t n, int shift, const u32* __restrict__ hist,
                             u32 nblk) {
    __shared__ u32 s_run[256];
    __shared__ u32 s_w[kThreads / 32][256];
    const int t = threadIdx.x, warp = t >> 5;
    s_run[t]          = hist[static_cast<size_t>(t) * nblk + blockIdx.x];
    const size_t base = blockIdx.x * kTile;
    for (int j = 0; j < kItems; ++j) {
#pragma unroll
        for (int w = 0; w < kThreads / 32; ++w)
            s_w[w][t] = 0;
        __syncthreads();
        const size_t i    = base + j * kThreads + t;
        const bool valid  = i < n;
        const u64 k       = valid ? kin[i] : 0;
        const u32 v       = valid ? vin[i] : 0;
        const u32 d       = valid ? static_cast<u32>((k >> shift) & 255u) : 256u;
        const u32 peers   = __match_any_sync(0xffffffffu, d);
        const u32 rank    = __popc(peers & lanemask_lt());
        if (valid && rank == 0)
            s_w[warp][d] = __popc(peers);
        __syncthreads();
        {
            u32 run = s_run[t];
#pragma unroll
            for (int w = 0; w < kThreads / 32; ++w) {
                const u32 c = s_w[w][t];
                s_w[w][t]   = run;
                run += c;
            }
            s_run[t] = run;
        }
        __syncthreads();
        if (valid) {
            const u32 pos = s_w[warp][d] + rank;
            kout[pos]     = k;
            vout[pos]     = v;
        }
        __syncthreads();
    }
}

__global__ void k_keys(const frost_giant* __restrict__ rows, const u32* __restrict__ perm, size_t n,
                       KeySpec spec, const u32* __restrict__ aux32, const u64* __restrict__ aux64,
                       const u32* __restrict__ keep, u64* __restrict__ keys) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= n)
        return;
    const u32 row       = perm[i];
    const bool kept     = keep == nullptr || keep[row] != 0;
    const frost_giant& g = rows[row];
    u64 key             = 0;
    for (int f = 0; f < spec.n; ++f) {
        u64 v;
        if (spec.f[f].kind == kKeyDropped)
            v = kept ? 0 : 1;
        else if (!kept)
            v = spec.f[f].lo;
        else
            v = field_value(spec.f[f].kind, g, row, aux32, aux64);
        key |= (v - spec.f[f].lo) << spec.f[f].shift;
    }
    keys[i] = key;
}

__device__ __forceinline__ u64 shfl_u64(u64 v, int o) {
    return __shfl_xor_sync(0xffffffffu, v, o);
}

__global__ void k_ranges(const frost_giant* __restrict__ rows, size_t n, RangeKinds kinds,
                         const u32* __restrict__ aux32, const u64* __restrict__ aux64,
                         const u32* __restrict__ keep, unsigned long long* out) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    const bool ok  = i < n && (keep == nullptr || keep[i] != 0);
    for (int k = 0; k < kinds.n; ++k) {
        u64 lo = ~u64{0}, hi = 0;
        if (ok) {
            lo = hi = field_value(kinds.kind[k], rows[i], static_cast<u32>(i), aux32, aux64);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const u64 l2 = shfl_u64(lo, o), h2 = shfl_u64(hi, o);
            lo           = l2 < lo ? l2 : lo;
            hi           = h2 > hi ? h2 : hi;
        }
        if ((threadIdx.x & 31) == 0 && lo <= hi) {
            atomicMin(out + 2 * k, static_cast<unsigned long long>(lo));
            atomicMax(out + 2 * k + 1, static_cast<unsigned long long>(hi));
        }
    }
}

/** Per tile: local exclusive scan and the tile sum. */
__global__ void k_scan_tiles(const u32* __restrict__ in, size_t n, u32* __restrict__ out,
                             u32* __restrict__ tile_sums) {
    __shared__ u32 ws[kThreads / 32];
    const size_t base = blockIdx.x * kTile + static_cast<size_t>(threadIdx.x) * kItems;
    u32 v[kItems];
    u32 s = 0;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        v[j] = base + j < n ? in[base + j] : 0u;
        s += v[j];
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    u32 x          = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const u32 y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o)
            x += y;
    }
    if (lane == 31)
        ws[w] = x;
    __syncthreads();
    if (w == 0) {
        u32 y = lane < kThreads / 32 ? ws[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const u32 z = __shfl_up_sync(0xffffffffu, y, o);
            if (lane >= o)
                y += z;
        }
        if (lane < kThreads / 32)
            ws[lane] = y;
    }
    __syncthreads();
    u32 run = x - s + (w > 0 ? ws[w - 1] : 0u);
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        if (base + j < n)
            out[base + j] = run;
        run += v[j];
    }
    if (threadIdx.x == kThreads - 1)
        tile_sums[blockIdx.x] = ws[kThreads / 32 - 1];
}

__global__ void k_scan_add(u32* __restrict__ out, size_t n, const u32* __restrict__ tile_sums) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n)
        out[i] += tile_sums[i / kTile];
}

__global__ void k_gather(const frost_giant* __restrict__ src, const u32* __restrict__ perm, size_t n,
                         frost_giant* __restrict__ dst) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n)
        dst[i] = src[perm[i]];
}

__global__ void k_compact(const frost_giant* __restrict__ src, const u32* __restrict__ flag,
                          const u32* __restrict__ pos, size_t n, frost_giant* __restrict__ dst) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n && flag[i] != 0)
        dst[pos[i]] = src[i];
}

// ---- ingest -------------------------------------------------------------------

__global__ void k_ingest(const frost_candidate* __restrict__ raw, size_t n, u64 samples_read, u64 nchans,
                         int flip, u64 boxcar_max, frost_giant* __restrict__ out, u32* __restrict__ keep,
                         unsigned long long* first_err, u32* nkept) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    bool kept      = false;
    if (i < n) {
        const frost_candidate r = raw[i];
        kept                    = r.peak_sample < samples_read;
        if (kept) {
            int kind = -1;
            if (r.chan_begin >= r.chan_end || r.chan_end > nchans)
                kind = 0;
            else if (r.beam_idx != 0 || r.width == 0 || r.width > boxcar_max ||
                     r.begin_sample > r.peak_sample || r.end_sample < r.peak_sample)
                kind = 1;
            if (kind >= 0)
                atomicMin(first_err, (static_cast<unsigned long long>(i) << 1) | static_cast<unsigned>(kind));
            frost_giant g;
            memset(&g, 0, sizeof(g));
            g.snr          = r.snr;
            g.samp_idx     = r.peak_sample;
            g.begin        = r.begin_sample;
            g.end          = r.end_sample < samples_read - 1 ? r.end_sample : samples_read - 1;
            g.filter_idx   = r.filter_idx;
            g.filter_width = r.width;
            g.dm_idx       = r.dm_idx;
            g.dm           = r.dm;
            g.f_low        = r.f_low_mhz;
            g.f_high       = r.f_high_mhz;
            g.chan_begin   = flip ? nchans - r.chan_end : r.chan_begin;
            g.chan_end     = flip ? nchans - 1 - r.chan_begin : static_cast<u64>(r.chan_end) - 1;
            g.plane        = static_cast<u64>(r.subband_level) * nchans + r.subband_idx;
            g.members      = 1;
            g.n_extents    = 1;
            out[i]         = g;
        }
        keep[i] = kept ? 1u : 0u;
    }
    const u32 b = __ballot_sync(0xffffffffu, kept);
    if ((threadIdx.x & 31) == 0 && b != 0)
        atomicAdd(nkept, static_cast<u32>(__popc(b)));
}

__global__ void k_plane_runs(const frost_giant* __restrict__ rows, size_t n, u64* run_plane, u32* run_start,
                             u32* nruns) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= n)
        return;
    if (i == 0 || rows[i].plane != rows[i - 1].plane) {
        const u32 s  = atomicAdd(nruns, 1u);
        run_plane[s] = rows[i].plane;
        run_start[s] = static_cast<u32>(i);
    }
}

__global__ void k_build_work(const frost_giant* __restrict__ inc, const frost_giant* __restrict__ pend,
                             const Seg* __restrict__ segs, int nseg, size_t nwork,
                             frost_giant* __restrict__ work, u32* __restrict__ seg_of) {
    const size_t w = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (w >= nwork)
        return;
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (segs[mid].work_start <= w)
            lo = mid;
        else
            hi = mid - 1;
    }
    const Seg sg = segs[lo];
    const u32 t  = static_cast<u32>(w - sg.work_start);
    work[w]      = t < sg.in_keep ? inc[sg.in_start + t] : pend[sg.pend_start + (t - sg.in_keep)];
    seg_of[w]    = static_cast<u32>(lo);
}

// ---- friends-of-friends -------------------------------------------------------

/** Columns of rows[perm[r]] in time order, plus the packed 16-byte key the
 * fast sweep reads: (samp - samp_lo, width, dm_idx, filter_idx), all
 * 32-bit. *c.general is set when some row does not fit that key or its
 * (plane, chan_begin, chan_end) differs from its segment's first row; the
 * general sweep then runs instead. */
__global__ void k_columns(const frost_giant* __restrict__ rows, const u32* __restrict__ perm,
                          const u32* __restrict__ seg_of, const u32* __restrict__ seg_lo, size_t n, u64 samp_lo,
                          Columns c) {
    const size_t r = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (r >= n)
        return;
    const u32 i          = perm[r];
    const frost_giant& g = rows[i];
    const u32 sg         = seg_of != nullptr ? seg_of[i] : 0u;
    const u64 width      = box_width(g.filter_width, g.filter_idx);
    c.samp[r]            = g.samp_idx;
    c.width[r]           = width;
    c.dm_idx[r]          = g.dm_idx;
    c.filter[r]          = g.filter_idx;
    c.cb[r]              = g.chan_begin;
    c.ce[r]              = g.chan_end;
    c.plane[r]           = g.plane;
    c.dm[r]              = g.dm;
    c.snr[r]             = g.snr;
    c.flo[r]             = g.f_low;
    c.fhi[r]             = g.f_high;
    c.idx[r]             = i;
    c.seg[r]             = sg;
    c.minidx[r]          = 0xFFFFFFFFu;
    const u64 rel        = g.samp_idx - samp_lo;
    const frost_giant& f = rows[perm[seg_lo != nullptr ? seg_lo[sg] : 0u]];
    const bool fits = g.samp_idx >= samp_lo && rel <= 0xFFFFFFFFull && width <= 0xFFFFFFFFull &&
                      g.dm_idx <= 0xFFFFFFFFull && g.filter_idx <= 0xFFFFFFFFull && g.plane == f.plane &&
                      g.chan_begin == f.chan_begin && g.chan_end == f.chan_end;
    if (!fits)
        atomicOr(c.general, 1u);
    c.key[r] = make_uint4(static_cast<u32>(rel), static_cast<u32>(width), static_cast<u32>(g.dm_idx),
                          static_cast<u32>(g.filter_idx));
}

__device__ __forceinline__ Pt column_pt(const Columns& c, size_t r) {
    return Pt{c.samp[r], c.filter[r], c.width[r], c.dm_idx[r], c.cb[r], c.ce[r], c.plane[r],
              c.dm[r],   c.snr[r],    c.flo[r],   c.fhi[r]};
}

__device__ __forceinline__ u32 absdiff32(u32 a, u32 b) { return a > b ? a - b : b - a; }

/** Fast sweep (every row fits the packed key and each segment has one
 * extent). One warp per time rank r tests the rows inside r's time reach in
 * r's segment, 32 at a time, forward (widths <= r's) and backward (widths
 * < r's) -- the pairs and orientation of the reference's sweep
 * (clustering.cpp:146-183). parent[] is over time ranks; a row already
 * hanging under r's root (one coalesced read per 32 rows) skips the rest. The
 * DM gate's bound (dm_smear * width * step) depends only on r, the wider
 * row, and is computed once. */
__global__ void k_chain_fast(Columns c, const u32* __restrict__ seg_lo, const u32* __restrict__ seg_hi, size_t n,
                             frost_cluster_tolerances tol, u32* parent) {
    const size_t r = (blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= n || *c.general != 0)
        return;
    volatile u32* p   = parent;
    const u32 sg      = c.seg[r];
    const size_t lo   = seg_lo != nullptr ? seg_lo[sg] : 0;
    const size_t hi   = seg_hi != nullptr ? seg_hi[sg] : n;
    const uint4 a     = c.key[r];
    const u64 reach   = time_reach(a.y, tol.time_tol);
    const bool gate   = tol.dm_smear > 0.0 && tol.tsamp > 0.0;
    const double step = gate ? dm_step(c.flo[r], c.fhi[r], static_cast<float>(tol.tsamp)) : 0.0;
    const bool open   = !gate || !(step > 0.0);
    const double lim  = tol.dm_smear * static_cast<double>(a.y) * step;
    const double dma  = static_cast<double>(c.dm[r]);
    const float snra  = c.snr[r];
    const u32 rr      = static_cast<u32>(r);
    u32 ra            = find_root(p, rr);
    auto test         = [&](size_t q, const uint4& b) {
        const u32 dd = absdiff32(a.z, b.z);
        if (dd > tol.dm_tol || absdiff32(a.w, b.w) > tol.filter_tol)
            return;
        if (p[q] == ra)
            return;
        if (!open && dd > 1) {
            const double ddm = abs_d(dma - static_cast<double>(c.dm[q]));
            double growth    = 1.0;
            if (tol.snr_floor > 0.0) {
                const double ratio = static_cast<double>(max_f(snra, c.snr[q])) / tol.snr_floor;
                growth             = max_d(1.0, sqrt(max_d(0.0, (ratio * ratio) - 1.0)));
            }
            if (!(ddm <= lim * growth))
                return;
        }
        const u32 qq = static_cast<u32>(q);
        if (find_root(p, qq) != ra)
            unite(p, rr, qq);
    };
    for (size_t q0 = r + 1; q0 < hi; q0 += 32) {
        const size_t q = q0 + lane;
        const bool ok  = q < hi;
        const uint4 b  = ok ? c.key[q] : make_uint4(0, 0, 0, 0);
        const bool in  = ok && static_cast<u64>(b.x - a.x) <= reach;
        const u32 m    = __ballot_sync(0xffffffffu, in);
        if (in && b.y <= a.y)
            test(q, b);
        if (m != 0xffffffffu)
            break;
        ra = find_root(p, ra);
    }
    ra = find_root(p, ra);
    for (size_t q0 = r; q0 > lo;) {
        const bool has = q0 > lo + static_cast<size_t>(lane);
        const size_t q = has ? q0 - 1 - lane : 0;
        const uint4 b  = has ? c.key[q] : make_uint4(0, 0, 0, 0);
        const bool in  = has && static_cast<u64>(a.x - b.x) <= reach;
        const u32 m    = __ballot_sync(0xffffffffu, in);
        if (in && b.y < a.y)
            test(q, b);
        if (m != 0xffffffffu)
            break;
        q0 -= 32;
        ra = find_root(p, ra);
    }
}

/** General sweep: 64-bit columns and the full coincidence test on each
 * pair; same pairs and orientation as the fast sweep. Runs only when
 * *c.general is set. */
__global__ void k_chain(Columns c, const u32* __restrict__ seg_lo, const u32* __restrict__ seg_hi, size_t n,
                        frost_cluster_tolerances tol, u32* parent) {
    const size_t r = (blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= n || *c.general == 0)
        return;
    volatile u32* p  = parent;
    const u32 sg     = c.seg[r];
    const size_t lo  = seg_lo != nullptr ? seg_lo[sg] : 0;
    const size_t hi  = seg_hi != nullptr ? seg_hi[sg] : n;
    const Pt a       = column_pt(c, r);
    const u64 reach  = time_reach(a.width, tol.time_tol);
    const u32 rr     = static_cast<u32>(r);
    u32 ra           = find_root(p, rr);
    auto test        = [&](size_t q) {
        if (absdiff(a.dm_idx, c.dm_idx[q]) > tol.dm_tol || absdiff(a.filter, c.filter[q]) > tol.filter_tol ||
            a.cb != c.cb[q] || a.ce != c.ce[q] || a.plane != c.plane[q])
            return;
        if (!dm_gate(a, column_pt(c, q), tol))
            return;
        const u32 qq = static_cast<u32>(q);
        if (find_root(p, qq) != ra)
            unite(p, rr, qq);
    };
    for (size_t q0 = r + 1; q0 < hi; q0 += 32) {
        const size_t q = q0 + lane;
        const bool in  = q < hi && c.samp[q] - a.samp <= reach;
        const u32 m    = __ballot_sync(0xffffffffu, in);
        if (in && c.width[q] <= a.width)
            test(q);
        if (m != 0xffffffffu)
            break;
        ra = find_root(p, ra);
    }
    ra = find_root(p, ra);
    for (size_t q0 = r; q0 > lo;) {
        const bool has = q0 > lo + static_cast<size_t>(lane);
        const size_t q = has ? q0 - 1 - lane : 0;
        const bool in  = has && a.samp - c.samp[q] <= reach;
        const u32 m    = __ballot_sync(0xffffffffu, in);
        if (in && c.width[q] < a.width)
            test(q);
        if (m != 0xffffffffu)
            break;
        q0 -= 32;
        ra = find_root(p, ra);
    }
}

/** Rank roots to row labels: each component's label is its smallest row
 * index (what the reference's union-find over row indices gives). */
__global__ void k_rank_min(u32* parent, const u32* __restrict__ idx, size_t n, u32* minidx) {
    const size_t r = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (r >= n)
        return;
    const u32 root = find_root(parent, static_cast<u32>(r));
    atomicMin(minidx + root, idx[r]);
}

__global__ void k_rank_label(u32* parent, const u32* __restrict__ idx, const u32* __restrict__ minidx, size_t n,
                             u32* __restrict__ label) {
    const size_t r = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (r < n)
        label[idx[r]] = minidx[find_root(parent, static_cast<u32>(r))];
}

__global__ void k_find_all(u32* parent, size_t n, u32* label) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n)
        label[i] = find_root(parent, static_cast<u32>(i));
}

// ---- seeded clustering ----------------------------------------------------------

template <bool kShared>
__global__ void k_seeded(const frost_giant* __restrict__ rows, const u32* __restrict__ tord,
                         const u32* __restrict__ sord, const u32* __restrict__ rank_of,
                         const u32* __restrict__ lo_of, const u32* __restrict__ hi_of,
                         frost_cluster_tolerances tol, u32* __restrict__ label, u32* gbitmap,
                         size_t bitmap_words) {
    extern __shared__ u32 s_bits[];
    __shared__ u64 s_wide[32];
    const u32 lo = lo_of[blockIdx.x], hi = hi_of[blockIdx.x];
    if (lo >= hi)
        return;
    const u32 n   = hi - lo;
    const u32 nw  = (n + 31) / 32;
    u32* bits     = kShared ? s_bits : gbitmap + blockIdx.x * bitmap_words;
    volatile u32* vbits = bits;
    for (u32 w = threadIdx.x; w < nw; w += blockDim.x)
        bits[w] = 0;
    u64 wide = 1;
    for (u32 i = lo + threadIdx.x; i < hi; i += blockDim.x)
        wide = max_u(wide, box_width(rows[i].filter_width, rows[i].filter_idx));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        wide = max_u(wide, shfl_u64(wide, o));
    if ((threadIdx.x & 31) == 0)
        s_wide[threadIdx.x >> 5] = wide;
    __syncthreads();
    wide = 1;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w)
        wide = max_u(wide, s_wide[w]);
    const u64 reach = time_reach(wide, tol.time_tol);
    for (u32 k = lo; k < hi; ++k) {
        const u32 seed = sord[k];
        const u32 sb   = seed - lo;
        if ((vbits[sb >> 5] >> (sb & 31)) & 1u)
            continue;
        __syncthreads();
        if (threadIdx.x == 0) {
            atomicOr(bits + (sb >> 5), 1u << (sb & 31));
            label[seed] = seed;
        }
        const Pt a     = pt_of(rows[seed]);
        const u32 rank = rank_of[seed];
        for (u32 q = rank + 1 + threadIdx.x; q < hi; q += blockDim.x) {
            const u32 j = tord[q];
            if (rows[j].samp_idx - a.samp > reach)
                break;
            const u32 jb = j - lo;
            if (!((vbits[jb >> 5] >> (jb & 31)) & 1u) && coincident(a, pt_of(rows[j]), tol)) {
                atomicOr(bits + (jb >> 5), 1u << (jb & 31));
                label[j] = seed;
            }
        }
        for (long long q = static_cast<long long>(rank) - 1 - threadIdx.x; q >= static_cast<long long>(lo);
             q -= blockDim.x) {
            const u32 j = tord[q];
            if (a.samp - rows[j].samp_idx > reach)
                break;
            const u32 jb = j - lo;
            if (!((vbits[jb >> 5] >> (jb & 31)) & 1u) && coincident(a, pt_of(rows[j]), tol)) {
                atomicOr(bits + (jb >> 5), 1u << (jb & 31));
                label[j] = seed;
            }
        }
        __syncthreads();
    }
}

__global__ void k_invert(const u32* __restrict__ perm, size_t n, u32* __restrict__ rank_of) {
    const size_t r = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (r < n)
        rank_of[perm[r]] = static_cast<u32>(r);
}

__global__ void k_seg_bounds(const u32* __restrict__ seg_of, size_t n, u32* lo, u32* hi) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= n)
        return;
    const u32 s = seg_of[i];
    if (i == 0 || seg_of[i - 1] != s)
        lo[s] = static_cast<u32>(i);
    if (i + 1 == n || seg_of[i + 1] != s)
        hi[s] = static_cast<u32>(i + 1);
}

// ---- merge --------------------------------------------------------------------------

__global__ void k_root_flags(const u32* __restrict__ label, size_t n, u32* __restrict__ flag) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n)
        flag[i] = label[i] == i ? 1u : 0u;
}

__device__ __forceinline__ void merge_accum_one(const frost_giant& g, u32 i, u32 grp, unsigned long long* best,
                                                u32* first, unsigned long long* sum) {
    atomicMin(first + grp, i);
    const unsigned long long key =
        (static_cast<unsigned long long>(ordered_bits(g.snr)) << 32) | (0xFFFFFFFFull - i);
    atomicMax(best + grp, key);
    atomicAdd(sum + grp, static_cast<unsigned long long>(g.members));
}

__global__ void k_merge_accum(const frost_giant* __restrict__ rows, const u32* __restrict__ label,
                              const u32* __restrict__ ord, size_t n, unsigned long long* best, u32* first,
                              unsigned long long* sum, u32* gmap) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i >= n)
        return;
    const u32 grp = ord[label[i]];
    merge_accum_one(rows[i], static_cast<u32>(i), grp, best, first, sum);
    if (gmap != nullptr)
        gmap[i] = grp;
}

__global__ void k_merge_accum_ord(const frost_giant* __restrict__ rows, const u32* __restrict__ ordv,
                                  size_t n, unsigned long long* best, u32* first, unsigned long long* sum) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n)
        merge_accum_one(rows[i], static_cast<u32>(i), ordv[i], best, first, sum);
}

/** The reference keeps the first member and replaces it only by a strictly
 * higher S/N: the first maximum, unless the first member's S/N is NaN (then
 * nothing compares greater and it stays). */
__global__ void k_merge_emit(const frost_giant* __restrict__ rows, size_t ngroups,
                             const unsigned long long* __restrict__ best, const u32* __restrict__ first,
                             const unsigned long long* __restrict__ sum, const u32* __restrict__ seg_of,
                             u32* __restrict__ seg_out, frost_giant* __restrict__ out) {
    const size_t g = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (g >= ngroups)
        return;
    const u32 f   = first[g];
    const float s = rows[f].snr;
    const u32 w   = (s != s) ? f : static_cast<u32>(0xFFFFFFFFull - (best[g] & 0xFFFFFFFFull));
    frost_giant o = rows[w];
    o.members     = sum[g];
    out[g]        = o;
    if (seg_of != nullptr && seg_out != nullptr)
        seg_out[g] = seg_of[f];
}

__global__ void k_heads(const u64* __restrict__ keys, size_t n, u32* __restrict__ heads) {
    const size_t k = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (k < n)
        heads[k] = (k == 0 || keys[k] != keys[k - 1]) ? 1u : 0u;
}

/** excl is the exclusive scan of heads: the value rank at sorted position
 * k is excl[k] + heads[k] - 1. */
__global__ void k_scatter_ord(const u32* __restrict__ perm, const u32* __restrict__ excl,
                              const u32* __restrict__ heads, size_t n, u32* __restrict__ ordv) {
    const size_t k = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (k < n)
        ordv[perm[k]] = excl[k] + heads[k] - 1u;
}

__global__ void k_seg_counts(const u32* __restrict__ flag, const u32* __restrict__ seg_of, size_t n,
                             u32* counts) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n && flag[i] != 0)
        atomicAdd(counts + seg_of[i], 1u);
}

// ---- retention ------------------------------------------------------------------------

__global__ void k_recent(const frost_giant* __restrict__ work, size_t n, const u32* __restrict__ gmap,
                         const u32* __restrict__ rmap, u64 watermark, u32* recent) {
    const size_t w = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (w < n && work[w].end >= watermark) {
        const u32 g = gmap[w];
        recent[rmap != nullptr ? rmap[g] : g] = 1u;
    }
}

__global__ void k_pending_flags(size_t n, const u32* __restrict__ gmap, const u32* __restrict__ rmap,
                                const u32* __restrict__ recent, int final_call, u32* __restrict__ pflag) {
    const size_t w = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (w >= n)
        return;
    const u32 g = gmap[w];
    pflag[w]    = final_call ? 0u : recent[rmap != nullptr ? rmap[g] : g];
}

__global__ void k_ready_flags(size_t n, const u32* __restrict__ recent, int final_call, u32* __restrict__ rflag) {
    const size_t g = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (g < n)
        rflag[g] = (final_call || recent[g] == 0) ? 1u : 0u;
}

// ---- sub-band dedup ---------------------------------------------------------------------

constexpr int kPairTile = 128;

__global__ void __launch_bounds__(kPairTile) k_dedup_pairs(const frost_giant* __restrict__ rows, size_t n,
                                                           frost_cluster_tolerances tol, float tsamp,
                                                           u32* parent) {
    __shared__ Pt tile[kPairTile];
    volatile u32* p = parent;
    const size_t i  = blockIdx.x * static_cast<size_t>(kPairTile) + threadIdx.x;
    const Pt a      = i < n ? pt_of(rows[i]) : Pt{};
    for (size_t j0 = blockIdx.x * static_cast<size_t>(kPairTile); j0 < n; j0 += kPairTile) {
        const size_t jl = j0 + threadIdx.x;
        if (jl < n)
            tile[threadIdx.x] = pt_of(rows[jl]);
        __syncthreads();
        if (i < n) {
            const size_t m = (n - j0) < static_cast<size_t>(kPairTile) ? n - j0 : kPairTile;
            for (size_t jj = 0; jj < m; ++jj) {
                const size_t j = j0 + jj;
                if (j > i && on_same_curve(a, tile[jj], tol, tsamp))
                    unite(p, static_cast<u32>(i), static_cast<u32>(j));
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kPairTile) k_first_match(const frost_giant* __restrict__ rows,
                                                           const u32* __restrict__ order, size_t n,
                                                           frost_cluster_tolerances tol, float tsamp,
                                                           u32* __restrict__ fm) {
    __shared__ Pt tile[kPairTile];
    const size_t k    = blockIdx.x * static_cast<size_t>(kPairTile) + threadIdx.x;
    const Pt b        = k < n ? pt_of(rows[order[k]]) : Pt{};
    u32 found         = k < n ? static_cast<u32>(k) : 0u;
    bool done         = k >= n;
    const size_t kmax = (blockIdx.x + 1) * static_cast<size_t>(kPairTile) < n
                            ? (blockIdx.x + 1) * static_cast<size_t>(kPairTile)
                            : n;
    for (size_t m0 = 0; m0 < kmax; m0 += kPairTile) {
        const size_t ml = m0 + threadIdx.x;
        if (ml < n)
            tile[threadIdx.x] = pt_of(rows[order[ml]]);
        __syncthreads();
        if (!done) {
            for (size_t mm = 0; mm < static_cast<size_t>(kPairTile); ++mm) {
                const size_t m = m0 + mm;
                if (m >= k)
                    break;
                if (on_same_curve(tile[mm], b, tol, tsamp)) {
                    found = static_cast<u32>(m);
                    done  = true;
                    break;
                }
            }
        }
        __syncthreads();
    }
    if (k < n)
        fm[k] = found;
}

__global__ void k_resolve_seeded(const u32* __restrict__ order, const u32* __restrict__ fm, size_t n,
                                 u32* __restrict__ group_of, u32* first) {
    const size_t k = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (k >= n)
        return;
    u32 r = static_cast<u32>(k);
    while (fm[r] != r)
        r = fm[r];
    const u32 g         = order[r];
    group_of[order[k]]  = g;
    atomicMin(first + g, order[k]);
}

__global__ void k_relabel(const u32* __restrict__ group_of, const u32* __restrict__ first, size_t n,
                          u32* __restrict__ label) {
    const size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (i < n)
        label[i] = first[group_of[i]];
}

__global__ void k_group_starts(const u32* __restrict__ perm, const u32* __restrict__ label,
                               const u32* __restrict__ ord, size_t n, u32* __restrict__ gstart) {
    const size_t k = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (k >= n)
        return;
    const u32 l = label[perm[k]];
    if (k == 0 || label[perm[k - 1]] != l)
        gstart[ord[l]] = static_cast<u32>(k);
}

__device__ __forceinline__ float best_snr_of(const frost_giant& g) {
    return g.snr_best > g.snr ? g.snr_best : g.snr;
}
__device__ __forceinline__ bool has_best_extent(const frost_giant& g) {
    return g.has_location_best != 0 || g.snr_best > g.snr;
}
__device__ __forceinline__ void strongest_location(const frost_giant& g, frost_giant& dst) {
    if (g.has_location_best != 0) {
        dst.loc_samp_idx     = g.loc_samp_idx;
        dst.loc_dm           = g.loc_dm;
        dst.loc_filter_width = g.loc_filter_width;
        dst.loc_f_low        = g.loc_f_low;
        dst.loc_f_high       = g.loc_f_high;
    } else {
        dst.loc_samp_idx     = g.samp_idx;
        dst.loc_dm           = g.dm;
        dst.loc_filter_width = box_width(g.filter_width, g.filter_idx);
        dst.loc_f_low        = g.f_low;
        dst.loc_f_high       = g.f_high;
    }
}

/** Sequential over a group's members in index order, exactly as
 * subband_dedup.cpp:271-313 folds them. */
__global__ void k_dedup_emit(const frost_giant* __restrict__ rows, const u32* __restrict__ perm,
                             const u32* __restrict__ gstart, size_t ngroups, size_t n,
                             frost_giant* __restrict__ out) {
    const size_t g = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    if (g >= ngroups)
        return;
    const u32 b = gstart[g];
    const u32 e = g + 1 < ngroups ? gstart[g + 1] : static_cast<u32>(n);
    const frost_giant& f0 = rows[perm[b]];
    frost_giant winner    = f0;
    frost_giant loc;
    strongest_location(f0, loc);
    float bsnr = best_snr_of(f0);
    u64 bbeg   = has_best_extent(f0) ? f0.best_chan_begin : f0.chan_begin;
    u64 bend   = has_best_extent(f0) ? f0.best_chan_end : f0.chan_end;
    for (u32 k = b + 1; k < e; ++k) {
        const frost_giant& c = rows[perm[k]];
        const u64 msum       = winner.members + c.members;
        const u64 sc = span_of(c.chan_begin, c.chan_end), sw = span_of(winner.chan_begin, winner.chan_end);
        if (sc != sw ? sc > sw : c.snr > winner.snr)
            winner = c;
        winner.members = msum;
        const float cb = best_snr_of(c);
        if (cb > bsnr) {
            bsnr = cb;
            bbeg = has_best_extent(c) ? c.best_chan_begin : c.chan_begin;
            bend = has_best_extent(c) ? c.best_chan_end : c.chan_end;
            strongest_location(c, loc);
        }
    }
    u64 next = 0;
    for (u32 k = b; k < e; ++k) {
        const frost_giant& c = rows[perm[k]];
        bool seen            = false;
        for (u32 q = b; q < k && !seen; ++q)
            seen = rows[perm[q]].chan_begin == c.chan_begin && rows[perm[q]].chan_end == c.chan_end;
        next += seen ? 0 : 1;
    }
    winner.n_extents         = next;
    winner.snr_best          = bsnr;
    winner.best_chan_begin   = bbeg;
    winner.best_chan_end     = bend;
    winner.has_location_best = 1;
    winner.loc_samp_idx      = loc.loc_samp_idx;
    winner.loc_dm            = loc.loc_dm;
    winner.loc_filter_width  = loc.loc_filter_width;
    winner.loc_f_low         = loc.loc_f_low;
    winner.loc_f_high        = loc.loc_f_high;
    out[g]                   = winner;
}

} // namespace

u64 launch_counter() { return g_launches.load(std::memory_order_relaxed); }

#define FB_PP_GRID(n) blocks_for(n), kThreads, 0, s

void launch_iota(u32* v, size_t n, cudaStream_t s) {
    if (n == 0)
        return;
    k_iota<<<FB_PP_GRID(n)>>>(v, n);
    FB_LAUNCH_CHECK();
    count();
}

void radix_sort(u64*& keys, u32*& vals, u64*& keys_alt, u32*& vals_alt, size_t n, int bits, u32* hist,
                cudaStream_t s) {
    if (n < 2)
        return;
    const u32 nblk = static_cast<u32>((n + kTile - 1) / kTile);
    for (int shift = 0; shift < bits; shift += 8) {
        k_rs_hist<<<nblk, kThreads, 0, s>>>(keys, n, shift, hist, nblk);
        FB_LAUNCH_CHECK();
        k_scan_single<<<1, 1024, 0, s>>>(hist, static_cast<size_t>(nblk) * 256, nullptr);
        FB_LAUNCH_CHECK();
        k_rs_scatter<<<nblk, kThreads, 0, s>>>(keys, vals, keys_alt, vals_alt, n, shift, hist, nblk);
        FB_LAUNCH_CHECK();
        count();
        count();
        count();
        std::swap(keys, keys_alt);
        std::swap(vals, vals_alt);
    }
}

void launch_keys(const frost_giant* rows, const u32* perm, size_t n, const KeySpec& spec, const u32* aux32,
                 const u64* aux64, const u32* keep, u64* keys, cudaStream_t s) {
    if (n == 0)
        return;
    k_keys<<<FB_PP_GRID(n)>>>(rows, perm, n, spec, aux32, aux64, keep, keys);
    FB_LAUNCH_CHECK();
    count();
}

void launch_ranges(const frost_giant* rows, size_t n, const RangeKinds& kinds, const u32* aux32,
                   const u64* aux64, const u32* keep, unsigned long long* out, cudaStream_t s) {
    if (n == 0)
        return;
    k_ranges<<<FB_PP_GRID(n)>>>(rows, n, kinds, aux32, aux64, keep, out);
    FB_LAUNCH_CHECK();
    count();
}

void exclusive_scan(const u32* in, u32* out, size_t n, u32* tile_sums, u32* total, cudaStream_t s) {
    if (n == 0) {
        FB_CUDA(cudaMemsetAsync(total, 0, sizeof(u32), s));
        return;
    }
    const unsigned nt = static_cast<unsigned>((n + kTile - 1) / kTile);
    k_scan_tiles<<<nt, kThreads, 0, s>>>(in, n, out, tile_sums);
    FB_LAUNCH_CHECK();
    k_scan_single<<<1, 1024, 0, s>>>(tile_sums, nt, total);
    FB_LAUNCH_CHECK();
    count();
    count();
    if (nt > 1) {
        k_scan_add<<<FB_PP_GRID(n)>>>(out, n, tile_sums);
        FB_LAUNCH_CHECK();
        count();
    }
}

void launch_gather(const frost_giant* src, const u32* perm, size_t n, frost_giant* dst, cudaStream_t s) {
    if (n == 0)
        return;
    k_gather<<<FB_PP_GRID(n)>>>(src, perm, n, dst);
    FB_LAUNCH_CHECK();
    count();
}

void launch_compact(const frost_giant* src, const u32* flag, const u32* pos, size_t n, frost_giant* dst,
                    cudaStream_t s) {
    if (n == 0)
        return;
    k_compact<<<FB_PP_GRID(n)>>>(src, flag, pos, n, dst);
    FB_LAUNCH_CHECK();
    count();
}

void launch_ingest(const frost_candidate* raw, size_t n, u64 samples_read, u64 nchans, int flip,
                   u64 boxcar_max, frost_giant* out, u32* keep, unsigned long long* first_err, u32* nkept,
                   cudaStream_t s) {
    if (n == 0)
        return;
    k_ingest<<<FB_PP_GRID(n)>>>(raw, n, samples_read, nchans, flip, boxcar_max, out, keep, first_err, nkept);
    FB_LAUNCH_CHECK();
    count();
}

void launch_plane_runs(const frost_giant* rows, size_t n, u64* run_plane, u32* run_start, u32* nruns,
                       cudaStream_t s) {
    if (n == 0)
        return;
    k_plane_runs<<<FB_PP_GRID(n)>>>(rows, n, run_plane, run_start, nruns);
    FB_LAUNCH_CHECK();
    count();
}

void launch_build_work(const frost_giant* inc, const frost_giant* pend, const Seg* segs, int nseg,
                       size_t nwork, frost_giant* work, u32* seg_of, cudaStream_t s) {
    if (nwork == 0)
        return;
    k_build_work<<<FB_PP_GRID(nwork)>>>(inc, pend, segs, nseg, nwork, work, seg_of);
    FB_LAUNCH_CHECK();
    count();
}

void launch_columns(const frost_giant* rows, const u32* perm, const u32* seg_of, const u32* seg_lo, size_t n,
                    u64 samp_lo, const Columns& c, cudaStream_t s) {
    FB_CUDA(cudaMemsetAsync(c.general, 0, sizeof(u32), s));
    if (n == 0)
        return;
    k_columns<<<FB_PP_GRID(n)>>>(rows, perm, seg_of, seg_lo, n, samp_lo, c);
    FB_LAUNCH_CHECK();
    count();
}

void launch_chain(const Columns& c, const u32* seg_lo, const u32* seg_hi, size_t n,
                  const frost_cluster_tolerances& tol, u32* parent, cudaStream_t s) {
    if (n < 2)
        return;
    k_chain_fast<<<blocks_for(n * 32), kThreads, 0, s>>>(c, seg_lo, seg_hi, n, tol, parent);
    FB_LAUNCH_CHECK();
    k_chain<<<blocks_for(n * 32), kThreads, 0, s>>>(c, seg_lo, seg_hi, n, tol, parent);
    FB_LAUNCH_CHECK();
    count();
    count();
}

void launch_rank_labels(u32* parent, const Columns& c, size_t n, u32* label, cudaStream_t s) {
    if (n == 0)
        return;
    k_rank_min<<<FB_PP_GRID(n)>>>(parent, c.idx, n, c.minidx);
    FB_LAUNCH_CHECK();
    k_rank_label<<<FB_PP_GRID(n)>>>(parent, c.idx, c.minidx, n, label);
    FB_LAUNCH_CHECK();
    count();
    count();
}

void launch_find_all(u32* parent, size_t n, u32* label, cudaStream_t s) {
    if (n == 0)
        return;
    k_find_all<<<FB_PP_GRID(n)>>>(parent, n, label);
    FB_LAUNCH_CHECK();
    count();
}

void launch_seeded(const frost_giant* rows, const u32* tord, const u32* sord, const u32* rank_of,
                   const u32* lo, const u32* hi, int nseg, const frost_cluster_tolerances& tol, u32* label,
                   u32* gbitmap, size_t bitmap_words, cudaStream_t s) {
    if (nseg == 0)
        return;
    constexpr size_t kSmemLimit = 200 * 1024;
    const size_t smem           = bitmap_words * sizeof(u32);
    if (smem <= kSmemLimit) {
        if (smem > 48 * 1024)
            allow_large_smem(reinterpret_cast<const void*>(&k_seeded<true>));
        k_seeded<true><<<nseg, kThreads, smem, s>>>(rows, tord, sord, rank_of, lo, hi, tol, label, nullptr,
                                                    bitmap_words);
    } else {
        k_seeded<false><<<nseg, kThreads, 0, s>>>(rows, tord, sord, rank_of, lo, hi, tol, label, gbitmap,
                                                  bitmap_words);
    }
    FB_LAUNCH_CHECK();
    count();
}

void launch_invert(const u32* perm, size_t n, u32* rank_of, cudaStream_t s) {
    if (n == 0)
        return;
    k_invert<<<FB_PP_GRID(n)>>>(perm, n, rank_of);
    FB_LAUNCH_CHECK();
    count();
}

void launch_seg_bounds(const u32* seg_of, size_t n, u32* lo, u32* hi, cudaStream_t s) {
    if (n == 0)
        return;
    k_seg_bounds<<<FB_PP_GRID(n)>>>(seg_of, n, lo, hi);
    FB_LAUNCH_CHECK();
    count();
}

void launch_root_flags(const u32* label, size_t n, u32* flag, cudaStream_t s) {
    if (n == 0)
        return;
    k_root_flags<<<FB_PP_GRID(n)>>>(label, n, flag);
    FB_LAUNCH_CHECK();
    count();
}

void launch_merge_accum(const frost_giant* rows, const u32* label, const u32* ord, size_t n,
                        unsigned long long* best, u32* first, unsigned long long* sum, u32* gmap,
                        cudaStream_t s) {
    if (n == 0)
        return;
    k_merge_accum<<<FB_PP_GRID(n)>>>(rows, label, ord, n, best, first, sum, gmap);
    FB_LAUNCH_CHECK();
    count();
}

void launch_merge_emit(const frost_giant* rows, size_t ngroups, const unsigned long long* best,
                       const u32* first, const unsigned long long* sum, const u32* seg_of, u32* seg_out,
                       frost_giant* out, cudaStream_t s) {
    if (ngroups == 0)
        return;
    k_merge_emit<<<FB_PP_GRID(ngroups)>>>(rows, ngroups, best, first, sum, seg_of, seg_out, out);
    FB_LAUNCH_CHECK();
    count();
}

void launch_heads(const u64* sorted_keys, size_t n, u32* heads, cudaStream_t s) {
    if (n == 0)
        return;
    k_heads<<<FB_PP_GRID(n)>>>(sorted_keys, n, heads);
    FB_LAUNCH_CHECK();
    count();
}

void launch_scatter_ord(const u32* perm, const u32* excl, const u32* heads, size_t n, u32* ordv,
                        cudaStream_t s) {
    if (n == 0)
        return;
    k_scatter_ord<<<FB_PP_GRID(n)>>>(perm, excl, heads, n, ordv);
    FB_LAUNCH_CHECK();
    count();
}

void launch_seg_counts(const u32* flag, const u32* seg_of, size_t n, u32* counts, cudaStream_t s) {
    if (n == 0)
        return;
    k_seg_counts<<<FB_PP_GRID(n)>>>(flag, seg_of, n, counts);
    FB_LAUNCH_CHECK();
    count();
}

void launch_merge_accum_ord(const frost_giant* rows, const u32* ordv, size_t n, unsigned long long* best,
                            u32* first, unsigned long long* sum, cudaStream_t s) {
    if (n == 0)
        return;
    k_merge_accum_ord<<<FB_PP_GRID(n)>>>(rows, ordv, n, best, first, sum);
    FB_LAUNCH_CHECK();
    count();
}

void launch_recent(const frost_giant* work, size_t n, const u32* gmap, const u32* rmap, u64 watermark,
                   u32* recent, cudaStream_t s) {
    if (n == 0)
        return;
    k_recent<<<FB_PP_GRID(n)>>>(work, n, gmap, rmap, watermark, recent);
    FB_LAUNCH_CHECK();
    count();
}

void launch_pending_flags(size_t n, const u32* gmap, const u32* rmap, const u32* recent, int final_call,
                          u32* pflag, cudaStream_t s) {
    if (n == 0)
        return;
    k_pending_flags<<<FB_PP_GRID(n)>>>(n, gmap, rmap, recent, final_call, pflag);
    FB_LAUNCH_CHECK();
    count();
}

void launch_ready_flags(size_t n, const u32* recent, int final_call, u32* rflag, cudaStream_t s) {
    if (n == 0)
        return;
    k_ready_flags<<<FB_PP_GRID(n)>>>(n, recent, final_call, rflag);
    FB_LAUNCH_CHECK();
    count();
}

void launch_dedup_pairs(const frost_giant* rows, size_t n, const frost_cluster_tolerances& tol, float tsamp,
                        u32* parent, cudaStream_t s) {
    if (n < 2)
        return;
    k_dedup_pairs<<<blocks_for(n, kPairTile), kPairTile, 0, s>>>(rows, n, tol, tsamp, parent);
    FB_LAUNCH_CHECK();
    count();
}

void launch_first_match(const frost_giant* rows, const u32* order, size_t n,
                        const frost_cluster_tolerances& tol, float tsamp, u32* fm, cudaStream_t s) {
    if (n == 0)
        return;
    k_first_match<<<blocks_for(n, kPairTile), kPairTile, 0, s>>>(rows, order, n, tol, tsamp, fm);
    FB_LAUNCH_CHECK();
    count();
}

void launch_resolve_seeded(const u32* order, const u32* fm, size_t n, u32* group_of, u32* first,
                           cudaStream_t s) {
    if (n == 0)
        return;
    k_resolve_seeded<<<FB_PP_GRID(n)>>>(order, fm, n, group_of, first);
    FB_LAUNCH_CHECK();
    count();
}

void launch_relabel(const u32* group_of, const u32* first, size_t n, u32* label, cudaStream_t s) {
    if (n == 0)
        return;
    k_relabel<<<FB_PP_GRID(n)>>>(group_of, first, n, label);
    FB_LAUNCH_CHECK();
    count();
}

void launch_group_starts(const u32* perm, const u32* label, const u32* ord, size_t n, u32* gstart,
                         cudaStream_t s) {
    if (n == 0)
        return;
    k_group_starts<<<FB_PP_GRID(n)>>>(perm, label, ord, n, gstart);
    FB_LAUNCH_CHECK();
    count();
}

void launch_dedup_emit(const frost_giant* rows, const u32* perm, const u32* gstart, size_t ngroups, size_t n,
                       frost_giant* out, cudaStream_t s) {
    if (ngroups == 0)
        return;
    k_dedup_emit<<<FB_PP_GRID(ngroups)>>>(rows, perm, gstart, ngroups, n, out);
    FB_LAUNCH_CHECK();
    count();
}

} // namespace fb::pp
