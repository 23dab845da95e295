// Streaming FDMT plan construction (see fdmt_plan.hpp for the rules).

#include "fdmt_plan.hpp"

#include <algorithm>
#include <cmath>
#include <functional>
#include <limits>
#include <string>

namespace fb::fdmt {

int32_t Node::row_of(int32_t d) const {
    const auto it = std::lower_bound(delays.begin(), delays.end(), d);
    if (it == delays.end() || *it != d)
        throw Error(FROST_ERR_INTERNAL, "FDMT plan: missing delay row " + std::to_string(d));
    return static_cast<int32_t>(it - delays.begin());
}

std::vector<int32_t> box_widths(uint64_t max_boxcar, float wtsp) {
    if (max_boxcar == 0 || max_boxcar > (uint64_t{1} << 20))
        invalid("boxcar: max_boxcar must be in [1, 2^20]");
    if (!is_finite(wtsp) || !(wtsp >= 1.0F))
        invalid("boxcar: wtsp must be a finite number >= 1");
    std::vector<int32_t> w{1};
    while (true) {
        const double next = std::ceil(static_cast<double>(wtsp) * w.back());
        const int64_t n   = std::max<int64_t>(static_cast<int64_t>(next), w.back() + 1);
        if (n > static_cast<int64_t>(max_boxcar))
            break;
        w.push_back(static_cast<int32_t>(n));
    }
    return w;
}

double window_box_variance(int32_t L, int32_t W, bool trapezoid) {
    std::vector<double> wgt(W, 1.0);
    if (trapezoid && W >= 3) {
        const int32_t e = (W + 1) / 4;
        for (int32_t i = 0; i < e; ++i) {
            wgt[i]         = 0.5;
            wgt[W - 1 - i] = 0.5;
        }
    }
    // m_k = sum_{i : 0 <= k - i < L} wgt[i] via a prefix sum over wgt.
    std::vector<double> pre(W + 1, 0.0);
    for (int32_t i = 0; i < W; ++i)
        pre[i + 1] = pre[i] + wgt[i];
    double g = 0.0;
    for (int32_t k = 0; k < W + L - 1; ++k) {
        const int32_t hi = std::min(k, W - 1);
        const int32_t lo = std::max(0, k - L + 1);
        const double m   = pre[hi + 1] - pre[lo];
        g += m * m;
    }
    return g;
}

double Plan::edge(int64_t c) const {
    const double bw = (m_cfg.f_max - m_cfg.f_min) / static_cast<double>(m_cfg.nchans);
    return m_cfg.f_min + static_cast<double>(c) * bw;
}

int32_t Plan::band_delay(double dm, double f_lo, double f_hi) const {
    const double d = kDispConst * dm * K(f_lo, f_hi) / m_cfg.tsamp;
    if (!(d >= 0.0) || d > 1.0e9)
        invalid("FDMT plan: delay out of range");
    return static_cast<int32_t>(std::llround(d));
}

void Plan::split_delay(const Node& n, int32_t d, int32_t& d_lo, int32_t& d_hi) const {
    const double ratio = K(n.f_mid, n.f_hi) / K(n.f_lo, n.f_hi);
    d_hi               = static_cast<int32_t>(std::llround(static_cast<double>(d) * ratio));
    d_lo               = d - d_hi;
}

int32_t Plan::build_tree(int32_t begin, int32_t end) {
    Node n;
    n.chan_begin = begin;
    n.chan_end   = end;
    n.f_lo       = edge(begin);
    n.f_hi       = edge(end);
    if (end - begin == 1) {
        m_nodes.push_back(n);
        return static_cast<int32_t>(m_nodes.size() - 1);
    }
    const int32_t mid = begin + (end - begin) / 2;
    int32_t lo        = build_tree(begin, mid);
    int32_t hi        = build_tree(mid, end);
    const int32_t h   = 1 + std::max(m_nodes[lo].height, m_nodes[hi].height);
    lo                = wrap(lo, h - 1);
    hi                = wrap(hi, h - 1);
    n.lo              = lo;
    n.hi              = hi;
    n.height          = h;
    n.f_mid           = edge(mid);
    m_nodes.push_back(n);
    return static_cast<int32_t>(m_nodes.size() - 1);
}

int32_t Plan::wrap(int32_t node, int32_t height) {
    while (m_nodes[node].height < height) {
        Node p;
        p.chan_begin = m_nodes[node].chan_begin;
        p.chan_end   = m_nodes[node].chan_end;
        p.f_lo       = m_nodes[node].f_lo;
        p.f_hi       = m_nodes[node].f_hi;
        p.lo         = node;
        p.hi         = -1;
        p.height     = m_nodes[node].height + 1;
        m_nodes.push_back(p);
        node = static_cast<int32_t>(m_nodes.size() - 1);
    }
    return node;
}

Plan::Plan(PlanConfig cfg) : m_cfg(std::move(cfg)) {
    const auto C = m_cfg.nchans;
    if (C < 2 || C > (uint64_t{1} << 20))
        invalid("FDMT plan: nchans must be in [2, 2^20]");
    if (!is_positive_finite(m_cfg.f_min) || !is_positive_finite(m_cfg.f_max) ||
        !(m_cfg.f_max > m_cfg.f_min))
        invalid("FDMT plan: band edges must be positive and ascending");
    if (!is_positive_finite(m_cfg.tsamp))
        invalid("FDMT plan: tsamp must be positive");
    if (m_cfg.dm_list.empty())
        invalid("FDMT plan: empty DM list");
    for (size_t i = 0; i < m_cfg.dm_list.size(); ++i) {
        if (!is_finite(m_cfg.dm_list[i]) || m_cfg.dm_list[i] < 0.0F)
            invalid("FDMT plan: DM trials must be finite and >= 0");
        if (i > 0 && !(m_cfg.dm_list[i] > m_cfg.dm_list[i - 1]))
            invalid("FDMT plan: DM trials must increase");
    }
    const uint64_t S = m_cfg.subband_depth;
    if (S > 8 || (uint64_t{2} << S) > C)
        invalid("FDMT plan: subband_depth " + std::to_string(S) + " needs at least " +
                std::to_string(uint64_t{2} << std::min<uint64_t>(S, 8)) + " channels");
    m_widths = box_widths(m_cfg.max_boxcar, m_cfg.wtsp);

    // Tree.
    m_nodes.reserve(4 * C);
    m_root   = build_tree(0, static_cast<int32_t>(C));
    m_levels = m_nodes[m_root].height;

    for (const float dm : m_cfg.dm_list)
        m_final_delays.push_back(band_delay(dm, m_cfg.f_min, m_cfg.f_max));
    m_dt_max = *std::max_element(m_final_delays.begin(), m_final_delays.end());

    // Regular nodes by tree depth (pass-through wrappers are transparent).
    std::vector<std::vector<int32_t>> by_depth(S + 2);
    std::function<int32_t(int32_t)> unwrap = [&](int32_t n) {
        while (m_nodes[n].hi < 0 && m_nodes[n].lo >= 0)
            n = m_nodes[n].lo;
        return n;
    };
    std::function<void(int32_t, uint64_t)> collect = [&](int32_t n, uint64_t depth) {
        n = unwrap(n);
        if (depth > S + 1)
            return;
        by_depth[depth].push_back(n);
        if (!m_nodes[n].leaf()) {
            collect(m_nodes[n].lo, depth + 1);
            collect(m_nodes[n].hi, depth + 1);
        }
    };
    collect(m_root, 0);

    // Planes: level s holds the 2^s tree bands then the 2^s - 1 staggered
    // bands across their boundaries (merges of adjacent level s+1 bands).
    auto add_plane = [&](int32_t node, int32_t level, int32_t idx, int32_t stag) {
        Plane p;
        p.node          = node;
        p.height        = m_nodes[node].height;
        p.subband_level = level;
        p.subband_idx   = idx;
        p.staggered     = stag;
        p.chan_begin    = m_nodes[node].chan_begin;
        p.chan_end      = m_nodes[node].chan_end;
        p.f_lo          = m_nodes[node].f_lo;
        p.f_hi          = m_nodes[node].f_hi;
        m_planes.push_back(std::move(p));
    };
    add_plane(m_root, 0, 0, 0);
    for (uint64_t s = 1; s <= S; ++s) {
        const auto& band = by_depth[s];
        const auto& half = by_depth[s + 1];
        for (size_t i = 0; i < band.size(); ++i)
            add_plane(band[i], static_cast<int32_t>(s), static_cast<int32_t>(i), 0);
        for (size_t i = 0; i + 1 < band.size(); ++i) {
            const int32_t a = half[2 * i + 1], b = half[2 * i + 2];
            Node n;
            n.chan_begin    = m_nodes[a].chan_begin;
            n.chan_end      = m_nodes[b].chan_end;
            n.f_lo          = m_nodes[a].f_lo;
            n.f_hi          = m_nodes[b].f_hi;
            n.f_mid         = m_nodes[b].f_lo;
            n.staggered     = 1;
            const int32_t h = 1 + std::max(m_nodes[a].height, m_nodes[b].height);
            const int32_t lo = wrap(a, h - 1);
            const int32_t hi = wrap(b, h - 1);
            n.lo            = lo;
            n.hi            = hi;
            n.height        = h;
            m_nodes.push_back(n);
            add_plane(static_cast<int32_t>(m_nodes.size() - 1), static_cast<int32_t>(s),
                      static_cast<int32_t>(band.size() + i), 1);
        }
    }
    m_levels = 0;
    for (const auto& n : m_nodes)
        m_levels = std::max(m_levels, n.height);

    // Searched rows: distinct delays of the DM list across each plane band.
    std::vector<std::vector<int32_t>> demand(m_nodes.size());
    for (auto& p : m_planes) {
        int32_t last = -1;
        for (size_t k = 0; k < m_cfg.dm_list.size(); ++k) {
            const int32_t d = band_delay(m_cfg.dm_list[k], p.f_lo, p.f_hi);
            if (d != last) {
                p.delay.push_back(d);
                p.dm.push_back(m_cfg.dm_list[k]);
                p.dm_index.push_back(static_cast<int32_t>(k));
                last = d;
            }
        }
        auto& dem = demand[p.node];
        dem.insert(dem.end(), p.delay.begin(), p.delay.end());
    }
    // Propagate demands top-down (every parent has a greater height).
    std::vector<int32_t> order(m_nodes.size());
    for (size_t i = 0; i < order.size(); ++i)
        order[i] = static_cast<int32_t>(i);
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t a, int32_t b) { return m_nodes[a].height > m_nodes[b].height; });
    for (const int32_t id : order) {
        auto& dem = demand[id];
        std::sort(dem.begin(), dem.end());
        dem.erase(std::unique(dem.begin(), dem.end()), dem.end());
        Node& n   = m_nodes[id];
        n.delays  = dem;
        if (n.leaf())
            continue;
        for (const int32_t d : n.delays) {
            if (n.hi < 0) {
                demand[n.lo].push_back(d);
            } else {
                int32_t dl, dh;
                split_delay(n, d, dl, dh);
                demand[n.lo].push_back(dl);
                demand[n.hi].push_back(dh);
            }
        }
    }

    // Level buffers: rows of every node of height h, in node order.
    m_level_rows.assign(m_levels + 1, 0);
    m_level_hist.assign(m_levels + 1, 0);
    m_row_ops.assign(m_levels + 1, {});
    for (auto& n : m_nodes) {
        if (n.height == 0 || n.delays.empty())
            continue;
        n.row_offset = m_level_rows[n.height];
        m_level_rows[n.height] += static_cast<int64_t>(n.delays.size());
    }
    for (int32_t id = 0; id < static_cast<int32_t>(m_nodes.size()); ++id) {
        const Node& n = m_nodes[id];
        if (n.height == 0 || n.delays.empty())
            continue;
        for (const int32_t d : n.delays) {
            int32_t dl = d, dh = 0;
            if (n.hi >= 0)
                split_delay(n, d, dl, dh);
            if (n.height == 1) {
                const Node& a = m_nodes[n.lo];
                LeafOp op{a.chan_begin, n.hi >= 0 ? m_nodes[n.hi].chan_begin : -1, dl, dh};
                m_leaf_ops.push_back(op);
                m_level_hist[0] = std::max(m_level_hist[0], dl + dh);
                m_max_leaf_len  = std::max({m_max_leaf_len, dl + 1, dh + 1});
            } else {
                const Node& a = m_nodes[n.lo];
                RowOp op{};
                op.lo_row = static_cast<int32_t>(a.row_offset + a.row_of(dl));
                op.hi_row = -1;
                op.shift  = n.hi >= 0 ? dl : 0;
                op.delay  = d;
                if (n.hi >= 0) {
                    const Node& b = m_nodes[n.hi];
                    op.hi_row     = static_cast<int32_t>(b.row_offset + b.row_of(dh));
                    m_level_hist[n.height - 1] = std::max(m_level_hist[n.height - 1], dl);
                }
                m_row_ops[n.height].push_back(op);
            }
        }
    }
    const int32_t wmax = m_widths.back();
    for (auto& p : m_planes) {
        const Node& n = m_nodes[p.node];
        for (const int32_t d : p.delay)
            p.level_row.push_back(n.row_offset + n.row_of(d));
        m_level_hist[p.height] = std::max(m_level_hist[p.height], wmax - 1);
    }
    if (m_levels < 1)
        invalid("FDMT plan: need at least two channels");
}

int64_t Plan::max_level_rows() const {
    int64_t r = 0;
    for (int h = 1; h <= m_levels; ++h)
        r = std::max(r, m_level_rows[h]);
    return r;
}

int32_t Plan::max_history() const {
    int32_t h = 0;
    for (int i = 0; i <= m_levels; ++i)
        h = std::max(h, m_level_hist[i]);
    return h;
}

void Plan::descend(int32_t node, int32_t d, uint16_t* out, int32_t base) const {
    const Node& n = m_nodes[node];
    if (n.leaf()) {
        out[n.chan_begin - base] = static_cast<uint16_t>(std::min(d + 1, 65535));
        return;
    }
    if (n.hi < 0) {
        descend(n.lo, d, out, base);
        return;
    }
    int32_t dl, dh;
    split_delay(n, d, dl, dh);
    descend(n.lo, dl, out, base);
    descend(n.hi, dh, out, base);
}

std::vector<uint16_t> Plan::leaf_lengths(int p) const {
    const Plane& pl       = m_planes[p];
    const int32_t nch     = pl.chan_end - pl.chan_begin;
    std::vector<uint16_t> out(pl.delay.size() * static_cast<size_t>(nch), 0);
    for (size_t r = 0; r < pl.delay.size(); ++r)
        descend(pl.node, pl.delay[r], out.data() + r * nch, pl.chan_begin);
    return out;
}

} // namespace fb::fdmt
