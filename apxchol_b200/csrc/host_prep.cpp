// Host-side factor preparation; see host_prep.hpp for the contract.
#include "host_prep.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <chrono>
#include <cstdio>
#include <exception>
#include <numeric>
#include <thread>

namespace apxb {

namespace {

// Per-column scale: max |off-diagonal| over [first+1, last) in double,
// stored fp32; 1.0f when the column has none (factor_drop.h:90-96).
float column_scale(const float* v, uint32_t first, uint32_t last) {
    double mx = 0.0;
    for (uint32_t p = first + 1; p < last; ++p) mx = std::max(mx, std::fabs(static_cast<double>(v[p])));
    return mx > 0.0 ? static_cast<float>(mx) : 1.0f;
}

// fp32 storage keep rule (omp.h:476-481): |v| >= rel*s and v != 0.
bool keep_offdiag(float v, float s, double rel) {
    return std::fabs(static_cast<double>(v)) >= rel * static_cast<double>(s) && v != 0.0f;
}

// Threads for a pass over `work` items: 1 below a million, else up to 8.
// APXB_PREP_THREADS=T (1..64) sets T whatever the size, so that tests can
// compare the threaded passes with the serial ones on small inputs.
unsigned prep_threads(uint64_t work) {
    if (const char* e = std::getenv("APXB_PREP_THREADS")) {
        const long t = std::strtol(e, nullptr, 10);
        if (t >= 1 && t <= 64) return static_cast<unsigned>(t);
    }
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    return work < (1u << 20) ? 1u : std::min(8u, hw);
}

// Column ranges of T threads with about equal entry counts: [jb[t], jb[t+1]).
template <class P>
std::vector<uint32_t> column_ranges(const P* ptr, uint32_t cols, unsigned T) {
    std::vector<uint32_t> jb(T + 1, cols);
    jb[0] = 0;
    const uint64_t total = ptr[cols] - ptr[0];
    for (unsigned t = 1; t < T; ++t) {
        const uint64_t target = ptr[0] + total * t / T;
        jb[t] = static_cast<uint32_t>(std::lower_bound(ptr, ptr + cols, target) - ptr);
        jb[t] = std::max(jb[t], jb[t - 1]);
    }
    return jb;
}

// Plan of one direction (see sweep_plan). level[r] = level of row r in this
// direction; (ptr, idx, val) = the canonical arrays of the direction (forward:
// CSR(L11), diagonal last; backward: CSC(L11), diagonal first).
// APXB_SEG_LEVEL_ROWS overrides kSegLevelRows (0 disables the serial segment).
uint32_t seg_level_rows_setting() {
    const char* e = std::getenv("APXB_SEG_LEVEL_ROWS");
    return e ? static_cast<uint32_t>(std::atoi(e)) : kSegLevelRows;
}

// Appends row r's entries re-laid (off-diagonals in the reference order, the
// diagonal last) to (oi, ov).
void relay_row(uint32_t r, bool forward, const std::vector<uint32_t>& ptr, const plan_vec<uint32_t>& idx,
               const plan_vec<float>& val, std::vector<uint32_t>& oi, std::vector<float>& ov) {
    const uint32_t b = ptr[r], en = ptr[r + 1];
    const uint32_t d = forward ? en - 1 : b;
    for (uint32_t p = b; p < en; ++p) {
        if (p == d) continue;
        oi.push_back(idx[p]); ov.push_back(val[p]);
    }
    oi.push_back(idx[d]); ov.push_back(val[d]);
}

// Rows grouped by (level, class): levels ascending, classes 0..n_cls-1, rows
// ascending inside a group -- one stable counting sort. cls[r] == n_cls leaves
// row r out. start[l * n_cls + c] is where group (l, c) begins in rows.
void group_rows(uint32_t m, const std::vector<int32_t>& level, int32_t n_levels, const std::vector<uint8_t>& cls,
                uint32_t n_cls, std::vector<uint32_t>& rows, std::vector<uint32_t>& start) {
    const size_t nk = static_cast<size_t>(n_levels) * n_cls;
    start.assign(nk + 1, 0);
    for (uint32_t r = 0; r < m; ++r)
        if (cls[r] < n_cls) start[static_cast<size_t>(level[r]) * n_cls + cls[r] + 1]++;
    for (size_t k = 0; k < nk; ++k) start[k + 1] += start[k];
    rows.resize(start[nk]);
    std::vector<uint32_t> cur(start.begin(), start.end() - 1);
    for (uint32_t r = 0; r < m; ++r)
        if (cls[r] < n_cls) rows[cur[static_cast<size_t>(level[r]) * n_cls + cls[r]]++] = r;
}

// val16 (fp16 storage, nullable): binary16 values beside val, re-laid the
// same way into plan.val16; such plans have no serial segment.
void build_plan(uint32_t m, const std::vector<int32_t>& level, int32_t n_levels, const std::vector<uint32_t>& bits,
                const std::vector<uint32_t>& ptr, const plan_vec<uint32_t>& idx, const plan_vec<float>& val,
                bool forward, bool contiguous, sweep_plan& plan, const plan_vec<uint16_t>* val16 = nullptr) {
    if (val16) contiguous = false;
    plan = sweep_plan{};
    // Serial segment: the trailing run (forward order) of small levels.
    int32_t seg_from = n_levels;   // in this direction's level numbering: forward [seg_from, n), backward [0, seg_to)
    int32_t seg_to = 0;
    const uint32_t seg_rows_max = seg_level_rows_setting();
    if (contiguous && seg_rows_max > 0) {
        std::vector<std::vector<uint32_t>> by_level(static_cast<size_t>(n_levels));
        for (uint32_t r = 0; r < m; ++r) by_level[level[r]].push_back(r);
        uint32_t rows = 0;
        int32_t nseg = 0;
        for (int32_t k = 0; k < n_levels; ++k) {            // k-th level from the forward end
            const int32_t l = forward ? n_levels - 1 - k : k;
            const uint32_t c = static_cast<uint32_t>(by_level[l].size());
            if (c > seg_rows_max || rows + c > kSegMaxRows) break;
            rows += c;
            ++nseg;
        }
        if (nseg >= static_cast<int32_t>(kSegMinLevels)) {
            if (forward) seg_from = n_levels - nseg;
            else seg_to = nseg;
        }
        auto in_seg = [&](int32_t l) { return forward ? l >= seg_from : l < seg_to; };
        if (seg_from < n_levels || seg_to > 0) {
            plan.seg_first = m;
            plan.seg_ptr.push_back(0);
            for (int32_t l = 0; l < n_levels; ++l) {
                if (!in_seg(l)) continue;
                const auto& lr = by_level[l];
                const uint32_t thin = lr.empty() ? 0u : (bits[lr[0] >> 5] >> (lr[0] & 31)) & 1u;
                plan.seg_lvl.push_back(static_cast<uint32_t>(plan.seg_row.size()) | (thin << 31));
                for (uint32_t r : lr) {
                    plan.seg_row.push_back(r);
                    plan.seg_first = std::min(plan.seg_first, r);
                    relay_row(r, forward, ptr, idx, val, plan.seg_idx, plan.seg_val);
                    plan.seg_ptr.push_back(static_cast<uint32_t>(plan.seg_idx.size()));
                }
            }
            plan.seg_levels = static_cast<uint32_t>(plan.seg_lvl.size());
            plan.seg_lvl.push_back(static_cast<uint32_t>(plan.seg_row.size()));
            plan.seg_rows = static_cast<uint32_t>(plan.seg_row.size());
        }
    }
    auto in_seg = [&](int32_t l) { return forward ? l >= seg_from : l < seg_to; };
    // items: (level, G) groups, G = 32, 16, 8, 4, 1 (classes 0..4), cut into 32/G rows
    constexpr uint32_t kCls = 5;
    std::vector<uint8_t> cls(m);
    std::vector<uint32_t> first_row(static_cast<size_t>(n_levels), kNoRow);   // a level's smallest row (its thin bit)
    for (uint32_t r = 0; r < m; ++r) {
        const uint32_t g = group_width(ptr[r + 1] - ptr[r] - 1);
        cls[r] = in_seg(level[r]) ? kCls : static_cast<uint8_t>(g == 1 ? 4 : 5 - __builtin_ctz(g));
        if (first_row[level[r]] == kNoRow) first_row[level[r]] = r;
    }
    std::vector<uint32_t> item_rows, start;
    group_rows(m, level, n_levels, cls, kCls, item_rows, start);
    for (int32_t l = 0; l < n_levels; ++l) {
        if (in_seg(l) || first_row[l] == kNoRow) continue;
        const uint32_t thin = (bits[first_row[l] >> 5] >> (first_row[l] & 31)) & 1u;
        for (uint32_t c = 0; c < kCls; ++c) {
            const size_t key = static_cast<size_t>(l) * kCls + c;
            const uint32_t lg = c == 4 ? 0u : 5u - c, cap = 32u >> lg;
            for (uint32_t q = start[key]; q < start[key + 1]; q += cap) {
                plan.info.push_back(std::min(cap, start[key + 1] - q) | (lg << 8) | (thin << 16));
                plan.item_level.push_back(l);
            }
        }
    }
    plan.n_items = static_cast<uint32_t>(plan.info.size());
    const size_t npos = static_cast<size_t>(plan.n_items) * 32;
    plan.ord.resize(npos);      // uninitialized: every position is written below
    plan.ptr.resize(npos + 1);
    // entry offsets, then the items filled on T threads (see build_batch_plan)
    std::vector<uint32_t> item_k(static_cast<size_t>(plan.n_items) + 1, 0);
    for (uint32_t c = 0; c < plan.n_items; ++c) item_k[c + 1] = item_k[c] + (plan.info[c] & 0xffu);
    std::vector<uint32_t> row_e(item_rows.size() + 1, 0);
    for (size_t k = 0; k < item_rows.size(); ++k) row_e[k + 1] = row_e[k] + (ptr[item_rows[k] + 1] - ptr[item_rows[k]]);
    const uint32_t total = row_e.back();
    plan.idx.resize(total);
    plan.val.resize(total);
    if (val16) plan.val16.resize(total);
    std::vector<uint32_t> item_e(static_cast<size_t>(plan.n_items) + 1);
    for (uint32_t c = 0; c <= plan.n_items; ++c) item_e[c] = row_e[item_k[c]];
    const unsigned T = prep_threads(total);
    const std::vector<uint32_t> cb = column_ranges(item_e.data(), plan.n_items, T);
    run_threads(T, [&](unsigned t) {
        for (uint32_t c = cb[t]; c < cb[t + 1]; ++c) {
            const uint32_t cnt = plan.info[c] & 0xffu;
            for (uint32_t sl = 0; sl < 32; ++sl) {
                const size_t pos = static_cast<size_t>(c) * 32 + sl;
                if (sl >= cnt) { plan.ord[pos] = kNoRow; plan.ptr[pos] = row_e[item_k[c] + cnt]; continue; }
                const uint32_t k = item_k[c] + sl, r = item_rows[k];
                uint32_t e = row_e[k];
                plan.ptr[pos] = e;
                plan.ord[pos] = r;
                const uint32_t b = ptr[r], en = ptr[r + 1];
                const uint32_t d = forward ? en - 1 : b;                 // diagonal slot
                for (uint32_t p = b; p < en; ++p) {
                    if (p == d) continue;
                    plan.idx[e] = idx[p]; plan.val[e] = val[p];
                    if (val16) plan.val16[e] = (*val16)[p];
                    ++e;
                }
                plan.idx[e] = idx[d]; plan.val[e] = val[d];             // diagonal last
                if (val16) plan.val16[e] = (*val16)[d];
            }
        }
    });
    plan.ptr[npos] = total;
    chunk_plan(plan);
}

// Plan invariants the kernels rely on (checked at every setup): every row is
// in exactly one slot; items hold 1..32/G rows of one level, in nondecreasing
// level order; every slot's entries end with its own diagonal.
std::string check_plan(uint32_t m, const std::vector<int32_t>& level, const sweep_plan& pl) {
    std::vector<uint8_t> seen(m, 0);
    int32_t prev = -1;
    for (uint32_t c = 0; c < pl.n_items; ++c) {
        const uint32_t cnt = pl.info[c] & 0xffu, lg = (pl.info[c] >> 8) & 0xffu;
        if (cnt == 0 || lg > 5 || lg == 1 || cnt > (32u >> lg)) return "bad plan item";
        int32_t l = -1;
        for (uint32_t s = 0; s < 32; ++s) {
            const size_t pos = static_cast<size_t>(c) * 32 + s;
            const uint32_t r = pl.ord[pos];
            if (s >= cnt) {
                if (r != kNoRow || pl.ptr[pos + 1] != pl.ptr[pos]) return "non-empty padding slot";
                continue;
            }
            if (r >= m || seen[r]) return "plan lists a row twice or out of range";
            seen[r] = 1;
            if (pl.ptr[pos + 1] <= pl.ptr[pos] || pl.idx[pl.ptr[pos + 1] - 1] != r) return "slot diagonal misplaced";
            if (l < 0) l = level[r];
            else if (level[r] != l) return "plan item spans two levels";
        }
        if (l < prev) return "plan items out of level order";
        prev = l;
    }
    if (pl.seg_rows) {
        if (pl.seg_first + pl.seg_rows != m) return "serial segment is not a suffix";
        for (uint32_t i = 0; i < pl.seg_rows; ++i) {
            const uint32_t r = pl.seg_row[i];
            if (r < pl.seg_first || r >= m || seen[r]) return "bad segment row";
            seen[r] = 1;
            if (pl.seg_ptr[i + 1] <= pl.seg_ptr[i] || pl.seg_idx[pl.seg_ptr[i + 1] - 1] != r)
                return "segment diagonal misplaced";
        }
        for (uint32_t l = 0; l < pl.seg_levels; ++l) {
            const uint32_t lo = pl.seg_lvl[l] & 0x7fffffffu, hi = pl.seg_lvl[l + 1] & 0x7fffffffu;
            if (hi < lo) return "bad segment level";
            for (uint32_t i = lo; i < hi; ++i)
                if (level[pl.seg_row[i]] != level[pl.seg_row[lo]]) return "segment level mixes levels";
        }
    }
    for (uint32_t r = 0; r < m; ++r)
        if (!seen[r]) return "plan misses row " + std::to_string(r);
    if (pl.chunk.empty() || pl.chunk.front() != 0 || pl.chunk.back() != pl.n_items) return "bad chunk table";
    for (size_t i = 0; i + 1 < pl.chunk.size(); ++i)
        if (pl.chunk[i + 1] <= pl.chunk[i] || pl.chunk[i + 1] - pl.chunk[i] > 8) return "bad chunk";
    return {};
}

// APXB_PREP_TRACE=1: the time of each preparation stage on stderr.
struct stage_clock {
    bool on = false;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    stage_clock() {
        const char* e = std::getenv("APXB_PREP_TRACE");
        on = e && *e && *e != '0';
    }
    void mark(const char* what) {
        if (!on) return;
        const auto t = std::chrono::steady_clock::now();
        std::fprintf(stderr, "[apxb prep] %-22s %8.2f ms\n", what,
                     std::chrono::duration<double, std::milli>(t - t0).count());
        t0 = t;
    }
};

void level_bits(const std::vector<int32_t>& level, int32_t n_levels, std::vector<uint32_t>& bits) {
    std::vector<uint32_t> cnt(static_cast<size_t>(n_levels) + 1, 0);
    for (int32_t l : level) cnt[l]++;
    bits.assign((level.size() + 31) / 32, 0u);
    for (size_t r = 0; r < level.size(); ++r)
        if (cnt[level[r]] <= kThinLevelRows) bits[r >> 5] |= 1u << (r & 31);
}

}  // namespace

void build_batch_plan(const prepared_factor& h, int dir, uint32_t col_lanes, sweep_plan& plan) {
    const bool forward = dir == 0;
    const uint32_t m = h.m;
    const std::vector<int32_t>& level = forward ? h.fwd_level : h.bck_level;
    const int32_t n_levels = forward ? h.fwd_levels : h.bck_levels;
    const std::vector<uint32_t>& ptr = forward ? h.csr_ptr : h.csc_ptr;
    const plan_vec<uint32_t>& idx = forward ? h.csr_idx : h.csc_idx;
    const plan_vec<float>& val = forward ? h.csr_val : h.csc_val;
    auto width = [&](uint32_t r) {
        const uint32_t len = ptr[r + 1] - ptr[r] - 1;
        uint32_t ge = 1;
        while (ge * col_lanes < 32 && ge * 8 < len) ge *= 2;
        return ge * col_lanes;
    };
    // items: (level, G) groups, G = 32, 16, ..., col_lanes (class c: G = 32 >> c),
    // cut into 32/G rows; rows ascending inside a group
    uint32_t n_cls = 1;
    while ((32u >> (n_cls - 1)) > col_lanes) ++n_cls;
    std::vector<uint8_t> cls(m);
    for (uint32_t r = 0; r < m; ++r) cls[r] = static_cast<uint8_t>(5 - __builtin_ctz(width(r)));
    std::vector<uint32_t> item_rows, start;
    group_rows(m, level, n_levels, cls, n_cls, item_rows, start);
    plan = sweep_plan{};
    for (int32_t l = 0; l < n_levels; ++l)
        for (uint32_t c = 0; c < n_cls; ++c) {
            const size_t key = static_cast<size_t>(l) * n_cls + c;
            const uint32_t lg = 5u - c, cap = 32u >> lg;
            for (uint32_t q = start[key]; q < start[key + 1]; q += cap) {
                plan.info.push_back(std::min(cap, start[key + 1] - q) | (lg << 8));
                plan.item_level.push_back(l);
            }
        }
    plan.n_items = static_cast<uint32_t>(plan.info.size());
    const size_t npos = static_cast<size_t>(plan.n_items) * 32;
    plan.ord.resize(npos);      // uninitialized: every position is written below
    plan.ptr.resize(npos + 1);
    // Entry offsets first (row k of item_rows starts at row_e[k], item c's rows
    // at item_k[c]), then the items are filled on T threads, each over a range
    // of items with about equal entry counts: the same arrays as one pass.
    std::vector<uint32_t> item_k(static_cast<size_t>(plan.n_items) + 1, 0);
    for (uint32_t c = 0; c < plan.n_items; ++c) item_k[c + 1] = item_k[c] + (plan.info[c] & 0xffu);
    std::vector<uint32_t> row_e(item_rows.size() + 1, 0);
    for (size_t k = 0; k < item_rows.size(); ++k) row_e[k + 1] = row_e[k] + (ptr[item_rows[k] + 1] - ptr[item_rows[k]]);
    const uint32_t total = row_e.back();
    plan.idx.resize(total);
    plan.val.resize(total);
    const plan_vec<uint16_t>* val16 = h.fp16 ? (forward ? &h.csr_h : &h.csc_h) : nullptr;
    if (val16) plan.val16.resize(total);
    std::vector<uint32_t> item_e(static_cast<size_t>(plan.n_items) + 1);
    for (uint32_t c = 0; c <= plan.n_items; ++c) item_e[c] = row_e[item_k[c]];
    const unsigned T = prep_threads(total);
    const std::vector<uint32_t> cb = column_ranges(item_e.data(), plan.n_items, T);
    run_threads(T, [&](unsigned t) {
        std::vector<std::pair<int32_t, uint32_t>> order;   // (dependency level, position in the row)
        for (uint32_t c = cb[t]; c < cb[t + 1]; ++c) {
            const uint32_t cnt = plan.info[c] & 0xffu;
            for (uint32_t sl = 0; sl < 32; ++sl) {
                const size_t pos = static_cast<size_t>(c) * 32 + sl;
                if (sl >= cnt) { plan.ord[pos] = kNoRow; plan.ptr[pos] = row_e[item_k[c] + cnt]; continue; }
                const uint32_t k = item_k[c] + sl, r = item_rows[k];
                uint32_t e = row_e[k];
                plan.ptr[pos] = e;
                plan.ord[pos] = r;
                const uint32_t b = ptr[r], en = ptr[r + 1];
                const uint32_t d = forward ? en - 1 : b;
                order.clear();
                for (uint32_t p = b; p < en; ++p)
                    if (p != d) order.emplace_back(level[idx[p]], p);
                std::sort(order.begin(), order.end(), [&](const auto& x, const auto& y) {
                    return x.first != y.first ? x.first < y.first : idx[x.second] < idx[y.second];
                });
                for (const auto& o : order) {
                    plan.idx[e] = idx[o.second];
                    plan.val[e] = val[o.second];
                    if (val16) plan.val16[e] = (*val16)[o.second];
                    ++e;
                }
                plan.idx[e] = idx[d]; plan.val[e] = val[d];
                if (val16) plan.val16[e] = (*val16)[d];
            }
        }
    });
    plan.ptr[npos] = total;
    chunk_plan(plan);
}

void chunk_plan(sweep_plan& p) {
    p.chunk.clear();
    uint32_t c = 0;
    while (c < p.n_items) {
        uint32_t e = c;
        while (e < p.n_items && p.item_level[e] == p.item_level[c]) ++e;
        const uint32_t per = std::max(1u, std::min(8u, (e - c) / 4096u));
        for (uint32_t s = c; s < e; s += per) p.chunk.push_back(s);
        c = e;
    }
    p.chunk.push_back(p.n_items);
}

std::string check_batch_plan(uint32_t m, const std::vector<int32_t>& level, const sweep_plan& pl, uint32_t col_lanes) {
    std::vector<uint8_t> seen(m, 0);
    int32_t prev = -1;
    if (pl.item_level.size() != pl.n_items || pl.info.size() != pl.n_items) return "bad batch plan sizes";
    for (uint32_t c = 0; c < pl.n_items; ++c) {
        const uint32_t cnt = pl.info[c] & 0xffu, lg = (pl.info[c] >> 8) & 0xffu;
        if (cnt == 0 || lg > 5 || (1u << lg) < col_lanes || cnt > (32u >> lg)) return "bad batch plan item";
        for (uint32_t s = 0; s < 32; ++s) {
            const size_t pos = static_cast<size_t>(c) * 32 + s;
            const uint32_t r = pl.ord[pos];
            if (s >= cnt) {
                if (r != kNoRow || pl.ptr[pos + 1] != pl.ptr[pos]) return "non-empty padding slot";
                continue;
            }
            if (r >= m || seen[r]) return "batch plan lists a row twice or out of range";
            seen[r] = 1;
            if (pl.ptr[pos + 1] <= pl.ptr[pos] || pl.idx[pl.ptr[pos + 1] - 1] != r) return "slot diagonal misplaced";
            if (level[r] != pl.item_level[c]) return "batch plan item level mismatch";
            for (uint32_t q = pl.ptr[pos]; q + 1 < pl.ptr[pos + 1]; ++q)
                if (pl.idx[q] >= m || level[pl.idx[q]] >= level[r]) return "batch plan dependency not older";
        }
        if (pl.item_level[c] < prev) return "batch plan items out of level order";
        prev = pl.item_level[c];
    }
    for (uint32_t r = 0; r < m; ++r)
        if (!seen[r]) return "batch plan misses row " + std::to_string(r);
    if (pl.chunk.empty() || pl.chunk.front() != 0 || pl.chunk.back() != pl.n_items) return "bad chunk table";
    for (size_t i = 0; i + 1 < pl.chunk.size(); ++i) {
        const uint32_t lo = pl.chunk[i], hi = pl.chunk[i + 1];
        if (hi <= lo || hi - lo > 8 || pl.item_level[hi - 1] != pl.item_level[lo]) return "bad chunk";
    }
    return {};
}

std::string prepare_factor(uint32_t n, const uint32_t* colptr, const uint32_t* rowidx, const float* vals,
                           const uint32_t* perm, bool sddm, const uint64_t* rounds, uint32_t n_rounds,
                           double drop_rel, prepared_factor& out, bool fp16) {
    if (n == 0) return "empty factor";
    if (!sddm && n < 2) return "a Laplacian factor needs n >= 2";
    const uint32_t m = sddm ? n : n - 1;
    out = prepared_factor{};
    out.n = n; out.m = m; out.sddm = sddm; out.fp16 = fp16;
    const double rel = drop_rel < 0.0 ? kDropRelDefault : drop_rel;

    stage_clock clk;
    // Validate the storage contract: colptr monotone, each column starts
    // with its diagonal, rows strictly ascending and < n.
    if (colptr[0] != 0) return "colptr[0] != 0";
    for (uint32_t j = 0; j < n; ++j) {
        const uint32_t b = colptr[j], e = colptr[j + 1];
        if (e <= b) return "column " + std::to_string(j) + " is empty (no diagonal)";
        if (rowidx[b] != j) return "column " + std::to_string(j) + " does not start with its diagonal";
        for (uint32_t p = b + 1; p < e; ++p)
            if (rowidx[p] <= rowidx[p - 1] || rowidx[p] >= n)
                return "column " + std::to_string(j) + " rows not ascending / out of range";
        if (!(vals[b] > 0.0f) || !std::isfinite(vals[b]))
            return "column " + std::to_string(j) + " has a non-positive or non-finite diagonal";
    }

    clk.mark("validate");
    // L11 (drop row n-1 for a Laplacian), then the compacting drop, written
    // straight into the CSC arrays; with fp16 storage each column is then
    // narrowed (cuda_host.h:202-232). Columns are independent: pass 1 counts
    // what each keeps, a prefix sum places them, pass 2 writes them -- on T
    // threads over column ranges (factor_drop.h:131-211 has the same shape).
    std::vector<uint32_t>& cp = out.csc_ptr;
    plan_vec<uint32_t>& ci = out.csc_idx;     // uninitialized on resize: pass 2 writes every entry
    plan_vec<float>& cv = out.csc_val;
    plan_vec<uint16_t>& ch = out.csc_h;
    cp.assign(static_cast<size_t>(m) + 1, 0);
    // a Laplacian's L11 leaves out row n-1: the column's last row when present
    auto col_end = [&](uint32_t j) {
        uint32_t e = colptr[j + 1];
        if (!sddm && e > colptr[j] + 1 && rowidx[e - 1] == n - 1) --e;
        return e;
    };
    // fp16 storage also drops what it would flush (cuda_host.h:135-139)
    auto kept = [&](float v, float s) { return keep_offdiag(v, s, rel) && !(fp16 && fp16_flushes(v / s)); };
    std::vector<float> col_s(m);
    const unsigned TD = prep_threads(colptr[m]);
    const std::vector<uint32_t> jd = column_ranges(colptr, m, TD);
    std::vector<uint64_t> nf_t(TD), dr_t(TD), df_t(TD), fl_t(TD);
    run_threads(TD, [&](unsigned t) {
        uint64_t nf = 0;
        for (uint32_t j = jd[t]; j < jd[t + 1]; ++j) {
            const uint32_t b = colptr[j], e = col_end(j);
            nf += e - b;
            float s = 1.0f;   // the column's scale, taken before the drop
            if (rel > 0.0 || fp16) {
                s = column_scale(vals, b, e);
                // fp16 storage: a scale whose 1/s or diagonal/s overflows fp32
                // falls back to 1, before the drop (cuda.h:287-301)
                if (fp16 && (!std::isfinite(1.0f / s) || !std::isfinite(vals[b] / s))) s = 1.0f;
            }
            col_s[j] = s;
            uint32_t k = e - b;
            if (rel > 0.0) {
                k = 1;                                     // the diagonal, first in the column
                for (uint32_t p = b + 1; p < e; ++p) k += kept(vals[p], s) ? 1u : 0u;
            }
            cp[j + 1] = k;
        }
        nf_t[t] = nf;
    });
    for (uint32_t j = 0; j < m; ++j) cp[j + 1] += cp[j];
    ci.resize(cp[m]);
    cv.resize(cp[m]);
    if (fp16) {
        ch.resize(cp[m]);
        out.diag16.resize(m);
        out.inv_scale.resize(m);
    }
    run_threads(TD, [&](unsigned t) {
        uint64_t dr = 0, df = 0, fl = 0;
        for (uint32_t j = jd[t]; j < jd[t + 1]; ++j) {
            const uint32_t b = colptr[j], e = col_end(j), first = cp[j];
            const float s = col_s[j];
            uint32_t o = first;
            if (rel > 0.0) {
                double dropped_sum = 0.0, kept_abs = 0.0;
                for (uint32_t p = b; p < e; ++p) {
                    const float v = vals[p];
                    if (p != b) {
                        if (!kept(v, s)) {
                            if (std::fabs(static_cast<double>(v)) >= rel * static_cast<double>(s)) ++df;
                            dropped_sum += static_cast<double>(v);
                            ++dr;
                            continue;
                        }
                        kept_abs += std::fabs(static_cast<double>(v));
                    }
                    ci[o] = rowidx[p]; cv[o] = v; ++o;
                }
                if (dropped_sum != 0.0 && kept_abs > 0.0) {
                    const double per_abs = dropped_sum / kept_abs;
                    for (uint32_t q = first + 1; q < o; ++q) {
                        const double v = static_cast<double>(cv[q]);
                        cv[q] = static_cast<float>(v + per_abs * std::fabs(v));
                    }
                }
            } else {
                for (uint32_t p = b; p < e; ++p) { ci[o] = rowidx[p]; cv[o] = vals[p]; ++o; }
            }
            if (fp16) {
                // off-diagonals as binary16(v / s); the diagonal as fp32 d / s
                // plus the column's rounding residual, so the stored column sums
                // to what the fp32 column sums to
                const float d = cv[first] / s;
                ch[first] = fp16_narrow(cv[first], s);      // the diagonal's slot (never read)
                double resid = 0.0;
                for (uint32_t q = first + 1; q < o; ++q) {
                    const float v = cv[q];
                    const uint16_t h = fp16_narrow(v, s);
                    ch[q] = h;
                    const float w = fp16_value(h);
                    if (v != 0.0f && w == 0.0f) ++fl;
                    resid += static_cast<double>(v) / static_cast<double>(s) - static_cast<double>(w);
                }
                out.diag16[j] = static_cast<float>(static_cast<double>(d) + resid);
                out.inv_scale[j] = 1.0f / s;
            }
        }
        dr_t[t] = dr; df_t[t] = df; fl_t[t] = fl;
    });
    uint64_t nnz_factor = 0, dropped = 0, dropped_flush = 0, flushed = 0;
    for (unsigned t = 0; t < TD; ++t) {
        nnz_factor += nf_t[t]; dropped += dr_t[t]; dropped_flush += df_t[t]; flushed += fl_t[t];
    }
    out.nnz_factor = nnz_factor;
    out.nnz_stored = ci.size();
    out.dropped = dropped;
    out.dropped_flush = dropped_flush;
    out.flushed = flushed;

    clk.mark("L11 + drop");
    // CSR by the column-order scatter: columns ascend within each row. On T
    // threads: thread t owns a range of columns (equal entry counts), counts
    // its entries per row, and scatters them at per-row offsets that follow the
    // ranges of threads 0..t-1 -- the same arrays the serial scatter makes.
    const uint64_t nnz = ci.size();
    out.csr_ptr.assign(static_cast<size_t>(m) + 1, 0);
    out.csr_idx.resize(nnz);
    out.csr_val.resize(nnz);
    if (fp16) out.csr_h.resize(nnz);
    {
        const unsigned T = prep_threads(nnz);
        const std::vector<uint32_t> jb = column_ranges(cp.data(), m, T);
        std::vector<std::vector<uint32_t>> cnt(T);
        run_threads(T, [&](unsigned t) {
            cnt[t].assign(m, 0);
            for (uint32_t p = cp[jb[t]]; p < cp[jb[t + 1]]; ++p) cnt[t][ci[p]]++;
        });
        // row lengths, row starts, then each thread's offset inside every row
        // (threads over row ranges)
        std::vector<uint32_t> len(m);
        run_threads(T, [&](unsigned t) {
            const uint32_t i1 = static_cast<uint32_t>(static_cast<uint64_t>(m) * (t + 1) / T);
            for (uint32_t i = static_cast<uint32_t>(static_cast<uint64_t>(m) * t / T); i < i1; ++i) {
                uint32_t c = 0;
                for (unsigned u = 0; u < T; ++u) c += cnt[u][i];
                len[i] = c;
            }
        });
        for (uint32_t i = 0; i < m; ++i) out.csr_ptr[i + 1] = out.csr_ptr[i] + len[i];
        run_threads(T, [&](unsigned t) {
            const uint32_t i1 = static_cast<uint32_t>(static_cast<uint64_t>(m) * (t + 1) / T);
            for (uint32_t i = static_cast<uint32_t>(static_cast<uint64_t>(m) * t / T); i < i1; ++i) {
                uint32_t acc = out.csr_ptr[i];
                for (unsigned u = 0; u < T; ++u) {
                    const uint32_t c = cnt[u][i];
                    cnt[u][i] = acc;
                    acc += c;
                }
            }
        });
        run_threads(T, [&](unsigned t) {
            std::vector<uint32_t>& cur = cnt[t];
            for (uint32_t j = jb[t]; j < jb[t + 1]; ++j)
                for (uint32_t p = cp[j]; p < cp[j + 1]; ++p) {
                    const uint32_t slot = cur[ci[p]]++;
                    out.csr_idx[slot] = j;
                    out.csr_val[slot] = cv[p];
                    if (fp16) out.csr_h[slot] = ch[p];
                }
        });
    }

    clk.mark("transpose");
    // Levels: round-as-level when the round bounds fit (omp.h:880-932), with
    // the bounds built as apx_cholesky::install_factor does
    // (preconditioner.h:247-258); else topological depths.
    std::vector<int32_t> fl(m), bl(m);
    bool done = false;
    if (n_rounds > 0) {
        std::vector<uint64_t> b(static_cast<size_t>(n_rounds) + 1, 0);
        uint64_t acc = 0;
        for (uint32_t r = 0; r < n_rounds; ++r) {
            acc += rounds[r];
            if (acc > m) acc = m;
            b[r + 1] = acc;
        }
        const uint64_t last = b[n_rounds];
        int32_t maxd = 0;
        uint32_t r = 0;
        for (uint32_t c = 0; c < m; ++c) {
            int32_t d;
            if (c >= last) {
                d = static_cast<int32_t>(n_rounds + (c - last));
            } else {
                while (r + 1 < n_rounds + 1 && c >= b[r + 1]) ++r;
                d = static_cast<int32_t>(r);
            }
            fl[c] = d;
            maxd = std::max(maxd, d);
        }
        for (uint32_t c = 0; c < m; ++c) bl[c] = maxd - fl[c];
        out.fwd_levels = out.bck_levels = maxd + 1;
        done = true;
    }
    if (!done) {
        int32_t maxf = 0, maxb = 0;
        for (uint32_t i = 0; i < m; ++i) {
            int32_t d = 0;
            for (uint32_t p = out.csr_ptr[i]; p + 1 < out.csr_ptr[i + 1]; ++p) d = std::max(d, fl[out.csr_idx[p]] + 1);
            fl[i] = d;
            maxf = std::max(maxf, d);
        }
        for (uint32_t j = m; j-- > 0;) {
            int32_t d = 0;
            for (uint32_t p = cp[j]; p < cp[j + 1]; ++p)
                if (ci[p] > j) d = std::max(d, bl[ci[p]] + 1);
            bl[j] = d;
            maxb = std::max(maxb, d);
        }
        out.fwd_levels = maxf + 1;
        out.bck_levels = maxb + 1;
    }
    level_bits(fl, out.fwd_levels, out.fwd_thin_bits);
    level_bits(bl, out.bck_levels, out.bck_thin_bits);
    clk.mark("levels");
    // Sweep plans (the kernels' layout), checked before anything is uploaded;
    // the two directions are independent and built on two threads.
    std::string bad[2];
    run_threads(2, [&](unsigned dir) {
        if (dir == 1) {
            build_plan(m, bl, out.bck_levels, out.bck_thin_bits, cp, ci, cv, false, done, out.bck_plan,
                       fp16 ? &ch : nullptr);
            bad[1] = check_plan(m, bl, out.bck_plan);
        } else {
            build_plan(m, fl, out.fwd_levels, out.fwd_thin_bits, out.csr_ptr, out.csr_idx, out.csr_val, true, done,
                       out.fwd_plan, fp16 ? &out.csr_h : nullptr);
            bad[0] = check_plan(m, fl, out.fwd_plan);
        }
    });
    for (int dir = 0; dir < 2; ++dir)
        if (!bad[dir].empty()) return "internal sweep plan error: " + bad[dir];
    out.fwd_level = std::move(fl);
    out.bck_level = std::move(bl);

    clk.mark("plans");
    // Permutation: must be a bijection of [0, n).
    out.perm.assign(perm, perm + n);
    {
        std::vector<uint8_t> seen(n, 0);
        for (uint32_t v = 0; v < n; ++v) {
            if (perm[v] >= n || seen[perm[v]]) return "perm is not a permutation of [0, n)";
            seen[perm[v]] = 1;
        }
    }
    return {};
}

std::string permute_operator(uint32_t n, const int32_t* colptr, const int32_t* rowidx, const double* vals,
                             const uint32_t* perm, std::vector<int32_t>& ptr, plan_vec<int32_t>& idx,
                             plan_vec<double>& val) {
    if (colptr[0] != 0) return "operator colptr[0] != 0";
    const int64_t nnz = colptr[n];
    if (nnz < 0 || nnz > INT32_MAX) return "operator nnz out of the int32 range";
    {
        std::vector<uint8_t> seen(n, 0);
        for (uint32_t v = 0; v < n; ++v) {
            if (perm[v] >= n || seen[perm[v]]) return "perm is not a permutation of [0, n)";
            seen[perm[v]] = 1;
        }
    }
    // A is symmetric, so its CSC column j is its CSR row j. Row perm[j] of
    // P A P^T holds the entries of row j with columns mapped through perm.
    ptr.assign(static_cast<size_t>(n) + 1, 0);
    for (uint32_t j = 0; j < n; ++j) {
        if (colptr[j + 1] < colptr[j]) return "operator colptr not monotone";
        ptr[perm[j] + 1] = colptr[j + 1] - colptr[j];
    }
    for (uint32_t i = 0; i < n; ++i) ptr[i + 1] += ptr[i];
    idx.resize(nnz);     // uninitialized: every entry is written below
    val.resize(nnz);
    // Rows are independent: T threads over column ranges of equal entry counts.
    const unsigned T = prep_threads(static_cast<uint64_t>(nnz));
    const std::vector<uint32_t> jb = column_ranges(colptr, n, T);
    std::vector<uint8_t> bad(T, 0);
    run_threads(T, [&](unsigned t) {
        std::vector<std::pair<int32_t, double>> row;
        for (uint32_t j = jb[t]; j < jb[t + 1]; ++j) {
            row.clear();
            for (int32_t p = colptr[j]; p < colptr[j + 1]; ++p) {
                const int32_t r = rowidx[p];
                if (r < 0 || static_cast<uint32_t>(r) >= n) { bad[t] = 1; return; }
                row.emplace_back(static_cast<int32_t>(perm[r]), vals[p]);
            }
            std::sort(row.begin(), row.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
            int32_t o = ptr[perm[j]];
            for (const auto& [c, v] : row) { idx[o] = c; val[o] = v; ++o; }
        }
    });
    for (unsigned t = 0; t < T; ++t)
        if (bad[t]) return "operator row index out of range";
    return {};
}

}  // namespace apxb
