// Host-side preparation of the factor for the sweep kernels.
//
// Produces the exact arrays the reference's CPU SpTRSV sweeps over
// (omp_sptrsv::setup_impl, include/apxchol/solver/sptrsv/omp.h:505-861):
//   * L11 = the leading m x m block of the factor (Laplacian: row/column n-1
//     dropped, omp.h:543-581);
//   * the compacting drop with column-sum compensation
//     (include/apxchol/solver/sptrsv/factor_drop.h:90-211), scale taken before
//     the drop (omp.h:627-650);
//   * CSC(L11) (the backward sweep, diagonal first) and CSR(L11) by the
//     column-order scatter (include/apxchol/solver/sptrsv/transpose.h:116-246;
//     diagonal last);
//   * the level of every row per direction -- from the elimination rounds
//     (omp.h:880-932) or the topological depth (omp.h:933-975) -- and from it
//     the per-row sum mode: rows of levels with <= 1024 rows use the 4-way
//     split sum, the others one serial sum (omp.h:32, 1094-1119, 1425-1445).
// With these the fp64 sweep kernels reproduce the reference's bytes.
#pragma once
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <new>
#include <string>
#include <thread>
#include <utility>
#include <vector>

namespace apxb {

constexpr uint32_t kThinLevelRows = 1024;   // kSpTRSVOMPThreshold, omp.h:32
constexpr double kDropRelDefault = 1e-4;    // kFactorDropRelDefault, factor_drop.h:70

// IEEE binary16 bit pattern of x, rounded to nearest even (overflow to
// infinity, subnormal results kept as subnormals).
inline uint16_t fp16_bits(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    const uint16_t sign = static_cast<uint16_t>((u >> 16) & 0x8000u);
    const uint32_t ax = u & 0x7fffffffu;
    if (ax >= 0x7f800000u)                                   // infinity, NaN (quiet, payload kept)
        return static_cast<uint16_t>(sign | 0x7c00u | (ax > 0x7f800000u ? 0x200u | ((ax >> 13) & 0x3ffu) : 0u));
    if (ax >= 0x477ff000u) return static_cast<uint16_t>(sign | 0x7c00u);   // >= 65520: rounds past 65504
    if (ax >= 0x38800000u) {                                 // >= 2^-14: a normal half
        const uint32_t v = ax - 0x38000000u;                 // exponent rebiased 127 -> 15
        return static_cast<uint16_t>(sign | ((v + 0xfffu + ((v >> 13) & 1u)) >> 13));
    }
    if (ax < 0x33000000u) return sign;                       // < 2^-25: rounds to zero
    // subnormal half: x / 2^-24 rounded to nearest even
    const uint32_t e = ax >> 23, mant = (ax & 0x7fffffu) | 0x800000u;
    const uint32_t shift = 126u - e;                          // 14 .. 24
    uint32_t q = mant >> shift;
    const uint32_t rem = mant & ((1u << shift) - 1u), half = 1u << (shift - 1u);
    if (rem > half || (rem == half && (q & 1u))) ++q;
    return static_cast<uint16_t>(sign | q);
}

// The value of a binary16 bit pattern (exact in fp32).
inline float fp16_value(uint16_t h) {
    const uint32_t sign = static_cast<uint32_t>(h & 0x8000u) << 16, e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
    uint32_t u;
    if (e == 0) {
        const float v = static_cast<float>(m) * 5.9604644775390625e-8f;   // m * 2^-24, exact
        std::memcpy(&u, &v, 4);
        u |= sign;
    } else if (e == 31) {
        u = sign | 0x7f800000u | (m << 13);
    } else {
        u = sign | ((e + 112u) << 23) | (m << 13);
    }
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// fp16 storage flushes x: it rounds to zero or to a subnormal (stored as zero).
inline bool fp16_flushes(float x) { return (fp16_bits(x) & 0x7c00u) == 0; }

// What the fp16 storage keeps for an entry v of a column with scale s:
// binary16(fp32(v) / s), subnormals flushed to signed zero
// (cuda_host.h:195-201).
inline uint16_t fp16_narrow(float v, float s) {
    const uint16_t h = fp16_bits(v / s);
    return (h & 0x7c00u) == 0 ? static_cast<uint16_t>(h & 0x8000u) : h;
}

// body(t) for t in [0, T), t = 0 on the calling thread. An exception thrown
// by any share is rethrown here after every thread has joined; when a thread
// cannot be started, the shares left run on the calling thread.
template <class F>
inline void run_threads(unsigned T, F&& body) {
    std::vector<std::exception_ptr> err(T);
    auto guarded = [&](unsigned t) {
        try {
            body(t);
        } catch (...) {
            err[t] = std::current_exception();
        }
    };
    std::vector<std::thread> th;
    th.reserve(T);
    unsigned started = 1;
    for (; started < T; ++started) {
        try {
            th.emplace_back(guarded, started);
        } catch (...) {
            break;
        }
    }
    guarded(0u);
    for (unsigned t = started; t < T; ++t) guarded(t);
    for (auto& x : th) x.join();
    for (auto& e : err)
        if (e) std::rethrow_exception(e);
}

// std::allocator whose value-less construct leaves the element uninitialized:
// resize() then costs no serial zero-fill, and the threads that write the
// array (every element) touch its pages first.
template <class T>
struct uninit_alloc : std::allocator<T> {
    template <class U>
    struct rebind { using other = uninit_alloc<U>; };
    uninit_alloc() = default;
    template <class U>
    uninit_alloc(const uninit_alloc<U>&) noexcept {}
    template <class U>
    void construct(U* p) noexcept { ::new (static_cast<void*>(p)) U; }
    template <class U, class... A>
    void construct(U* p, A&&... a) { ::new (static_cast<void*>(p)) U(std::forward<A>(a)...); }
};
template <class T>
using plan_vec = std::vector<T, uninit_alloc<T>>;

// Execution plan of one sweep direction, in the layout the dataflow kernels
// read.
//  * Rows are scheduled level by level; inside a level by lane-group width G
//    (the lanes that share one row: 1, 4, 8, 16 or 32 -- 1 for rows of <= 8
//    off-diagonals, else the smallest with 8 * G >= row length), widest first.
//    Rows of one level never depend on each other, so any order inside a
//    level gives the same result.
//  * A work item is up to 32 / G rows of one level and one G. Item c owns the
//    32 "positions" 32c .. 32c+31; slot s < count holds one row.
//  * Per position: `ord` = the row (kNoRow for an empty slot), and the row's
//    entries re-laid in processing order: off-diagonals in the reference's
//    order (forward: CSR row, columns ascending; backward: CSC column, rows
//    ascending), then the diagonal last, at [ptr[pos], ptr[pos + 1]).
//  * `info[c]` = count | log2(G) << 8 | thin << 16 (thin: the level uses the
//    4-way split sum; a level property, so uniform in an item).
//  * The serial segment (round-as-level factors only): the run of small
//    levels at the end of the elimination (the forward sweep's last levels,
//    the backward sweep's first), at most kSegLevelRows rows each. One thread
//    block solves it level by level through shared memory and __syncthreads,
//    which is far cheaper per level than a cross-SM dependency hop. Its rows
//    are the suffix [seg_first, m); `seg_row` lists them in processing order,
//    `seg_lvl` holds each level's start in that list (seg_levels + 1 words,
//    bit 31 = thin level), and their entries are re-laid like the items'
//    (`seg_ptr` per listed row, diagonal last).
struct sweep_plan {
    uint32_t n_items = 0;
    std::vector<int32_t> item_level;   // level of each item (host side; batch plans)
    std::vector<uint32_t> chunk;       // claim units of batch plans: chunk c = items [chunk[c], chunk[c+1])
    std::vector<uint32_t> info;
    plan_vec<uint32_t> ord;
    plan_vec<uint32_t> ptr;
    plan_vec<uint32_t> idx;
    plan_vec<float> val;
    plan_vec<uint16_t> val16;          // fp16 storage: the binary16 values, same layout as val
    uint32_t seg_first = 0, seg_rows = 0, seg_levels = 0;
    std::vector<uint32_t> seg_row, seg_lvl, seg_ptr, seg_idx;
    std::vector<float> seg_val;
};

// The serial segment is off by default (APXB_SEG_LEVEL_ROWS=<rows> enables it):
// on the factors measured so far the cross-SM dataflow hop beat it.
constexpr uint32_t kSegLevelRows = 0;    // a level joins the serial segment when it has <= this many rows
constexpr uint32_t kSegMaxRows = 4096;   // segment values stay in shared memory (fp64: 32 KB)
constexpr uint32_t kSegMinLevels = 8;    // fewer small trailing levels than this: no segment

constexpr uint32_t kNoRow = 0xffffffffu;

struct prepared_factor {
    uint32_t n = 0, m = 0;
    bool sddm = false;
    uint64_t nnz_factor = 0;     // L11 before the drop
    uint64_t nnz_stored = 0;     // after the drop
    uint64_t dropped = 0;
    // forward: CSR(L11), diagonal last in each row
    std::vector<uint32_t> csr_ptr;
    plan_vec<uint32_t> csr_idx;
    plan_vec<float> csr_val;
    // backward: CSC(L11), diagonal first in each column
    std::vector<uint32_t> csc_ptr;
    plan_vec<uint32_t> csc_idx;
    plan_vec<float> csc_val;
    // per-row 4-way-sum flag, bit-packed (bit r&31 of word r>>5)
    std::vector<uint32_t> fwd_thin_bits, bck_thin_bits;
    int32_t fwd_levels = 0, bck_levels = 0;
    std::vector<uint32_t> perm;  // perm[original] = position
    std::vector<int32_t> fwd_level, bck_level;   // level of every row per direction
    sweep_plan fwd_plan, bck_plan;
    // fp16 storage (the reference's cuda_sptrsv default, cuda.h:131-163;
    // cuda_host.h:16-34): column j is stored scaled by 1 / s_j (s_j the
    // pre-drop max |off-diagonal|; 1 when 1/s_j or L_jj/s_j overflows fp32),
    // off-diagonals as binary16, the diagonal as fp32 L_jj / s_j plus the
    // column's rounding residual. The forward sweep on the scaled factor
    // returns D y; the backward reads its input times inv_scale^2 (in fp64).
    bool fp16 = false;
    uint64_t dropped_flush = 0;                // off-diagonals dropped only because fp16 flushes them
    uint64_t flushed = 0;                      // stored off-diagonals v != 0 whose binary16 is zero
    plan_vec<uint16_t> csr_h, csc_h;           // binary16 values, same layout as csr_val / csc_val
    std::vector<float> diag16;                 // per row j: fp32(L_jj) / s_j + rounding residual
    std::vector<float> inv_scale;              // per row j: fp32(1 / s_j)
};

// Lane-group width for a row with `len` off-diagonals (see sweep_plan).
inline uint32_t group_width(uint32_t len) {
    if (len <= 8) return 1;
    uint32_t g = 4;
    while (g < 32 && g * 8 < len) g *= 2;
    return g;
}

// Work plan of the batched fp32 sweep with k right-hand sides per row (the
// column-lane kernels). Same item layout as sweep_plan, except:
//  * a row gets G = C * ge lanes: C column lanes, each holding min(k, 4) of the
//    k columns (C = k / min(k, 4)), times ge entry lanes (the smallest power
//    of two with 8 * ge >= off-diagonals, C * ge <= 32), so every lane keeps
//    up to 8 entries of 16-byte gathers in flight;
//  * a row's off-diagonals are ordered by the level of the row they depend on,
//    oldest first (ties by column), then the diagonal: consumed in order, a
//    row then waits only at its end, on its newest dependencies;
//  * item_level holds each item's level; chunk (see chunk_plan) the claim units;
//  * fp16 factors: val16 holds the binary16 values in the same layout (the
//    diagonal slot's is not read: the sweep divides by diag16 of the row).
// The fp32 sweep need not follow the reference's sum order (it has a
// tolerance); this order is fixed, so results stay deterministic.
void build_batch_plan(const prepared_factor& h, int dir, uint32_t col_lanes, sweep_plan& out);
// Claim units over a plan's items (in level order): consecutive items of one
// level, max(1, min(8, items of the level / 4096)) per unit, so large levels
// take one work-counter claim per several items while every warp stays busy.
void chunk_plan(sweep_plan& p);
// Invariants of a batch plan (rows once each, items in level order within one
// level, G >= col_lanes, diagonal last, chunks cover the items).
std::string check_batch_plan(uint32_t m, const std::vector<int32_t>& level, const sweep_plan& p, uint32_t col_lanes);

// Returns an empty string on success, else the reason the factor was rejected.
// fp16: also build the fp16 storage (prepared_factor::fp16); its drop then
// also removes the off-diagonals fp16 flushes (cuda_host.h:128-139).
std::string prepare_factor(uint32_t n, const uint32_t* colptr, const uint32_t* rowidx, const float* vals,
                           const uint32_t* perm, bool sddm, const uint64_t* rounds, uint32_t n_rounds,
                           double drop_rel, prepared_factor& out, bool fp16 = false);

// Full symmetric CSR of P A P^T (rows sorted) from A's full symmetric CSC and
// perm (what cuda_pcg::setup builds, include/apxchol/solver/pcg_cuda.h:304-404).
std::string permute_operator(uint32_t n, const int32_t* colptr, const int32_t* rowidx, const double* vals,
                             const uint32_t* perm, std::vector<int32_t>& ptr, plan_vec<int32_t>& idx,
                             plan_vec<double>& val);

}  // namespace apxb
