// Device entropy coding and assembly (see entropy.cuh for the data model).
//
// Token and context semantics follow the reference encoder exactly: AC
// tokens as src/entropy.cu:649-681 with the contexts of src/ac_context.h and
// the fixed 32-cluster map; DC residuals with the modular Gradient predictor
// inside each DC group (src/entropy.cu:114-124); AcMetadata samples YtoX,
// YtoB, strategy row, quant-field row and EPF zeros under the Zero predictor
// (src/entropy.cu:252-274); hybrid-uint (4,2,0) tokens; prefix codes from
// prefix_code.cuh; section layout and headers as src/frame_encoder.cu:88-292
// and src/bitstream/{frame_assembly,codestream,container}.cc.
//
// AC block-channels are tokenised one warp per item: each lane takes one scan
// position of a 32-position chunk, and ballots plus prefix counts give every
// lane the reference's sequential state at its position (non-zeros left,
// previous-coefficient flag), so a chunk's tokens, contexts, bit lengths and
// bit offsets come out in one step. Every other item (header blobs, DC
// residuals, AcMetadata samples) takes one thread.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstring>

#include "entropy.cuh"
#include "jxl_constants.cuh"
#include "prefix_code.cuh"

namespace jxb {
namespace {

constexpr unsigned kFull = 0xffffffffu;

// Token channel order Y, X, B over planes stored X, Y, B.
__device__ __forceinline__ int phys_channel(int p) { return p == 0 ? 1 : (p == 1 ? 0 : 2); }

// Section holding `item`, searched in sections [lo, hi].
__device__ __forceinline__ int find_section(const Section* secs, int lo, int hi, std::uint32_t item) {
    while (lo < hi) {
        const int mid{(lo + hi + 1) >> 1};
        if (__ldg(&secs[mid].first) <= item) {
            lo = mid;
        } else {
            hi = mid - 1;
        }
    }
    return lo;
}

struct GroupGeom {
    int bx0, by0, gw, gh;
};

__device__ __forceinline__ GroupGeom ac_group_geom(const EntropyDev& e, int g) {
    GroupGeom r;
    r.bx0 = (g % e.xg) * kAcGroupBlocks;
    r.by0 = (g / e.xg) * kAcGroupBlocks;
    r.gw = min(kAcGroupBlocks, e.bw - r.bx0);
    r.gh = min(kAcGroupBlocks, e.bh - r.by0);
    return r;
}

__device__ __forceinline__ GroupGeom dc_group_geom(const EntropyDev& e, int g) {
    GroupGeom r;
    r.bx0 = (g % e.xdg) * kDcGroupBlocks;
    r.by0 = (g / e.xdg) * kDcGroupBlocks;
    r.gw = min(kDcGroupBlocks, e.bw - r.bx0);
    r.gh = min(kDcGroupBlocks, e.bh - r.by0);
    return r;
}

enum TokTable : int { kTabDc = 1, kTabAm = 2 };

__device__ __forceinline__ int misc_hi(const EntropyDev& e) { return e.ndc + 1; }

// ---- items other than AC block-channels -------------------------------------------

// Visits the bits of one non-AC item in stream order: blob(bytes, nbits),
// varlen(v), count_field(group, nbits), epf(group), first_block(group),
// token(table, group, symbol, extra_bits, extra_value).
template <class V>
__device__ void visit_misc(const EntropyDev& e, std::uint32_t item, V& v) {
    const int s{find_section(e.sections, 0, misc_hi(e), item)};
    const Section sec{e.sections[s]};
    const std::uint32_t j{item - sec.first};
    if (sec.kind == kSecDcGlobal) {
        v.blob(e.dc_global, e.dc_global_bits);
        return;
    }
    if (sec.kind == kSecAcGlobal) {
        if (j == 0) {
            v.blob(e.ac_prefix, e.ac_prefix_bits);
        } else if (j <= 32) {
            v.varlen(e.ac_alpha[j - 1] - 1);
        } else {
            v.blob(e.desc + (j - 33) * kDescBytes, e.desc_bits[j - 33]);
        }
        return;
    }
    const int g{sec.group};
    const GroupGeom gg{dc_group_geom(e, g)};
    const std::uint32_t n{static_cast<std::uint32_t>(gg.gw * gg.gh)};
    if (j == 0) {
        v.blob(e.pre_const, e.pre_const_bits);
        return;
    }
    if (j == 1) {
        v.blob(e.desc + (32 + g) * kDescBytes, e.desc_bits[32 + g]);
        return;
    }
    if (j < 2 + 3 * n) {
        const std::uint32_t sidx{j - 2};
        const int c{phys_channel(static_cast<int>(sidx / n))};
        const std::uint32_t bp{sidx % n};
        const int bx{gg.bx0 + static_cast<int>(bp % gg.gw)};
        const int by{gg.by0 + static_cast<int>(bp / gg.gw)};
        const std::int32_t* plane{e.dc + static_cast<std::size_t>(c) * e.nblocks};
        const std::size_t blk{static_cast<std::size_t>(by) * e.bw + bx};
        const bool hl{bx > gg.bx0};
        const bool ht{by > gg.by0};
        const std::int32_t w{hl ? plane[blk - 1] : 0};
        const std::int32_t nn{ht ? plane[blk - e.bw] : 0};
        const std::int32_t nw{(hl && ht) ? plane[blk - e.bw - 1] : 0};
        const std::int32_t pred{gradient_predict(hl, ht, w, nn, nw)};
        std::uint32_t tok, nb, bits;
        hybrid_uint(pack_signed(plane[blk] - pred), tok, nb, bits);
        v.token(kTabDc, g, tok, nb, bits);
        return;
    }
    if (j == 2 + 3 * n) {
        v.count_field(g, ceil_log2_u(n));
        return;
    }
    if (j == 3 + 3 * n) {
        v.blob(e.mid_const, e.mid_const_bits);
        return;
    }
    if (j == 4 + 3 * n) {
        v.blob(e.desc + (32 + e.ndc + g) * kDescBytes, e.desc_bits[32 + e.ndc + g]);
        return;
    }
    const std::uint32_t m{j - (5 + 3 * n)};
    const int cw{(gg.gw + 7) / 8};
    const int ch{(gg.gh + 7) / 8};
    const std::uint32_t cwch{static_cast<std::uint32_t>(cw * ch)};
    std::int32_t val{0};
    if (m < 2 * cwch) {
        const std::uint32_t t{m < cwch ? m : m - cwch};
        const std::size_t tile{static_cast<std::size_t>(gg.by0 / 8 + static_cast<int>(t) / cw) * e.cmw +
                               gg.bx0 / 8 + static_cast<int>(t) % cw};
        val = m < cwch ? e.ytox[tile] : e.ytob[tile];
    } else if (m < 2 * cwch + 2 * n) {
        const std::uint32_t r{m - 2 * cwch};
        const std::uint32_t b{r % n};
        const std::size_t blk{static_cast<std::size_t>(gg.by0 + static_cast<int>(b) / gg.gw) * e.bw +
                              gg.bx0 + static_cast<int>(b) % gg.gw};
        const int side{e.acs[blk]};
        if (side == 0) return;
        if (r < n) {
            val = raw_strategy(side);
            v.first_block(g);
        } else {
            val = e.qf[blk] - 1;
        }
    } else {
        v.epf(g);
        return;
    }
    std::uint32_t tok, nb, bits;
    hybrid_uint(pack_signed(val), tok, nb, bits);
    v.token(kTabAm, g, tok, nb, bits);
}

// ---- AC block-channels: one CTA per stripe staged in shared memory -------------------

constexpr int kAcThreads = 256;
constexpr int kAcWarps = kAcThreads / 32;
constexpr int kStripeItems = 3 * kStripeRows * kAcGroupBlocks;  // 384
constexpr int kRowSlots = kAcGroupBlocks * kCoeffsPerBlock;      // 2048
// AC token symbols are hybrid-uint (4, 2, 0) tokens of values below 2^16
// (packed int16 coefficients, counts up to 1008): at most 63.
constexpr int kAcSymbols = 64;
constexpr int kWindowWords = 4096;  // 16 KB of output bits assembled per CTA

__device__ __forceinline__ unsigned long long prefix_at(const EntropyDev& e, std::uint32_t i) {
    if (i >= e.total_items) return e.tile_off[e.num_tiles];
    return e.tile_off[i / kScanTile] + e.item_pre[i];
}

// ORs `n` (<= 32) bits of `v` at bit position `pos` of a zeroed word array in
// shared or global memory.
__device__ __forceinline__ void put_bits_at(unsigned int* words, unsigned long long pos, std::uint32_t n,
                                            std::uint32_t v) {
    while (n > 0) {
        const unsigned long long wi{pos >> 5};
        const std::uint32_t off{static_cast<std::uint32_t>(pos & 31)};
        const std::uint32_t take{n < 32 - off ? n : 32 - off};
        const std::uint32_t chunk{take == 32 ? v : (v & ((1u << take) - 1u))};
        if (chunk != 0) atomicOr(&words[wi], chunk << off);
        v = take == 32 ? 0 : v >> take;
        n -= take;
        pos += take;
    }
}

// A stripe's inputs in shared memory: the three coefficient planes of its
// block rows (row stride kRowSlots), the natural orders, strategies and
// non-zero counts (nzn row 0 is the block row above the stripe).
// Rows of the zero-density cluster table, padded to 16 bytes.
constexpr int kZdRow = (kZeroDensityCount + 15) & ~15;
constexpr int kCoeffCtxBytes = 64 + 64 + 2 * kZdRow;
// The context tables every stripe CTA stages (layout of StripeStage's
// nz_ctx .. zd_cluster), filled on each device by entropy_kernels_init.
__device__ __align__(16) std::uint8_t g_coeff_ctx[kCoeffCtxBytes];

struct StripeStage {
    std::int16_t coef[3][kStripeRows][kRowSlots];
    std::uint16_t order[64 + 256 + 1024];
    std::uint16_t nzc[3][kStripeRows][kAcGroupBlocks];
    std::uint8_t nzn[3][kStripeRows + 1][kAcGroupBlocks];
    std::int8_t acs[kStripeRows][kAcGroupBlocks];
    std::uint16_t active[kStripeItems];  // items with coefficient tokens
    std::uint32_t aux[kStripeItems];     // per-item bits (bits pass) or bit offset (emit pass)
    // The coefficient-token context as table lookups (a copy of
    // g_coeff_ctx): coeff_nz_ctx and coeff_freq_ctx of 1..63, and the
    // cluster of zero-density context z for luma (row 0) and chroma (row 1)
    // block contexts.
    alignas(16) std::uint8_t nz_ctx[64];
    std::uint8_t freq_ctx[64];
    std::uint8_t zd_cluster[2][kZdRow];
    int nactive;
};

// Asynchronous global -> shared copies (cp.async, sm_80 and later): a thread
// issues all of its copies before waiting once for them (cp_async_wait_all).
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    const unsigned dst{static_cast<unsigned>(__cvta_generic_to_shared(smem_dst))};
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gmem_src) {
    const unsigned dst{static_cast<unsigned>(__cvta_generic_to_shared(smem_dst))};
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// The caller's barrier after this publishes the stage to the whole CTA.
__device__ void stage_stripe(const EntropyDev& e, const Stripe& st, const GroupGeom& gg, StripeStage& s) {
    const int tid{static_cast<int>(threadIdx.x)};
    const int vpr{gg.gw * (kCoeffsPerBlock * 2 / 16)};  // 16-byte vectors per block row
    for (int c{0}; c < 3; ++c) {
        const std::int16_t* plane{e.ac + static_cast<std::size_t>(c) * e.nblocks * kCoeffsPerBlock};
        for (int r{0}; r < st.rows; ++r) {
            const std::size_t blk0{static_cast<std::size_t>(gg.by0 + st.r0 + r) * e.bw + gg.bx0};
            const uint4* src{reinterpret_cast<const uint4*>(plane + blk0 * kCoeffsPerBlock)};
            uint4* dst{reinterpret_cast<uint4*>(&s.coef[c][r][0])};
            for (int v{tid}; v < vpr; v += kAcThreads) cp_async16(&dst[v], &src[v]);
        }
    }
    for (int i{tid}; i < (64 + 256 + 1024) / 2; i += kAcThreads) {
        cp_async4(&reinterpret_cast<std::uint32_t*>(s.order)[i], &reinterpret_cast<const std::uint32_t*>(e.order)[i]);
    }
    const int cells{st.rows * gg.gw};
    for (int i{tid}; i < cells; i += kAcThreads) {
        const int r{i / gg.gw};
        const int x{i - r * gg.gw};
        const std::size_t blk{static_cast<std::size_t>(gg.by0 + st.r0 + r) * e.bw + gg.bx0 + x};
        s.acs[r][x] = e.acs[blk];
        for (int c{0}; c < 3; ++c) {
            const std::size_t cb{static_cast<std::size_t>(c) * e.nblocks + blk};
            s.nzc[c][r][x] = e.nzc[cb];
            s.nzn[c][r + 1][x] = e.nzn[cb];
            if (r == 0) s.nzn[c][0][x] = st.r0 > 0 ? e.nzn[cb - e.bw] : 0;
        }
    }
    static_assert(kCoeffCtxBytes % 16 == 0 && offsetof(StripeStage, zd_cluster) + 2 * kZdRow ==
                                                   offsetof(StripeStage, nz_ctx) + kCoeffCtxBytes,
                  "context tables: one contiguous 16-byte-aligned copy");
    for (int i{tid}; i < kCoeffCtxBytes / 16; i += kAcThreads) {
        cp_async16(reinterpret_cast<uint4*>(s.nz_ctx) + i, reinterpret_cast<const uint4*>(g_coeff_ctx) + i);
    }
    if (tid == 0) s.nactive = 0;
    cp_async_wait_all();
}

// Stripe-local item j: block (bx, by) of the stripe, plane c.
struct StripeItem {
    int c, bx, by, n;
    std::uint32_t nz;
};

__device__ __forceinline__ StripeItem stripe_item(const StripeStage& s, int gw, int j) {
    StripeItem it;
    const int bidx{j / 3};
    it.c = phys_channel(j - 3 * bidx);
    it.by = bidx / gw;
    it.bx = bidx - it.by * gw;
    it.n = s.acs[it.by][it.bx];
    it.nz = it.n != 0 ? s.nzc[it.c][it.by][it.bx] : 0u;
    return it;
}

// Count token of a non-covered item: cluster from the non-zero prediction of
// the group-local top and left neighbours (src/entropy.cu:649-652).
__device__ __forceinline__ void count_token(const StripeStage& s, const Stripe& st, const StripeItem& it, int& cl,
                                            std::uint32_t& tok, std::uint32_t& nb, std::uint32_t& bits) {
    const bool hl{it.bx > 0};
    const bool ht{st.r0 + it.by > 0};
    const std::uint32_t top{ht ? s.nzn[it.c][it.by][it.bx] : 0u};
    const std::uint32_t left{hl ? s.nzn[it.c][it.by + 1][it.bx - 1] : 0u};
    cl = context_cluster(nonzero_context(predict_nonzeros(hl, ht, top, left), block_ctx(it.c, it.n)));
    hybrid_uint(it.nz, tok, nb, bits);
}

// Calls f(has, cluster, symbol, extra_bits, extra_value) with all 32 lanes
// once per 32-position chunk of the item's scan, one coefficient token per
// lane in stream order. Ballots give each lane the reference's sequential
// state at its position (src/entropy.cu:653-680): a position is coded while
// non-zeros remain before it, and its context uses that count and whether the
// previous coefficient was non-zero.
template <class F>
__device__ void coeff_tokens(const StripeStage& s, const StripeItem& it, int lane, F&& f) {
    const int n{it.n};
    const int side{n >> 3};
    const int lside{side == 1 ? 0 : (side == 2 ? 1 : 2)};
    const std::uint32_t covered{static_cast<std::uint32_t>(side * side)};
    const std::uint32_t size{static_cast<std::uint32_t>(n * n)};
    const std::uint32_t l2{static_cast<std::uint32_t>(2 * lside)};
    const int bctx{block_ctx(it.c, n)};
    const std::uint16_t* ord{s.order + (n == 8 ? 0 : (n == 16 ? 64 : 320))};
    const std::int16_t* plane{&s.coef[it.c][it.by][it.bx * kCoeffsPerBlock]};
    std::uint32_t remaining{it.nz};
    std::uint32_t prev{it.nz > size / 16 ? 0u : 1u};
    const unsigned below{(1u << lane) - 1u};
    for (std::uint32_t k0{covered}; k0 < size && remaining > 0; k0 += 32) {
        const std::uint32_t k{k0 + static_cast<std::uint32_t>(lane)};
        std::int32_t val{0};
        if (k < size) {
            const int raw{ord[k]};
            const int q{raw >> 6};
            const int qy{q >> lside};
            const int qx{q & (side - 1)};
            // Transforms start at multiples of their size inside the group, so
            // the covered blocks lie in the stripe; planes that break this
            // layout read zeros instead of leaving the staged area.
            if (it.by + qy < kStripeRows && it.bx + qx < kAcGroupBlocks) {
                val = plane[qy * kRowSlots + qx * kCoeffsPerBlock + (raw & 63)];
            }
        }
        const unsigned nzmask{__ballot_sync(kFull, val != 0)};
        const std::uint32_t left{remaining - static_cast<std::uint32_t>(__popc(nzmask & below))};
        const std::uint32_t p{lane == 0 ? prev : ((nzmask >> (lane - 1)) & 1u)};
        const bool has{k < size && left > 0};
        std::uint32_t tok{0}, nb{0}, bits{0};
        int cl{0};
        if (has) {
            // context_cluster(coeff_context(bctx, left, k, covered, l2, p)):
            // the context is the block context's zero-density base plus z,
            // and its cluster depends only on z and luma/chroma. coeff_nz_ctx
            // is constant from 33 on, so the clamp to 63 changes nothing; z
            // stays below kZeroDensityCount whenever the item's count is its
            // non-zeros, and the clamp keeps the lookup in the table otherwise.
            const std::uint32_t nzi{min((left + covered - 1) >> l2, 63u)};
            const std::uint32_t z{min((static_cast<std::uint32_t>(s.nz_ctx[nzi]) + s.freq_ctx[k >> l2]) * 2 + p,
                                      static_cast<std::uint32_t>(kZeroDensityCount - 1))};
            cl = s.zd_cluster[bctx < 7 ? 0 : 1][z];
            hybrid_uint(pack_signed(val), tok, nb, bits);
        }
        f(has, cl, tok, nb, bits);
        remaining -= static_cast<std::uint32_t>(__popc(nzmask));
        prev = (nzmask >> 31) & 1u;
    }
}

__device__ __forceinline__ std::uint32_t warp_sum(std::uint32_t v) {
#pragma unroll
    for (int off{16}; off > 0; off >>= 1) v += __shfl_xor_sync(kFull, v, off);
    return v;
}

__device__ __forceinline__ std::uint32_t warp_incl_scan(std::uint32_t v, int lane) {
#pragma unroll
    for (int off{1}; off < 32; off <<= 1) {
        const std::uint32_t t{__shfl_up_sync(kFull, v, off)};
        if (lane >= off) v += t;
    }
    return v;
}

// An AC token in 32 bits: symbol (6 bits), cluster (5), extra-bit count (4)
// and extra bits (at most 13: packed coefficients stay below 2^16).
__device__ __forceinline__ std::uint32_t pack_ac_token(int cl, std::uint32_t sym, std::uint32_t nb,
                                                       std::uint32_t bits) {
    return (bits << 15) | (nb << 11) | (static_cast<std::uint32_t>(cl) << 6) | sym;
}
__device__ __forceinline__ std::uint32_t token_table_index(std::uint32_t t) {
    return ((t >> 6) & 31u) * 256u + (t & 63u);
}
__device__ __forceinline__ std::uint32_t token_extra_count(std::uint32_t t) { return (t >> 11) & 15u; }
__device__ __forceinline__ std::uint32_t token_extra_bits(std::uint32_t t) { return t >> 15; }

// Number of coefficient tokens of an item: the scan positions from `covered`
// through its last non-zero coefficient, exactly those on which
// coeff_tokens reports `has` (all positions to the end of the transform when
// the staged coefficients hold fewer non-zeros than the item's count).
__device__ std::uint32_t coeff_extent(const StripeStage& s, const StripeItem& it, int lane) {
    const int n{it.n};
    const int side{n >> 3};
    const int lside{side == 1 ? 0 : (side == 2 ? 1 : 2)};
    const std::uint32_t covered{static_cast<std::uint32_t>(side * side)};
    const std::uint32_t size{static_cast<std::uint32_t>(n * n)};
    const std::uint16_t* ord{s.order + (n == 8 ? 0 : (n == 16 ? 64 : 320))};
    const std::int16_t* plane{&s.coef[it.c][it.by][it.bx * kCoeffsPerBlock]};
    std::uint32_t remaining{it.nz};
    if (remaining == 0) return 0;
    const unsigned upto{(2u << lane) - 1u};  // lanes 0..lane
    for (std::uint32_t k0{covered}; k0 < size; k0 += 32) {
        const std::uint32_t k{k0 + static_cast<std::uint32_t>(lane)};
        std::int32_t val{0};
        if (k < size) {
            const int raw{ord[k]};
            const int q{raw >> 6};
            const int qy{q >> lside};
            const int qx{q & (side - 1)};
            if (it.by + qy < kStripeRows && it.bx + qx < kAcGroupBlocks) {
                val = plane[qy * kRowSlots + qx * kCoeffsPerBlock + (raw & 63)];
            }
        }
        const unsigned m{__ballot_sync(kFull, val != 0)};
        const std::uint32_t pc{static_cast<std::uint32_t>(__popc(m))};
        if (pc >= remaining) {
            // The lane holding the remaining-th non-zero of this chunk.
            const bool last{val != 0 && static_cast<std::uint32_t>(__popc(m & upto)) == remaining};
            const unsigned who{__ballot_sync(kFull, last)};
            return k0 + static_cast<std::uint32_t>(__ffs(who) - 1) - covered + 1;
        }
        remaining -= pc;
    }
    return size - covered;
}

// Exclusive scan over a CTA of kAcThreads threads; `warp_sums` holds
// kAcWarps + 1 words and receives the total in its last entry.
__device__ std::uint32_t cta_exclusive_scan(std::uint32_t v, std::uint32_t* warp_sums, std::uint32_t& total) {
    const int lane{static_cast<int>(threadIdx.x) & 31};
    const int warp{static_cast<int>(threadIdx.x) >> 5};
    const std::uint32_t incl{warp_incl_scan(v, lane)};
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const std::uint32_t ws{lane < kAcWarps ? warp_sums[lane] : 0u};
        const std::uint32_t wi{warp_incl_scan(ws, lane)};
        if (lane < kAcWarps) warp_sums[lane] = wi - ws;
        if (lane == kAcWarps - 1) warp_sums[kAcWarps] = wi;
    }
    __syncthreads();
    const std::uint32_t off{warp_sums[warp] + incl - v};
    total = warp_sums[kAcWarps];
    __syncthreads();
    return off;
}

// ---- pass 1: histograms ---------------------------------------------------------

// One CTA per stripe: the stripe's coefficient planes are read once, its
// tokens counted into the 32-cluster histogram and written, in stream order,
// to a run of the token pool that the stripe reserves once it knows their
// number (count tokens first sized, then the coefficient extents).
__device__ __forceinline__ void ac_tok_body(const EntropyDev& e, const unsigned blk, const unsigned nblk) {
    extern __shared__ __align__(16) unsigned char ac_smem[];
    StripeStage& s{*reinterpret_cast<StripeStage*>(ac_smem)};
    std::uint32_t* hist{reinterpret_cast<std::uint32_t*>(ac_smem + sizeof(StripeStage))};  // [32][64]
    __shared__ std::uint32_t sh_scan[kAcWarps + 1];
    __shared__ std::uint32_t sh_base;
    __shared__ int sh_stored;
    const int tid{static_cast<int>(threadIdx.x)};
    const int lane{tid & 31};
    const Stripe st{e.stripes[blk]};
    const GroupGeom gg{ac_group_geom(e, st.group)};
    for (int i{tid}; i < kNumClusters * kAcSymbols; i += kAcThreads) hist[i] = 0;
    stage_stripe(e, st, gg, s);
    __syncthreads();
    const int nitems{3 * st.rows * gg.gw};
    for (int j{tid}; j < nitems; j += kAcThreads) {
        const StripeItem it{stripe_item(s, gg.gw, j)};
        if (it.n == 0) {
            s.aux[j] = 0;
            continue;
        }
        int cl;
        std::uint32_t tok, nb, bits;
        count_token(s, st, it, cl, tok, nb, bits);
        atomicAdd(&hist[cl * kAcSymbols + tok], 1u);
        s.aux[j] = 1;
        if (it.nz != 0) s.active[atomicAdd(&s.nactive, 1)] = static_cast<std::uint16_t>(j);
    }
    __syncthreads();
    for (int a{tid >> 5}; a < s.nactive; a += kAcWarps) {
        const int j{s.active[a]};
        const std::uint32_t ext{coeff_extent(s, stripe_item(s, gg.gw, j), lane)};
        if (lane == 0) s.aux[j] += ext;
    }
    __syncthreads();
    // Token offsets of the items: each thread scans two adjacent items.
    const int j0{2 * tid};
    const std::uint32_t c0{j0 < nitems ? s.aux[j0] : 0u};
    const std::uint32_t c1{j0 + 1 < nitems ? s.aux[j0 + 1] : 0u};
    std::uint32_t total{0};
    const std::uint32_t off{cta_exclusive_scan(c0 + c1, sh_scan, total)};
    if (j0 < nitems) s.aux[j0] = off;
    if (j0 + 1 < nitems) s.aux[j0 + 1] = off + c0;
    if (tid == 0) {
        std::uint32_t base{0};
        bool stored{true};
        if (total != 0) {
            base = atomicAdd(e.tok_count, total);
            stored = base <= e.tok_capacity && total <= e.tok_capacity - base;
        }
        sh_base = base;
        sh_stored = stored ? 1 : 0;
        e.stripe_tok[2 * blk] = stored ? base : kNoTokens;
        e.stripe_tok[2 * blk + 1] = total;
    }
    __syncthreads();
    const bool stored{sh_stored != 0};
    std::uint32_t* pool{e.tok_pool + sh_base};
    if (stored) {
        for (int j{tid}; j < nitems; j += kAcThreads) {
            const StripeItem it{stripe_item(s, gg.gw, j)};
            if (it.n == 0) continue;
            int cl;
            std::uint32_t tok, nb, bits;
            count_token(s, st, it, cl, tok, nb, bits);
            pool[s.aux[j]] = pack_ac_token(cl, tok, nb, bits);
        }
    }
    for (int a{tid >> 5}; a < s.nactive; a += kAcWarps) {
        const int j{s.active[a]};
        const StripeItem it{stripe_item(s, gg.gw, j)};
        std::uint32_t* dst{pool + s.aux[j] + 1 + static_cast<std::uint32_t>(lane)};
        coeff_tokens(s, it, lane, [&](bool has, int cl, std::uint32_t sym, std::uint32_t nb, std::uint32_t bits) {
            const unsigned key{has ? static_cast<unsigned>(cl * kAcSymbols + sym) : 0xffffffffu};
            const unsigned peers{__match_any_sync(kFull, key)};
            if (has && (__ffs(peers) - 1) == lane) atomicAdd(&hist[key], static_cast<unsigned>(__popc(peers)));
            if (has && stored) *dst = pack_ac_token(cl, sym, nb, bits);
            dst += 32;
        });
    }
    __syncthreads();
    for (int i{tid}; i < kNumClusters * kAcSymbols; i += kAcThreads) {
        if (hist[i]) atomicAdd(&e.ac_hist[(i / kAcSymbols) * 256 + i % kAcSymbols], hist[i]);
    }
}

struct HistVisitor {
    std::uint32_t* sh_g;      // [2 slots][2 tables][256]
    std::uint32_t* sh_fb;     // [2 slots]
    int g0, g1;
    const EntropyDev* e;
    __device__ void blob(const std::uint8_t*, std::uint32_t) {}
    __device__ void varlen(std::uint32_t) {}
    __device__ void count_field(int, unsigned) {}
    __device__ void epf(int) {}
    __device__ void first_block(int g) {
        if (g == g0) {
            atomicAdd(&sh_fb[0], 1u);
        } else if (g == g1) {
            atomicAdd(&sh_fb[1], 1u);
        } else {
            atomicAdd(&e->fb_count[g], 1u);
        }
    }
    __device__ void token(int tab, int g, std::uint32_t sym, std::uint32_t, std::uint32_t) {
        const int t{tab == kTabDc ? 0 : 1};
        if (g == g0) {
            atomicAdd(&sh_g[t * 256 + sym], 1u);
        } else if (g == g1) {
            atomicAdd(&sh_g[(2 + t) * 256 + sym], 1u);
        } else {
            atomicAdd(&(t == 0 ? e->dc_hist : e->am_hist)[g * 256 + sym], 1u);
        }
    }
};

// Other items per CTA of the item passes (256 threads, two items each).
constexpr std::uint32_t kMiscItemsPerBlock = 512;
constexpr int kMiscPerThread = 2;

__device__ __forceinline__ void misc_hist_body(const EntropyDev& e, const unsigned blk, const unsigned nblk) {
    extern __shared__ __align__(16) unsigned char misc_smem[];
    std::uint32_t* sh_g{reinterpret_cast<std::uint32_t*>(misc_smem)};  // [4 * 256]
    std::uint32_t* sh_fb{sh_g + 4 * 256};                              // [2]
    if (threadIdx.x < 2) sh_fb[threadIdx.x] = 0;
    for (int i{static_cast<int>(threadIdx.x)}; i < 4 * 256; i += blockDim.x) sh_g[i] = 0;
    const std::uint32_t first{blk * kMiscItemsPerBlock};
    const std::uint32_t last{min(first + kMiscItemsPerBlock, e.ac_first) - 1};
    const Section s0{e.sections[find_section(e.sections, 0, misc_hi(e), first)]};
    const Section s1{e.sections[find_section(e.sections, 0, misc_hi(e), last)]};
    HistVisitor v{sh_g, sh_fb, s0.kind == kSecDcGroup ? s0.group : -1,
                  s1.kind == kSecDcGroup && s1.group != s0.group ? s1.group : -2, &e};
    __syncthreads();
#pragma unroll
    for (int k{0}; k < kMiscPerThread; ++k) {
        const std::uint32_t item{first + threadIdx.x + k * blockDim.x};
        if (item < e.ac_first) visit_misc(e, item, v);
    }
    __syncthreads();
    for (int i{static_cast<int>(threadIdx.x)}; i < 4 * 256; i += blockDim.x) {
        const int slot{i >> 9};
        const int t{(i >> 8) & 1};
        const int g{slot == 0 ? v.g0 : v.g1};
        if (sh_g[i] && g >= 0) atomicAdd(&(t == 0 ? e.dc_hist : e.am_hist)[g * 256 + (i & 255)], sh_g[i]);
    }
    if (threadIdx.x < 2) {
        const int g{threadIdx.x == 0 ? v.g0 : v.g1};
        if (g >= 0 && sh_fb[threadIdx.x]) atomicAdd(&e.fb_count[g], sh_fb[threadIdx.x]);
    }
}

// ---- pass 2: prefix codes ---------------------------------------------------------

struct WarpCodeSmem {
    std::uint32_t hist[256];
    std::uint32_t cnt[256];            // leaf counts in rank order (count floor 1)
    std::uint16_t leaf_sym[256];       // symbol of the leaf of each rank
    std::uint16_t floor_sym[256];      // symbols of the clamped leaves in descending order
    std::uint8_t depth[256];
    std::uint16_t bits[256];
    std::uint16_t used[256];           // compacted list of used symbols
    std::uint32_t len_count[18];       // depths per code length (canonical codes, header)
    std::uint32_t len_next[18];
    alignas(4) std::uint8_t desc[kDescBytes];
    CodeLengthScratch cl;
    // One tree per lane, lane-interleaved: internal node counts, heights and
    // every node's parent, for the count floor 2^lane.
    std::uint32_t icnt[256 * 32];
    std::uint8_t height[256 * 32];
    std::int16_t parent[512 * 32];
};

// Depths for a histogram with at least two used symbols, equal to the
// reference's serial construction (src/bitstream/prefix_code.cc:65-125):
// leaves ranked by (count ascending, symbol descending), two-queue merge (a
// leaf wins ties), the whole construction repeated with the count floor
// doubled until no depth exceeds `limit`.
//
// Warp-cooperative: the used symbols are compacted and ranked once. Raising
// the floor to F only clamps the smallest counts to F - 1, so the leaves of
// floor F are the same ranks with counts max(count, F - 1), the clamped ones
// (count <= F - 1, a prefix of the ranks) re-ordered by descending symbol.
// Every lane runs the merge for its own floor 2^lane at once, without
// branches, recording parents and internal heights; the smallest floor whose
// tree is no higher than `limit` is the one the serial loop stops at, and its
// leaves are walked to the root.
//
// hist[0..length) is read, depth[] of the used symbols written (the caller
// zeroes the rest); the rest of `s` other than hist and depth is scratch. A
// single used symbol gets depth 1, as the serial builder gives it.
__device__ void warp_create_tree(WarpCodeSmem& s, const std::uint32_t* hist, int length, int limit,
                                 std::uint8_t* depth, int lane) {
    int n{0};
    for (int base{0}; base < length; base += 32) {
        const int sym{base + lane};
        const bool used{sym < length && hist[sym] != 0};
        const unsigned m{__ballot_sync(kFull, used)};
        if (used) s.used[n + __popc(m & ((1u << lane) - 1u))] = static_cast<std::uint16_t>(sym);
        n += __popc(m);
    }
    __syncwarp();
    if (n < 2) {
        if (n == 1 && lane == 0) depth[s.used[0]] = 1;
        __syncwarp();
        return;
    }
    for (int i{lane}; i < n; i += 32) {
        const int sym{s.used[i]};
        const std::uint32_t c{hist[sym]};
        int rank{0};
        for (int t{0}; t < n; ++t) {
            const int ts{s.used[t]};
            const std::uint32_t ct{hist[ts]};
            rank += (ct < c || (ct == c && ts > sym)) ? 1 : 0;
        }
        s.cnt[rank] = c;
        s.leaf_sym[rank] = static_cast<std::uint16_t>(sym);
    }
    __syncwarp();
    // Lane L: floor 2^L, leaf r has count max(cnt[r], 2^L - 1).
    constexpr std::uint32_t kInf{0xffffffffu};
    const std::uint32_t fm1{lane == 31 ? 0x7fffffffu : (1u << lane) - 1u};
    std::uint32_t* icnt{s.icnt + lane};
    std::uint8_t* height{s.height + lane};
    std::int16_t* parent{s.parent + lane};
    int i{0};
    int j{0};
    for (int t{0}; t < n - 1; ++t) {
        int node[2];
        std::uint32_t sum{0};
        int h{0};
#pragma unroll
        for (int k{0}; k < 2; ++k) {
            const std::uint32_t li{i < n ? max(s.cnt[i < n ? i : 0], fm1) : kInf};
            const std::uint32_t lj{j < t ? icnt[32 * (j < t ? j : 0)] : kInf};
            const bool leaf{li <= lj};
            node[k] = leaf ? i : n + j;
            // Saturating: only floors far above any that can fit reach it.
            const std::uint32_t v{leaf ? li : lj};
            sum = sum > kInf - 1u - v ? kInf - 1u : sum + v;
            const int hk{leaf ? 0 : static_cast<int>(height[32 * (j < t ? j : 0)])};
            h = max(h, hk);
            i += leaf ? 1 : 0;
            j += leaf ? 0 : 1;
        }
        icnt[32 * t] = sum;
        height[32 * t] = static_cast<std::uint8_t>(h + 1);
        parent[32 * node[0]] = static_cast<std::int16_t>(n + t);
        parent[32 * node[1]] = static_cast<std::int16_t>(n + t);
    }
    const int root_h{static_cast<int>(height[32 * (n - 2)])};
    const unsigned fit{__ballot_sync(kFull, root_h <= limit)};
    __syncwarp();
    const int best{__ffs(fit) - 1};  // a floor of 2^31 leaves every count equal: always fits
    // Leaves clamped at the chosen floor, in descending symbol order.
    const std::uint32_t bm1{best == 31 ? 0x7fffffffu : (1u << best) - 1u};
    int m{0};
    for (int base{0}; base < n; base += 32) {
        const int r{base + lane};
        m += __popc(__ballot_sync(kFull, r < n && s.cnt[r] <= bm1));
    }
    for (int q{lane}; q < m; q += 32) {
        const int sym{s.leaf_sym[q]};
        int rank{0};
        for (int t{0}; t < m; ++t) rank += s.leaf_sym[t] > sym ? 1 : 0;
        s.floor_sym[rank] = static_cast<std::uint16_t>(sym);
    }
    __syncwarp();
    const std::int16_t* bp{s.parent + best};
    const int root{2 * n - 2};
    for (int r{lane}; r < n; r += 32) {
        int d{0};
        for (int v{r}; v != root; v = bp[32 * v]) ++d;
        depth[r < m ? s.floor_sym[r] : s.leaf_sym[r]] = static_cast<std::uint8_t>(d);
    }
    __syncwarp();
}

// Canonical codes of depth[0..len) (canonical_codes in prefix_code.cuh),
// warp-cooperative: codes of equal length are handed out in symbol order.
__device__ void warp_canonical_codes(WarpCodeSmem& s, const std::uint8_t* depth, int len, std::uint16_t* bits,
                                     int lane) {
    if (lane < 18) s.len_count[lane] = 0;
    __syncwarp();
    for (int base{0}; base < len; base += 32) {
        const int sym{base + lane};
        const int d{sym < len ? depth[sym] : 0};
        const unsigned peers{__match_any_sync(kFull, d)};
        if (d != 0 && (__ffs(peers) - 1) == lane) s.len_count[d] += static_cast<std::uint32_t>(__popc(peers));
    }
    __syncwarp();
    if (lane == 0) {
        std::uint32_t code{0};
        s.len_next[0] = 0;
        for (int i{1}; i < 16; ++i) {
            code = (code + (i - 1 == 0 ? 0u : s.len_count[i - 1])) << 1;
            s.len_next[i] = code;
        }
    }
    __syncwarp();
    const unsigned below{(1u << lane) - 1u};
    for (int base{0}; base < len; base += 32) {
        const int sym{base + lane};
        const int d{sym < len ? depth[sym] : 0};
        const unsigned peers{__match_any_sync(kFull, d)};
        const std::uint32_t code{d != 0 ? s.len_next[d] + static_cast<std::uint32_t>(__popc(peers & below)) : 0u};
        __syncwarp();
        if (d != 0 && (__ffs(peers) - 1) == lane) s.len_next[d] += static_cast<std::uint32_t>(__popc(peers));
        if (sym < len) bits[sym] = d != 0 ? static_cast<std::uint16_t>(__brev(code) >> (32 - d)) : 0;
        __syncwarp();
    }
}

// ORs `n` (<= 32) bits of `v` at bit `pos` of a zeroed little-endian byte
// buffer held as 32-bit words; bits at or past `cap` are dropped.
__device__ __forceinline__ void or_bits(std::uint8_t* buf, std::uint32_t pos, std::uint32_t n, std::uint32_t v,
                                        std::uint32_t cap) {
    if (n == 0) return;
    if (n < 32) v &= (1u << n) - 1u;
    unsigned int* words{reinterpret_cast<unsigned int*>(buf)};
    const std::uint32_t off{pos & 31u};
    if (pos < cap) atomicOr(&words[pos >> 5], v << off);
    if (off + n > 32 && pos + (32 - off) < cap) atomicOr(&words[(pos >> 5) + 1], v >> (32 - off));
}

// store_complex (prefix_code.cuh) with the per-symbol depth codes written by
// the whole warp: lane 0 builds the code-length code and writes its part of
// the header, then every lane places its symbols' codes at offsets from a
// warp scan.
__device__ void warp_store_complex(WarpCodeSmem& s, int num, BitSink& w, int lane) {
    int new_len{0};
    for (int i{lane}; i < num; i += 32) {
        if (s.depth[i] != 0) new_len = i + 1;
    }
#pragma unroll
    for (int off{16}; off > 0; off >>= 1) new_len = max(new_len, __shfl_xor_sync(kFull, new_len, off));
    CodeLengthScratch& scr{s.cl};
    if (lane < 18) scr.hist[lane] = 0;
    __syncwarp();
    for (int base{0}; base < new_len; base += 32) {
        const int i{base + lane};
        const int d{i < new_len ? s.depth[i] : -1};
        const unsigned peers{__match_any_sync(kFull, d)};
        if (d >= 0 && (__ffs(peers) - 1) == lane) scr.hist[d] += static_cast<std::uint32_t>(__popc(peers));
    }
    __syncwarp();
    // The code-length code: the same construction (limit 5) and canonical
    // codes, across the warp.
    if (lane < 18) {
        scr.cl_depth[lane] = 0;
        scr.cl_bits[lane] = 0;
    }
    __syncwarp();
    warp_create_tree(s, scr.hist, 18, 5, scr.cl_depth, lane);
    warp_canonical_codes(s, scr.cl_depth, 18, scr.cl_bits, lane);
    std::uint32_t pos{0};
    if (lane == 0) {
        std::uint32_t* hist{scr.hist};
        int num_codes{0};
        int code{0};
        for (int i{0}; i < 18; ++i) {
            if (hist[i]) {
                if (num_codes == 0) {
                    code = i;
                    num_codes = 1;
                } else if (num_codes == 1) {
                    num_codes = 2;
                    break;
                }
            }
        }
        std::uint8_t* cl_depth{scr.cl_depth};
        constexpr std::uint8_t kOrder[18]{1, 2, 3, 4, 0, 5, 17, 6, 16, 7, 8, 9, 10, 11, 12, 13, 14, 15};
        constexpr std::uint8_t kSym[6]{0, 7, 3, 2, 1, 15};
        constexpr std::uint8_t kLen[6]{2, 4, 3, 2, 2, 4};
        int to_store{18};
        if (num_codes > 1) {
            for (; to_store > 0; --to_store) {
                if (cl_depth[kOrder[to_store - 1]] != 0) break;
            }
        }
        std::uint32_t skip{0};
        if (cl_depth[kOrder[0]] == 0 && cl_depth[kOrder[1]] == 0) {
            skip = 2;
            if (cl_depth[kOrder[2]] == 0) skip = 3;
        }
        w.put(2, skip);
        for (int i{static_cast<int>(skip)}; i < to_store; ++i) {
            const int l{cl_depth[kOrder[i]]};
            w.put(kLen[l], kSym[l]);
        }
        if (num_codes == 1) cl_depth[code] = 0;
        pos = w.pos;
    }
    pos = __shfl_sync(kFull, pos, 0);
    __syncwarp();
    const std::uint32_t cap{w.cap};
    for (int base{0}; base < new_len; base += 32) {
        const int i{base + lane};
        const int d{i < new_len ? s.depth[i] : 0};
        const std::uint32_t n{i < new_len ? scr.cl_depth[d] : 0u};
        const std::uint32_t incl{warp_incl_scan(n, lane)};
        or_bits(w.buf, pos + incl - n, n, scr.cl_bits[d], cap);
        pos += __shfl_sync(kFull, incl, 31);
    }
    __syncwarp();
    if (lane == 0) {
        if (pos > cap) w.overflow = true;
        w.pos = pos;
    }
}

// build_and_store for s.hist[0..length) (src/bitstream/prefix_code.cc:387-426);
// the header goes to w (lane 0's copy holds the final position).
__device__ void warp_build_and_store(WarpCodeSmem& s, int length, BitSink& w, int lane) {
    int s4[4]{0, 0, 0, 0};
    int count{0};
    for (int base{0}; base < length && count <= 4; base += 32) {
        const int sym{base + lane};
        unsigned m{__ballot_sync(kFull, sym < length && s.hist[sym] != 0)};
        while (m != 0 && count <= 4) {
            if (count < 4) s4[count] = base + __ffs(m) - 1;
            ++count;
            m &= m - 1;
        }
    }
    if (count <= 1) {
        if (lane == 0) {
            w.put(4, 1);
            w.put(alphabet_bits(length), static_cast<std::uint32_t>(s4[0]));
        }
        __syncwarp();
        return;
    }
    warp_create_tree(s, s.hist, length, 15, s.depth, lane);
    warp_canonical_codes(s, s.depth, length, s.bits, lane);
    if (count <= 4) {
        if (lane == 0) store_code_header(count, s4, length, s.depth, w, s.cl);
        __syncwarp();
        return;
    }
    warp_store_complex(s, length, w, lane);
}

// One single-warp CTA per histogram (the 32 AC clusters, then the DC and the
// AcMetadata histogram of every DC group): the construction is a long serial
// chain on lane 0, so each chain gets an SM to itself.
__device__ __forceinline__ void codes_body(const EntropyDev& e, const unsigned blk, const unsigned nblk) {
    extern __shared__ __align__(16) unsigned char code_smem[];
    const int lane{static_cast<int>(threadIdx.x) & 31};
    WarpCodeSmem& s{*reinterpret_cast<WarpCodeSmem*>(code_smem)};
    int idx;
    const std::uint32_t* src;
    std::uint8_t* dst_depth;
    std::uint16_t* dst_bits;
    bool clustered;
    std::uint32_t extra0{0};
    if (blk < kNumClusters) {
        const int c{static_cast<int>(blk)};
        idx = c;
        src = e.ac_hist + c * 256;
        dst_depth = e.ac_depth + c * 256;
        dst_bits = e.ac_bits + c * 256;
        clustered = true;
    } else {
        const int g{(static_cast<int>(blk) - kNumClusters) >> 1};
        const int warp{(static_cast<int>(blk) - kNumClusters) & 1};
        if (warp == 0) {
            idx = 32 + g;
            src = e.dc_hist + g * 256;
            dst_depth = e.dc_depth + g * 256;
            dst_bits = e.dc_bits + g * 256;
        } else {
            idx = 32 + e.ndc + g;
            src = e.am_hist + g * 256;
            dst_depth = e.am_depth + g * 256;
            dst_bits = e.am_bits + g * 256;
            const GroupGeom gg{dc_group_geom(e, g)};
            extra0 = static_cast<std::uint32_t>(gg.gw * gg.gh);  // EPF zeros
        }
        clustered = false;
    }
    std::uint32_t hv[8];
#pragma unroll
    for (int k{0}; k < 8; ++k) hv[k] = src[lane + 32 * k];  // all eight loads in flight at once
#pragma unroll
    for (int k{0}; k < 8; ++k) {
        const int i{lane + 32 * k};
        s.hist[i] = hv[k] + (i == 0 ? extra0 : 0u);
        s.depth[i] = 0;
        s.bits[i] = 0;
    }
    for (int i{lane}; i < kDescBytes / 4; i += 32) reinterpret_cast<std::uint32_t*>(s.desc)[i] = 0;
    __syncwarp();
    int alpha{1};
    for (int i{lane}; i < 256; i += 32) {
        if (s.hist[i]) alpha = i + 1;
    }
#pragma unroll
    for (int off{16}; off > 0; off >>= 1) alpha = max(alpha, __shfl_xor_sync(kFull, alpha, off));
    BitSink w{s.desc, 0, kDescBytes * 8, false};
    if (!clustered && lane == 0) {
        // Single-context prefix histogram header (src/bitstream/histogram_writer.cc:59-83).
        w.put(1, 0);
        w.put(1, 1);
        put_uint_config(w, 4, 2, 0);
        put_var_len_u16(w, static_cast<std::uint32_t>(alpha - 1));
    }
    if (clustered && lane == 0) e.ac_alpha[idx] = static_cast<std::uint32_t>(alpha);
    if (alpha > 1) warp_build_and_store(s, alpha, w, lane);
    __syncwarp();
    std::uint32_t nbits{w.overflow ? 0u : w.pos};
    nbits = __shfl_sync(kFull, nbits, 0);
    if (lane == 0) e.desc_bits[idx] = nbits;
    std::uint8_t* d{e.desc + idx * kDescBytes};
    for (int i{lane}; i < kDescBytes; i += 32) d[i] = s.desc[i];
    for (int i{lane}; i < 256; i += 32) {
        dst_depth[i] = s.depth[i];
        dst_bits[i] = s.bits[i];
    }
}

// One histogram through the device builder (test hook): `length` symbols,
// depths, codes and the header (simple or code-length-code form) out.
__global__ void __launch_bounds__(32) prefix_code_test_kernel(const std::uint32_t* hist, int length,
                                                              std::uint8_t* depth, std::uint16_t* bits,
                                                              std::uint8_t* header, std::uint32_t* nbits) {
    extern __shared__ __align__(16) unsigned char code_smem[];
    const int lane{static_cast<int>(threadIdx.x) & 31};
    WarpCodeSmem& s{*reinterpret_cast<WarpCodeSmem*>(code_smem)};
    for (int i{lane}; i < 256; i += 32) {
        s.hist[i] = i < length ? hist[i] : 0u;
        s.depth[i] = 0;
        s.bits[i] = 0;
    }
    for (int i{lane}; i < kDescBytes; i += 32) s.desc[i] = 0;
    __syncwarp();
    BitSink w{s.desc, 0, kDescBytes * 8, false};
    warp_build_and_store(s, length, w, lane);
    __syncwarp();
    for (int i{lane}; i < length; i += 32) {
        depth[i] = s.depth[i];
        bits[i] = s.bits[i];
    }
    for (int i{lane}; i < kDescBytes; i += 32) header[i] = s.desc[i];
    if (lane == 0) *nbits = w.overflow ? 0xffffffffu : w.pos;
}

// ---- pass 3: bit lengths and scan ----------------------------------------------------

// Which stripes a launch of the AC bit-length or emission pass takes: those
// whose tokens are stored (no staging, small shared memory) or the others
// (staged coefficients, tokenised again).
enum StripeSet : int { kStoredStripes = 0, kUnstoredStripes = 1 };

template <int kSet>
__device__ __forceinline__ void ac_bits_body(const EntropyDev& e, const unsigned blk, const unsigned nblk) {
    extern __shared__ __align__(16) unsigned char ac_smem[];
    StripeStage& s{*reinterpret_cast<StripeStage*>(ac_smem)};
    __shared__ std::uint32_t sh_sum[kAcWarps];
    const int tid{static_cast<int>(threadIdx.x)};
    const int lane{tid & 31};
    const Stripe st{e.stripes[blk]};
    const GroupGeom gg{ac_group_geom(e, st.group)};
    const std::uint32_t tbase{e.stripe_tok[2 * blk]};
    if ((tbase != kNoTokens) != (kSet == kStoredStripes)) return;
    if (tbase != kNoTokens) {
        // Stored tokens: the stripe's whole length goes on its first item
        // (the scan only needs sums at stripe and section starts).
        const std::uint32_t ntok{e.stripe_tok[2 * blk + 1]};
        const std::uint32_t* pool{e.tok_pool + tbase};
        std::uint32_t sum{0};
        for (std::uint32_t t{static_cast<std::uint32_t>(tid)}; t < ntok; t += kAcThreads) {
            const std::uint32_t tk{pool[t]};
            sum += __ldg(&e.ac_depth[token_table_index(tk)]) + token_extra_count(tk);
        }
        sum = warp_sum(sum);
        if (lane == 0) sh_sum[tid >> 5] = sum;
        __syncthreads();
        const int nitems{3 * st.rows * gg.gw};
        std::uint32_t total{0};
        for (int w{0}; w < kAcWarps; ++w) total += sh_sum[w];
        for (int j{tid}; j < nitems; j += kAcThreads) e.item_bits[st.item0 + j] = j == 0 ? total : 0u;
        return;
    }
    stage_stripe(e, st, gg, s);
    __syncthreads();
    const int nitems{3 * st.rows * gg.gw};
    for (int j{tid}; j < nitems; j += kAcThreads) {
        const StripeItem it{stripe_item(s, gg.gw, j)};
        std::uint32_t b{0};
        if (it.n != 0) {
            int cl;
            std::uint32_t tok, nb, bits;
            count_token(s, st, it, cl, tok, nb, bits);
            b = __ldg(&e.ac_depth[cl * 256 + tok]) + nb;
            if (it.nz != 0) s.active[atomicAdd(&s.nactive, 1)] = static_cast<std::uint16_t>(j);
        }
        s.aux[j] = b;
    }
    __syncthreads();
    for (int a{tid >> 5}; a < s.nactive; a += kAcWarps) {
        const int j{s.active[a]};
        const StripeItem it{stripe_item(s, gg.gw, j)};
        std::uint32_t total{0};
        coeff_tokens(s, it, lane, [&](bool has, int cl, std::uint32_t sym, std::uint32_t nb, std::uint32_t) {
            if (has) total += __ldg(&e.ac_depth[cl * 256 + sym]) + nb;
        });
        total = warp_sum(total);
        if (lane == 0) s.aux[j] += total;
    }
    __syncthreads();
    for (int j{tid}; j < nitems; j += kAcThreads) e.item_bits[st.item0 + j] = s.aux[j];
}

struct BitsVisitor {
    const EntropyDev* e;
    std::uint32_t total;
    __device__ void blob(const std::uint8_t*, std::uint32_t nbits) { total += nbits; }
    __device__ void varlen(std::uint32_t v) {
        if (v == 0) {
            total += 1;
        } else {
            unsigned nb{0};
            for (std::uint32_t x{v}; x > 1; x >>= 1) ++nb;
            total += 5 + nb;
        }
    }
    __device__ void count_field(int, unsigned nbits) { total += nbits; }
    __device__ void epf(int g) { total += e->am_depth[g * 256]; }
    __device__ void first_block(int) {}
    __device__ void token(int tab, int g, std::uint32_t sym, std::uint32_t nb, std::uint32_t) {
        total += (tab == kTabDc ? e->dc_depth : e->am_depth)[g * 256 + sym] + nb;
    }
};

__device__ __forceinline__ void misc_bits_body(const EntropyDev& e, const unsigned blk, const unsigned nblk) {
#pragma unroll
    for (int k{0}; k < kMiscPerThread; ++k) {
        const std::uint32_t item{blk * kMiscItemsPerBlock + threadIdx.x + k * blockDim.x};
        if (item >= e.ac_first) return;
        BitsVisitor v{&e, 0};
        visit_misc(e, item, v);
        e.item_bits[item] = v.total;
    }
}

// Exclusive scan of item_bits inside tiles of kScanTile items (1024 threads x 4).
__device__ __forceinline__ void scan_tile_body(const EntropyDev& e, const unsigned blk, const unsigned nblk) {
    __shared__ std::uint32_t warp_sums[32];
    const std::uint32_t base{blk * kScanTile + threadIdx.x * 4};
    std::uint32_t v[4];
    std::uint32_t local{0};
#pragma unroll
    for (int k{0}; k < 4; ++k) {
        v[k] = base + k < e.total_items ? e.item_bits[base + k] : 0u;
        local += v[k];
    }
    const int lane{static_cast<int>(threadIdx.x) & 31};
    const int warp{static_cast<int>(threadIdx.x) >> 5};
    std::uint32_t incl{local};
#pragma unroll
    for (int off{1}; off < 32; off <<= 1) {
        const std::uint32_t t{__shfl_up_sync(kFull, incl, off)};
        if (lane >= off) incl += t;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const std::uint32_t ws{warp_sums[lane]};
        std::uint32_t wi{ws};
#pragma unroll
        for (int off{1}; off < 32; off <<= 1) {
            const std::uint32_t t{__shfl_up_sync(kFull, wi, off)};
            if (lane >= off) wi += t;
        }
        warp_sums[lane] = wi - ws;
        if (lane == 31) e.tile_sum[blk] = wi;
    }
    __syncthreads();
    std::uint32_t run{warp_sums[warp] + incl - local};
#pragma unroll
    for (int k{0}; k < 4; ++k) {
        if (base + k < e.total_items) e.item_pre[base + k] = run;
        run += v[k];
    }
}

__device__ __forceinline__ void scan_top_body(const EntropyDev& e, const unsigned blk, const unsigned nblk) {
    __shared__ unsigned long long warp_sums[32];
    __shared__ unsigned long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane{static_cast<int>(threadIdx.x) & 31};
    const int warp{static_cast<int>(threadIdx.x) >> 5};
    for (std::uint32_t base{0}; base < e.num_tiles; base += 1024) {
        const std::uint32_t i{base + threadIdx.x};
        const unsigned long long x{i < e.num_tiles ? e.tile_sum[i] : 0ull};
        unsigned long long incl{x};
#pragma unroll
        for (int off{1}; off < 32; off <<= 1) {
            const unsigned long long t{__shfl_up_sync(kFull, incl, off)};
            if (lane >= off) incl += t;
        }
        if (lane == 31) warp_sums[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const unsigned long long ws{warp_sums[lane]};
            unsigned long long wi{ws};
#pragma unroll
            for (int off{1}; off < 32; off <<= 1) {
                const unsigned long long t{__shfl_up_sync(kFull, wi, off)};
                if (lane >= off) wi += t;
            }
            warp_sums[lane] = wi - ws;
        }
        __syncthreads();
        if (i < e.num_tiles) e.tile_off[i] = carry + warp_sums[warp] + incl - x;
        __syncthreads();
        if (threadIdx.x == 1023) carry += warp_sums[31] + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) e.tile_off[e.num_tiles] = carry;
}


// ---- pass 4: layout --------------------------------------------------------------

struct U32Dist {
    bool direct;
    std::uint32_t v;
    std::uint32_t extra;
};

__device__ void put_u32(BitSink& w, const U32Dist* d, std::uint32_t value) {
    std::uint32_t best{0};
    std::uint32_t best_bits{64};
    for (std::uint32_t s{0}; s < 4; ++s) {
        if (d[s].direct) {
            if (d[s].v == value) {
                best = s;
                best_bits = 2;
                break;
            }
            continue;
        }
        if (value < d[s].v || static_cast<unsigned long long>(value) >=
                                  static_cast<unsigned long long>(d[s].v) + (1ull << d[s].extra)) {
            continue;
        }
        if (2 + d[s].extra < best_bits) {
            best = s;
            best_bits = 2 + d[s].extra;
        }
    }
    w.put(2, best);
    if (!d[best].direct) w.put(d[best].extra, value - d[best].v);
}

constexpr int kLayoutThreads = 256;

// TOC entry of a section of `bytes` bytes: U32 with selectors 0 + 10 bits,
// 1024 + 14, 17408 + 22, 4211712 + 30 (src/bitstream/codestream.cc:16-18, 91-98);
// the smallest selector that holds the value, as one LSB-first field.
__device__ __forceinline__ void toc_entry(std::uint32_t bytes, std::uint32_t& nbits, std::uint32_t& field) {
    std::uint32_t sel;
    std::uint32_t base;
    std::uint32_t extra;
    if (bytes < 1024u) {
        sel = 0; base = 0; extra = 10;
    } else if (bytes < 17408u) {
        sel = 1; base = 1024; extra = 14;
    } else if (bytes < 4211712u) {
        sel = 2; base = 17408; extra = 22;
    } else {
        sel = 3; base = 4211712; extra = 30;
    }
    nbits = 2 + extra;
    field = sel | ((bytes - base) << 2);
}

// Block-wide exclusive scan of one 64-bit value per thread; returns the
// thread's offset and sets `total`.
__device__ unsigned long long block_scan(unsigned long long v, unsigned long long* warp_sums,
                                         unsigned long long& total) {
    const int lane{static_cast<int>(threadIdx.x) & 31};
    const int warp{static_cast<int>(threadIdx.x) >> 5};
    unsigned long long incl{v};
#pragma unroll
    for (int off{1}; off < 32; off <<= 1) {
        const unsigned long long t{__shfl_up_sync(kFull, incl, off)};
        if (lane >= off) incl += t;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const int nw{static_cast<int>(blockDim.x) >> 5};
        const unsigned long long ws{lane < nw ? warp_sums[lane] : 0ull};
        unsigned long long wi{ws};
#pragma unroll
        for (int off{1}; off < 32; off <<= 1) {
            const unsigned long long t{__shfl_up_sync(kFull, wi, off)};
            if (lane >= off) wi += t;
        }
        if (lane < nw) warp_sums[lane] = wi - ws;
        if (lane == nw - 1) warp_sums[32] = wi;
    }
    __syncthreads();
    const unsigned long long off{warp_sums[warp] + incl - v};
    total = warp_sums[32];
    __syncthreads();
    return off;
}

// Sizes the sections, then writes the codestream headers and frame header
// (one thread), the TOC (every thread its own entries, placed by a scan of
// their bit lengths), the container framing and the section positions
// (src/bitstream/codestream.cc:57-135, src/bitstream/container.cc:35-62).
// Dynamic shared memory: the section sizes, then the header words
// (layout_head_bytes).
__device__ __forceinline__ void layout_body(const EntropyDev& e, const unsigned blk, const unsigned nblk) {
    extern __shared__ __align__(16) unsigned char layout_smem[];
    __shared__ unsigned long long scan_sums[33];
    __shared__ unsigned long long sh_start, sh_status, sh_head;
    __shared__ std::uint32_t sh_toc_start;
    auto* sec_bytes{reinterpret_cast<std::uint32_t*>(layout_smem)};
    const std::uint32_t head_cap{layout_head_bytes(e.nsec)};
    std::uint8_t* head{layout_smem + layout_sizes_bytes(e.nsec)};
    auto* head_words{reinterpret_cast<unsigned int*>(head)};
    const int tid{static_cast<int>(threadIdx.x)};
    for (std::uint32_t i{static_cast<std::uint32_t>(tid)}; i < head_cap / 4; i += kLayoutThreads) head_words[i] = 0;
    // With one AC group the four sections are one combined TOC entry: their
    // bits follow each other with no padding between them
    // (tools/bitstream/vardct_frame.cc:414-449).
    const bool single{e.nac == 1};
    const int ntoc{single ? 1 : e.nsec};
    if (single) {
        if (tid == 0) {
            const unsigned long long bits{prefix_at(e, e.total_items) - prefix_at(e, 0)};
            sec_bytes[0] = static_cast<std::uint32_t>((bits + 7) / 8);
        }
    } else {
        for (int s{tid}; s < e.nsec; s += kLayoutThreads) {
            const Section sec{e.sections[s]};
            const unsigned long long bits{prefix_at(e, sec.first + sec.count) - prefix_at(e, sec.first)};
            sec_bytes[s] = static_cast<std::uint32_t>((bits + 7) / 8);
        }
    }
    __syncthreads();
    if (tid == 0) {
        BitSink w{head, 0, head_cap * 8, false};
        const U32Dist dim[4]{{false, 1, 9}, {false, 1, 13}, {false, 1, 18}, {false, 1, 30}};
        w.put(8, 0xFF);
        w.put(8, 0x0A);
        const std::uint32_t W{static_cast<std::uint32_t>(e.width)};
        const std::uint32_t H{static_cast<std::uint32_t>(e.height)};
        const bool small{W % 8 == 0 && H % 8 == 0 && W <= 256 && H <= 256};
        w.put(1, small ? 1 : 0);
        if (small) w.put(5, H / 8 - 1); else put_u32(w, dim, H);
        w.put(3, 0);
        if (small) w.put(5, W / 8 - 1); else put_u32(w, dim, W);
        w.put(1, 1);  // ImageMetadata all_default
        w.put(1, 1);  // transform data all_default
        w.pos = (w.pos + 7) & ~7u;
        // FrameHeader: regular VarDCT frame, upsampling 1, x/b qm scale 2, one
        // pass, no custom size, replace blending, last, unnamed, default loop filter.
        w.put(1, 0);
        w.put(2, 0);
        w.put(1, 0);
        w.put(2, 0);
        w.put(2, 0);
        w.put(3, 2);
        w.put(3, 2);
        w.put(2, 0);
        w.put(1, 0);
        w.put(2, 0);
        w.put(1, 1);
        w.put(2, 0);
        w.put(1, 1);
        w.put(2, 0);
        w.put(1, 0);  // TOC without permutation
        w.pos = (w.pos + 7) & ~7u;
        sh_toc_start = w.pos;
    }
    __syncthreads();
    // Each thread takes a contiguous run of TOC entries.
    const int per{(ntoc + kLayoutThreads - 1) / kLayoutThreads};
    const int lo{min(ntoc, tid * per)};
    const int hi{min(ntoc, lo + per)};
    unsigned long long my_bits{0};
    unsigned long long my_bytes{0};
    for (int s{lo}; s < hi; ++s) {
        std::uint32_t nb, field;
        toc_entry(sec_bytes[s], nb, field);
        my_bits += nb;
        my_bytes += sec_bytes[s];
    }
    unsigned long long toc_bits{0};
    unsigned long long body{0};
    const unsigned long long bit_off{block_scan(my_bits, scan_sums, toc_bits)};
    const unsigned long long byte_off{block_scan(my_bytes, scan_sums, body)};
    {
        unsigned long long p{sh_toc_start + bit_off};
        for (int s{lo}; s < hi; ++s) {
            std::uint32_t nb, field;
            toc_entry(sec_bytes[s], nb, field);
            const std::uint32_t off{static_cast<std::uint32_t>(p & 31)};
            atomicOr(&head_words[p >> 5], field << off);
            if (off + nb > 32) atomicOr(&head_words[(p >> 5) + 1], field >> (32 - off));
            p += nb;
        }
    }
    __syncthreads();
    if (tid == 0) {
        const unsigned long long head_bytes{(sh_toc_start + toc_bits + 7) / 8};
        const unsigned long long cs{head_bytes + body};
        const bool large{cs >= 0x100000000ull - 8};
        const unsigned long long framing{32ull + (large ? 16 : 8)};
        const unsigned long long total{framing + cs};
        sh_head = head_bytes;
        sh_start = framing + head_bytes;
        sh_status = total > e.out_capacity ? 1ull : 0ull;
        e.result[0] = total;
        e.result[1] = sh_start;
        e.result[2] = sh_status;
        if (sh_status == 0) {
            const std::uint8_t hdr[32]{0, 0, 0, 0x0c, 'J', 'X', 'L', ' ', 0x0d, 0x0a, 0x87, 0x0a, 0, 0, 0, 0x14,
                                       'f', 't', 'y', 'p', 'j', 'x', 'l', ' ', 0, 0, 0, 0, 'j', 'x', 'l', ' '};
            for (int i{0}; i < 32; ++i) e.out[i] = hdr[i];
            std::size_t at{32};
            const unsigned long long box{cs + (large ? 16 : 8)};
            const std::uint32_t sf{large ? 1u : static_cast<std::uint32_t>(box)};
            for (int i{0}; i < 4; ++i) e.out[at++] = static_cast<std::uint8_t>(sf >> (8 * (3 - i)));
            e.out[at++] = 'j';
            e.out[at++] = 'x';
            e.out[at++] = 'l';
            e.out[at++] = 'c';
            if (large) {
                for (int i{0}; i < 8; ++i) e.out[at++] = static_cast<std::uint8_t>(box >> (8 * (7 - i)));
            }
        }
    }
    __syncthreads();
    if (sh_status != 0) return;
    if (single) {
        const unsigned long long base{prefix_at(e, 0)};
        for (int s{tid}; s < e.nsec; s += kLayoutThreads) {
            e.sec_pos[s] = sh_start * 8 + (prefix_at(e, e.sections[s].first) - base);
        }
    } else {
        unsigned long long pos{sh_start + byte_off};
        for (int s{lo}; s < hi; ++s) {
            e.sec_pos[s] = pos * 8;
            pos += sec_bytes[s];
        }
    }
    const unsigned long long framing{sh_start - sh_head};
    for (unsigned long long i{static_cast<unsigned long long>(tid)}; i < sh_head; i += kLayoutThreads) {
        e.out[framing + i] = head[i];
    }
}

__device__ __forceinline__ void zero_body_body(const EntropyDev& e, const unsigned blk, const unsigned nblk) {
    if (e.result[2] != 0) return;
    const unsigned long long start{e.result[1]};
    const unsigned long long end{e.result[0]};
    const unsigned long long a{(start + 15) & ~15ull};
    const unsigned long long stride{static_cast<unsigned long long>(nblk) * blockDim.x};
    const unsigned long long tid{static_cast<unsigned long long>(blk) * blockDim.x + threadIdx.x};
    if (tid < a - start && start + tid < end) e.out[start + tid] = 0;
    const unsigned long long nvec{end > a ? (end - a) / 16 : 0};
    uint4* v{reinterpret_cast<uint4*>(e.out + a)};
    for (unsigned long long i{tid}; i < nvec; i += stride) v[i] = make_uint4(0, 0, 0, 0);
    const unsigned long long tail{a + nvec * 16};
    if (tail + tid < end && tid < 16) e.out[tail + tid] = 0;
}

// ---- pass 5: emission ------------------------------------------------------------

// Copies a window of `nwords` assembled words to global word w0 onward. The
// first and last words can share bits with neighbouring items and are ORed
// in; every word between lies wholly inside the window's bit range and is
// stored.
__device__ void flush_window(const unsigned int* win, int nwords, unsigned int* gwords, unsigned long long w0) {
    for (int i{static_cast<int>(threadIdx.x)}; i < nwords; i += blockDim.x) {
        const unsigned int v{win[i]};
        if (i == 0 || i == nwords - 1) {
            if (v != 0) atomicOr(&gwords[w0 + i], v);
        } else {
            gwords[w0 + i] = v;
        }
    }
}

// Writes a stripe's tokens. The stripe's bits are contiguous in its section;
// they are assembled in a shared-memory window and written out with plain
// stores (global atomics only when the stripe exceeds the window).
template <int kSet>
__device__ __forceinline__ void ac_emit_body(const EntropyDev& e, const unsigned blk, const unsigned nblk) {
    extern __shared__ __align__(16) unsigned char ac_smem[];
    StripeStage& s{*reinterpret_cast<StripeStage*>(ac_smem)};
    // Stored stripes need no staging: their window starts the allocation.
    unsigned int* win{reinterpret_cast<unsigned int*>(ac_smem + (kSet == kStoredStripes ? 0 : sizeof(StripeStage)))};
    __shared__ unsigned long long sh_start;
    __shared__ unsigned long long sh_p0;
    __shared__ int sh_words;
    if (e.result[2] != 0) return;
    const int tid{static_cast<int>(threadIdx.x)};
    const int lane{tid & 31};
    const Stripe st{e.stripes[blk]};
    const GroupGeom gg{ac_group_geom(e, st.group)};
    const int nitems{3 * st.rows * gg.gw};
    if ((e.stripe_tok[2 * blk] != kNoTokens) != (kSet == kStoredStripes)) return;
    if (kSet == kUnstoredStripes) stage_stripe(e, st, gg, s);
    if (tid == 0) {
        const Section sec{e.sections[st.section]};
        const unsigned long long p0{prefix_at(e, st.item0)};
        const unsigned long long start{e.sec_pos[st.section] + (p0 - prefix_at(e, sec.first))};
        const unsigned long long bits{prefix_at(e, st.item0 + static_cast<std::uint32_t>(nitems)) - p0};
        const unsigned long long nw{bits == 0 ? 0ull : ((start + bits + 31) >> 5) - (start >> 5)};
        sh_start = start;
        sh_p0 = p0;
        sh_words = nw <= static_cast<unsigned long long>(kWindowWords) ? static_cast<int>(nw) : -1;
    }
    __syncthreads();
    const int nwords{sh_words};
    for (int i{tid}; i < nwords; i += kAcThreads) win[i] = 0;
    unsigned int* words{nwords >= 0 ? win : reinterpret_cast<unsigned int*>(e.out)};
    const unsigned long long base{nwords >= 0 ? (sh_start & 31) : sh_start};
    const std::uint32_t tbase{e.stripe_tok[2 * blk]};
    if (tbase != kNoTokens) {
        // Stored tokens in stream order: their lengths, a CTA scan for their
        // offsets, and their bits, kAcThreads * kPer tokens per round.
        __shared__ std::uint32_t sh_scan[kAcWarps + 1];
        constexpr int kPer{4};
        const std::uint32_t ntok{e.stripe_tok[2 * blk + 1]};
        const std::uint32_t* pool{e.tok_pool + tbase};
        __syncthreads();
        unsigned long long run{base};
        for (std::uint32_t t0{0}; t0 < ntok; t0 += kAcThreads * kPer) {
            std::uint32_t tk[kPer];
            std::uint32_t len[kPer];
            std::uint32_t local{0};
#pragma unroll
            for (int i{0}; i < kPer; ++i) {
                const std::uint32_t t{t0 + static_cast<std::uint32_t>(tid) * kPer + i};
                tk[i] = t < ntok ? pool[t] : 0u;
                len[i] = t < ntok ? __ldg(&e.ac_depth[token_table_index(tk[i])]) + token_extra_count(tk[i]) : 0u;
                local += len[i];
            }
            std::uint32_t total{0};
            unsigned long long at{run + cta_exclusive_scan(local, sh_scan, total)};
#pragma unroll
            for (int i{0}; i < kPer; ++i) {
                if (len[i] == 0) continue;
                const std::uint32_t idx{token_table_index(tk[i])};
                const std::uint32_t d{__ldg(&e.ac_depth[idx])};
                put_bits_at(words, at, d, __ldg(&e.ac_bits[idx]));
                const std::uint32_t nb{token_extra_count(tk[i])};
                if (nb) put_bits_at(words, at + d, nb, token_extra_bits(tk[i]));
                at += len[i];
            }
            run += total;
        }
        __syncthreads();
        if (nwords > 0) flush_window(win, nwords, reinterpret_cast<unsigned int*>(e.out), sh_start >> 5);
        return;
    }
    for (int j{tid}; j < nitems; j += kAcThreads) {
        s.aux[j] = static_cast<std::uint32_t>(prefix_at(e, st.item0 + static_cast<std::uint32_t>(j)) - sh_p0);
    }
    __syncthreads();
    for (int j{tid}; j < nitems; j += kAcThreads) {
        const StripeItem it{stripe_item(s, gg.gw, j)};
        if (it.n == 0) continue;
        int cl;
        std::uint32_t tok, nb, bits;
        count_token(s, st, it, cl, tok, nb, bits);
        const std::uint32_t d{__ldg(&e.ac_depth[cl * 256 + tok])};
        const unsigned long long at{base + s.aux[j]};
        put_bits_at(words, at, d, __ldg(&e.ac_bits[cl * 256 + tok]));
        if (nb) put_bits_at(words, at + d, nb, bits);
        if (it.nz != 0) {
            s.active[atomicAdd(&s.nactive, 1)] = static_cast<std::uint16_t>(j);
            s.aux[j] += d + nb;  // coefficient tokens start after the count token
        }
    }
    __syncthreads();
    for (int a{tid >> 5}; a < s.nactive; a += kAcWarps) {
        const int j{s.active[a]};
        const StripeItem it{stripe_item(s, gg.gw, j)};
        unsigned long long pos{base + s.aux[j]};
        coeff_tokens(s, it, lane, [&](bool has, int cl, std::uint32_t sym, std::uint32_t nb, std::uint32_t bits) {
            const std::uint32_t d{has ? __ldg(&e.ac_depth[cl * 256 + sym]) : 0u};
            const std::uint32_t tb{has ? d + nb : 0u};
            const std::uint32_t incl{warp_incl_scan(tb, lane)};
            if (has) {
                const unsigned long long at{pos + incl - tb};
                put_bits_at(words, at, d, __ldg(&e.ac_bits[cl * 256 + sym]));
                if (nb) put_bits_at(words, at + d, nb, bits);
            }
            pos += __shfl_sync(kFull, incl, 31);
        });
    }
    __syncthreads();
    if (nwords > 0) flush_window(win, nwords, reinterpret_cast<unsigned int*>(e.out), sh_start >> 5);
}

// A header blob long enough to be written by the whole CTA (the AcGlobal
// prefix with its context map runs to tens of thousands of bits).
struct DeferredBlob {
    unsigned int* words;
    unsigned long long pos;
    const std::uint8_t* src;  // 4-byte aligned, readable in whole words
    std::uint32_t nbits;
};
constexpr int kMaxDeferred = 32;
constexpr std::uint32_t kDeferBits = 256;

struct EmitVisitor {
    const EntropyDev* e;
    unsigned int* words;
    unsigned long long pos;
    DeferredBlob* deferred{nullptr};
    int* ndeferred{nullptr};
    __device__ void put(std::uint32_t n, std::uint32_t v) {
        if (n == 0) return;
        if (n < 32) v &= (1u << n) - 1u;
        put_bits_at(words, pos, n, v);
        pos += n;
    }
    __device__ void blob(const std::uint8_t* b, std::uint32_t nbits) {
        if (deferred != nullptr && nbits > kDeferBits) {
            const int k{atomicAdd(ndeferred, 1)};
            if (k < kMaxDeferred) {
                deferred[k] = DeferredBlob{words, pos, b, nbits};
                pos += nbits;
                return;
            }
        }
        std::uint32_t i{0};
        for (; i + 32 <= nbits; i += 32) {
            put(32, static_cast<std::uint32_t>(b[i >> 3]) | (static_cast<std::uint32_t>(b[(i >> 3) + 1]) << 8) |
                        (static_cast<std::uint32_t>(b[(i >> 3) + 2]) << 16) |
                        (static_cast<std::uint32_t>(b[(i >> 3) + 3]) << 24));
        }
        for (; i + 8 <= nbits; i += 8) put(8, b[i >> 3]);
        if (i < nbits) put(nbits - i, b[i >> 3]);
    }
    __device__ void varlen(std::uint32_t v) {
        if (v == 0) {
            put(1, 0);
            return;
        }
        put(1, 1);
        unsigned nb{0};
        for (std::uint32_t x{v}; x > 1; x >>= 1) ++nb;
        put(4, nb);
        put(nb, v - (1u << nb));
    }
    __device__ void count_field(int g, unsigned nbits) { put(nbits, e->fb_count[g] - 1); }
    __device__ void epf(int g) { put(e->am_depth[g * 256], e->am_bits[g * 256]); }
    __device__ void first_block(int) {}
    __device__ void token(int tab, int g, std::uint32_t sym, std::uint32_t nb, std::uint32_t bits) {
        const std::uint8_t* d{tab == kTabDc ? e->dc_depth : e->am_depth};
        const std::uint16_t* c{tab == kTabDc ? e->dc_bits : e->am_bits};
        put(d[g * 256 + sym], c[g * 256 + sym]);
        if (nb) put(nb, bits);
    }
};

constexpr int kMiscWindowWords = 2048;

// One thread per non-AC item; the bits of the block's items that share the
// first item's section are assembled in a shared-memory window.
__device__ __forceinline__ void misc_emit_body(const EntropyDev& e, const unsigned blk, const unsigned nblk) {
    extern __shared__ __align__(16) unsigned char misc_smem[];
    unsigned int* win{reinterpret_cast<unsigned int*>(misc_smem)};                              // [kMiscWindowWords]
    DeferredBlob* deferred{reinterpret_cast<DeferredBlob*>(misc_smem + kMiscWindowWords * 4)};  // [kMaxDeferred]
    __shared__ unsigned long long sh_start;
    __shared__ std::uint32_t sh_end;
    __shared__ int sh_words;
    __shared__ int sh_ndeferred;
    if (e.result[2] != 0) return;
    const std::uint32_t first{blk * kMiscItemsPerBlock};
    if (threadIdx.x == 0) {
        sh_ndeferred = 0;
        const int s0{find_section(e.sections, 0, misc_hi(e), first)};
        const Section sec{e.sections[s0]};
        const std::uint32_t end{min(min(first + kMiscItemsPerBlock, sec.first + sec.count), e.ac_first)};
        const unsigned long long p0{prefix_at(e, first)};
        const unsigned long long start{e.sec_pos[s0] + (p0 - prefix_at(e, sec.first))};
        const unsigned long long bits{prefix_at(e, end) - p0};
        const unsigned long long nw{bits == 0 ? 0ull : ((start + bits + 31) >> 5) - (start >> 5)};
        sh_start = start;
        sh_end = end;
        sh_words = nw <= static_cast<unsigned long long>(kMiscWindowWords) ? static_cast<int>(nw) : -1;
    }
    __syncthreads();
    const int nwords{sh_words};
    for (int i{static_cast<int>(threadIdx.x)}; i < nwords; i += blockDim.x) win[i] = 0;
    __syncthreads();
#pragma unroll
    for (int k{0}; k < kMiscPerThread; ++k) {
        const std::uint32_t item{first + threadIdx.x + k * blockDim.x};
        if (item < e.ac_first) {
            const int s{find_section(e.sections, 0, misc_hi(e), item)};
            const Section sec{e.sections[s]};
            const unsigned long long pos{e.sec_pos[s] + (prefix_at(e, item) - prefix_at(e, sec.first))};
            const bool in_window{nwords >= 0 && item < sh_end};
            EmitVisitor v{&e, in_window ? win : reinterpret_cast<unsigned int*>(e.out),
                          in_window ? pos - ((sh_start >> 5) << 5) : pos, deferred, &sh_ndeferred};
            visit_misc(e, item, v);
        }
    }
    __syncthreads();
    // Long blobs, one 32-bit word of each per thread.
    const int nd{min(sh_ndeferred, kMaxDeferred)};
    for (int k{0}; k < nd; ++k) {
        const DeferredBlob d{deferred[k]};
        const auto* src{reinterpret_cast<const std::uint32_t*>(d.src)};
        for (std::uint32_t w{threadIdx.x}; 32 * w < d.nbits; w += blockDim.x) {
            const std::uint32_t n{min(32u, d.nbits - 32 * w)};
            std::uint32_t v{src[w]};
            if (n < 32) v &= (1u << n) - 1u;
            put_bits_at(d.words, d.pos + 32ull * w, n, v);
        }
    }
    __syncthreads();
    if (nwords > 0) flush_window(win, nwords, reinterpret_cast<unsigned int*>(e.out), sh_start >> 5);
}

// Clears a frame's histograms and counters (the first step of every encode).
// Zeroes a frame's histograms, first-block counts and token-pool fill; block
// blk of nblk takes every nblk-th 256-word stretch.
__device__ __forceinline__ void clear_body(const EntropyDev& e, unsigned blk, unsigned nblk) {
    const unsigned stride{nblk * blockDim.x};
    const unsigned t0{blk * blockDim.x + threadIdx.x};
    for (unsigned i{t0}; i < static_cast<unsigned>(kNumClusters * 256); i += stride) e.ac_hist[i] = 0;
    for (unsigned i{t0}; i < static_cast<unsigned>(e.ndc) * 256u; i += stride) {
        e.dc_hist[i] = 0;
        e.am_hist[i] = 0;
    }
    for (unsigned i{t0}; i < static_cast<unsigned>(e.ndc); i += stride) e.fb_count[i] = 0;
    if (t0 == 0) *e.tok_count = 0;
}

// Blocks of a frame's clear: one per 32 DC groups (8192 histogram words each).
__host__ __device__ constexpr unsigned clear_blocks(int ndc) { return 1u + static_cast<unsigned>(ndc) / 32u; }

// ---- kernels: one frame per launch, and every frame of a batch per launch -----------

// Blocks of a single-frame launch of the body-zeroing pass.
constexpr unsigned kZeroBlocks = 296;
// Blocks per frame of the body-zeroing pass in a batched launch.
constexpr unsigned kZeroBlocksBatched = 32;

#define JXB_ENTROPY_KERNELS(NAME, BOUNDS, PHASE, NBLK)                                                     \
    __global__ void BOUNDS NAME##_kernel(const __grid_constant__ EntropyDev e) {                              \
        NAME##_body(e, blockIdx.x, gridDim.x);                                                                \
    }                                                                                                         \
    __global__ void BOUNDS NAME##_batch_kernel(const __grid_constant__ EntropyBatch b) {                      \
        const int f{batch_frame(b, PHASE, blockIdx.x)};                                                      \
        NAME##_body(b.frames[f], blockIdx.x - b.begin[PHASE][f], NBLK);                                       \
    }

// Frame of block `blk` of a batched launch of `phase` (binary search over the
// frames' first blocks).
__device__ __forceinline__ int batch_frame(const EntropyBatch& b, int phase, unsigned blk) {
    int lo{0};
    int hi{b.nframes - 1};
    while (lo < hi) {
        const int mid{(lo + hi + 1) >> 1};
        if (b.begin[phase][mid] <= blk) {
            lo = mid;
        } else {
            hi = mid - 1;
        }
    }
    return lo;
}

// The three item passes run the AC stripes (blocks 0 .. nstripes - 1, the
// long ones, scheduled first) and the other items (the blocks after them) as
// one launch: the two kinds are independent within a pass.
__device__ __forceinline__ void tokens_body(const EntropyDev& e, const unsigned blk, const unsigned nblk) {
    if (blk < static_cast<unsigned>(e.nstripes)) {
        ac_tok_body(e, blk, nblk);
    } else {
        misc_hist_body(e, blk - static_cast<unsigned>(e.nstripes), nblk);
    }
}
__device__ __forceinline__ void lengths_body(const EntropyDev& e, const unsigned blk, const unsigned nblk) {
    if (blk < static_cast<unsigned>(e.nstripes)) {
        ac_bits_body<kStoredStripes>(e, blk, nblk);
    } else {
        misc_bits_body(e, blk - static_cast<unsigned>(e.nstripes), nblk);
    }
}
__device__ __forceinline__ void emit_body(const EntropyDev& e, const unsigned blk, const unsigned nblk) {
    if (blk < static_cast<unsigned>(e.nstripes)) {
        ac_emit_body<kStoredStripes>(e, blk, nblk);
    } else {
        misc_emit_body(e, blk - static_cast<unsigned>(e.nstripes), nblk);
    }
}
// Stripes whose tokens did not fit the pool, with their coefficients staged
// (their CTAs return at once for stored stripes).
__device__ __forceinline__ void lengths_unstored_body(const EntropyDev& e, const unsigned blk, const unsigned nblk) {
    ac_bits_body<kUnstoredStripes>(e, blk, nblk);
}
__device__ __forceinline__ void emit_unstored_body(const EntropyDev& e, const unsigned blk, const unsigned nblk) {
    ac_emit_body<kUnstoredStripes>(e, blk, nblk);
}

JXB_ENTROPY_KERNELS(tokens, __launch_bounds__(kAcThreads), kPhaseItems, 0u)
JXB_ENTROPY_KERNELS(codes, __launch_bounds__(32), kPhaseCodes, 0u)
JXB_ENTROPY_KERNELS(lengths, __launch_bounds__(kAcThreads), kPhaseItems, 0u)
JXB_ENTROPY_KERNELS(scan_tile, __launch_bounds__(1024), kPhaseScan, 0u)
JXB_ENTROPY_KERNELS(scan_top, __launch_bounds__(1024), kPhaseFrame, 0u)
JXB_ENTROPY_KERNELS(layout, __launch_bounds__(kLayoutThreads), kPhaseFrame, 0u)
JXB_ENTROPY_KERNELS(zero_body, __launch_bounds__(256), kPhaseZero, kZeroBlocksBatched)
JXB_ENTROPY_KERNELS(emit, __launch_bounds__(kAcThreads), kPhaseItems, 0u)
// Stripes whose tokens did not fit the pool are rare, so their passes run on
// a few resident CTAs that skip the stored stripes with one load each.
constexpr unsigned kUnstoredCtas = 148;

// Every stripe adds its token count to the pool fill whether or not it fits,
// so a frame has an unstored stripe exactly when its final fill exceeds the
// capacity; a frame without one is passed over after one load.
__device__ __forceinline__ bool frame_all_stored(const EntropyDev& e) { return *e.tok_count <= e.tok_capacity; }

#define JXB_UNSTORED_KERNELS(NAME)                                                                         \
    __global__ void __launch_bounds__(kAcThreads) NAME##_kernel(const __grid_constant__ EntropyDev e) {       \
        if (frame_all_stored(e)) return;                                                                      \
        for (unsigned s{blockIdx.x}; s < static_cast<unsigned>(e.nstripes); s += gridDim.x) {                 \
            if (e.stripe_tok[2 * s] != kNoTokens) continue;                                                   \
            NAME##_body(e, s, 0u);                                                                            \
            __syncthreads();                                                                                  \
        }                                                                                                     \
    }                                                                                                         \
    __global__ void __launch_bounds__(kAcThreads) NAME##_batch_kernel(const __grid_constant__ EntropyBatch b) { \
        const unsigned total{b.begin[kPhaseStripes][b.nframes]};                                              \
        for (unsigned i{blockIdx.x}; i < total; i += gridDim.x) {                                             \
            const int f{batch_frame(b, kPhaseStripes, i)};                                                    \
            if (frame_all_stored(b.frames[f])) {                                                              \
                /* on to this block's last stripe of frame f */                                               \
                i += (b.begin[kPhaseStripes][f + 1] - 1 - i) / gridDim.x * gridDim.x;                         \
                continue;                                                                                     \
            }                                                                                                 \
            const unsigned s{i - b.begin[kPhaseStripes][f]};                                                  \
            if (b.frames[f].stripe_tok[2 * s] != kNoTokens) continue;                                         \
            NAME##_body(b.frames[f], s, 0u);                                                                  \
            __syncthreads();                                                                                  \
        }                                                                                                     \
    }

JXB_UNSTORED_KERNELS(lengths_unstored)
JXB_UNSTORED_KERNELS(emit_unstored)
#undef JXB_UNSTORED_KERNELS
#undef JXB_ENTROPY_KERNELS

__global__ void __launch_bounds__(256) clear_kernel(const __grid_constant__ EntropyDev e) {
    clear_body(e, blockIdx.x, gridDim.x);
}
__global__ void __launch_bounds__(256) clear_batch_kernel(const __grid_constant__ EntropyBatch b) {
    clear_body(b.frames[blockIdx.x], 0u, 1u);
}

constexpr std::size_t kHistSmem{sizeof(StripeStage) + kNumClusters * kAcSymbols * sizeof(std::uint32_t)};
constexpr std::size_t kBitsSmem{sizeof(StripeStage)};
constexpr std::size_t kEmitSmem{sizeof(StripeStage) + kWindowWords * sizeof(unsigned int)};
// Emission of stored stripes and other items: the larger of their windows.
constexpr std::size_t kEmitStoredSmem{kWindowWords * sizeof(unsigned int) >
                                              kMiscWindowWords * sizeof(unsigned int) + kMaxDeferred * sizeof(DeferredBlob)
                                          ? kWindowWords * sizeof(unsigned int)
                                          : kMiscWindowWords * sizeof(unsigned int) + kMaxDeferred * sizeof(DeferredBlob)};
// The other items' passes share these launches and their shared memory.
static_assert(kHistSmem >= (4 * 256 + 2) * sizeof(std::uint32_t), "token pass shared memory");


}  // namespace

static_assert(sizeof(EntropyBatch) <= 32000, "a batched entropy launch's parameters exceed the kernel parameter limit");

bool entropy_launch(const EntropyDev& e, void* stream) {
    if (e.nsec > kMaxSections) return false;
    cudaStream_t st{static_cast<cudaStream_t>(stream)};
    const unsigned misc{(e.ac_first + kMiscItemsPerBlock - 1) / kMiscItemsPerBlock};
    const unsigned stripes{static_cast<unsigned>(e.nstripes)};
    const std::uint32_t layout_smem{layout_sizes_bytes(e.nsec) + layout_head_bytes(e.nsec)};
    clear_kernel<<<clear_blocks(e.ndc), 256, 0, st>>>(e);  // histograms, first-block counts, pool fill
    tokens_kernel<<<stripes + misc, kAcThreads, kHistSmem, st>>>(e);
    codes_kernel<<<kNumClusters + 2 * e.ndc, 32, sizeof(WarpCodeSmem), st>>>(e);
    lengths_kernel<<<stripes + misc, kAcThreads, 0, st>>>(e);
    lengths_unstored_kernel<<<kUnstoredCtas, kAcThreads, kBitsSmem, st>>>(e);
    scan_tile_kernel<<<e.num_tiles, 1024, 0, st>>>(e);
    scan_top_kernel<<<1, 1024, 0, st>>>(e);
    layout_kernel<<<1, kLayoutThreads, layout_smem, st>>>(e);
    zero_body_kernel<<<kZeroBlocks, 256, 0, st>>>(e);
    emit_kernel<<<stripes + misc, kAcThreads, kEmitStoredSmem, st>>>(e);
    emit_unstored_kernel<<<kUnstoredCtas, kAcThreads, kEmitSmem, st>>>(e);
    return cudaGetLastError() == cudaSuccess;
}

void entropy_batch_plan(EntropyBatch& b) {
    for (int p{0}; p < kEntropyPhases; ++p) b.begin[p][0] = 0;
    for (int f{0}; f < b.nframes; ++f) {
        const EntropyDev& e{b.frames[f]};
        const std::uint32_t per[kEntropyPhases]{static_cast<std::uint32_t>(e.nstripes) +
                                                     (e.ac_first + kMiscItemsPerBlock - 1) / kMiscItemsPerBlock,
                                                 static_cast<std::uint32_t>(kNumClusters + 2 * e.ndc), e.num_tiles,
                                                 1u, kZeroBlocksBatched, static_cast<std::uint32_t>(e.nstripes)};
        for (int p{0}; p < kEntropyPhases; ++p) b.begin[p][f + 1] = b.begin[p][f] + per[p];
    }
}

bool entropy_batch_launch(const EntropyBatch& b, void* stream) {
    if (b.nframes <= 0 || b.nframes > kEntropyBatchFrames) return false;
    std::uint32_t layout_smem{0};
    for (int f{0}; f < b.nframes; ++f) {
        const EntropyDev& e{b.frames[f]};
        if (e.nsec > kMaxSections) return false;
        layout_smem = std::max(layout_smem, layout_sizes_bytes(e.nsec) + layout_head_bytes(e.nsec));
    }
    cudaStream_t st{static_cast<cudaStream_t>(stream)};
    const int nf{b.nframes};
    const unsigned items{b.begin[kPhaseItems][nf]};
    clear_batch_kernel<<<static_cast<unsigned>(nf), 256, 0, st>>>(b);
    tokens_batch_kernel<<<items, kAcThreads, kHistSmem, st>>>(b);
    codes_batch_kernel<<<b.begin[kPhaseCodes][nf], 32, sizeof(WarpCodeSmem), st>>>(b);
    lengths_batch_kernel<<<items, kAcThreads, 0, st>>>(b);
    lengths_unstored_batch_kernel<<<kUnstoredCtas, kAcThreads, kBitsSmem, st>>>(b);
    scan_tile_batch_kernel<<<b.begin[kPhaseScan][nf], 1024, 0, st>>>(b);
    scan_top_batch_kernel<<<static_cast<unsigned>(nf), 1024, 0, st>>>(b);
    layout_batch_kernel<<<static_cast<unsigned>(nf), kLayoutThreads, layout_smem, st>>>(b);
    zero_body_batch_kernel<<<b.begin[kPhaseZero][nf], 256, 0, st>>>(b);
    emit_batch_kernel<<<items, kAcThreads, kEmitStoredSmem, st>>>(b);
    emit_unstored_batch_kernel<<<kUnstoredCtas, kAcThreads, kEmitSmem, st>>>(b);
    return cudaGetLastError() == cudaSuccess;
}

bool prefix_code_test(const std::uint32_t* hist, int length, std::uint8_t* depth, std::uint16_t* bits,
                      std::uint8_t* header, std::size_t header_cap, std::uint32_t* nbits) {
    if (length < 1 || length > 256 || header_cap < static_cast<std::size_t>(kDescBytes)) return false;
    unsigned char* dev{nullptr};
    const std::size_t bytes{256 * 4 + 256 + 256 * 2 + kDescBytes + 4};
    if (cudaMalloc(&dev, bytes) != cudaSuccess) return false;
    auto* dh{reinterpret_cast<std::uint32_t*>(dev)};
    auto* dd{dev + 1024};
    auto* db{reinterpret_cast<std::uint16_t*>(dev + 1280)};
    auto* dhead{dev + 1792};
    auto* dn{reinterpret_cast<std::uint32_t*>(dev + 1792 + kDescBytes)};
    bool ok{cudaFuncSetAttribute(prefix_code_test_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(sizeof(WarpCodeSmem))) == cudaSuccess &&
            cudaMemcpy(dh, hist, static_cast<std::size_t>(length) * 4, cudaMemcpyHostToDevice) == cudaSuccess};
    if (ok) {
        prefix_code_test_kernel<<<1, 32, sizeof(WarpCodeSmem)>>>(dh, length, dd, db, dhead, dn);
        ok = cudaGetLastError() == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess &&
             cudaMemcpy(depth, dd, static_cast<std::size_t>(length), cudaMemcpyDeviceToHost) == cudaSuccess &&
             cudaMemcpy(bits, db, static_cast<std::size_t>(length) * 2, cudaMemcpyDeviceToHost) == cudaSuccess &&
             cudaMemcpy(header, dhead, kDescBytes, cudaMemcpyDeviceToHost) == cudaSuccess &&
             cudaMemcpy(nbits, dn, 4, cudaMemcpyDeviceToHost) == cudaSuccess;
    }
    cudaFree(dev);
    return ok;
}

bool entropy_kernels_init() {
    std::uint8_t ctx[kCoeffCtxBytes]{};
    for (int i{1}; i < 64; ++i) {
        ctx[i] = static_cast<std::uint8_t>(coeff_nz_ctx(static_cast<std::uint32_t>(i)));
        ctx[64 + i] = static_cast<std::uint8_t>(coeff_freq_ctx(static_cast<std::uint32_t>(i)));
    }
    for (int g{0}; g < 2; ++g) {
        for (int z{0}; z < kZeroDensityCount; ++z) {
            // Block context 0 stands for every luma context, 7 for every chroma one.
            ctx[128 + g * kZdRow + z] = static_cast<std::uint8_t>(context_cluster(
                static_cast<std::uint32_t>(kNumBlockCtx * kNonZeroBuckets + kZeroDensityCount * (7 * g) + z)));
        }
    }
    if (cudaMemcpyToSymbol(g_coeff_ctx, ctx, sizeof(ctx)) != cudaSuccess) return false;
    return cudaFuncSetAttribute(codes_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(sizeof(WarpCodeSmem))) == cudaSuccess &&
           cudaFuncSetAttribute(layout_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(kLayoutSmemLimit)) == cudaSuccess &&
           cudaFuncSetAttribute(tokens_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(kHistSmem)) == cudaSuccess &&
           cudaFuncSetAttribute(lengths_unstored_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(kBitsSmem)) == cudaSuccess &&
           cudaFuncSetAttribute(emit_unstored_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(kEmitSmem)) == cudaSuccess &&
           cudaFuncSetAttribute(codes_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(sizeof(WarpCodeSmem))) == cudaSuccess &&
           cudaFuncSetAttribute(layout_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(kLayoutSmemLimit)) == cudaSuccess &&
           cudaFuncSetAttribute(tokens_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(kHistSmem)) == cudaSuccess &&
           cudaFuncSetAttribute(lengths_unstored_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(kBitsSmem)) == cudaSuccess &&
           cudaFuncSetAttribute(emit_unstored_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(kEmitSmem)) == cudaSuccess;
}

}  // namespace jxb
