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

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "entropy.cuh"
#include "jxl_constants.cuh"
#include "prefix_code.cuh"

namespace jxb {
namespace {

// Token channel order Y, X, B over planes stored X, Y, B.
__device__ __forceinline__ int phys_channel(int p) { return p == 0 ? 1 : (p == 1 ? 0 : 2); }

__device__ __forceinline__ int find_section(const Section* secs, int nsec, std::uint32_t item) {
    int lo{0};
    int hi{nsec - 1};
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

// Table selectors for tokens.
enum TokTable : int { kTabAc = 0, kTabDc = 1, kTabAm = 2 };

// Visits the bits of one item in stream order. The visitor receives
//   blob(bytes, nbits), raw(nbits, value),
//   token(table, index, symbol, extra_bits, extra_value, hist_weight_flag)
// where `index` is the AC cluster or the DC group.
template <class V>
__device__ void visit_item(const EntropyDev& e, std::uint32_t item, V& v) {
    const int s{find_section(e.sections, e.nsec, item)};
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
    if (sec.kind == kSecAcGroup) {
        const GroupGeom gg{ac_group_geom(e, sec.group)};
        const int bidx{static_cast<int>(j / 3)};
        const int c{phys_channel(static_cast<int>(j % 3))};
        const int bx{gg.bx0 + bidx % gg.gw};
        const int by{gg.by0 + bidx / gg.gw};
        const std::size_t blk{static_cast<std::size_t>(by) * e.bw + bx};
        const int n{e.acs[blk]};
        if (n == 0) return;
        const std::size_t cb{static_cast<std::size_t>(c) * e.nblocks};
        const std::uint32_t nz{e.nzc[cb + blk]};
        const bool hl{bx > gg.bx0};
        const bool ht{by > gg.by0};
        const std::uint32_t top{ht ? e.nzn[cb + blk - e.bw] : 0u};
        const std::uint32_t left{hl ? e.nzn[cb + blk - 1] : 0u};
        const int bctx{block_ctx(c, n)};
        std::uint32_t tok, nb, bits;
        hybrid_uint(nz, tok, nb, bits);
        v.token(kTabAc, context_cluster(nonzero_context(predict_nonzeros(hl, ht, top, left), bctx)),
                tok, nb, bits);
        if (nz == 0) return;
        const int side{n >> 3};
        const std::uint32_t covered{static_cast<std::uint32_t>(side * side)};
        const std::uint32_t size{static_cast<std::uint32_t>(n * n)};
        const std::uint32_t l2{n == 16 ? 2u : (n == 32 ? 4u : 0u)};
        const std::uint16_t* ord{e.order + (n == 8 ? 0 : (n == 16 ? 64 : 320))};
        const std::int16_t* plane{e.ac + static_cast<std::size_t>(c) * e.nblocks * kCoeffsPerBlock};
        std::uint32_t remaining{nz};
        std::uint32_t prev{nz > size / 16 ? 0u : 1u};
        for (std::uint32_t k{covered}; k < size && remaining > 0; ++k) {
            const int raw{__ldg(&ord[k])};
            const std::int32_t val{plane[covered_slot(n, bx, by, e.bw, raw)]};
            const std::uint32_t ctx{coeff_context(bctx, remaining, k, covered, l2, prev)};
            hybrid_uint(pack_signed(val), tok, nb, bits);
            v.token(kTabAc, context_cluster(ctx), tok, nb, bits);
            prev = val != 0 ? 1u : 0u;
            remaining -= prev;
        }
        return;
    }
    // DC group.
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

// ---- pass 1: histograms ---------------------------------------------------------

struct HistVisitor {
    std::uint32_t* sh_ac;     // [32][256] shared
    std::uint32_t* sh_g;      // [2][2][256] shared: slot x (dc, am)
    std::uint32_t* sh_fb;     // [2] shared first-block counts per slot
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
    __device__ void token(int tab, int idx, std::uint32_t sym, std::uint32_t, std::uint32_t) {
        if (tab == kTabAc) {
            atomicAdd(&sh_ac[idx * 256 + sym], 1u);
            return;
        }
        const int t{tab == kTabDc ? 0 : 1};
        if (idx == g0) {
            atomicAdd(&sh_g[(0 * 2 + t) * 256 + sym], 1u);
        } else if (idx == g1) {
            atomicAdd(&sh_g[(1 * 2 + t) * 256 + sym], 1u);
        } else {
            atomicAdd(&(t == 0 ? e->dc_hist : e->am_hist)[idx * 256 + sym], 1u);
        }
    }
};

__global__ void __launch_bounds__(256) hist_kernel(EntropyDev e) {
    __shared__ std::uint32_t sh_ac[kNumClusters * 256];
    __shared__ std::uint32_t sh_g[4 * 256];
    __shared__ std::uint32_t sh_fb[2];
    if (threadIdx.x < 2) sh_fb[threadIdx.x] = 0;
    for (int i{static_cast<int>(threadIdx.x)}; i < kNumClusters * 256; i += blockDim.x) sh_ac[i] = 0;
    for (int i{static_cast<int>(threadIdx.x)}; i < 4 * 256; i += blockDim.x) sh_g[i] = 0;
    const std::uint32_t first{blockIdx.x * blockDim.x};
    const std::uint32_t last{min(first + blockDim.x, e.total_items) - 1};
    const Section s0{e.sections[find_section(e.sections, e.nsec, first)]};
    const Section s1{e.sections[find_section(e.sections, e.nsec, last)]};
    HistVisitor v{sh_ac, sh_g, sh_fb, s0.kind == kSecDcGroup ? s0.group : -1,
                  s1.kind == kSecDcGroup && s1.group != s0.group ? s1.group : -2, &e};
    __syncthreads();
    const std::uint32_t item{first + threadIdx.x};
    if (item < e.total_items) visit_item(e, item, v);
    __syncthreads();
    for (int i{static_cast<int>(threadIdx.x)}; i < kNumClusters * 256; i += blockDim.x) {
        if (sh_ac[i]) atomicAdd(&e.ac_hist[i], sh_ac[i]);
    }
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
    HuffNode pool[2 * 256 + 4];
    std::uint8_t level[2 * 256 + 4];
    std::uint8_t depth[256];
    std::uint16_t bits[256];
};

// Depths for a histogram with at least two used symbols, warp-cooperative:
// each lane ranks its symbols by (clamped count ascending, symbol descending),
// which is the order the reference's stable sort produces from leaves pushed
// in descending symbol order; lane 0 merges and assigns levels.
__device__ void warp_create_tree(WarpCodeSmem& s, int length, int limit, int lane) {
    for (std::uint32_t floor{1};; floor *= 2) {
        int mine{0};
        for (int sym{lane}; sym < length; sym += 32) {
            if (s.hist[sym]) ++mine;
        }
        int n{mine};
#pragma unroll
        for (int off{16}; off > 0; off >>= 1) n += __shfl_xor_sync(0xffffffffu, n, off);
        for (int sym{lane}; sym < length; sym += 32) {
            const std::uint32_t h{s.hist[sym]};
            if (!h) continue;
            const std::uint32_t c{h > floor - 1 ? h : floor - 1};
            int rank{0};
            for (int t{0}; t < length; ++t) {
                const std::uint32_t ht{s.hist[t]};
                if (!ht) continue;
                const std::uint32_t ct{ht > floor - 1 ? ht : floor - 1};
                rank += (ct < c || (ct == c && t > sym)) ? 1 : 0;
            }
            s.pool[rank].count = c;
            s.pool[rank].left = -1;
            s.pool[rank].right_or_value = static_cast<std::int16_t>(sym);
        }
        __syncwarp();
        int mx{0};
        if (lane == 0) {
            merge_pool(s.pool, n);
            for (int i{0}; i < length; ++i) s.depth[i] = 0;
            depths_from_pool(s.pool, n, s.level, s.depth);
            for (int i{0}; i < length; ++i) mx = s.depth[i] > mx ? s.depth[i] : mx;
        }
        mx = __shfl_sync(0xffffffffu, mx, 0);
        __syncwarp();
        if (mx <= limit) return;
    }
}

// build_and_store for histogram s.hist[0..length), warp-cooperative; lane 0
// writes the header into w. Leaves depth/bits in s.
__device__ void warp_build_and_store(WarpCodeSmem& s, int length, BitSink& w, int lane) {
    for (int i{lane}; i < 256; i += 32) {
        s.depth[i] = 0;
        s.bits[i] = 0;
    }
    __syncwarp();
    int s4[4]{0, 0, 0, 0};
    int count{0};
    if (lane == 0) count = symbol_census(s.hist, length, s4);
    count = __shfl_sync(0xffffffffu, count, 0);
    if (count <= 1) {
        if (lane == 0) {
            w.put(4, 1);
            w.put(alphabet_bits(length), static_cast<std::uint32_t>(s4[0]));
        }
        __syncwarp();
        return;
    }
    warp_create_tree(s, length, 15, lane);
    if (lane == 0) {
        canonical_codes(s.depth, length, s.bits);
        store_code_header(count, s4, length, s.depth, w);
    }
    __syncwarp();
}

__global__ void __launch_bounds__(512) codes_kernel(EntropyDev e) {
    extern __shared__ __align__(16) unsigned char code_smem[];
    const int warp{static_cast<int>(threadIdx.x) >> 5};
    const int lane{static_cast<int>(threadIdx.x) & 31};
    WarpCodeSmem& s{reinterpret_cast<WarpCodeSmem*>(code_smem)[warp]};
    int idx;          // description slot
    const std::uint32_t* src;
    std::uint8_t* dst_depth;
    std::uint16_t* dst_bits;
    bool clustered;
    std::uint32_t extra0{0};
    if (blockIdx.x < 2) {
        const int c{static_cast<int>(blockIdx.x) * 16 + warp};
        idx = c;
        src = e.ac_hist + c * 256;
        dst_depth = e.ac_depth + c * 256;
        dst_bits = e.ac_bits + c * 256;
        clustered = true;
    } else {
        if (warp >= 2) return;
        const int g{static_cast<int>(blockIdx.x) - 2};
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
    for (int i{lane}; i < 256; i += 32) s.hist[i] = src[i] + (i == 0 ? extra0 : 0u);
    std::uint8_t* d{e.desc + idx * kDescBytes};
    for (int i{lane}; i < kDescBytes; i += 32) d[i] = 0;
    __syncwarp();
    int alpha{1};
    for (int i{lane}; i < 256; i += 32) {
        if (s.hist[i]) alpha = i + 1;
    }
#pragma unroll
    for (int off{16}; off > 0; off >>= 1) alpha = max(alpha, __shfl_xor_sync(0xffffffffu, alpha, off));
    BitSink w{d, 0, kDescBytes * 8, false};
    if (clustered) {
        if (lane == 0) e.ac_alpha[idx] = static_cast<std::uint32_t>(alpha);
        if (alpha > 1) {
            warp_build_and_store(s, alpha, w, lane);
        } else {
            for (int i{lane}; i < 256; i += 32) {
                s.depth[i] = 0;
                s.bits[i] = 0;
            }
            __syncwarp();
        }
    } else {
        // Single-context prefix histogram (src/bitstream/histogram_writer.cc:59-83).
        if (lane == 0) {
            w.put(1, 0);
            w.put(1, 1);
            put_uint_config(w, 4, 2, 0);
            put_var_len_u16(w, static_cast<std::uint32_t>(alpha - 1));
        }
        w.pos = __shfl_sync(0xffffffffu, w.pos, 0);
        if (alpha > 1) {
            warp_build_and_store(s, alpha, w, lane);
        } else {
            for (int i{lane}; i < 256; i += 32) {
                s.depth[i] = 0;
                s.bits[i] = 0;
            }
            __syncwarp();
        }
    }
    if (lane == 0) e.desc_bits[idx] = w.overflow ? 0u : w.pos;
    for (int i{lane}; i < 256; i += 32) {
        dst_depth[i] = s.depth[i];
        dst_bits[i] = s.bits[i];
    }
}

// ---- pass 3: bit lengths and scan ----------------------------------------------------

struct BitsVisitor {
    const EntropyDev* e;
    unsigned long long total;
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
    __device__ void token(int tab, int idx, std::uint32_t sym, std::uint32_t nb, std::uint32_t) {
        const std::uint8_t* d{tab == kTabAc ? e->ac_depth : (tab == kTabDc ? e->dc_depth : e->am_depth)};
        total += d[idx * 256 + sym] + nb;
    }
};

__global__ void __launch_bounds__(256) bits_kernel(EntropyDev e) {
    const std::uint32_t item{blockIdx.x * blockDim.x + threadIdx.x};
    if (item >= e.total_items) return;
    BitsVisitor v{&e, 0};
    visit_item(e, item, v);
    e.item_bits[item] = static_cast<std::uint32_t>(v.total);
}

// Exclusive scan of item_bits inside tiles of kScanTile items (1024 threads x 4).
__global__ void __launch_bounds__(1024) scan_tile_kernel(EntropyDev e) {
    __shared__ std::uint32_t warp_sums[32];
    const std::uint32_t base{blockIdx.x * kScanTile + threadIdx.x * 4};
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
        const std::uint32_t t{__shfl_up_sync(0xffffffffu, incl, off)};
        if (lane >= off) incl += t;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        std::uint32_t ws{warp_sums[lane]};
        std::uint32_t wi{ws};
#pragma unroll
        for (int off{1}; off < 32; off <<= 1) {
            const std::uint32_t t{__shfl_up_sync(0xffffffffu, wi, off)};
            if (lane >= off) wi += t;
        }
        warp_sums[lane] = wi - ws;
        if (lane == 31) e.tile_sum[blockIdx.x] = wi;
    }
    __syncthreads();
    std::uint32_t run{warp_sums[warp] + incl - local};
#pragma unroll
    for (int k{0}; k < 4; ++k) {
        if (base + k < e.total_items) e.item_pre[base + k] = run;
        run += v[k];
    }
}

__global__ void __launch_bounds__(1024) scan_top_kernel(EntropyDev e) {
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
            const unsigned long long t{__shfl_up_sync(0xffffffffu, incl, off)};
            if (lane >= off) incl += t;
        }
        if (lane == 31) warp_sums[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const unsigned long long ws{warp_sums[lane]};
            unsigned long long wi{ws};
#pragma unroll
            for (int off{1}; off < 32; off <<= 1) {
                const unsigned long long t{__shfl_up_sync(0xffffffffu, wi, off)};
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

__device__ __forceinline__ unsigned long long prefix_at(const EntropyDev& e, std::uint32_t i) {
    if (i >= e.total_items) return e.tile_off[e.num_tiles];
    return e.tile_off[i / kScanTile] + e.item_pre[i];
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

constexpr int kHeadBytes = 8192;

// Single thread: sizes the sections, writes the container framing, codestream
// headers, frame header and TOC (src/bitstream/codestream.cc:57-135,
// src/bitstream/container.cc:35-62) and places the sections.
__global__ void layout_kernel(EntropyDev e) {
    __shared__ __align__(16) std::uint8_t head[kHeadBytes];
    if (threadIdx.x != 0) return;
    for (int i{0}; i < kHeadBytes; ++i) head[i] = 0;
    BitSink w{head, 0, kHeadBytes * 8, false};
    const U32Dist dim[4]{{false, 1, 9}, {false, 1, 13}, {false, 1, 18}, {false, 1, 30}};
    const U32Dist toc[4]{{false, 0, 10}, {false, 1024, 14}, {false, 17408, 22}, {false, 4211712, 30}};
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
    // TOC without permutation.
    w.put(1, 0);
    w.pos = (w.pos + 7) & ~7u;
    unsigned long long body{0};
    for (int s{0}; s < e.nsec; ++s) {
        const Section sec{e.sections[s]};
        const unsigned long long bits{prefix_at(e, sec.first + sec.count) - prefix_at(e, sec.first)};
        const unsigned long long bytes{(bits + 7) / 8};
        put_u32(w, toc, static_cast<std::uint32_t>(bytes));
        e.sec_pos[s] = body;  // relative to the body start for now
        body += bytes;
    }
    w.pos = (w.pos + 7) & ~7u;
    const unsigned long long head_bytes{w.pos / 8};
    const unsigned long long cs{head_bytes + body};
    const bool large{cs >= 0x100000000ull - 8};
    const unsigned long long framing{32ull + (large ? 16 : 8)};
    const unsigned long long total{framing + cs};
    unsigned long long status{w.overflow ? 2ull : 0ull};
    if (total > e.out_capacity) status = 1;
    e.result[0] = total;
    e.result[1] = framing + head_bytes;
    e.result[2] = status;
    if (status != 0) return;
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
    for (unsigned long long i{0}; i < head_bytes; ++i) e.out[at++] = head[i];
    for (int s{0}; s < e.nsec; ++s) e.sec_pos[s] += framing + head_bytes;
}

__global__ void zero_body_kernel(EntropyDev e) {
    if (e.result[2] != 0) return;
    const unsigned long long start{e.result[1]};
    const unsigned long long end{e.result[0]};
    const unsigned long long a{(start + 15) & ~15ull};
    const unsigned long long stride{static_cast<unsigned long long>(gridDim.x) * blockDim.x};
    const unsigned long long tid{static_cast<unsigned long long>(blockIdx.x) * blockDim.x + threadIdx.x};
    if (tid < a - start && start + tid < end) e.out[start + tid] = 0;
    const unsigned long long nvec{end > a ? (end - a) / 16 : 0};
    uint4* v{reinterpret_cast<uint4*>(e.out + a)};
    for (unsigned long long i{tid}; i < nvec; i += stride) v[i] = make_uint4(0, 0, 0, 0);
    const unsigned long long tail{a + nvec * 16};
    if (tail + tid < end && tid < 16) e.out[tail + tid] = 0;
}

// ---- pass 5: emission ------------------------------------------------------------

struct EmitVisitor {
    const EntropyDev* e;
    unsigned int* words;
    unsigned long long pos;
    __device__ void put(std::uint32_t n, std::uint32_t v) {
        if (n == 0) return;
        if (n < 32) v &= (1u << n) - 1u;
        while (n > 0) {
            const unsigned long long wi{pos >> 5};
            const std::uint32_t off{static_cast<std::uint32_t>(pos & 31)};
            const std::uint32_t take{n < 32 - off ? n : 32 - off};
            const std::uint32_t chunk{take == 32 ? v : (v & ((1u << take) - 1u))};
            atomicOr(&words[wi], chunk << off);
            v = take == 32 ? 0 : v >> take;
            n -= take;
            pos += take;
        }
    }
    __device__ void blob(const std::uint8_t* b, std::uint32_t nbits) {
        std::uint32_t i{0};
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
    __device__ void token(int tab, int idx, std::uint32_t sym, std::uint32_t nb, std::uint32_t bits) {
        const std::uint8_t* d{tab == kTabAc ? e->ac_depth : (tab == kTabDc ? e->dc_depth : e->am_depth)};
        const std::uint16_t* c{tab == kTabAc ? e->ac_bits : (tab == kTabDc ? e->dc_bits : e->am_bits)};
        put(d[idx * 256 + sym], c[idx * 256 + sym]);
        if (nb) put(nb, bits);
    }
};

__global__ void __launch_bounds__(256) emit_kernel(EntropyDev e) {
    if (e.result[2] != 0) return;
    const std::uint32_t item{blockIdx.x * blockDim.x + threadIdx.x};
    if (item >= e.total_items) return;
    const int s{find_section(e.sections, e.nsec, item)};
    const Section sec{e.sections[s]};
    const unsigned long long rel{prefix_at(e, item) - prefix_at(e, sec.first)};
    EmitVisitor v{&e, reinterpret_cast<unsigned int*>(e.out), e.sec_pos[s] * 8 + rel};
    visit_item(e, item, v);
}

// ---- host-side constant blobs ------------------------------------------------------

struct HostBits {
    std::vector<std::uint8_t> buf;
    BitSink w;
    HostBits() : buf(1 << 16, 0), w{nullptr, 0, (1u << 16) * 8, false} { w.buf = buf.data(); }
    std::vector<std::uint8_t> bytes() const {
        return std::vector<std::uint8_t>(buf.begin(), buf.begin() + (w.pos + 7) / 8);
    }
};

// Single-histogram description with the serial builder (small alphabets).
void host_prefix_histograms(BitSink& w, const std::uint32_t* hist, int length, int num_contexts,
                            std::uint32_t se, std::uint32_t msb, std::uint32_t lsb, std::uint8_t* depth,
                            std::uint16_t* bits) {
    w.put(1, 0);
    if (num_contexts > 1) {
        w.put(1, 1);
        w.put(2, 0);
    }
    w.put(1, 1);
    put_uint_config(w, se, msb, lsb);
    put_var_len_u16(w, static_cast<std::uint32_t>(length - 1));
    for (int i{0}; i < length; ++i) {
        depth[i] = 0;
        bits[i] = 0;
    }
    if (length > 1) {
        std::vector<HuffNode> pool(2 * length + 4);
        std::vector<std::uint8_t> level(2 * length + 4);
        build_and_store_serial(hist, length, depth, bits, w, pool.data(), level.data());
    }
}

// Hybrid-uint split with an arbitrary configuration.
void host_hybrid(std::uint32_t v, std::uint32_t se, std::uint32_t msb, std::uint32_t lsb,
                 std::uint32_t& tok, std::uint32_t& nb, std::uint32_t& bits) {
    const std::uint32_t split{1u << se};
    if (v < split) {
        tok = v;
        nb = 0;
        bits = 0;
        return;
    }
    std::uint32_t n{31};
    while (!((v >> n) & 1u)) --n;
    const std::uint32_t m{v - (1u << n)};
    tok = split + ((n - se) << (msb + lsb)) + ((m >> (n - msb)) << lsb) + (m & ((1u << lsb) - 1u));
    nb = n - msb - lsb;
    bits = (v >> lsb) & ((1u << nb) - 1u);
}

// Complex context map (src/bitstream/context_map.cc:127-164).
void host_context_map_complex(BitSink& w, const std::vector<std::uint8_t>& map, bool mtf) {
    std::vector<std::uint8_t> sym(map.size());
    std::uint8_t order[256];
    for (int i{0}; i < 256; ++i) order[i] = static_cast<std::uint8_t>(i);
    for (std::size_t i{0}; i < map.size(); ++i) {
        if (!mtf) {
            sym[i] = map[i];
            continue;
        }
        int r{0};
        while (order[r] != map[i]) ++r;
        sym[i] = static_cast<std::uint8_t>(r);
        const std::uint8_t v{order[r]};
        for (; r > 0; --r) order[r] = order[r - 1];
        order[0] = v;
    }
    std::uint32_t hist[16]{};
    for (std::uint8_t s : sym) {
        std::uint32_t t, nb, b;
        host_hybrid(s, 2, 0, 1, t, nb, b);
        ++hist[t];
    }
    int alpha{1};
    for (int i{0}; i < 16; ++i) {
        if (hist[i]) alpha = i + 1;
    }
    w.put(1, 0);
    w.put(1, mtf ? 1 : 0);
    std::uint8_t depth[16];
    std::uint16_t bits[16];
    host_prefix_histograms(w, hist, alpha, 1, 2, 0, 1, depth, bits);
    for (std::uint8_t s : sym) {
        std::uint32_t t, nb, b;
        host_hybrid(s, 2, 0, 1, t, nb, b);
        w.put(depth[t], bits[t]);
        if (nb) w.put(nb, b);
    }
}

// Modular group header + single-leaf tree (src/bitstream/frame_assembly.cc:150-175).
void host_modular_tree(BitSink& w, bool gradient) {
    w.put(1, 0);
    w.put(1, 1);
    w.put(2, 0);
    const std::uint32_t tokens[5]{0, gradient ? 5u : 0u, 0, 0, 0};
    std::uint32_t hist[16]{};
    int len{1};
    for (std::uint32_t t : tokens) {
        ++hist[t];
        len = std::max(len, static_cast<int>(t) + 1);
    }
    std::uint8_t depth[16];
    std::uint16_t bits[16];
    host_prefix_histograms(w, hist, len, 6, 4, 2, 0, depth, bits);
    for (std::uint32_t t : tokens) w.put(depth[t], bits[t]);
}

void append_bits(BitSink& dst, const BitSink& src) { dst.put_bits(src.buf, src.pos); }

}  // namespace

std::size_t worst_case_output(std::uint32_t width, std::uint32_t height) {
    const std::size_t bw{width / 8u};
    const std::size_t bh{height / 8u};
    const std::size_t nac{((bw + 31) / 32) * ((bh + 31) / 32)};
    const std::size_t ndc{((bw + 255) / 256) * ((bh + 255) / 256)};
    return 3 * bw * bh * 384 + 48 * bw * bh + (nac + ndc) * 2048 + 16384;
}

std::vector<std::uint8_t> dc_global_bits(std::uint32_t global_scale, std::uint32_t quant_dc,
                                         std::uint32_t* nbits) {
    HostBits hb;
    BitSink& w{hb.w};
    auto u32 = [&](const std::uint32_t (*d)[3], std::uint32_t value) {
        std::uint32_t best{0};
        std::uint32_t best_bits{64};
        for (std::uint32_t s{0}; s < 4; ++s) {
            if (d[s][0]) {
                if (d[s][1] == value) {
                    best = s;
                    best_bits = 2;
                    break;
                }
                continue;
            }
            if (value < d[s][1] || static_cast<unsigned long long>(value) >=
                                       static_cast<unsigned long long>(d[s][1]) + (1ull << d[s][2])) {
                continue;
            }
            if (2 + d[s][2] < best_bits) {
                best = s;
                best_bits = 2 + d[s][2];
            }
        }
        w.put(2, best);
        if (!d[best][0]) w.put(d[best][2], value - d[best][1]);
    };
    const std::uint32_t gs_enc[4][3]{{0, 1, 11}, {0, 2049, 11}, {0, 4097, 12}, {0, 8193, 16}};
    const std::uint32_t qdc_enc[4][3]{{1, 16, 0}, {0, 1, 5}, {0, 1, 8}, {0, 1, 16}};
    w.put(1, 1);
    u32(gs_enc, global_scale);
    u32(qdc_enc, quant_dc);
    w.put(1, 1);
    w.put(1, 1);
    w.put(1, 0);
    w.pos = (w.pos + 7) & ~7u;
    *nbits = w.pos;
    return hb.bytes();
}

EntropyHostPlan entropy_plan(int width, int height) {
    EntropyHostPlan p;
    const int bw{width / 8};
    const int bh{height / 8};
    const int xg{(bw + 31) / 32};
    const int yg{(bh + 31) / 32};
    const int xdg{(bw + 255) / 256};
    const int ydg{(bh + 255) / 256};
    std::uint32_t at{0};
    p.sections.push_back({at, 1, kSecDcGlobal, 0});
    at += 1;
    for (int g{0}; g < xdg * ydg; ++g) {
        const int gw{std::min(256, bw - (g % xdg) * 256)};
        const int gh{std::min(256, bh - (g / xdg) * 256)};
        const std::uint32_t n{static_cast<std::uint32_t>(gw * gh)};
        const std::uint32_t cwch{static_cast<std::uint32_t>(((gw + 7) / 8) * ((gh + 7) / 8))};
        const std::uint32_t cnt{5 + 6 * n + 2 * cwch};
        p.sections.push_back({at, cnt, kSecDcGroup, g});
        at += cnt;
    }
    p.sections.push_back({at, 65, kSecAcGlobal, 0});
    at += 65;
    for (int g{0}; g < xg * yg; ++g) {
        const int gw{std::min(32, bw - (g % xg) * 32)};
        const int gh{std::min(32, bh - (g / xg) * 32)};
        const std::uint32_t cnt{static_cast<std::uint32_t>(3 * gw * gh)};
        p.sections.push_back({at, cnt, kSecAcGroup, g});
        at += cnt;
    }
    p.total_items = at;

    {
        HostBits hb;
        hb.w.put(2, 0);  // extra_precision
        host_modular_tree(hb.w, true);
        p.pre_const = hb.bytes();
        p.pre_const_bits = hb.w.pos;
    }
    {
        HostBits hb;
        host_modular_tree(hb.w, false);
        p.mid_const = hb.bytes();
        p.mid_const_bits = hb.w.pos;
    }
    {
        HostBits hb;
        BitSink& w{hb.w};
        w.put(1, 1);                                                       // dequant all_default
        w.put(ceil_log2_u(static_cast<std::uint32_t>(xg * yg)), 0);        // num_histograms - 1
        w.put(2, 2);                                                       // used_orders = 0
        w.put(1, 0);                                                       // lz77 disabled
        std::vector<std::uint8_t> map(kNumAcContexts);
        for (int i{0}; i < kNumAcContexts; ++i) {
            map[i] = static_cast<std::uint8_t>(context_cluster(static_cast<std::uint32_t>(i)));
        }
        HostBits a;
        HostBits b;
        host_context_map_complex(a.w, map, false);
        host_context_map_complex(b.w, map, true);
        append_bits(w, b.w.pos < a.w.pos ? b.w : a.w);
        w.put(1, 1);  // use_prefix_code
        for (int c{0}; c < kNumClusters; ++c) put_uint_config(w, 4, 2, 0);
        p.ac_prefix = hb.bytes();
        p.ac_prefix_bits = w.pos;
    }
    // Natural coefficient orders (src/coeff_order.cc:10-43), concatenated 8|16|32.
    for (int n : {8, 16, 32}) {
        const int cx{n / 8};
        std::vector<std::uint16_t> out(static_cast<std::size_t>(n) * n);
        int cur{cx * cx};
        for (int i{0}; i < n; ++i) {
            for (int jj{0}; jj <= i; ++jj) {
                int x{jj};
                int y{i - jj};
                if (i & 1) std::swap(x, y);
                const int val{(x < cx && y < cx) ? y * cx + x : cur++};
                out[val] = static_cast<std::uint16_t>(y * n + x);
            }
        }
        for (int ip{n - 1}; ip > 0; --ip) {
            const int i{ip - 1};
            for (int jj{0}; jj <= i; ++jj) {
                int x{n - 1 - (i - jj)};
                int y{n - 1 - jj};
                if (i & 1) std::swap(x, y);
                out[cur++] = static_cast<std::uint16_t>(y * n + x);
            }
        }
        p.order.insert(p.order.end(), out.begin(), out.end());
    }
    return p;
}

bool entropy_launch(const EntropyDev& e, void* stream) {
    cudaStream_t st{static_cast<cudaStream_t>(stream)};
    if (cudaMemsetAsync(e.ac_hist, 0, kNumClusters * 256 * sizeof(std::uint32_t), st) != cudaSuccess ||
        cudaMemsetAsync(e.dc_hist, 0, static_cast<std::size_t>(e.ndc) * 256 * sizeof(std::uint32_t), st) != cudaSuccess ||
        cudaMemsetAsync(e.am_hist, 0, static_cast<std::size_t>(e.ndc) * 256 * sizeof(std::uint32_t), st) != cudaSuccess ||
        cudaMemsetAsync(e.fb_count, 0, static_cast<std::size_t>(e.ndc) * sizeof(std::uint32_t), st) != cudaSuccess) {
        return false;
    }
    const unsigned items{e.total_items};
    hist_kernel<<<(items + 255) / 256, 256, 0, st>>>(e);
    const std::size_t code_smem{sizeof(WarpCodeSmem) * 16};
    codes_kernel<<<2 + e.ndc, 512, code_smem, st>>>(e);
    bits_kernel<<<(items + 255) / 256, 256, 0, st>>>(e);
    scan_tile_kernel<<<e.num_tiles, 1024, 0, st>>>(e);
    scan_top_kernel<<<1, 1024, 0, st>>>(e);
    layout_kernel<<<1, 32, 0, st>>>(e);
    zero_body_kernel<<<296, 256, 0, st>>>(e);
    emit_kernel<<<(items + 255) / 256, 256, 0, st>>>(e);
    return cudaGetLastError() == cudaSuccess;
}

bool entropy_kernels_init() {
    return cudaFuncSetAttribute(codes_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(sizeof(WarpCodeSmem) * 16)) == cudaSuccess;
}

}  // namespace jxb
