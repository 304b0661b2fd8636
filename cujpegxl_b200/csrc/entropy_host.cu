// Host side of the entropy stage: the per-geometry section table, the
// constant header blobs (modular tree headers, AcGlobal prefix with the fixed
// context map), the natural coefficient orders and the DcGlobal section.
// Every blob is written with the same prefix-code builder as the device
// (prefix_code.cuh), so the bits equal the reference's host writer
// (src/bitstream/*.cc).

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "entropy.cuh"
#include "jxl_constants.cuh"
#include "prefix_code.cuh"

namespace jxb {
namespace {


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
    // Unpadded: a separate DcGlobal section is padded by the layout, and in
    // the combined single-group section the DcGroup follows bit for bit.
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
    p.ac_first = at;
    for (int g{0}; g < xg * yg; ++g) {
        const int gw{std::min(32, bw - (g % xg) * 32)};
        const int gh{std::min(32, bh - (g / xg) * 32)};
        const std::uint32_t cnt{static_cast<std::uint32_t>(3 * gw * gh)};
        const int sec{static_cast<int>(p.sections.size())};
        for (int r0{0}; r0 < gh; r0 += kStripeRows) {
            const int rows{std::min(kStripeRows, gh - r0)};
            p.stripes.push_back({at + static_cast<std::uint32_t>(3 * gw * r0), sec, static_cast<std::uint16_t>(g),
                                 static_cast<std::uint8_t>(r0), static_cast<std::uint8_t>(rows)});
        }
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

}  // namespace jxb
