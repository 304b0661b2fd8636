// A JPEG XL decoder for the subset this encoder writes, on the host: ISOBMFF
// container, codestream and frame headers, TOC, prefix-coded histograms and
// context maps, modular DC and AcMetadata groups (single-leaf trees with the
// Gradient and Zero predictors), VarDCT AC groups with DCT8/16/32, CfL,
// LLF from DC, inverse DCT, the decoder's 3x3 gaborish and XYB -> sRGB.
//
// It checks decodability of the output (every header field and section is
// parsed and every section must end exactly where the TOC says) and measures
// quality (PSNR of the luma). Reconstruction is the plain dequantisation of the
// format: the optional decoder-side refinements of libjxl (quantisation-bias
// adjustment, adaptive DC smoothing) are not applied, and the edge-preserving
// filter is a no-op for the all-zero sharpness this encoder writes.
//
// Anything outside the subset (other transforms, LZ77, modular transforms,
// ...) is reported as an error rather than decoded.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "jxl_constants.cuh"
#include "subset_decoder.h"

namespace jxb {
namespace {

#include "jxl_dequant_tables.inc"

struct DecodeError {
    std::string what;
};

[[noreturn]] void fail(const std::string& what) { throw DecodeError{what}; }

// ---- bits ------------------------------------------------------------------

class BitReader {
public:
    BitReader(const std::uint8_t* data, std::size_t size) : data_{data}, size_{size} {}

    std::uint32_t read(int nbits) {
        std::uint32_t v{0};
        for (int i{0}; i < nbits; ++i) v |= static_cast<std::uint32_t>(bit()) << i;
        return v;
    }
    int bit() {
        if (pos_ >= 8 * size_) fail("read past the end of a section");
        const int b{(data_[pos_ >> 3] >> (pos_ & 7)) & 1};
        ++pos_;
        return b;
    }
    std::uint32_t peek4() const {
        std::uint32_t v{0};
        for (int i{0}; i < 4; ++i) {
            const std::size_t p{pos_ + static_cast<std::size_t>(i)};
            if (p < 8 * size_) v |= static_cast<std::uint32_t>((data_[p >> 3] >> (p & 7)) & 1) << i;
        }
        return v;
    }
    void skip(int nbits) { pos_ += static_cast<std::size_t>(nbits); }
    void align() { pos_ = (pos_ + 7) & ~static_cast<std::size_t>(7); }
    std::size_t bits_read() const { return pos_; }
    std::size_t byte_pos() const { return (pos_ + 7) / 8; }

private:
    const std::uint8_t* data_;
    std::size_t size_;
    std::size_t pos_{0};
};

void expect(BitReader& br, int nbits, std::uint32_t value, const char* field) {
    const std::uint32_t v{br.read(nbits)};
    if (v != value) fail(std::string("unsupported ") + field + " = " + std::to_string(v));
}

struct U32Dist {
    bool direct;
    std::uint32_t v;
    int bits;
};

std::uint32_t read_u32(BitReader& br, const U32Dist (&d)[4]) {
    const U32Dist& s{d[br.read(2)]};
    return s.direct ? s.v : s.v + br.read(s.bits);
}

std::uint32_t read_varlen_u16(BitReader& br) {
    if (!br.bit()) return 0;
    const int nb{static_cast<int>(br.read(4))};
    return (1u << nb) + br.read(nb);
}

int ceil_log2(std::uint32_t x) {
    int b{0};
    while ((1u << b) < x) ++b;
    return b;
}

std::int32_t unpack_signed(std::uint32_t v) {
    return (v & 1u) ? -static_cast<std::int32_t>((v >> 1) + 1) : static_cast<std::int32_t>(v >> 1);
}

// ---- prefix codes ------------------------------------------------------------

struct PrefixCode {
    int single{-1};                      // symbol of a zero-length code, or -1
    int count[16]{};
    std::vector<std::uint16_t> sorted;   // symbols by (length, value)

    void build(const std::vector<std::uint8_t>& depth) {
        sorted.clear();
        std::fill(std::begin(count), std::end(count), 0);
        int used{0};
        int last{0};
        for (std::size_t s{0}; s < depth.size(); ++s) {
            if (depth[s] > 15) fail("code length above 15");
            if (depth[s]) {
                ++count[depth[s]];
                ++used;
                last = static_cast<int>(s);
            }
        }
        if (used == 0) fail("empty prefix code");
        for (int l{1}; l < 16; ++l) {
            for (std::size_t s{0}; s < depth.size(); ++s) {
                if (depth[s] == l) sorted.push_back(static_cast<std::uint16_t>(s));
            }
        }
        if (used == 1) single = last;
    }

    int decode(BitReader& br) const {
        if (single >= 0) return single;
        int code{0};
        int first{0};
        int index{0};
        for (int l{1}; l < 16; ++l) {
            code |= br.bit();
            const int c{count[l]};
            if (code - first < c) return sorted[static_cast<std::size_t>(index + code - first)];
            index += c;
            first = (first + c) << 1;
            code <<= 1;
        }
        fail("invalid prefix code word");
    }
};

PrefixCode single_symbol(int s) {
    PrefixCode pc;
    pc.single = s;
    return pc;
}

// Brotli-style prefix code header (simple form or code-length code).
PrefixCode read_prefix_code(BitReader& br, int alphabet) {
    if (alphabet == 1) return single_symbol(0);
    const int alphabet_bits{ceil_log2(static_cast<std::uint32_t>(alphabet))};
    const std::uint32_t hskip{br.read(2)};
    std::vector<std::uint8_t> depth(static_cast<std::size_t>(alphabet), 0);
    if (hskip == 1) {
        const int nsym{static_cast<int>(br.read(2)) + 1};
        int sym[4];
        for (int i{0}; i < nsym; ++i) {
            sym[i] = static_cast<int>(br.read(alphabet_bits));
            if (sym[i] >= alphabet) fail("simple-code symbol outside the alphabet");
        }
        if (nsym == 1) return single_symbol(sym[0]);
        if (nsym == 2) {
            depth[sym[0]] = 1;
            depth[sym[1]] = 1;
        } else if (nsym == 3) {
            depth[sym[0]] = 1;
            depth[sym[1]] = 2;
            depth[sym[2]] = 2;
        } else if (br.bit() == 0) {
            for (int i{0}; i < 4; ++i) depth[sym[i]] = 2;
        } else {
            depth[sym[0]] = 1;
            depth[sym[1]] = 2;
            depth[sym[2]] = 3;
            depth[sym[3]] = 3;
        }
        PrefixCode pc;
        pc.build(depth);
        return pc;
    }
    constexpr int kOrder[18]{1, 2, 3, 4, 0, 5, 17, 6, 16, 7, 8, 9, 10, 11, 12, 13, 14, 15};
    std::vector<std::uint8_t> cl(18, 0);
    int space{32};
    int num_codes{0};
    for (int i{static_cast<int>(hskip)}; i < 18 && space > 0; ++i) {
        // Static code of the code-length-code lengths 0..5 (LSB first):
        // 00 -> 0, 0111 -> 1, 011 -> 2, 10 -> 3, 01 -> 4, 1111 -> 5.
        const std::uint32_t v{br.peek4()};
        int l;
        if ((v & 3u) == 0u) {
            l = 0;
            br.skip(2);
        } else if ((v & 3u) == 2u) {
            l = 3;
            br.skip(2);
        } else if ((v & 3u) == 1u) {
            l = 4;
            br.skip(2);
        } else if ((v & 4u) == 0u) {
            l = 2;
            br.skip(3);
        } else if ((v & 8u) == 0u) {
            l = 1;
            br.skip(4);
        } else {
            l = 5;
            br.skip(4);
        }
        cl[static_cast<std::size_t>(kOrder[i])] = static_cast<std::uint8_t>(l);
        if (l) {
            space -= 32 >> l;
            ++num_codes;
        }
    }
    if (num_codes != 1 && space != 0) fail("incomplete code-length code");
    PrefixCode clc;
    clc.build(cl);
    int sym_space{32768};
    for (int s{0}; s < alphabet && sym_space > 0; ++s) {
        const int l{clc.decode(br)};
        if (l > 15) fail("repeat codes are outside the subset");
        depth[static_cast<std::size_t>(s)] = static_cast<std::uint8_t>(l);
        if (l) sym_space -= 32768 >> l;
    }
    if (sym_space != 0) fail("incomplete prefix code");
    PrefixCode pc;
    pc.build(depth);
    return pc;
}

// ---- entropy codes -----------------------------------------------------------

struct HybridConfig {
    std::uint32_t split_exponent, msb, lsb;
};

HybridConfig read_uint_config(BitReader& br) {
    HybridConfig c{};
    c.split_exponent = br.read(ceil_log2(16));
    if (c.split_exponent == 15) return c;
    c.msb = br.read(ceil_log2(c.split_exponent + 1));
    c.lsb = br.read(ceil_log2(c.split_exponent - c.msb + 1));
    return c;
}

std::uint32_t hybrid_decode(BitReader& br, const HybridConfig& c, std::uint32_t token) {
    const std::uint32_t split{1u << c.split_exponent};
    if (token < split) return token;
    const std::uint32_t nbits{c.split_exponent - (c.msb + c.lsb) + ((token - split) >> (c.msb + c.lsb))};
    if (nbits > 30) fail("hybrid-uint value out of range");
    const std::uint32_t low{token & ((1u << c.lsb) - 1u)};
    const std::uint32_t hi{((token >> c.lsb) & ((1u << c.msb) - 1u)) | (1u << c.msb)};
    return (((hi << nbits) | br.read(static_cast<int>(nbits))) << c.lsb) | low;
}

struct EntropyCode {
    std::vector<std::uint8_t> ctx_map;
    std::vector<HybridConfig> cfg;
    std::vector<PrefixCode> codes;

    std::uint32_t read(BitReader& br, std::size_t ctx) const {
        const std::uint8_t cl{ctx_map[ctx]};
        const std::uint32_t tok{static_cast<std::uint32_t>(codes[cl].decode(br))};
        return hybrid_decode(br, cfg[cl], tok);
    }
};

EntropyCode read_entropy_code(BitReader& br, std::size_t num_contexts);

std::vector<std::uint8_t> read_context_map(BitReader& br, std::size_t n) {
    std::vector<std::uint8_t> map(n, 0);
    if (br.bit()) {
        const int bits{static_cast<int>(br.read(2))};
        for (std::size_t i{0}; i < n; ++i) map[i] = static_cast<std::uint8_t>(br.read(bits));
        return map;
    }
    const bool mtf{br.bit() != 0};
    const EntropyCode nested{read_entropy_code(br, 1)};
    for (std::size_t i{0}; i < n; ++i) {
        const std::uint32_t v{nested.read(br, 0)};
        if (v > 255) fail("context map entry out of range");
        map[i] = static_cast<std::uint8_t>(v);
    }
    if (mtf) {
        std::uint8_t order[256];
        for (int i{0}; i < 256; ++i) order[i] = static_cast<std::uint8_t>(i);
        for (std::size_t i{0}; i < n; ++i) {
            const int r{map[i]};
            const std::uint8_t v{order[r]};
            for (int k{r}; k > 0; --k) order[k] = order[k - 1];
            order[0] = v;
            map[i] = v;
        }
    }
    return map;
}

EntropyCode read_entropy_code(BitReader& br, std::size_t num_contexts) {
    if (br.bit()) fail("LZ77 is outside the subset");
    EntropyCode ec;
    ec.ctx_map = num_contexts > 1 ? read_context_map(br, num_contexts) : std::vector<std::uint8_t>(1, 0);
    const int clusters{*std::max_element(ec.ctx_map.begin(), ec.ctx_map.end()) + 1};
    if (!br.bit()) fail("ANS-coded histograms are outside the subset");
    for (int c{0}; c < clusters; ++c) ec.cfg.push_back(read_uint_config(br));
    std::vector<int> alphabet;
    for (int c{0}; c < clusters; ++c) alphabet.push_back(static_cast<int>(read_varlen_u16(br)) + 1);
    for (int c{0}; c < clusters; ++c) ec.codes.push_back(read_prefix_code(br, alphabet[static_cast<std::size_t>(c)]));
    return ec;
}

// ---- modular groups -----------------------------------------------------------

// Group header and a single-leaf tree; returns the leaf's predictor.
int read_modular_single_leaf(BitReader& br) {
    expect(br, 1, 0, "use_global_tree");
    expect(br, 1, 1, "wp_header.all_default");
    expect(br, 2, 0, "nb_transforms");
    const EntropyCode tree{read_entropy_code(br, 6)};
    if (tree.read(br, 1) != 0) fail("only single-leaf trees are in the subset");
    const std::uint32_t predictor{tree.read(br, 2)};
    if (unpack_signed(tree.read(br, 3)) != 0 || tree.read(br, 4) != 0 || tree.read(br, 5) != 0) {
        fail("leaf offset/multiplier outside the subset");
    }
    if (predictor != 0 && predictor != 5) fail("predictor outside the subset");
    return static_cast<int>(predictor);
}

struct Frame {
    int width{0}, height{0}, bw{0}, bh{0};
    std::uint32_t global_scale{0}, quant_dc{0};
    std::vector<std::int32_t> dc;      // [3][B] planes X, Y, B
    std::vector<std::int8_t> acs;      // [B] side at first blocks, 0 covered
    std::vector<std::int32_t> qf;      // [B] at first blocks
    std::vector<std::int8_t> ytox, ytob;  // [T]
    std::vector<std::int32_t> ac;      // [3][B*64] covered-block slots
    int tiles_x{0};
};

int phys_of(int token_channel) { return token_channel == 0 ? 1 : (token_channel == 1 ? 0 : 2); }

void read_dc_group(BitReader& br, Frame& f, int g) {
    const int xdg{(f.bw + kDcGroupBlocks - 1) / kDcGroupBlocks};
    const int bx0{(g % xdg) * kDcGroupBlocks};
    const int by0{(g / xdg) * kDcGroupBlocks};
    const int gw{std::min(kDcGroupBlocks, f.bw - bx0)};
    const int gh{std::min(kDcGroupBlocks, f.bh - by0)};
    const int n{gw * gh};
    const int nb{f.bw * f.bh};
    expect(br, 2, 0, "extra_precision");
    if (read_modular_single_leaf(br) != 5) fail("DC must use the Gradient predictor");
    const EntropyCode dcc{read_entropy_code(br, 1)};
    for (int tc{0}; tc < 3; ++tc) {
        std::int32_t* plane{f.dc.data() + static_cast<std::size_t>(phys_of(tc)) * nb};
        for (int y{0}; y < gh; ++y) {
            for (int x{0}; x < gw; ++x) {
                const std::size_t blk{static_cast<std::size_t>(by0 + y) * f.bw + bx0 + x};
                const bool hl{x > 0};
                const bool ht{y > 0};
                const std::int32_t w{hl ? plane[blk - 1] : 0};
                const std::int32_t nn{ht ? plane[blk - f.bw] : 0};
                const std::int32_t nw{(hl && ht) ? plane[blk - f.bw - 1] : 0};
                plane[blk] = gradient_predict(hl, ht, w, nn, nw) + unpack_signed(dcc.read(br, 0));
            }
        }
    }
    const int count{static_cast<int>(br.read(ceil_log2(static_cast<std::uint32_t>(n)))) + 1};
    if (read_modular_single_leaf(br) != 0) fail("AcMetadata must use the Zero predictor");
    const EntropyCode am{read_entropy_code(br, 1)};
    const int cw{(gw + 7) / 8};
    const int ch{(gh + 7) / 8};
    for (int k{0}; k < 2; ++k) {
        std::vector<std::int8_t>& map{k == 0 ? f.ytox : f.ytob};
        for (int t{0}; t < cw * ch; ++t) {
            const std::int32_t v{unpack_signed(am.read(br, 0))};
            if (v < -128 || v > 127) fail("CfL map value out of range");
            map[static_cast<std::size_t>(bx0 / 8 + by0 / 8 * f.tiles_x + (t / cw) * f.tiles_x + t % cw)] =
                static_cast<std::int8_t>(v);
        }
    }
    std::vector<std::int32_t> strategy(static_cast<std::size_t>(count));
    std::vector<std::int32_t> qfm1(static_cast<std::size_t>(count));
    for (int i{0}; i < count; ++i) strategy[static_cast<std::size_t>(i)] = unpack_signed(am.read(br, 0));
    for (int i{0}; i < count; ++i) qfm1[static_cast<std::size_t>(i)] = unpack_signed(am.read(br, 0));
    for (int i{0}; i < n; ++i) {
        if (unpack_signed(am.read(br, 0)) != 0) fail("non-zero EPF sharpness is outside the subset");
    }
    // Place the strategies: raster order over the group, each listed
    // transform at the next position no earlier transform covers.
    std::vector<std::uint8_t> covered(static_cast<std::size_t>(n), 0);
    int next{0};
    for (int y{0}; y < gh; ++y) {
        for (int x{0}; x < gw; ++x) {
            if (covered[static_cast<std::size_t>(y * gw + x)]) continue;
            if (next >= count) fail("fewer strategies than uncovered blocks");
            const std::int32_t raw{strategy[static_cast<std::size_t>(next)]};
            const int side{raw == 0 ? 8 : (raw == 4 ? 16 : (raw == 5 ? 32 : 0))};
            if (side == 0) fail("transform outside the subset (only DCT8, DCT16, DCT32)");
            const int s{side / 8};
            if (x + s > gw || y + s > gh) fail("transform crosses the group");
            for (int dy{0}; dy < s; ++dy) {
                for (int dx{0}; dx < s; ++dx) {
                    if (covered[static_cast<std::size_t>((y + dy) * gw + x + dx)]) fail("overlapping transforms");
                    covered[static_cast<std::size_t>((y + dy) * gw + x + dx)] = 1;
                    f.acs[static_cast<std::size_t>(by0 + y + dy) * f.bw + bx0 + x + dx] = 0;
                }
            }
            const std::size_t blk{static_cast<std::size_t>(by0 + y) * f.bw + bx0 + x};
            f.acs[blk] = static_cast<std::int8_t>(side);
            f.qf[blk] = qfm1[static_cast<std::size_t>(next)] + 1;
            ++next;
        }
    }
    if (next != count) fail("more strategies than transforms");
}

void read_ac_group(BitReader& br, Frame& f, int g, const EntropyCode& ac, const std::vector<std::uint16_t>& order) {
    const int xg{(f.bw + kAcGroupBlocks - 1) / kAcGroupBlocks};
    const int bx0{(g % xg) * kAcGroupBlocks};
    const int by0{(g / xg) * kAcGroupBlocks};
    const int gw{std::min(kAcGroupBlocks, f.bw - bx0)};
    const int gh{std::min(kAcGroupBlocks, f.bh - by0)};
    const std::size_t nb{static_cast<std::size_t>(f.bw) * f.bh};
    // Normalised non-zero counts over the group, per channel.
    std::vector<std::uint32_t> nzn(static_cast<std::size_t>(3 * gw * gh), 0);
    for (int y{0}; y < gh; ++y) {
        for (int x{0}; x < gw; ++x) {
            const std::size_t blk{static_cast<std::size_t>(by0 + y) * f.bw + bx0 + x};
            const int n{f.acs[blk]};
            if (n == 0) continue;
            const int side{n / 8};
            const std::uint32_t covered{static_cast<std::uint32_t>(side * side)};
            const std::uint32_t size{static_cast<std::uint32_t>(n * n)};
            const std::uint32_t l2{n == 16 ? 2u : (n == 32 ? 4u : 0u)};
            const std::uint16_t* ord{order.data() + (n == 8 ? 0 : (n == 16 ? 64 : 320))};
            for (int tc{0}; tc < 3; ++tc) {
                const int c{phys_of(tc)};
                std::uint32_t* nz_c{nzn.data() + static_cast<std::size_t>(c) * gw * gh};
                const bool hl{x > 0};
                const bool ht{y > 0};
                const std::uint32_t top{ht ? nz_c[(y - 1) * gw + x] : 0u};
                const std::uint32_t left{hl ? nz_c[y * gw + x - 1] : 0u};
                const int bctx{block_ctx(c, n)};
                const std::uint32_t nz{ac.read(br, nonzero_context(predict_nonzeros(hl, ht, top, left), bctx))};
                if (nz > size - covered) fail("non-zero count above the transform's AC size");
                const std::uint32_t norm{(nz + covered - 1) >> l2};
                for (int dy{0}; dy < side; ++dy) {
                    for (int dx{0}; dx < side; ++dx) nz_c[(y + dy) * gw + x + dx] = norm;
                }
                std::int32_t* plane{f.ac.data() + static_cast<std::size_t>(c) * nb * kCoeffsPerBlock};
                std::uint32_t remaining{nz};
                std::uint32_t prev{nz > size / 16 ? 0u : 1u};
                for (std::uint32_t k{covered}; k < size && remaining > 0; ++k) {
                    const std::uint32_t ctx{coeff_context(bctx, remaining, k, covered, l2, prev)};
                    const std::int32_t v{unpack_signed(ac.read(br, ctx))};
                    plane[covered_slot(n, static_cast<std::size_t>(bx0 + x), static_cast<std::size_t>(by0 + y),
                                       static_cast<std::size_t>(f.bw), ord[k])] = v;
                    prev = v != 0 ? 1u : 0u;
                    remaining -= prev;
                }
                if (remaining != 0) fail("non-zero count not reached");
            }
        }
    }
}

// Natural coefficient orders 8 | 16 | 32 (the decoder's default order).
std::vector<std::uint16_t> natural_orders() {
    std::vector<std::uint16_t> all;
    for (int n : {8, 16, 32}) {
        const int cx{n / 8};
        std::vector<std::uint16_t> out(static_cast<std::size_t>(n) * n);
        int cur{cx * cx};
        for (int i{0}; i < n; ++i) {
            for (int j{0}; j <= i; ++j) {
                int x{j};
                int y{i - j};
                if (i & 1) std::swap(x, y);
                const int val{(x < cx && y < cx) ? y * cx + x : cur++};
                out[static_cast<std::size_t>(val)] = static_cast<std::uint16_t>(y * n + x);
            }
        }
        for (int ip{n - 1}; ip > 0; --ip) {
            const int i{ip - 1};
            for (int j{0}; j <= i; ++j) {
                int x{n - 1 - (i - j)};
                int y{n - 1 - j};
                if (i & 1) std::swap(x, y);
                out[static_cast<std::size_t>(cur++)] = static_cast<std::uint16_t>(y * n + x);
            }
        }
        all.insert(all.end(), out.begin(), out.end());
    }
    return all;
}

// ---- codestream -----------------------------------------------------------------

std::vector<std::uint8_t> codestream_of(const std::uint8_t* data, std::size_t size) {
    if (size >= 2 && data[0] == 0xFF && data[1] == 0x0A) return std::vector<std::uint8_t>(data, data + size);
    static const std::uint8_t kSig[12]{0, 0, 0, 0x0c, 'J', 'X', 'L', ' ', 0x0d, 0x0a, 0x87, 0x0a};
    if (size < 12 || std::memcmp(data, kSig, 12) != 0) fail("not a JPEG XL file");
    std::size_t at{12};
    while (at + 8 <= size) {
        std::uint64_t box{0};
        for (int i{0}; i < 4; ++i) box = (box << 8) | data[at + static_cast<std::size_t>(i)];
        const bool jxlc{std::memcmp(data + at + 4, "jxlc", 4) == 0};
        std::size_t head{8};
        if (box == 1) {
            if (at + 16 > size) fail("truncated box");
            box = 0;
            for (int i{0}; i < 8; ++i) box = (box << 8) | data[at + 8 + static_cast<std::size_t>(i)];
            head = 16;
        } else if (box == 0) {
            box = size - at;
        }
        if (box < head || at + box > size) fail("box size out of range");
        if (jxlc) return std::vector<std::uint8_t>(data + at + head, data + at + box);
        at += box;
    }
    fail("no jxlc box");
}

void read_headers(BitReader& br, Frame& f) {
    expect(br, 8, 0xFF, "signature");
    expect(br, 8, 0x0A, "signature");
    const U32Dist dim[4]{{false, 1, 9}, {false, 1, 13}, {false, 1, 18}, {false, 1, 30}};
    const bool small{br.bit() != 0};
    f.height = small ? static_cast<int>(br.read(5) + 1) * 8 : static_cast<int>(read_u32(br, dim));
    expect(br, 3, 0, "ratio");
    f.width = small ? static_cast<int>(br.read(5) + 1) * 8 : static_cast<int>(read_u32(br, dim));
    expect(br, 1, 1, "ImageMetadata.all_default");
    expect(br, 1, 1, "CustomTransformData.all_default");
    br.align();
    if (f.width % 8 || f.height % 8) fail("frame sizes must be multiples of 8");
    expect(br, 1, 0, "FrameHeader.all_default");
    expect(br, 2, 0, "frame_type");
    expect(br, 1, 0, "encoding (VarDCT)");
    expect(br, 2, 0, "flags");
    expect(br, 2, 0, "upsampling");
    expect(br, 3, 2, "x_qm_scale");
    expect(br, 3, 2, "b_qm_scale");
    expect(br, 2, 0, "num_passes");
    expect(br, 1, 0, "custom_size_or_origin");
    expect(br, 2, 0, "blending mode");
    expect(br, 1, 1, "is_last");
    expect(br, 2, 0, "name length");
    expect(br, 1, 1, "RestorationFilter.all_default");
    expect(br, 2, 0, "extensions");
}

}  // namespace

// Parses every section of `data` into the frame's quantised planes.
void parse_frame(const std::uint8_t* data, std::size_t size, Frame& f) {
    const std::vector<std::uint8_t> cs{codestream_of(data, size)};
    BitReader br{cs.data(), cs.size()};
    read_headers(br, f);
    f.bw = f.width / 8;
    f.bh = f.height / 8;
    const int nb{f.bw * f.bh};
    const int xg{(f.bw + kAcGroupBlocks - 1) / kAcGroupBlocks};
    const int nac{xg * ((f.bh + kAcGroupBlocks - 1) / kAcGroupBlocks)};
    const int xdg{(f.bw + kDcGroupBlocks - 1) / kDcGroupBlocks};
    const int ndc{xdg * ((f.bh + kDcGroupBlocks - 1) / kDcGroupBlocks)};
    f.tiles_x = (f.bw + 7) / 8;
    const int tiles{f.tiles_x * ((f.bh + 7) / 8)};
    f.dc.assign(static_cast<std::size_t>(3) * nb, 0);
    f.acs.assign(static_cast<std::size_t>(nb), -1);
    f.qf.assign(static_cast<std::size_t>(nb), 0);
    f.ytox.assign(static_cast<std::size_t>(tiles), 0);
    f.ytob.assign(static_cast<std::size_t>(tiles), 0);
    f.ac.assign(static_cast<std::size_t>(3) * nb * kCoeffsPerBlock, 0);

    // TOC: DcGlobal, the DC groups, AcGlobal, the AC groups; with one AC
    // group a single entry for all four, read as one bit stream.
    expect(br, 1, 0, "TOC permutation");
    br.align();
    const U32Dist toc_dist[4]{{false, 0, 10}, {false, 1024, 14}, {false, 17408, 22}, {false, 4211712, 30}};
    const bool single{nac == 1};
    const int nsec{single ? 1 : 2 + ndc + nac};
    std::vector<std::size_t> sec_size(static_cast<std::size_t>(nsec));
    for (int s{0}; s < nsec; ++s) sec_size[static_cast<std::size_t>(s)] = read_u32(br, toc_dist);
    br.align();
    std::size_t at{br.byte_pos()};
    std::vector<std::size_t> sec_at(static_cast<std::size_t>(nsec));
    for (int s{0}; s < nsec; ++s) {
        sec_at[static_cast<std::size_t>(s)] = at;
        at += sec_size[static_cast<std::size_t>(s)];
    }
    if (at != cs.size()) fail("TOC does not cover the codestream exactly");
    auto section = [&](int s) {
        return BitReader{cs.data() + sec_at[static_cast<std::size_t>(s)], sec_size[static_cast<std::size_t>(s)]};
    };
    BitReader whole{section(0)};
    // The reader of logical section s: its own TOC section, or the combined one.
    auto part = [&](int s, BitReader& own) -> BitReader& {
        if (single) return whole;
        own = section(s);
        return own;
    };
    auto finish = [&](const BitReader& r, int s) {
        if (single) return;
        if (r.byte_pos() != sec_size[static_cast<std::size_t>(s)]) {
            fail("section " + std::to_string(s) + " ends at byte " + std::to_string(r.byte_pos()) + " of " +
                 std::to_string(sec_size[static_cast<std::size_t>(s)]));
        }
    };

    {  // DcGlobal
        BitReader own{whole};
        BitReader& r{part(0, own)};
        expect(r, 1, 1, "LF dequantisation all_default");
        const U32Dist gs[4]{{false, 1, 11}, {false, 2049, 11}, {false, 4097, 12}, {false, 8193, 16}};
        const U32Dist qdc[4]{{true, 16, 0}, {false, 1, 5}, {false, 1, 8}, {false, 1, 16}};
        f.global_scale = read_u32(r, gs);
        f.quant_dc = read_u32(r, qdc);
        expect(r, 1, 1, "block context map is_default");
        expect(r, 1, 1, "colour correlation all_default");
        expect(r, 1, 0, "global modular tree");
        finish(r, 0);
    }
    for (int g{0}; g < ndc; ++g) {
        BitReader own{whole};
        BitReader& r{part(1 + g, own)};
        read_dc_group(r, f, g);
        finish(r, 1 + g);
    }
    for (int b{0}; b < nb; ++b) {
        if (f.acs[static_cast<std::size_t>(b)] < 0) fail("block without a transform");
    }
    const std::vector<std::uint16_t> order{natural_orders()};
    EntropyCode ac;
    {  // AcGlobal
        BitReader own{whole};
        BitReader& r{part(1 + ndc, own)};
        expect(r, 1, 1, "dequantisation matrices all_default");
        expect(r, ceil_log2(static_cast<std::uint32_t>(nac)), 0, "num_histograms - 1");
        const U32Dist used[4]{{true, 0x5F, 0}, {true, 0x13, 0}, {true, 0, 0}, {false, 0, 13}};
        if (read_u32(r, used) != 0) fail("custom coefficient orders are outside the subset");
        ac = read_entropy_code(r, static_cast<std::size_t>(kNumAcContexts));
        finish(r, 1 + ndc);
    }
    for (int g{0}; g < nac; ++g) {
        BitReader own{whole};
        BitReader& r{part(2 + ndc + g, own)};
        read_ac_group(r, f, g, ac, order);
        finish(r, 2 + ndc + g);
    }
    if (single && whole.byte_pos() != sec_size[0]) {
        fail("combined section ends at byte " + std::to_string(whole.byte_pos()) + " of " +
             std::to_string(sec_size[0]));
    }
}

// Reconstructs the image of a parsed frame as XYB planes and sRGB planes in
// [0, 1].
void reconstruct(const Frame& f, std::vector<float>* xyb, std::vector<float>* srgb) {
    const int nb{f.bw * f.bh};
    const int W{f.width};
    const int H{f.height};
    const double gsf{static_cast<double>(f.global_scale) / 65536.0};
    const double dc_scale{gsf * f.quant_dc};
    const double dcq[3]{4096.0 * dc_scale, 512.0 * dc_scale, 256.0 * dc_scale};
    xyb->assign(static_cast<std::size_t>(3) * W * H, 0.0f);
    const double s16[2]{1.0, 0.901764195028874394};
    const double s32[4]{1.0, 0.974886821136879522, 0.901764195028874394, 0.787054918159101335};
    for (int by{0}; by < f.bh; ++by) {
        for (int bx{0}; bx < f.bw; ++bx) {
            const std::size_t blk{static_cast<std::size_t>(by) * f.bw + bx};
            const int n{f.acs[blk]};
            if (n == 0) continue;
            const int m{n / 8};
            const std::size_t tile{static_cast<std::size_t>(by / 8) * f.tiles_x + bx / 8};
            const double ytox{f.ytox[tile] / 84.0};
            const double ytob{f.ytob[tile] / 84.0 + 1.0};
            const double qgsf{f.qf[blk] * gsf};
            const int si{n == 8 ? 0 : (n == 16 ? 1 : 2)};
            std::vector<double> coef(static_cast<std::size_t>(3) * n * n, 0.0);
            for (int raw{0}; raw < n * n; ++raw) {
                const int fx{raw / n};
                const int fy{raw % n};
                if (fx < m && fy < m) continue;
                const std::size_t slot{covered_slot(n, static_cast<std::size_t>(bx), static_cast<std::size_t>(by),
                                                    static_cast<std::size_t>(f.bw), raw)};
                double v[3];
                for (int c{0}; c < 3; ++c) {
                    const std::uint32_t* wbits{si == 0 ? kDequantBits8[c] : (si == 1 ? kDequantBits16[c] : kDequantBits32[c])};
                    float w;
                    std::memcpy(&w, &wbits[raw], 4);
                    v[c] = f.ac[static_cast<std::size_t>(c) * nb * kCoeffsPerBlock + slot] * static_cast<double>(w) / qgsf;
                }
                coef[static_cast<std::size_t>(raw)] = v[0] + ytox * v[1];
                coef[static_cast<std::size_t>(n * n + raw)] = v[1];
                coef[static_cast<std::size_t>(2 * n * n + raw)] = v[2] + ytob * v[1];
            }
            // LLF corner from the DC of the covered 8x8 positions.
            for (int oy{0}; oy < m; ++oy) {
                for (int ox{0}; ox < m; ++ox) {
                    const std::size_t b2{static_cast<std::size_t>(by + oy) * f.bw + bx + ox};
                    const double y{f.dc[nb + b2] / dcq[1]};
                    const double dcv[3]{f.dc[b2] / dcq[0], y, f.dc[2 * static_cast<std::size_t>(nb) + b2] / dcq[2] + y};
                    for (int fx{0}; fx < m; ++fx) {
                        for (int fy{0}; fy < m; ++fy) {
                            if (m == 1) {
                                for (int c{0}; c < 3; ++c) coef[static_cast<std::size_t>(c * n * n)] = dcv[c];
                                continue;
                            }
                            const double on_x{(fx == 0 ? std::sqrt(1.0 / m) : std::sqrt(2.0 / m)) *
                                              std::cos(M_PI * (ox + 0.5) * fx / m)};
                            const double on_y{(fy == 0 ? std::sqrt(1.0 / m) : std::sqrt(2.0 / m)) *
                                              std::cos(M_PI * (oy + 0.5) * fy / m)};
                            const double* sc{m == 2 ? s16 : s32};
                            const double k{on_x * on_y / (m * sc[fx] * sc[fy])};
                            for (int c{0}; c < 3; ++c) coef[static_cast<std::size_t>(c * n * n + fx * n + fy)] += k * dcv[c];
                        }
                    }
                }
            }
            // Inverse DCT: p[y][x] = N sum O[fx][x] O[fy][y] c[fx][fy] (orthonormal O).
            std::vector<double> basis(static_cast<std::size_t>(n) * n);
            for (int k{0}; k < n; ++k) {
                for (int t{0}; t < n; ++t) {
                    basis[static_cast<std::size_t>(k * n + t)] =
                        (k == 0 ? std::sqrt(1.0 / n) : std::sqrt(2.0 / n)) * std::cos(M_PI * (t + 0.5) * k / n);
                }
            }
            std::vector<double> tmp(static_cast<std::size_t>(n) * n);
            for (int c{0}; c < 3; ++c) {
                const double* cc{coef.data() + static_cast<std::size_t>(c) * n * n};
                for (int fx{0}; fx < n; ++fx) {       // tmp[fx][y] = sum_fy O[fy][y] c[fx][fy]
                    for (int y{0}; y < n; ++y) {
                        double s{0.0};
                        for (int fy{0}; fy < n; ++fy) s += basis[static_cast<std::size_t>(fy * n + y)] * cc[fx * n + fy];
                        tmp[static_cast<std::size_t>(fx * n + y)] = s;
                    }
                }
                for (int y{0}; y < n; ++y) {
                    for (int x{0}; x < n; ++x) {
                        double s{0.0};
                        for (int fx{0}; fx < n; ++fx) s += basis[static_cast<std::size_t>(fx * n + x)] * tmp[static_cast<std::size_t>(fx * n + y)];
                        const int px{bx * 8 + x};
                        const int py{by * 8 + y};
                        (*xyb)[(static_cast<std::size_t>(c) * H + py) * W + px] = static_cast<float>(n * s);
                    }
                }
            }
        }
    }
    // Decoder gaborish: 3x3 smoothing with the format's default weights,
    // edges clamped.
    {
        const double w1{0.115169525};
        const double w2{0.061248592};
        const double norm{1.0 / (1.0 + 4.0 * w1 + 4.0 * w2)};
        std::vector<float> out(xyb->size());
        for (int c{0}; c < 3; ++c) {
            const float* p{xyb->data() + static_cast<std::size_t>(c) * W * H};
            auto at2 = [&](int x, int y) {
                x = std::min(std::max(x, 0), W - 1);
                y = std::min(std::max(y, 0), H - 1);
                return static_cast<double>(p[static_cast<std::size_t>(y) * W + x]);
            };
            for (int y{0}; y < H; ++y) {
                for (int x{0}; x < W; ++x) {
                    const double e{at2(x - 1, y) + at2(x + 1, y) + at2(x, y - 1) + at2(x, y + 1)};
                    const double d{at2(x - 1, y - 1) + at2(x + 1, y - 1) + at2(x - 1, y + 1) + at2(x + 1, y + 1)};
                    out[(static_cast<std::size_t>(c) * H + y) * W + x] = static_cast<float>((at2(x, y) + w1 * e + w2 * d) * norm);
                }
            }
        }
        xyb->swap(out);
    }
    // XYB -> linear RGB -> sRGB.
    const double m[9]{kM00, kM01, kM02, kM10, kM11, kM12, kM20, kM21, kM22};
    const double det{m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) + m[2] * (m[3] * m[7] - m[4] * m[6])};
    const double inv[9]{(m[4] * m[8] - m[5] * m[7]) / det, (m[2] * m[7] - m[1] * m[8]) / det, (m[1] * m[5] - m[2] * m[4]) / det,
                        (m[5] * m[6] - m[3] * m[8]) / det, (m[0] * m[8] - m[2] * m[6]) / det, (m[2] * m[3] - m[0] * m[5]) / det,
                        (m[3] * m[7] - m[4] * m[6]) / det, (m[1] * m[6] - m[0] * m[7]) / det, (m[0] * m[4] - m[1] * m[3]) / det};
    srgb->assign(static_cast<std::size_t>(3) * W * H, 0.0f);
    const std::size_t P{static_cast<std::size_t>(W) * H};
    for (std::size_t i{0}; i < P; ++i) {
        const double X{(*xyb)[i]};
        const double Y{(*xyb)[P + i]};
        const double B{(*xyb)[2 * P + i]};
        double mix[3]{Y + X, Y - X, B};
        for (double& v : mix) {
            const double t{v - static_cast<double>(kNegCbrtBias)};
            v = t * t * t - static_cast<double>(kOpsinBias);
        }
        for (int c{0}; c < 3; ++c) {
            double lin{inv[3 * c] * mix[0] + inv[3 * c + 1] * mix[1] + inv[3 * c + 2] * mix[2]};
            lin = std::min(std::max(lin, 0.0), 1.0);
            const double e{lin <= 0.0031308 ? 12.92 * lin : 1.055 * std::pow(lin, 1.0 / 2.4) - 0.055};
            (*srgb)[static_cast<std::size_t>(c) * P + i] = static_cast<float>(e);
        }
    }
}

}  // namespace jxb

extern "C" {

int jxlsubset_decode_planes(const uint8_t* data, size_t size, uint32_t* width, uint32_t* height, int16_t* ac,
                            int32_t* dc, int8_t* acs, int32_t* qf, int8_t* ytox, int8_t* ytob,
                            uint32_t* global_scale, uint32_t* quant_dc, size_t capacity_blocks, char* error,
                            size_t error_size) {
    try {
        jxb::Frame f;
        jxb::parse_frame(data, size, f);
        *width = static_cast<uint32_t>(f.width);
        *height = static_cast<uint32_t>(f.height);
        *global_scale = f.global_scale;
        *quant_dc = f.quant_dc;
        const std::size_t nb{static_cast<std::size_t>(f.bw) * f.bh};
        if (nb > capacity_blocks) return 2;
        if (ac != nullptr) {
            for (std::size_t i{0}; i < f.ac.size(); ++i) ac[i] = static_cast<int16_t>(f.ac[i]);
        }
        if (dc != nullptr) std::memcpy(dc, f.dc.data(), f.dc.size() * sizeof(int32_t));
        if (acs != nullptr) std::memcpy(acs, f.acs.data(), f.acs.size());
        if (qf != nullptr) {
            for (std::size_t i{0}; i < nb; ++i) qf[i] = f.acs[i] != 0 ? f.qf[i] : 0;
        }
        if (ytox != nullptr) std::memcpy(ytox, f.ytox.data(), f.ytox.size());
        if (ytob != nullptr) std::memcpy(ytob, f.ytob.data(), f.ytob.size());
        return 0;
    } catch (const jxb::DecodeError& e) {
        if (error != nullptr && error_size > 0) std::snprintf(error, error_size, "%s", e.what.c_str());
        return 1;
    } catch (const std::exception& e) {
        if (error != nullptr && error_size > 0) std::snprintf(error, error_size, "%s", e.what());
        return 1;
    }
}

int jxlsubset_decode(const uint8_t* data, size_t size, uint32_t* width, uint32_t* height, float* xyb, float* srgb,
                     size_t capacity_pixels, char* error, size_t error_size) {
    try {
        jxb::Frame f;
        jxb::parse_frame(data, size, f);
        *width = static_cast<uint32_t>(f.width);
        *height = static_cast<uint32_t>(f.height);
        const std::size_t p{static_cast<std::size_t>(f.width) * f.height};
        if (p > capacity_pixels) return 2;
        std::vector<float> x;
        std::vector<float> s;
        jxb::reconstruct(f, &x, &s);
        if (xyb != nullptr) std::memcpy(xyb, x.data(), 3 * p * sizeof(float));
        if (srgb != nullptr) std::memcpy(srgb, s.data(), 3 * p * sizeof(float));
        return 0;
    } catch (const jxb::DecodeError& e) {
        if (error != nullptr && error_size > 0) std::snprintf(error, error_size, "%s", e.what.c_str());
        return 1;
    } catch (const std::exception& e) {
        if (error != nullptr && error_size > 0) std::snprintf(error, error_size, "%s", e.what());
        return 1;
    }
}

}  // extern "C"
