// Length-limited canonical prefix codes and their JPEG XL header, usable from
// host and device code.
//
// Bit-exact with the reference's libjxl-derived builder
// (src/bitstream/prefix_code.cc:36-426): leaves are taken in descending
// symbol order, stably sorted by count (so equal counts keep descending symbol
// order), merged with the two-queue method, and the whole construction is
// retried with the count floor doubled until no depth exceeds the limit.
// Codes are canonical and stored bit-reversed for the LSB-first writer. The
// header is the simple form for at most four used symbols and otherwise the
// code-length-code form, in which every depth is sent as its own symbol (the
// reference never emits run-length codes for these alphabets).
#pragma once

#include <cstdint>

#include "jxl_constants.cuh"

namespace jxb {

// LSB-first bit sink over a zero-initialised byte buffer. Writes past `cap`
// bits are dropped and flagged.
struct BitSink {
    std::uint8_t* buf;
    std::uint32_t pos;
    std::uint32_t cap;
    bool overflow;

    JX_HD void put(std::uint32_t n, std::uint32_t v) {
        if (n == 0) return;
        if (pos + n > cap) {
            overflow = true;
            pos += n;
            return;
        }
        if (n < 32) v &= (1u << n) - 1u;
        while (n > 0) {
            const std::uint32_t off{pos & 7u};
            const std::uint32_t take{n < 8u - off ? n : 8u - off};
            buf[pos >> 3] = static_cast<std::uint8_t>(buf[pos >> 3] | ((v & ((1u << take) - 1u)) << off));
            v >>= take;
            n -= take;
            pos += take;
        }
    }

    // Appends `nbits` bits from an LSB-first byte buffer.
    JX_HD void put_bits(const std::uint8_t* src, std::uint32_t nbits) {
        std::uint32_t i{0};
        for (; i + 8 <= nbits; i += 8) put(8, src[i >> 3]);
        if (i < nbits) put(nbits - i, src[i >> 3]);
    }
};

struct HuffNode {
    std::uint32_t count;
    std::int16_t left;
    std::int16_t right_or_value;
};

JX_HD unsigned ceil_log2_u(std::uint32_t x) {
    unsigned b{0};
    if (x <= 1) return 0;
    for (std::uint32_t v{x - 1}; v != 0; v >>= 1) ++b;
    return b;
}

// Depths from a finished node pool: children always precede their parent,
// so one reverse pass from the root (index 2n-1) assigns every level.
JX_HD void depths_from_pool(const HuffNode* pool, int n, std::uint8_t* level, std::uint8_t* depth) {
    level[2 * n - 1] = 0;
    for (int p{2 * n - 1}; p > n; --p) {
        const HuffNode& nd{pool[p]};
        level[nd.left] = static_cast<std::uint8_t>(level[p] + 1);
        level[nd.right_or_value] = static_cast<std::uint8_t>(level[p] + 1);
    }
    for (int i{0}; i < n; ++i) depth[pool[i].right_or_value] = level[i];
}

// Two-queue merge over n sorted leaves in pool[0..n) (pool holds 2n+2 entries).
JX_HD void merge_pool(HuffNode* pool, int n) {
    const HuffNode sentinel{0xffffffffu, -1, -1};
    int size{n};
    pool[size++] = sentinel;
    pool[size++] = sentinel;
    int i{0};
    int j{n + 1};
    for (int k{n - 1}; k != 0; --k) {
        int left;
        int right;
        if (pool[i].count <= pool[j].count) { left = i; ++i; } else { left = j; ++j; }
        if (pool[i].count <= pool[j].count) { right = i; ++i; } else { right = j; ++j; }
        const int end{size - 1};
        pool[end].count = pool[left].count + pool[right].count;
        pool[end].left = static_cast<std::int16_t>(left);
        pool[end].right_or_value = static_cast<std::int16_t>(right);
        pool[size++] = sentinel;
    }
}

// Serial construction for small alphabets (insertion sort). `pool` holds at
// least 2*length+4 nodes and `level` at least 2*length+4 bytes.
JX_HD void create_tree_serial(const std::uint32_t* hist, int length, int limit, std::uint8_t* depth,
                              HuffNode* pool, std::uint8_t* level) {
    for (std::uint32_t floor{1};; floor *= 2) {
        int n{0};
        for (int s{length - 1}; s >= 0; --s) {
            if (hist[s] != 0) {
                const std::uint32_t c{hist[s] > floor - 1 ? hist[s] : floor - 1};
                pool[n].count = c;
                pool[n].left = -1;
                pool[n].right_or_value = static_cast<std::int16_t>(s);
                ++n;
            }
        }
        if (n == 1) {
            depth[pool[0].right_or_value] = 1;
            return;
        }
        for (int a{1}; a < n; ++a) {
            const HuffNode t{pool[a]};
            int b{a};
            while (b > 0 && pool[b - 1].count > t.count) {
                pool[b] = pool[b - 1];
                --b;
            }
            pool[b] = t;
        }
        merge_pool(pool, n);
        for (int s{0}; s < length; ++s) depth[s] = 0;
        depths_from_pool(pool, n, level, depth);
        int mx{0};
        for (int s{0}; s < length; ++s) mx = depth[s] > mx ? depth[s] : mx;
        if (mx <= limit) return;
    }
}

JX_HD std::uint16_t reverse_bits16(int nbits, std::uint32_t v) {
    std::uint32_t r{0};
    for (int i{0}; i < nbits; ++i) r |= ((v >> i) & 1u) << (nbits - 1 - i);
    return static_cast<std::uint16_t>(r);
}

JX_HD void canonical_codes(const std::uint8_t* depth, int len, std::uint16_t* bits) {
    std::uint32_t bl_count[16]{};
    std::uint32_t next_code[16]{};
    for (int i{0}; i < len; ++i) ++bl_count[depth[i]];
    bl_count[0] = 0;
    std::uint32_t code{0};
    for (int i{1}; i < 16; ++i) {
        code = (code + bl_count[i - 1]) << 1;
        next_code[i] = code;
    }
    for (int i{0}; i < len; ++i) {
        bits[i] = depth[i] ? reverse_bits16(depth[i], next_code[depth[i]]++) : 0;
    }
}

// Working arrays of the code-length code (kept in shared memory by the
// device builder, on the stack by host callers).
struct CodeLengthScratch {
    std::uint32_t hist[18];
    std::uint8_t cl_depth[18];
    std::uint16_t cl_bits[18];
    HuffNode pool[40];
    std::uint8_t level[40];
};

// Header of a code with more than four used symbols (code-length-code form).
JX_HD void store_complex(const std::uint8_t* depths, int num, BitSink& w, CodeLengthScratch& scr) {
    int new_len{num};
    while (new_len > 0 && depths[new_len - 1] == 0) --new_len;
    std::uint32_t* hist{scr.hist};
    for (int i{0}; i < 18; ++i) hist[i] = 0;
    for (int i{0}; i < new_len; ++i) ++hist[depths[i]];
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
    std::uint16_t* cl_bits{scr.cl_bits};
    for (int i{0}; i < 18; ++i) {
        cl_depth[i] = 0;
        cl_bits[i] = 0;
    }
    create_tree_serial(hist, 18, 5, cl_depth, scr.pool, scr.level);
    canonical_codes(cl_depth, 18, cl_bits);
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
    for (int i{0}; i < new_len; ++i) w.put(cl_depth[depths[i]], cl_bits[depths[i]]);
}

// Used-symbol census of a histogram: returns the number of non-zero entries
// (counting stops once it exceeds four) and the first four of them.
JX_HD int symbol_census(const std::uint32_t* hist, int length, int* s4) {
    int count{0};
    for (int i{0}; i < length; ++i) {
        if (hist[i]) {
            if (count < 4) {
                s4[count] = i;
            } else if (count > 4) {
                break;
            }
            ++count;
        }
    }
    return count;
}

JX_HD unsigned alphabet_bits(int length) {
    unsigned b{0};
    for (unsigned c{static_cast<unsigned>(length - 1)}; c; c >>= 1) ++b;
    return b;
}

// Header for a code whose depths are already built (count >= 2).
JX_HD void store_code_header(int count, int* s4, int length, const std::uint8_t* depth, BitSink& w,
                             CodeLengthScratch& scr) {
    const unsigned max_bits{alphabet_bits(length)};
    if (count <= 4) {
        w.put(2, 1);
        w.put(2, static_cast<std::uint32_t>(count - 1));
        for (int i{0}; i < count; ++i) {
            for (int j{i + 1}; j < count; ++j) {
                if (depth[s4[j]] < depth[s4[i]]) {
                    const int t{s4[j]};
                    s4[j] = s4[i];
                    s4[i] = t;
                }
            }
        }
        for (int i{0}; i < count; ++i) w.put(max_bits, static_cast<std::uint32_t>(s4[i]));
        if (count == 4) w.put(1, depth[s4[0]] == 1 ? 1 : 0);
    } else {
        store_complex(depth, length, w, scr);
    }
}

// Whole build_and_store for a small alphabet with the serial tree builder.
JX_HD void build_and_store_serial(const std::uint32_t* hist, int length, std::uint8_t* depth,
                                  std::uint16_t* bits, BitSink& w, HuffNode* pool, std::uint8_t* level) {
    for (int i{0}; i < length; ++i) {
        depth[i] = 0;
        bits[i] = 0;
    }
    int s4[4]{0, 0, 0, 0};
    const int count{symbol_census(hist, length, s4)};
    if (count <= 1) {
        w.put(4, 1);
        w.put(alphabet_bits(length), static_cast<std::uint32_t>(s4[0]));
        return;
    }
    create_tree_serial(hist, length, 15, depth, pool, level);
    canonical_codes(depth, length, bits);
    CodeLengthScratch scr;
    store_code_header(count, s4, length, depth, w, scr);
}

// Hybrid-uint configuration fields (src/bitstream/histogram_writer.cc:74-81),
// log_alpha_size 15.
JX_HD void put_uint_config(BitSink& w, std::uint32_t se, std::uint32_t msb, std::uint32_t lsb) {
    w.put(ceil_log2_u(16), se);
    if (se == 15) return;
    w.put(ceil_log2_u(se + 1), msb);
    w.put(ceil_log2_u(se - msb + 1), lsb);
}

JX_HD void put_var_len_u16(BitSink& w, std::uint32_t n) {
    if (n == 0) {
        w.put(1, 0);
        return;
    }
    w.put(1, 1);
    unsigned nb{0};
    for (std::uint32_t v{n}; v > 1; v >>= 1) ++nb;
    w.put(4, nb);
    w.put(nb, n - (1u << nb));
}

}  // namespace jxb
