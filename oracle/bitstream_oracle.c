/* CPU restatement of the reference encoder's entropy coding and frame
 * assembly (test infrastructure only: checker and CPU baseline).
 *
 * Restates, from the quantised planes to the .jxl file, m-pilia/cujpegxl's
 *   LSB-first bit writer ............ src/bitstream/bit_writer.h:17-60
 *   U32/U64 field coders ............ src/bitstream/field_coder.h:131-222
 *   hybrid uint (4,2,0) ............. src/bitstream/hybrid_uint.h:15-41
 *   length-limited Huffman + header . src/bitstream/prefix_code.cc:36-426
 *   context map (best form) ......... src/bitstream/context_map.cc:74-199
 *   histogram containers ............ src/bitstream/histogram_writer.cc:59-128
 *   AC tokens and contexts .......... src/entropy.cu:649-681, src/ac_context.h,
 *                                     tools/bitstream/vardct_frame.cc:262-351
 *   DcGroup / AcMetadata modular ... src/entropy.cu:227-341, tools/bitstream/modular.cc,
 *                                     src/bitstream/frame_assembly.cc:150-302
 *   DcGlobal, AcGlobal .............. src/bitstream/frame_assembly.cc:202-238
 *   headers, frame header, TOC ...... src/bitstream/codestream.cc:57-135
 *   ISOBMFF container ............... src/bitstream/container.cc:8-62
 *   section order / orchestration ... src/frame_encoder.cu:88-292
 * The per-block quant field enters the AcMetadata QF row as the production
 * device coder does (src/entropy.cu:270-271).
 */

#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

/* ---- bit writer ---- */

typedef struct {
    uint8_t* buf;
    size_t cap;
    size_t bits;
} BW;

static void bw_init(BW* w) { w->cap = 1024; w->buf = (uint8_t*)calloc(w->cap, 1); w->bits = 0; }
static void bw_free(BW* w) { free(w->buf); }
static void bw_put(BW* w, unsigned n, uint64_t v) {
    while ((w->bits + n + 7) / 8 + 8 > w->cap) {
        const size_t nc = w->cap * 2;
        w->buf = (uint8_t*)realloc(w->buf, nc);
        memset(w->buf + w->cap, 0, nc - w->cap);
        w->cap = nc;
    }
    for (unsigned i = 0; i < n; ++i) {
        if ((v >> i) & 1u) w->buf[(w->bits + i) >> 3] |= (uint8_t)(1u << ((w->bits + i) & 7));
    }
    w->bits += n;
}
static void bw_pad(BW* w) { w->bits = (w->bits + 7) & ~(size_t)7; bw_put(w, 0, 0); }
static size_t bw_bytes(const BW* w) { return (w->bits + 7) / 8; }
/* Appends another writer's bits. */
static void bw_append(BW* w, const BW* o) {
    for (size_t i = 0; i < o->bits; i += 8) {
        const unsigned n = o->bits - i < 8 ? (unsigned)(o->bits - i) : 8u;
        bw_put(w, n, o->buf[i >> 3] & ((1u << n) - 1u));
    }
}

/* ---- field coders ---- */

typedef struct { int direct; uint32_t v; uint32_t extra; } Distr;
#define VAL(x) {1, (x), 0}
#define BO(b, o) {0, (o), (b)}

static void write_u32(BW* w, const Distr d[4], uint32_t value) {
    uint32_t best = 0, best_bits = 64;
    for (uint32_t s = 0; s < 4; ++s) {
        if (d[s].direct) {
            if (d[s].v == value) { best = s; best_bits = 2; break; }
            continue;
        }
        if (value < d[s].v || (uint64_t)value >= (uint64_t)d[s].v + (1ull << d[s].extra)) continue;
        if (2 + d[s].extra < best_bits) { best = s; best_bits = 2 + d[s].extra; }
    }
    bw_put(w, 2, best);
    if (!d[best].direct) bw_put(w, d[best].extra, value - d[best].v);
}

static void write_u64_zero(BW* w) { bw_put(w, 2, 0); }

static unsigned ceil_log2(size_t x) {
    unsigned b = 0;
    if (x <= 1) return 0;
    for (size_t v = x - 1; v; v >>= 1) ++b;
    return b;
}

/* ---- hybrid uint ---- */

static void hybrid(uint32_t v, uint32_t se, uint32_t msb, uint32_t lsb, uint32_t* tok, uint32_t* nb,
                   uint32_t* bits) {
    const uint32_t split = 1u << se;
    if (v < split) { *tok = v; *nb = 0; *bits = 0; return; }
    uint32_t n = 31;
    while (!((v >> n) & 1u)) --n;
    const uint32_t m = v - (1u << n);
    *tok = split + ((n - se) << (msb + lsb)) + ((m >> (n - msb)) << lsb) + (m & ((1u << lsb) - 1u));
    *nb = n - msb - lsb;
    *bits = (v >> lsb) & ((1u << *nb) - 1u);
}

static uint32_t pack_signed(int32_t v) { return ((uint32_t)v << 1) ^ (uint32_t)(v >> 31); }

/* ---- Huffman ---- */

typedef struct { uint32_t count; int16_t left; int16_t right_or_value; } HNode;

static void set_depth(int p, const HNode* pool, uint8_t* depth, uint8_t level) {
    if (pool[p].left >= 0) {
        set_depth(pool[p].left, pool, depth, level + 1);
        set_depth(pool[p].right_or_value, pool, depth, level + 1);
    } else {
        depth[pool[p].right_or_value] = level;
    }
}

static void create_tree(const uint32_t* data, size_t length, int limit, uint8_t* depth) {
    HNode* tree = (HNode*)malloc(sizeof(HNode) * (2 * length + 4));
    for (uint32_t count_limit = 1;; count_limit *= 2) {
        size_t n = 0;
        for (size_t i = length; i != 0;) {
            --i;
            if (data[i]) {
                const uint32_t c = data[i] > count_limit - 1 ? data[i] : count_limit - 1;
                tree[n].count = c; tree[n].left = -1; tree[n].right_or_value = (int16_t)i; ++n;
            }
        }
        if (n == 1) { depth[tree[0].right_or_value] = 1; break; }
        /* stable insertion sort by count */
        for (size_t i = 1; i < n; ++i) {
            const HNode t = tree[i];
            size_t j = i;
            while (j > 0 && tree[j - 1].count > t.count) { tree[j] = tree[j - 1]; --j; }
            tree[j] = t;
        }
        const HNode sentinel = {0xffffffffu, -1, -1};
        size_t size = n;
        tree[size++] = sentinel;
        tree[size++] = sentinel;
        size_t i = 0, j = n + 1;
        for (size_t k = n - 1; k != 0; --k) {
            size_t left, right;
            if (tree[i].count <= tree[j].count) { left = i; ++i; } else { left = j; ++j; }
            if (tree[i].count <= tree[j].count) { right = i; ++i; } else { right = j; ++j; }
            const size_t end = size - 1;
            tree[end].count = tree[left].count + tree[right].count;
            tree[end].left = (int16_t)left;
            tree[end].right_or_value = (int16_t)right;
            tree[size++] = sentinel;
        }
        set_depth((int)(2 * n - 1), tree, depth, 0);
        uint8_t mx = 0;
        for (size_t s = 0; s < length; ++s) mx = depth[s] > mx ? depth[s] : mx;
        if (mx <= limit) break;
    }
    free(tree);
}

static uint16_t reverse_bits(int nbits, uint16_t bits) {
    uint16_t r = 0;
    for (int i = 0; i < nbits; ++i) r = (uint16_t)(r | (((bits >> i) & 1u) << (nbits - 1 - i)));
    return r;
}

static void depths_to_codes(const uint8_t* depth, size_t len, uint16_t* bits) {
    uint16_t bl_count[16] = {0}, next_code[16] = {0};
    for (size_t i = 0; i < len; ++i) ++bl_count[depth[i]];
    bl_count[0] = 0;
    int code = 0;
    for (int i = 1; i < 16; ++i) { code = (code + bl_count[i - 1]) << 1; next_code[i] = (uint16_t)code; }
    for (size_t i = 0; i < len; ++i)
        if (depth[i]) bits[i] = reverse_bits(depth[i], next_code[depth[i]]++);
}

static void store_complex(const uint8_t* depths, size_t num, BW* w) {
    size_t new_len = num;
    while (new_len > 0 && depths[new_len - 1] == 0) --new_len;
    /* every depth is emitted as its own code-length symbol (no run-length codes) */
    uint32_t hist[18] = {0};
    for (size_t i = 0; i < new_len; ++i) ++hist[depths[i]];
    int num_codes = 0, code = 0;
    for (int i = 0; i < 18; ++i)
        if (hist[i]) {
            if (num_codes == 0) { code = i; num_codes = 1; }
            else if (num_codes == 1) { num_codes = 2; break; }
        }
    uint8_t cl_depth[18] = {0};
    uint16_t cl_bits[18] = {0};
    create_tree(hist, 18, 5, cl_depth);
    depths_to_codes(cl_depth, 18, cl_bits);
    static const uint8_t kOrder[18] = {1, 2, 3, 4, 0, 5, 17, 6, 16, 7, 8, 9, 10, 11, 12, 13, 14, 15};
    static const uint8_t kSym[6] = {0, 7, 3, 2, 1, 15};
    static const uint8_t kLen[6] = {2, 4, 3, 2, 2, 4};
    size_t to_store = 18;
    if (num_codes > 1)
        for (; to_store > 0; --to_store)
            if (cl_depth[kOrder[to_store - 1]] != 0) break;
    unsigned skip = 0;
    if (cl_depth[kOrder[0]] == 0 && cl_depth[kOrder[1]] == 0) {
        skip = 2;
        if (cl_depth[kOrder[2]] == 0) skip = 3;
    }
    bw_put(w, 2, skip);
    for (size_t i = skip; i < to_store; ++i) {
        const unsigned l = cl_depth[kOrder[i]];
        bw_put(w, kLen[l], kSym[l]);
    }
    if (num_codes == 1) cl_depth[code] = 0;
    for (size_t i = 0; i < new_len; ++i) bw_put(w, cl_depth[depths[i]], cl_bits[depths[i]]);
}

static void build_and_store(const uint32_t* hist, size_t length, uint8_t* depth, uint16_t* bits, BW* w) {
    memset(depth, 0, length);
    memset(bits, 0, length * 2);
    size_t count = 0, s4[4] = {0, 0, 0, 0};
    for (size_t i = 0; i < length; ++i)
        if (hist[i]) {
            if (count < 4) s4[count] = i;
            else if (count > 4) break;
            ++count;
        }
    unsigned max_bits = 0;
    for (size_t c = length - 1; c; c >>= 1) ++max_bits;
    if (count <= 1) {
        bw_put(w, 4, 1);
        bw_put(w, max_bits, s4[0]);
        return;
    }
    create_tree(hist, length, 15, depth);
    depths_to_codes(depth, length, bits);
    if (count <= 4) {
        bw_put(w, 2, 1);
        bw_put(w, 2, count - 1);
        for (size_t i = 0; i < count; ++i)
            for (size_t j = i + 1; j < count; ++j)
                if (depth[s4[j]] < depth[s4[i]]) { const size_t t = s4[j]; s4[j] = s4[i]; s4[i] = t; }
        for (size_t i = 0; i < count; ++i) bw_put(w, max_bits, s4[i]);
        if (count == 4) bw_put(w, 1, depth[s4[0]] == 1 ? 1 : 0);
    } else {
        store_complex(depth, length, w);
    }
}

size_t oracle_huffman(const uint32_t* hist, size_t len, uint8_t* depth, uint16_t* bits, uint8_t* out,
                      size_t cap) {
    BW w;
    bw_init(&w);
    build_and_store(hist, len, depth, bits, &w);
    if (out) memcpy(out, w.buf, bw_bytes(&w) < cap ? bw_bytes(&w) : cap);
    const size_t n = w.bits;
    bw_free(&w);
    return n;
}

/* ---- histogram containers ---- */

static void uint_config(BW* w, uint32_t se, uint32_t msb, uint32_t lsb) {
    bw_put(w, ceil_log2(15 + 1), se);
    if (se == 15) return;
    bw_put(w, ceil_log2(se + 1), msb);
    bw_put(w, ceil_log2(se - msb + 1), lsb);
}

static void var_len_u16(BW* w, size_t n) {
    if (n == 0) { bw_put(w, 1, 0); return; }
    bw_put(w, 1, 1);
    unsigned nb = 0;
    for (size_t v = n; v > 1; v >>= 1) ++nb;
    bw_put(w, 4, nb);
    bw_put(w, nb, n - ((size_t)1 << nb));
}

/* One prefix-coded histogram for `num_contexts` contexts (all clustered). */
static void prefix_histograms(BW* w, const uint32_t* hist, size_t length, size_t num_contexts,
                              uint32_t se, uint32_t msb, uint32_t lsb, uint8_t* depth, uint16_t* bits) {
    bw_put(w, 1, 0);
    if (num_contexts > 1) { bw_put(w, 1, 1); bw_put(w, 2, 0); }
    bw_put(w, 1, 1);
    uint_config(w, se, msb, lsb);
    var_len_u16(w, length - 1);
    memset(depth, 0, length);
    memset(bits, 0, length * 2);
    if (length > 1) build_and_store(hist, length, depth, bits, w);
}

static int ac_cluster_of(uint32_t ctx) {
    const uint32_t count = 15 * 37;
    if (ctx < count) {
        const uint32_t bucket = ctx / 15;
        const int group = (int)(ctx % 15) < 7 ? 0 : 1;
        const int band = bucket < 4 ? 0 : (bucket < 12 ? 1 : (bucket < 24 ? 2 : 3));
        return group * 4 + band;
    }
    const uint32_t rel = ctx - count;
    const int group = (int)(rel / 458) < 7 ? 0 : 1;
    const uint32_t z = rel % 458;
    static const uint16_t kEdges[11] = {32, 64, 96, 128, 160, 200, 240, 280, 328, 376, 424};
    int band = 11;
    for (int i = 0; i < 11; ++i) if (z < kEdges[i]) { band = i; break; }
    return 8 + group * 12 + band;
}

static void context_map_complex(BW* w, const uint8_t* map, size_t n, int mtf) {
    uint32_t hist[16] = {0};
    uint8_t* sym = (uint8_t*)malloc(n);
    uint8_t order[256];
    for (int i = 0; i < 256; ++i) order[i] = (uint8_t)i;
    for (size_t i = 0; i < n; ++i) {
        if (!mtf) { sym[i] = map[i]; continue; }
        size_t r = 0;
        while (order[r] != map[i]) ++r;
        sym[i] = (uint8_t)r;
        const uint8_t v = order[r];
        for (; r > 0; --r) order[r] = order[r - 1];
        order[0] = v;
    }
    for (size_t i = 0; i < n; ++i) {
        uint32_t t, nb, b;
        hybrid(sym[i], 2, 0, 1, &t, &nb, &b);
        ++hist[t];
    }
    size_t alpha = 1;
    for (size_t i = 0; i < 16; ++i) if (hist[i]) alpha = i + 1;
    bw_put(w, 1, 0);
    bw_put(w, 1, mtf ? 1 : 0);
    uint8_t depth[16];
    uint16_t bits[16];
    prefix_histograms(w, hist, alpha, 1, 2, 0, 1, depth, bits);
    for (size_t i = 0; i < n; ++i) {
        uint32_t t, nb, b;
        hybrid(sym[i], 2, 0, 1, &t, &nb, &b);
        bw_put(w, depth[t], bits[t]);
        if (nb) bw_put(w, nb, b);
    }
    free(sym);
}

/* AcGlobal context map for the fixed 7425 -> 32 clustering (more than 8
 * clusters, so the simple form is never eligible). */
static void ac_context_map(BW* w) {
    static uint8_t map[7425];
    for (uint32_t i = 0; i < 7425; ++i) map[i] = (uint8_t)ac_cluster_of(i);
    BW a, b;
    bw_init(&a);
    bw_init(&b);
    context_map_complex(&a, map, 7425, 0);
    context_map_complex(&b, map, 7425, 1);
    bw_append(w, b.bits < a.bits ? &b : &a);
    bw_free(&a);
    bw_free(&b);
}

/* ---- AC tokens ---- */

static const uint32_t* natural_order(int n) {
    static uint32_t o[3][1024];
    static int ready = 0;
    if (!ready) {
        for (int si = 0; si < 3; ++si) {
            const size_t N = (size_t)8 << si, cx = N / 8;
            size_t cur = cx * cx;
            for (size_t i = 0; i < N; ++i)
                for (size_t j = 0; j <= i; ++j) {
                    size_t x = j, y = i - j;
                    if (i & 1) { const size_t t = x; x = y; y = t; }
                    const size_t val = (x < cx && y < cx) ? y * cx + x : cur++;
                    o[si][val] = (uint32_t)(y * N + x);
                }
            for (size_t ip = N - 1; ip > 0; --ip) {
                const size_t i = ip - 1;
                for (size_t j = 0; j <= i; ++j) {
                    size_t x = N - 1 - (i - j), y = N - 1 - j;
                    if (i & 1) { const size_t t = x; x = y; y = t; }
                    o[si][cur++] = (uint32_t)(y * N + x);
                }
            }
        }
        ready = 1;
    }
    return o[n == 8 ? 0 : (n == 16 ? 1 : 2)];
}

static size_t slot_of(int n, size_t bx, size_t by, size_t bw, uint32_t raw) {
    const size_t side = (size_t)n / 8, q = raw / 64;
    return ((by + q / side) * bw + bx + q % side) * 64 + raw % 64;
}

typedef struct { uint8_t cluster; uint16_t sym; uint8_t nb; uint32_t bits; } Tok;
typedef struct { Tok* t; size_t n, cap; } TokVec;
static void tv_push(TokVec* v, Tok t) {
    if (v->n == v->cap) { v->cap = v->cap ? v->cap * 2 : 4096; v->t = (Tok*)realloc(v->t, v->cap * sizeof(Tok)); }
    v->t[v->n++] = t;
}

static void ac_emit(TokVec* out, uint32_t* hist, uint32_t value, uint32_t ctx) {
    uint32_t s, nb, b;
    hybrid(value, 4, 2, 0, &s, &nb, &b);
    const int cl = ac_cluster_of(ctx);
    ++hist[cl * 256 + s];
    Tok t = {(uint8_t)cl, (uint16_t)s, (uint8_t)nb, b};
    tv_push(out, t);
}

static void tokenize_ac_group(int bwi, const int16_t* ac, const int8_t* acs, size_t nblocks, size_t bx0,
                              size_t by0, size_t gbw, size_t gbh, uint32_t* hist, TokVec* out) {
    const size_t bw = (size_t)bwi;
    const int chan[3] = {1, 0, 2};
    int32_t* nzg = (int32_t*)calloc(3 * gbw * gbh, sizeof(int32_t));
    for (size_t sy = 0; sy < gbh; ++sy)
        for (size_t sx = 0; sx < gbw; ++sx) {
            const int n = acs[(by0 + sy) * bw + bx0 + sx];
            if (n == 0) continue;
            const size_t cx = (size_t)n / 8, cb = cx * cx, sz = (size_t)n * n;
            const uint32_t l2 = n == 16 ? 2 : (n == 32 ? 4 : 0);
            const uint32_t* ord = natural_order(n);
            for (int p = 0; p < 3; ++p) {
                const int c = chan[p];
                const int16_t* pl = ac + (size_t)c * nblocks * 64;
                int32_t nz = 0;
                for (size_t k = cb; k < sz; ++k)
                    if (pl[slot_of(n, bx0 + sx, by0 + sy, bw, ord[k])] != 0) ++nz;
                const int32_t norm = (int32_t)(((uint32_t)nz + cb - 1) >> l2);
                for (size_t dy = 0; dy < cx; ++dy)
                    for (size_t dx = 0; dx < cx; ++dx) nzg[c * gbw * gbh + (sy + dy) * gbw + sx + dx] = norm;
            }
        }
    for (size_t sy = 0; sy < gbh; ++sy)
        for (size_t sx = 0; sx < gbw; ++sx) {
            const size_t gx = bx0 + sx, gy = by0 + sy;
            const int n = acs[gy * bw + gx];
            if (n == 0) continue;
            const size_t cb = ((size_t)n / 8) * ((size_t)n / 8), sz = (size_t)n * n;
            const uint32_t l2 = n == 16 ? 2 : (n == 32 ? 4 : 0);
            const uint32_t* ord = natural_order(n);
            for (int p = 0; p < 3; ++p) {
                const int c = chan[p];
                const int16_t* pl = ac + (size_t)c * nblocks * 64;
                uint32_t nzeros = 0;
                for (size_t k = cb; k < sz; ++k)
                    if (pl[slot_of(n, gx, gy, bw, ord[k])] != 0) ++nzeros;
                const int bctx = c == 1 ? (n == 8 ? 0 : 2) : (n == 8 ? 7 : 9);
                const int hl = sx > 0, ht = sy > 0;
                const uint32_t top = ht ? (uint32_t)nzg[c * gbw * gbh + (sy - 1) * gbw + sx] : 0;
                const uint32_t left = hl ? (uint32_t)nzg[c * gbw * gbh + sy * gbw + sx - 1] : 0;
                uint32_t pred;
                if (!hl) pred = ht ? top : 32u;
                else if (!ht) pred = left;
                else pred = (top + left + 1) / 2;
                const uint32_t pz = pred >= 64 ? 64 : pred;
                const uint32_t nzctx = (pz < 8 ? pz : 4 + pz / 2) * 15 + (uint32_t)bctx;
                ac_emit(out, hist, nzeros, nzctx);
                const uint32_t off = 15 * 37 + 458 * (uint32_t)bctx;
                uint32_t remaining = nzeros;
                uint32_t prev = nzeros > sz / 16 ? 0u : 1u;
                for (size_t k = cb; k < sz && remaining > 0; ++k) {
                    const int32_t v = pl[slot_of(n, gx, gy, bw, ord[k])];
                    const uint32_t left_nz = (remaining + (uint32_t)cb - 1) >> l2;
                    const uint32_t kk = (uint32_t)k >> l2;
                    uint32_t nzc, fc;
                    if (left_nz < 2) nzc = 0; else if (left_nz < 3) nzc = 31; else if (left_nz < 5) nzc = 62;
                    else if (left_nz < 9) nzc = 93; else if (left_nz < 13) nzc = 123; else if (left_nz < 21) nzc = 152;
                    else if (left_nz < 33) nzc = 180; else nzc = 206;
                    if (kk < 16) fc = kk - 1; else if (kk < 32) fc = 15 + (kk - 16) / 2; else fc = 23 + (kk - 32) / 4;
                    ac_emit(out, hist, pack_signed(v), off + (nzc + fc) * 2 + prev);
                    prev = v != 0 ? 1u : 0u;
                    remaining -= prev;
                }
            }
        }
    free(nzg);
}

/* ---- modular images ---- */

typedef struct { size_t w, h; const int32_t* px; } Chan;

static void modular_header_and_tokens(BW* w, const Chan* ch, int nch, int gradient) {
    bw_put(w, 1, 0);
    bw_put(w, 1, 1);
    bw_put(w, 2, 0);
    /* single-leaf MA tree: property 0, predictor, offset 0, mul_log 0, mul_bits 0 */
    const uint32_t tree_tok[5] = {0, gradient ? 5u : 0u, 0, 0, 0};
    uint32_t th[16] = {0};
    size_t tl = 1;
    for (int i = 0; i < 5; ++i) { ++th[tree_tok[i]]; if (tree_tok[i] + 1 > tl) tl = tree_tok[i] + 1; }
    uint8_t td[16];
    uint16_t tb[16];
    prefix_histograms(w, th, tl, 6, 4, 2, 0, td, tb);
    for (int i = 0; i < 5; ++i) bw_put(w, td[tree_tok[i]], tb[tree_tok[i]]);
    /* residual tokens */
    size_t total = 0;
    for (int c = 0; c < nch; ++c) total += ch[c].w * ch[c].h;
    uint32_t* tok = (uint32_t*)malloc(sizeof(uint32_t) * (total ? total : 1));
    uint32_t hist[256] = {0};
    size_t k = 0, alpha = 0;
    for (int c = 0; c < nch; ++c) {
        if (ch[c].w == 0 || ch[c].h == 0) continue;
        for (size_t y = 0; y < ch[c].h; ++y)
            for (size_t x = 0; x < ch[c].w; ++x) {
                const int32_t v = ch[c].px[y * ch[c].w + x];
                int32_t pred = 0;
                if (gradient) {
                    const int hl = x > 0, ht = y > 0;
                    const int32_t wv = hl ? ch[c].px[y * ch[c].w + x - 1] : 0;
                    const int32_t nv = ht ? ch[c].px[(y - 1) * ch[c].w + x] : 0;
                    const int32_t nw = (hl && ht) ? ch[c].px[(y - 1) * ch[c].w + x - 1] : 0;
                    const int32_t left = hl ? wv : (ht ? nv : 0);
                    const int32_t top = ht ? nv : left;
                    const int32_t tlv = (hl && ht) ? nw : left;
                    const int32_t lo = left < top ? left : top, hi = left < top ? top : left;
                    pred = tlv < lo ? hi : (tlv > hi ? lo : (int32_t)((int64_t)left + top - tlv));
                }
                tok[k++] = pack_signed(v - pred);
            }
    }
    for (size_t i = 0; i < k; ++i) {
        uint32_t s, nb, b;
        hybrid(tok[i], 4, 2, 0, &s, &nb, &b);
        ++hist[s];
        if (s + 1 > alpha) alpha = s + 1;
    }
    if (alpha == 0) { alpha = 1; hist[0] = 1; }
    uint8_t depth[256];
    uint16_t bits[256];
    prefix_histograms(w, hist, alpha, 1, 4, 2, 0, depth, bits);
    for (size_t i = 0; i < k; ++i) {
        uint32_t s, nb, b;
        hybrid(tok[i], 4, 2, 0, &s, &nb, &b);
        bw_put(w, depth[s], bits[s]);
        if (nb) bw_put(w, nb, b);
    }
    free(tok);
}

/* ---- frame assembly ---- */

static const Distr kDimEnc[4] = {BO(9, 1), BO(13, 1), BO(18, 1), BO(30, 1)};
static const Distr kTocDist[4] = {BO(10, 0), BO(14, 1024), BO(22, 17408), BO(30, 4211712)};
static const Distr kGsEnc[4] = {BO(11, 1), BO(11, 2049), BO(12, 4097), BO(16, 8193)};
static const Distr kQdcEnc[4] = {VAL(16), BO(5, 1), BO(8, 1), BO(16, 1)};
static const Distr kOrderEnc[4] = {VAL(0x5F), VAL(0x13), VAL(0), BO(13, 0)};

size_t oracle_assemble(int width, int height, const int16_t* ac, const int32_t* dc, const int8_t* acs,
                       const int32_t* qf, const int8_t* ytox, const int8_t* ytob, uint32_t gs,
                       uint32_t qdc, uint8_t* out, size_t cap) {
    const size_t W = (size_t)width, H = (size_t)height, bw = W / 8, bh = H / 8, nb = bw * bh;
    const size_t xg = (bw + 31) / 32, yg = (bh + 31) / 32, nac = xg * yg;
    const size_t xdg = (bw + 255) / 256, ydg = (bh + 255) / 256, ndc = xdg * ydg;
    const size_t cmw = (bw + 7) / 8;
    /* One AC group: DcGlobal, the DcGroup, AcGlobal and the AcGroup are one
     * combined section, concatenated bit by bit and padded once at its end,
     * with a single TOC entry (tools/bitstream/vardct_frame.cc:414-449). */
    const int single = nac == 1;
    const size_t nsec = 2 + ndc + nac;
    BW* sec = (BW*)calloc(nsec, sizeof(BW));
    for (size_t i = 0; i < nsec; ++i) bw_init(&sec[i]);
#define SECTION_END(w) do { if (!single) bw_pad(w); } while (0)

    /* DcGlobal */
    bw_put(&sec[0], 1, 1);
    write_u32(&sec[0], kGsEnc, gs);
    write_u32(&sec[0], kQdcEnc, qdc);
    bw_put(&sec[0], 1, 1);
    bw_put(&sec[0], 1, 1);
    bw_put(&sec[0], 1, 0);
    SECTION_END(&sec[0]);

    /* DcGroups */
    for (size_t g = 0; g < ndc; ++g) {
        BW* w = &sec[1 + g];
        const size_t bx0 = (g % xdg) * 256, by0 = (g / xdg) * 256;
        const size_t dgw = bw - bx0 < 256 ? bw - bx0 : 256, dgh = bh - by0 < 256 ? bh - by0 : 256;
        int32_t* dch = (int32_t*)malloc(sizeof(int32_t) * 3 * dgw * dgh);
        const int phys[3] = {1, 0, 2};
        for (int p = 0; p < 3; ++p)
            for (size_t y = 0; y < dgh; ++y)
                for (size_t x = 0; x < dgw; ++x)
                    dch[p * dgw * dgh + y * dgw + x] = dc[phys[p] * nb + (by0 + y) * bw + bx0 + x];
        Chan dcc[3] = {{dgw, dgh, dch}, {dgw, dgh, dch + dgw * dgh}, {dgw, dgh, dch + 2 * dgw * dgh}};
        bw_put(w, 2, 0);
        modular_header_and_tokens(w, dcc, 3, 1);
        const size_t cw = (dgw + 7) / 8, chh = (dgh + 7) / 8;
        int32_t* meta = (int32_t*)calloc(2 * cw * chh + 2 * dgw * dgh + dgw * dgh, sizeof(int32_t));
        for (size_t y = 0; y < chh; ++y)
            for (size_t x = 0; x < cw; ++x) {
                const size_t t = (by0 / 8 + y) * cmw + bx0 / 8 + x;
                meta[y * cw + x] = ytox[t];
                meta[cw * chh + y * cw + x] = ytob[t];
            }
        int32_t* aq = meta + 2 * cw * chh;
        size_t count = 0;
        for (size_t y = 0; y < dgh; ++y)
            for (size_t x = 0; x < dgw; ++x) {
                const size_t blk = (by0 + y) * bw + bx0 + x;
                if (acs[blk] == 0) continue;
                ++count;
            }
        size_t i = 0;
        for (size_t y = 0; y < dgh; ++y)
            for (size_t x = 0; x < dgw; ++x) {
                const size_t blk = (by0 + y) * bw + bx0 + x;
                const int n = acs[blk];
                if (n == 0) continue;
                aq[i] = n == 16 ? 4 : (n == 32 ? 5 : 0);
                aq[count + i] = qf[blk] - 1;
                ++i;
            }
        int32_t* epf = aq + 2 * count;
        Chan mc[4] = {{cw, chh, meta}, {cw, chh, meta + cw * chh}, {count, 2, aq}, {dgw, dgh, epf}};
        bw_put(w, ceil_log2(dgw * dgh), (uint32_t)(count - 1));
        modular_header_and_tokens(w, mc, 4, 0);
        SECTION_END(w);
        free(meta);
        free(dch);
    }

    /* AC groups: tokenize all, pooled clustered histogram, then AcGlobal. */
    uint32_t* hist = (uint32_t*)calloc(32 * 256, sizeof(uint32_t));
    TokVec* gt = (TokVec*)calloc(nac, sizeof(TokVec));
    for (size_t g = 0; g < nac; ++g) {
        const size_t bx0 = (g % xg) * 32, by0 = (g / xg) * 32;
        const size_t gbw = bw - bx0 < 32 ? bw - bx0 : 32, gbh = bh - by0 < 32 ? bh - by0 : 32;
        tokenize_ac_group((int)bw, ac, acs, nb, bx0, by0, gbw, gbh, hist, &gt[g]);
    }
    BW* acg = &sec[1 + ndc];
    bw_put(acg, 1, 1);
    bw_put(acg, ceil_log2(nac), 0);
    write_u32(acg, kOrderEnc, 0);
    bw_put(acg, 1, 0);
    ac_context_map(acg);
    bw_put(acg, 1, 1);
    for (int c = 0; c < 32; ++c) uint_config(acg, 4, 2, 0);
    size_t alpha[32];
    for (int c = 0; c < 32; ++c) {
        size_t a = 1;
        for (size_t s = 0; s < 256; ++s) if (hist[c * 256 + s]) a = s + 1;
        alpha[c] = a;
        var_len_u16(acg, a - 1);
    }
    uint8_t* depth = (uint8_t*)calloc(32 * 256, 1);
    uint16_t* bits = (uint16_t*)calloc(32 * 256, 2);
    for (int c = 0; c < 32; ++c)
        if (alpha[c] > 1) build_and_store(hist + c * 256, alpha[c], depth + c * 256, bits + c * 256, acg);
    SECTION_END(acg);
    for (size_t g = 0; g < nac; ++g) {
        BW* w = &sec[2 + ndc + g];
        for (size_t i = 0; i < gt[g].n; ++i) {
            const Tok* t = &gt[g].t[i];
            bw_put(w, depth[t->cluster * 256 + t->sym], bits[t->cluster * 256 + t->sym]);
            if (t->nb) bw_put(w, t->nb, t->bits);
        }
        SECTION_END(w);
        free(gt[g].t);
    }
    free(gt);
    free(hist);
    free(depth);
    free(bits);
#undef SECTION_END
    size_t nout = nsec;
    if (single) {
        for (size_t i = 1; i < nsec; ++i) bw_append(&sec[0], &sec[i]);
        bw_pad(&sec[0]);
        nout = 1;
    }

    /* Codestream head. */
    BW head;
    bw_init(&head);
    bw_put(&head, 8, 0xFF);
    bw_put(&head, 8, 0x0A);
    const int small = (W % 8 == 0 && H % 8 == 0 && W <= 256 && H <= 256);
    bw_put(&head, 1, small);
    if (small) bw_put(&head, 5, H / 8 - 1); else write_u32(&head, kDimEnc, (uint32_t)H);
    bw_put(&head, 3, 0);
    if (small) bw_put(&head, 5, W / 8 - 1); else write_u32(&head, kDimEnc, (uint32_t)W);
    bw_put(&head, 1, 1);
    bw_put(&head, 1, 1);
    bw_pad(&head);
    bw_put(&head, 1, 0);       /* all_default */
    bw_put(&head, 2, 0);       /* frame_type regular */
    bw_put(&head, 1, 0);       /* VarDCT */
    write_u64_zero(&head);     /* flags */
    bw_put(&head, 2, 0);       /* upsampling 1 */
    bw_put(&head, 3, 2);       /* x_qm_scale */
    bw_put(&head, 3, 2);       /* b_qm_scale */
    bw_put(&head, 2, 0);       /* num_passes 1 */
    bw_put(&head, 1, 0);       /* custom size/origin */
    bw_put(&head, 2, 0);       /* blending mode replace */
    bw_put(&head, 1, 1);       /* is_last */
    bw_put(&head, 2, 0);       /* name length 0 */
    bw_put(&head, 1, 1);       /* loop filter all default */
    write_u64_zero(&head);     /* extensions */
    bw_put(&head, 1, 0);       /* TOC: no permutation */
    bw_pad(&head);
    size_t body = 0;
    for (size_t i = 0; i < nout; ++i) {
        write_u32(&head, kTocDist, (uint32_t)bw_bytes(&sec[i]));
        body += bw_bytes(&sec[i]);
    }
    bw_pad(&head);

    const size_t cs = bw_bytes(&head) + body;
    static const uint8_t kHdr[32] = {0, 0, 0, 0x0c, 'J', 'X', 'L', ' ', 0x0d, 0x0a, 0x87, 0x0a, 0, 0, 0, 0x14,
                                     'f', 't', 'y', 'p', 'j', 'x', 'l', ' ', 0, 0, 0, 0, 'j', 'x', 'l', ' '};
    const int large = cs >= 0x100000000ull - 8;
    const size_t total = 32 + (large ? 16 : 8) + cs;
    uint8_t* file = (uint8_t*)malloc(total);
    memcpy(file, kHdr, 32);
    size_t at = 32;
    const uint64_t box = (uint64_t)cs + (large ? 16 : 8);
    const uint32_t sf = large ? 1u : (uint32_t)box;
    for (int i = 0; i < 4; ++i) file[at++] = (uint8_t)(sf >> (8 * (3 - i)));
    file[at++] = 'j'; file[at++] = 'x'; file[at++] = 'l'; file[at++] = 'c';
    if (large) for (int i = 0; i < 8; ++i) file[at++] = (uint8_t)(box >> (8 * (7 - i)));
    memcpy(file + at, head.buf, bw_bytes(&head));
    at += bw_bytes(&head);
    for (size_t i = 0; i < nout; ++i) { memcpy(file + at, sec[i].buf, bw_bytes(&sec[i])); at += bw_bytes(&sec[i]); }
    if (out) memcpy(out, file, total < cap ? total : cap);
    free(file);
    bw_free(&head);
    for (size_t i = 0; i < nsec; ++i) bw_free(&sec[i]);
    free(sec);
    return total;
}

size_t oracle_encode(const OracleFrame* in, float distance, uint8_t* out, size_t cap, int threads) {
    const size_t W = (size_t)in->width, H = (size_t)in->height, nb = (W / 8) * (H / 8);
    const size_t nt = ((W / 8 + 7) / 8) * ((H / 8 + 7) / 8);
    OracleOutputs o;
    memset(&o, 0, sizeof(o));
    o.ac = (int16_t*)malloc(sizeof(int16_t) * 3 * nb * 64);
    o.dc = (int32_t*)malloc(sizeof(int32_t) * 3 * nb);
    o.acs = (int8_t*)malloc(nb);
    o.qf = (int32_t*)malloc(sizeof(int32_t) * nb);
    o.ytox = (int8_t*)malloc(nt);
    o.ytob = (int8_t*)malloc(nt);
    o.nzn = (uint8_t*)malloc(3 * nb);
    o.nzc = (uint16_t*)malloc(sizeof(uint16_t) * 3 * nb);
    size_t n = 0;
    if (oracle_frontend(in, distance, &o, threads) == 0) {
        OracleScalars sc;
        oracle_scalars(distance, &sc);
        n = oracle_assemble(in->width, in->height, o.ac, o.dc, o.acs, o.qf, o.ytox, o.ytob, sc.global_scale,
                            sc.quant_dc, out, cap);
    }
    free(o.ac); free(o.dc); free(o.acs); free(o.qf); free(o.ytox); free(o.ytob); free(o.nzn); free(o.nzc);
    return n;
}
