// lavision_codecs.cpp -- libpivb_lavision: the byte-serial codecs of LaVision
// DaVis image containers, decoded on the host straight into the caller's
// (page-locked) buffer, from where the frames go to the GPU for the pixel
// unpack, the intensity scale and the float conversion (pivb_unpack_pixels_dev).
//
// Each codec is a sequential byte stream (a variable-length token grammar, an
// LZ77 block, a Deflate stream) with one stream per frame or per file, so there
// is no parallelism inside a stream for a GPU to use; the host decodes frames of
// different files or streams in parallel (every entry point is re-entrant and
// holds no state; ctypes releases the GIL around each call).
//
//   * DaVis token stream (.im7 pack 1, .set "IMX" entries):
//     pivtools_core/image_handling/readers/davis_tokens.py:46-127 (grammar:
//     int8 delta; 0x80 lo hi absolute; 0x7f n (lo hi)*n absolutes; 0x81 signed
//     4-bit deltas, high nibble first, ended only by a low nibble 8).
//   * LZ4 block (.im7 pack 20, .set "LZ4" entries): the published LZ4 block
//     format (token: literal length in the high nibble, match length - 4 in
//     the low nibble, 255-continued; little-endian 16-bit match offset),
//     decoded to exactly the size the frame geometry needs
//     (im7_reader.py:270-291).
//   * zlib (.im7 pack 2 row/frame blocks, .set "Zlib" entries): RFC 1950 /
//     RFC 1951 streams through this library's own Deflate decoder (below), with
//     the reference's checks on where the stream ends (im7_reader.py:569-594,
//     set_reader.py:1601-1633); the system zlib serves only the probe of a
//     file's first block.
#include <stdint.h>
#include <string.h>
#include <zlib.h>

#define PIV_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

// Token-stream status codes (davis_tokens.py:35-38).
constexpr int TOK_OK = 0, TOK_TRUNCATED = 1, TOK_OVERRUN = 2, TOK_RANGE = 3;
constexpr long long U16_MAX = 65535;

}  // namespace

// Decode npix values of a DaVis token stream, starting at byte *off with running
// value *prev; on return *off is the byte after the last token read, *prev the
// running value after the last value written and *written the values written.
// Returns 0, or 1 (the input ended inside a token), 2 (a 0x7f run would write
// past npix), 3 (the running value left 0..65535), or -1 for bad arguments.
// Mirrors davis_tokens.py:46-127.
PIV_EXPORT int pivb_davis_tokens_decode(const uint8_t *data, long long n, long long *off, long long *prev,
                                        uint16_t *out, long long npix, long long *written)
{
    if (!data || !off || !prev || !out || !written || n < 0 || npix < 0 || *off < 0) return -1;
    long long o = *off, p = *prev, i = 0;
    int status = TOK_OK;
    while (i < npix) {
        if (o >= n) { status = TOK_TRUNCATED; break; }
        const long long b = data[o++];
        if (b == 0x81) {
            bool stop = false;
            while (i < npix && !stop) {
                if (o >= n) { status = TOK_TRUNCATED; break; }
                const long long byte = data[o++];
                const long long hi = byte >> 4;
                p += hi >= 8 ? hi - 16 : hi;
                if (p < 0 || p > U16_MAX) { status = TOK_RANGE; break; }
                out[i++] = (uint16_t)p;
                if (i >= npix) break;
                const long long lo = byte & 0xF;
                if (lo == 8) { stop = true; break; }
                p += lo >= 8 ? lo - 16 : lo;
                if (p < 0 || p > U16_MAX) { status = TOK_RANGE; break; }
                out[i++] = (uint16_t)p;
            }
            if (status != TOK_OK) break;
        } else if (b == 0x80) {
            if (o + 2 > n) { status = TOK_TRUNCATED; break; }
            p = (long long)data[o] | ((long long)data[o + 1] << 8);
            o += 2;
            out[i++] = (uint16_t)p;
        } else if (b == 0x7F) {
            if (o >= n) { status = TOK_TRUNCATED; break; }
            const long long cnt = data[o++];
            if (i + cnt > npix) { status = TOK_OVERRUN; break; }
            if (o + 2 * cnt > n) { status = TOK_TRUNCATED; break; }
            for (long long k = 0; k < cnt; ++k) {
                p = (long long)data[o] | ((long long)data[o + 1] << 8);
                o += 2;
                out[i++] = (uint16_t)p;
            }
        } else {
            p += b >= 128 ? b - 256 : b;
            if (p < 0 || p > U16_MAX) { status = TOK_RANGE; break; }
            out[i++] = (uint16_t)p;
        }
    }
    *off = o;
    *prev = p;
    *written = i;
    return status;
}

// Decode one raw LZ4 block (no frame header, no size prefix) of n bytes into dst,
// which must receive exactly `expected` bytes.  Returns 0, 1 (the block is
// malformed: a sequence cut off, a zero or out-of-range match offset, output
// beyond `expected`), 2 (the block decodes to fewer than `expected` bytes) or -1
// for bad arguments.
PIV_EXPORT int pivb_lz4_block_decode(const uint8_t *src, long long n, uint8_t *dst, long long expected)
{
    if (!src || !dst || n < 0 || expected < 0) return -1;
    const uint8_t *ip = src, *const iend = src + n;
    long long w = 0;
    if (n == 0) return expected == 0 ? 0 : 2;
    for (;;) {
        if (ip >= iend) return 1;
        const unsigned token = *ip++;
        long long lit = token >> 4;
        if (lit == 15) {
            unsigned s;
            do {
                if (ip >= iend) return 1;
                s = *ip++;
                lit += s;
            } while (s == 255);
        }
        if (lit > iend - ip || lit > expected - w) return 1;
        memcpy(dst + w, ip, (size_t)lit);
        ip += lit;
        w += lit;
        if (ip == iend) break;                 // the last sequence holds literals only
        if (iend - ip < 2) return 1;
        const long long offset = (long long)ip[0] | ((long long)ip[1] << 8);
        ip += 2;
        if (offset == 0 || offset > w) return 1;
        long long mlen = token & 15;
        if (mlen == 15) {
            unsigned s;
            do {
                if (ip >= iend) return 1;
                s = *ip++;
                mlen += s;
            } while (s == 255);
        }
        mlen += 4;
        if (mlen > expected - w) return 1;
        uint8_t *d = dst + w;
        const uint8_t *m = d - offset;
        if (offset >= mlen) {
            memcpy(d, m, (size_t)mlen);
        } else {
            for (long long k = 0; k < mlen; ++k) d[k] = m[k];     // overlapping: byte order matters
        }
        w += mlen;
    }
    return w == expected ? 0 : 2;
}

// ---------------------------------------------------------------------------
// zlib streams (RFC 1950 wrapper around RFC 1951 Deflate), decoded to an exact
// size with this library's own decoder.  Canonical Huffman codes are looked up
// in a root table indexed by the next 10 (literal/length) or 8 (distance) input
// bits, least-significant bit first, with second-level tables for longer codes;
// a 64-bit bit buffer is refilled eight bytes at a time while at least 16 input
// bytes remain and a byte at a time near the end, where it supplies zero bytes
// past the input and counts them, so a code that reaches past the input reads
// as a truncated stream.  Matches copy eight bytes at a time when the distance
// allows.  The results and the status codes are those of zlib's inflate() driven
// to exactly `expected` bytes (checked against the system zlib on streams of
// every block type, level, strategy and window size, and on their truncations,
// bit flips, trailing bytes and wrong sizes); per-row .im7 streams decode about
// 1.7x faster than through zlib, which spends a third of a 4 KB row in its
// table set-up and checksum.
namespace {

// ---- table entries: bits 0-7 code length (total, root + second level), 8-11 kind,
// 12-15 extra bits (length/distance) or second-level index bits, 16-31 value
enum : uint32_t { K_LIT = 0, K_LEN = 1, K_EOB = 2, K_SUB = 3, K_BAD = 4, K_DIST = 5 };
constexpr uint32_t ent(uint32_t kind, uint32_t extra, uint32_t value, uint32_t nbits)
{
    return nbits | (kind << 8) | (extra << 12) | (value << 16);
}
inline uint32_t e_bits(uint32_t e) { return e & 0xff; }
inline uint32_t e_kind(uint32_t e) { return (e >> 8) & 0xf; }
inline uint32_t e_extra(uint32_t e) { return (e >> 12) & 0xf; }
inline uint32_t e_val(uint32_t e) { return e >> 16; }

// RFC 1951 3.2.5: length symbols 257..285 and distance symbols 0..29
constexpr uint16_t kLenBase[29] = {3, 4, 5, 6, 7, 8, 9, 10, 11, 13, 15, 17, 19, 23, 27,
                                   31, 35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
constexpr uint8_t kLenExtra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
constexpr uint16_t kDistBase[30] = {1, 2, 3, 4, 5, 7, 9, 13, 17, 25, 33, 49, 65, 97, 129,
                                    193, 257, 385, 513, 769, 1025, 1537, 2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
constexpr uint8_t kDistExtra[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};
// order of the code-length code lengths in a dynamic block header
constexpr uint8_t kClOrder[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};

constexpr int kLitRoot = 10, kDistRoot = 8, kClRoot = 7;
constexpr int kLitCap = (1 << kLitRoot) + 288 * 32, kDistCap = (1 << kDistRoot) + 32 * 128, kClCap = 1 << kClRoot;

inline uint32_t lit_value(int s)
{
    if (s < 256) return ent(K_LIT, 0, (uint32_t)s, 0);
    if (s == 256) return ent(K_EOB, 0, 0, 0);
    if (s <= 285) return ent(K_LEN, kLenExtra[s - 257], kLenBase[s - 257], 0);
    return ent(K_BAD, 0, 0, 0);
}
inline uint32_t dist_value(int s)
{
    return s < 30 ? ent(K_DIST, kDistExtra[s], kDistBase[s], 0) : ent(K_BAD, 0, 0, 0);
}
inline uint32_t cl_value(int s) { return ent(K_LIT, 0, (uint32_t)s, 0); }

// 8-bit reversal table
struct Rev8 {
    uint8_t t[256];
    constexpr Rev8() : t()
    {
        for (int v = 0; v < 256; ++v) {
            int r = 0;
            for (int k = 0; k < 8; ++k) r |= ((v >> k) & 1) << (7 - k);
            t[v] = (uint8_t)r;
        }
    }
};
constexpr Rev8 kRev8{};
// the low `len` bits of c, reversed (Deflate sends Huffman codes most-significant bit first)
inline uint32_t reverse_bits(uint32_t c, int len)
{
    return ((uint32_t)kRev8.t[c & 0xff] << 8 | kRev8.t[(c >> 8) & 0xff]) >> (16 - len);
}

// Canonical Huffman decode table for n code lengths (RFC 1951 3.2.2): a root
// table of 2^root entries indexed by the next root input bits, second-level
// tables for longer codes.  Returns 0, or 1 for a set that is over-subscribed,
// or incomplete other than a lone code of length 1 (allowed where allow_single),
// or empty (allowed where allow_empty: every entry then decodes as invalid).
template <uint32_t (*VALUE)(int)>
int build_table(const uint8_t *lens, int n, int root, uint32_t *tab, int cap, bool allow_single, bool allow_empty)
{
    int count[16] = {0};
    for (int s = 0; s < n; ++s) count[lens[s]]++;
    count[0] = 0;
    int left = 1, maxlen = 0;
    for (int l = 1; l <= 15; ++l) {
        left = (left << 1) - count[l];
        if (left < 0) return 1;
        if (count[l]) maxlen = l;
    }
    const int rsize = 1 << root;
    if (maxlen == 0) {
        if (!allow_empty) return 1;
        for (int k = 0; k < rsize; ++k) tab[k] = ent(K_BAD, 0, 0, 1);
        return 0;
    }
    if (left > 0) {
        if (!(allow_single && maxlen == 1)) return 1;
        for (int k = 0; k < rsize; ++k) tab[k] = ent(K_BAD, 0, 0, 1);
    }
    // symbols in canonical order (by length, then value) with their reversed codes
    int offs[17];
    offs[1] = 0;
    for (int l = 1; l <= 15; ++l) offs[l + 1] = offs[l] + count[l];
    const int total = offs[16];
    uint16_t sym[288];
    {
        int at[16];
        memcpy(at, offs, sizeof(at));
        for (int s = 0; s < n; ++s)
            if (lens[s]) sym[at[lens[s]]++] = (uint16_t)s;
    }
    uint32_t rev[288];
    uint8_t len[288];
    {
        uint32_t code = 0;
        int idx = 0;
        for (int l = 1; l <= maxlen; ++l, code <<= 1)
            for (int j = 0; j < count[l]; ++j, ++idx, ++code) {
                rev[idx] = reverse_bits(code, l);
                len[idx] = (uint8_t)l;
            }
    }
    const int nshort = offs[root + 1 > 16 ? 16 : root + 1];
    for (int idx = 0; idx < nshort; ++idx) {
        const uint32_t e = VALUE(sym[idx]) | len[idx];
        for (uint32_t k = rev[idx]; k < (uint32_t)rsize; k += 1u << len[idx]) tab[k] = e;
    }
    // longer codes: those under one root prefix are consecutive in canonical
    // order, and the last of them is the longest, which sizes their table
    int used = rsize;
    for (int idx = nshort; idx < total;) {
        const uint32_t prefix = rev[idx] & (uint32_t)(rsize - 1);
        int g = idx + 1;
        while (g < total && (rev[g] & (uint32_t)(rsize - 1)) == prefix) ++g;
        const int sb = len[g - 1] - root;
        if (used + (1 << sb) > cap) return 1;
        tab[prefix] = ent(K_SUB, (uint32_t)sb, (uint32_t)used, (uint32_t)root);
        for (; idx < g; ++idx) {
            const uint32_t e = VALUE(sym[idx]) | len[idx];
            for (uint32_t k = rev[idx] >> root; k < (1u << sb); k += 1u << (len[idx] - root)) tab[used + k] = e;
        }
        used += 1 << sb;
    }
    return 0;
}

struct FixedTables {
    uint32_t lit[kLitCap];
    uint32_t dist[kDistCap];
    FixedTables()
    {
        uint8_t l[288];
        for (int s = 0; s < 288; ++s) l[s] = s < 144 ? 8 : s < 256 ? 9 : s < 280 ? 7 : 8;
        build_table<lit_value>(l, 288, kLitRoot, lit, kLitCap, false, false);
        uint8_t d[32];
        for (int s = 0; s < 32; ++s) d[s] = 5;
        build_table<dist_value>(d, 32, kDistRoot, dist, kDistCap, false, false);
    }
};

const FixedTables &fixed_tables()
{
    static const FixedTables t;
    return t;
}

// LSB-first bit reader over [p, end).  `bb` holds `bc` unread bits (and, above
// them, possibly later input bits already loaded); past the end it supplies
// zero bytes, counted in `over`: a decode that consumed any of them (bc < over)
// ran off the input.
struct Bits {
    const uint8_t *p, *end;
    uint64_t bb = 0;
    int bc = 0;
    int over = 0;
    inline void refill()
    {
        if (end - p >= 8) {
            uint64_t w;
            memcpy(&w, p, 8);
            bb |= w << bc;
            p += (63 - bc) >> 3;
            bc |= 56;
        } else {
            while (bc <= 56) {
                if (p < end) bb |= (uint64_t)*p++ << bc;
                else over += 8;
                bc += 8;
            }
        }
    }
    inline uint32_t peek(int n) const { return (uint32_t)(bb & ((1ull << n) - 1)); }
    inline void drop(int n) { bb >>= n; bc -= n; }
    inline bool overrun() const { return bc < over; }
    // byte position of the next unread whole byte (after align())
    inline const uint8_t *byte_pos() const { return p - ((bc - over) >> 3); }
    inline void align() { drop(bc & 7); }
};

inline uint32_t lookup(const uint32_t *tab, int root, uint64_t bb)
{
    uint32_t e = tab[bb & ((1u << root) - 1)];
    if (e_kind(e) == K_SUB) e = tab[e_val(e) + ((uint32_t)(bb >> root) & ((1u << e_extra(e)) - 1))];
    return e;
}

enum { ST_OK = 0, ST_BAD = 1, ST_LONG = 2, ST_TRUNC = 3, ST_SHORT = 4, ST_TRAIL = 5 };

// Code lengths of a dynamic block (RFC 1951 3.2.7) into lit/dist tables.
int read_dynamic(Bits &b, uint32_t *lit, uint32_t *dist)
{
    b.refill();
    const int nlen = (int)b.peek(5) + 257;
    const int ndist = (int)(b.bb >> 5 & 31) + 1;
    const int ncl = (int)(b.bb >> 10 & 15) + 4;
    b.drop(14);
    if (b.overrun()) return ST_TRUNC;
    if (nlen > 286 || ndist > 30) return ST_BAD;
    uint8_t cl[19] = {0};
    for (int k = 0; k < ncl; ++k) {
        if (b.bc < 3) b.refill();
        cl[kClOrder[k]] = (uint8_t)b.peek(3);
        b.drop(3);
    }
    if (b.overrun()) return ST_TRUNC;
    uint32_t cltab[kClCap];
    if (build_table<cl_value>(cl, 19, kClRoot, cltab, kClCap, false, false)) return ST_BAD;
    uint8_t lens[286 + 30];
    const int total = nlen + ndist;
    int i = 0;
    while (i < total) {
        if (b.bc < 7 + 7) b.refill();
        const uint32_t e = cltab[b.peek(kClRoot)];
        b.drop((int)e_bits(e));
        const int sym = (int)e_val(e);
        int rep = 0, val = 0;
        if (sym < 16) {
            if (b.overrun()) return ST_TRUNC;
            lens[i++] = (uint8_t)sym;
            continue;
        } else if (sym == 16) {
            rep = 3 + (int)b.peek(2); b.drop(2);
            if (b.overrun()) return ST_TRUNC;
            if (i == 0) return ST_BAD;
            val = lens[i - 1];
        } else if (sym == 17) {
            rep = 3 + (int)b.peek(3); b.drop(3);
        } else {
            rep = 11 + (int)b.peek(7); b.drop(7);
        }
        if (b.overrun()) return ST_TRUNC;
        if (i + rep > total) return ST_BAD;
        memset(lens + i, val, (size_t)rep);
        i += rep;
    }
    if (lens[256] == 0) return ST_BAD;
    if (build_table<lit_value>(lens, nlen, kLitRoot, lit, kLitCap, true, false)) return ST_BAD;
    if (build_table<dist_value>(lens + nlen, ndist, kDistRoot, dist, kDistCap, true, true)) return ST_BAD;
    return ST_OK;
}

// Copy len bytes from dist back; ahead of `out` at least 8 spare bytes may be
// overwritten when `room` allows (fast path).
inline void copy_match(uint8_t *out, uint32_t dist, uint32_t len, bool fast)
{
    const uint8_t *src = out - dist;
    if (fast && dist >= 8) {
        uint8_t *o = out, *oe = out + len;
        do { memcpy(o, src, 8); o += 8; src += 8; } while (o < oe);
    } else if (dist == 1) {
        memset(out, src[0], len);
    } else {
        for (uint32_t k = 0; k < len; ++k) out[k] = src[k];
    }
}

// One Huffman-coded block.  Returns ST_OK at its end-of-block code.
int decode_block(Bits &b, const uint32_t *lit, const uint32_t *dist, uint8_t *const start, uint8_t *&out,
                 uint8_t *const oend)
{
    uint8_t *o = out;
    {
        // fast loop: at least 16 input bytes and 266 output bytes left.  The bit
        // reader is a local copy here, so the byte stores to the output cannot
        // alias it and it stays in registers.
        Bits L = b;
        for (;;) {
            if (L.end - L.p < 16 || oend - o < 258 + 8) break;
            L.refill();
            uint32_t e = lookup(lit, kLitRoot, L.bb);
            if (e_kind(e) == K_LIT) {
                L.drop((int)e_bits(e));
                *o++ = (uint8_t)e_val(e);
                e = lookup(lit, kLitRoot, L.bb);
                if (e_kind(e) == K_LIT) {
                    L.drop((int)e_bits(e));
                    *o++ = (uint8_t)e_val(e);
                    e = lookup(lit, kLitRoot, L.bb);
                    if (e_kind(e) == K_LIT) {
                        L.drop((int)e_bits(e));
                        *o++ = (uint8_t)e_val(e);
                        continue;
                    }
                }
                L.refill();
            }
            if (e_kind(e) == K_LEN) {
                L.drop((int)e_bits(e));
                const uint32_t len = e_val(e) + L.peek((int)e_extra(e));
                L.drop((int)e_extra(e));
                const uint32_t d = lookup(dist, kDistRoot, L.bb);
                L.drop((int)e_bits(d));
                if (e_kind(d) != K_DIST) { b = L; out = o; return ST_BAD; }
                const uint32_t dd = e_val(d) + L.peek((int)e_extra(d));
                L.drop((int)e_extra(d));
                if (dd > (uint32_t)(o - start)) { b = L; out = o; return ST_BAD; }
                copy_match(o, dd, len, true);
                o += len;
                continue;
            }
            L.drop((int)e_bits(e));
            b = L;
            out = o;
            return e_kind(e) == K_EOB ? ST_OK : ST_BAD;
        }
        b = L;
    }
    // careful loop: every code checked against the end of the input and output
    for (;;) {
        b.refill();
        const uint32_t e = lookup(lit, kLitRoot, b.bb);
        b.drop((int)e_bits(e));
        if (b.overrun()) { out = o; return ST_TRUNC; }
        const uint32_t k = e_kind(e);
        if (k == K_LIT) {
            if (o == oend) { out = o; return ST_LONG; }
            *o++ = (uint8_t)e_val(e);
            continue;
        }
        if (k == K_EOB) { out = o; return ST_OK; }
        if (k != K_LEN) { out = o; return ST_BAD; }
        const uint32_t len = e_val(e) + b.peek((int)e_extra(e));
        b.drop((int)e_extra(e));
        if (b.overrun()) { out = o; return ST_TRUNC; }
        b.refill();
        const uint32_t d = lookup(dist, kDistRoot, b.bb);
        b.drop((int)e_bits(d));
        if (b.overrun()) { out = o; return ST_TRUNC; }
        if (e_kind(d) != K_DIST) { out = o; return ST_BAD; }
        const uint32_t dd = e_val(d) + b.peek((int)e_extra(d));
        b.drop((int)e_extra(d));
        if (b.overrun()) { out = o; return ST_TRUNC; }
        if (dd > (uint32_t)(o - start)) { out = o; return ST_BAD; }
        if ((uint32_t)(oend - o) < len) { out = o; return ST_LONG; }
        copy_match(o, dd, len, false);
        o += len;
    }
}

// Adler-32 (RFC 1950 8.2) in blocks of at most 5552 bytes, the most whose sums
// stay within 32 bits before the modulo; 16 bytes at a time: s2 gains 16 s1
// plus the bytes weighted 16..1, s1 the bytes' sum.
uint32_t adler32_of(const uint8_t *p, size_t n)
{
    uint32_t s1 = 1, s2 = 0;
    while (n) {
        size_t blk = n < 5552 ? n : 5552;
        n -= blk;
        while (blk >= 16) {
            uint32_t a = 0, w = 0;
            for (int k = 0; k < 16; ++k) {
                a += p[k];
                w += (uint32_t)(16 - k) * p[k];
            }
            s2 += 16 * s1 + w;
            s1 += a;
            p += 16;
            blk -= 16;
        }
        while (blk--) {
            s1 += *p++;
            s2 += s1;
        }
        s1 %= 65521;
        s2 %= 65521;
    }
    return s2 << 16 | s1;
}

}  // namespace

// Inflate one zlib (RFC 1950) stream of n bytes into dst, which must receive
// exactly `expected` bytes, and the stream must end (its end marker) at its last
// byte.  Returns 0, 1 (not a valid stream), 2 (more than `expected` bytes),
// 3 (no end marker: truncated), 4 (fewer than `expected` bytes), 5 (bytes
// follow the end marker), or -1 for bad arguments.
PIV_EXPORT int pivb_zlib_inflate_exact(const uint8_t *src, long long n, uint8_t *dst, long long expected)
{
    if (!src || (!dst && expected > 0) || n < 0 || expected < 0) return -1;
    if (n < 2) return ST_TRUNC;
    const uint32_t cmf = src[0], flg = src[1];
    if ((cmf * 256 + flg) % 31 != 0 || (cmf & 15) != 8 || (cmf >> 4) > 7 || (flg & 0x20)) return ST_BAD;
    Bits b;
    b.p = src + 2;
    b.end = src + n;
    uint8_t *const start = dst, *out = dst, *const oend = dst + expected;
    uint32_t lit[kLitCap], dist[kDistCap];
    for (;;) {
        b.refill();
        const uint32_t final_ = b.peek(1), type = (uint32_t)(b.bb >> 1 & 3);
        b.drop(3);
        if (b.overrun()) return ST_TRUNC;
        int rc;
        if (type == 0) {
            b.align();
            const uint8_t *q = b.byte_pos();
            b.bb = 0; b.bc = 0; b.over = 0; b.p = q;
            if (b.end - q < 4) return ST_TRUNC;
            const uint32_t len = q[0] | (uint32_t)q[1] << 8, nlen = q[2] | (uint32_t)q[3] << 8;
            if (len != (~nlen & 0xffffu)) return ST_BAD;
            q += 4;
            const long long have = b.end - q, room = oend - out;
            const long long k = have < (long long)len ? have : (long long)len;
            if (room < k) return ST_LONG;
            if (k) memcpy(out, q, (size_t)k);
            out += k;
            if (k < (long long)len) return ST_TRUNC;
            b.p = q + len;
            rc = ST_OK;
        } else if (type == 1) {
            const FixedTables &f = fixed_tables();
            rc = decode_block(b, f.lit, f.dist, start, out, oend);
        } else if (type == 2) {
            rc = read_dynamic(b, lit, dist);
            if (rc == ST_OK) rc = decode_block(b, lit, dist, start, out, oend);
        } else {
            return ST_BAD;
        }
        if (rc != ST_OK) return rc;
        if (final_) break;
    }
    b.align();
    const uint8_t *q = b.byte_pos();
    if (b.end - q < 4) return ST_TRUNC;
    const uint32_t want = (uint32_t)q[0] << 24 | (uint32_t)q[1] << 16 | (uint32_t)q[2] << 8 | q[3];
    const long long produced = out - start;
    const uint32_t a = adler32_of(start, (size_t)produced);
    if (a != want) return ST_BAD;
    if (produced != expected) return ST_SHORT;
    return q + 4 != b.end ? ST_TRAIL : ST_OK;
}

// Inflate at most `cap` bytes from the start of one zlib stream (the reference's
// probe of the first pack-2 block, im7_reader.py:534-566).  Returns the bytes
// produced, or -1 if the stream is not valid up to there.
PIV_EXPORT long long pivb_zlib_inflate_prefix(const uint8_t *src, long long n, uint8_t *dst, long long cap)
{
    if (!src || !dst || n < 0 || cap < 0) return -1;
    z_stream zs;
    memset(&zs, 0, sizeof(zs));
    if (inflateInit(&zs) != Z_OK) return -1;
    zs.next_in = const_cast<Bytef *>(src);
    zs.avail_in = (uInt)n;
    zs.next_out = dst;
    zs.avail_out = (uInt)cap;
    const int rc = inflate(&zs, Z_SYNC_FLUSH);
    const long long produced = (long long)zs.total_out;
    inflateEnd(&zs);
    if (rc == Z_DATA_ERROR || rc == Z_NEED_DICT || rc == Z_STREAM_ERROR || rc == Z_MEM_ERROR) return -1;
    return produced;
}

#include <atomic>
#include <thread>
#include <vector>

// A run of int32-size-prefixed zlib blocks (.im7 pack 2) in one buffer: skip
// `skip_before` blocks, inflate the next n_blocks (each exactly block_bytes,
// ending at its declared size) into dst on up to n_threads host threads, then
// skip `skip_after` blocks.  *consumed receives the bytes walked (where the
// attribute records begin when every block of the file was walked).  Returns 0;
// -1 for bad arguments; -2 if a size prefix is cut off, not positive or runs
// past the buffer (*err_block = its index); or, for the first block (by index)
// that does not inflate as required, 10 + its pivb_zlib_inflate_exact code with
// *err_block = its index among the n_blocks.
PIV_EXPORT int pivb_zlib_blocks_decode(const uint8_t *buf, long long n, long long skip_before, long long n_blocks,
                                       long long skip_after, uint8_t *dst, long long block_bytes, int n_threads,
                                       long long *consumed, long long *err_block)
{
    if (!buf || n < 0 || skip_before < 0 || n_blocks < 0 || skip_after < 0 || block_bytes < 0 ||
        (n_blocks > 0 && !dst) || !consumed || !err_block)
        return -1;
    std::vector<long long> start((size_t)n_blocks), size((size_t)n_blocks);
    long long pos = 0;
    const long long total = skip_before + n_blocks + skip_after;
    for (long long b = 0; b < total; ++b) {
        if (n - pos < 4) { *err_block = b; return -2; }
        int32_t s;
        memcpy(&s, buf + pos, 4);
        pos += 4;
        if (s <= 0 || s > n - pos) { *err_block = b; return -2; }
        if (b >= skip_before && b < skip_before + n_blocks) {
            start[(size_t)(b - skip_before)] = pos;
            size[(size_t)(b - skip_before)] = s;
        }
        pos += s;
    }
    *consumed = pos;
    std::atomic<long long> next{0};
    std::vector<int> code((size_t)n_blocks, 0);
    auto work = [&]() {
        for (long long b = next.fetch_add(1); b < n_blocks; b = next.fetch_add(1))
            code[(size_t)b] = pivb_zlib_inflate_exact(buf + start[(size_t)b], size[(size_t)b],
                                                      dst + b * block_bytes, block_bytes);
    };
    const int nt = n_threads < 1 ? 1 : (n_threads > 64 ? 64 : n_threads);
    if (nt == 1 || n_blocks < 2) {
        work();
    } else {
        std::vector<std::thread> pool;
        for (int t = 0; t < nt; ++t) pool.emplace_back(work);
        for (auto &th : pool) th.join();
    }
    for (long long b = 0; b < n_blocks; ++b)
        if (code[(size_t)b]) {
            *err_block = b;
            return 10 + code[(size_t)b];
        }
    return 0;
}
