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
//   * zlib (.im7 pack 2 row/frame blocks, .set "Zlib" entries): RFC 1950
//     streams through the system zlib, with the reference's checks on where the
//     stream ends (im7_reader.py:569-594, set_reader.py:1601-1633).
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

// Inflate one zlib (RFC 1950) stream of n bytes into dst, which must receive
// exactly `expected` bytes, and the stream must end (its end marker) at its last
// byte.  Returns 0, 1 (not a valid stream), 2 (more than `expected` bytes),
// 3 (no end marker: truncated), 4 (fewer than `expected` bytes), 5 (bytes
// follow the end marker), or -1 for bad arguments.
PIV_EXPORT int pivb_zlib_inflate_exact(const uint8_t *src, long long n, uint8_t *dst, long long expected)
{
    if (!src || (!dst && expected > 0) || n < 0 || expected < 0) return -1;
    z_stream zs;
    memset(&zs, 0, sizeof(zs));
    if (inflateInit(&zs) != Z_OK) return 1;
    uint8_t spare;
    zs.next_in = const_cast<Bytef *>(src);
    zs.avail_in = (uInt)n;
    zs.next_out = dst;
    zs.avail_out = (uInt)expected;
    int rc = inflate(&zs, Z_FINISH);
    int result;
    if (rc == Z_STREAM_END) {
        result = (long long)zs.total_out != expected ? 4 : (zs.avail_in != 0 ? 5 : 0);
    } else if (rc == Z_DATA_ERROR || rc == Z_NEED_DICT || rc == Z_STREAM_ERROR || rc == Z_MEM_ERROR) {
        result = 1;
    } else if (zs.avail_out == 0) {
        // output full before the end marker: one more byte tells "longer" from
        // "ends exactly here"
        zs.next_out = &spare;
        zs.avail_out = 1;
        rc = inflate(&zs, Z_FINISH);
        if ((long long)zs.total_out > expected) result = 2;
        else if (rc == Z_STREAM_END) result = zs.avail_in != 0 ? 5 : 0;
        else if (rc == Z_DATA_ERROR || rc == Z_NEED_DICT || rc == Z_STREAM_ERROR) result = 1;
        else result = 3;
    } else {
        result = 3;                                // input used up before the end marker
    }
    inflateEnd(&zs);
    return result;
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
