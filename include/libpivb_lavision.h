/* libpivb_lavision -- the byte-serial codecs of LaVision DaVis containers, on
 * the host (no GPU code): each decodes one stream into a caller buffer (page-
 * locked memory, from which the payload goes to the GPU for
 * pivb_unpack_pixels_dev, libpivb_pass.h).  Every entry point is re-entrant and
 * keeps no state.  The reference decodes these in Python (numba, python-lz4,
 * zlib); there is no C counterpart to bind, so each declaration names the
 * reference function it replaces. */
#ifndef LIBPIVB_LAVISION_H
#define LIBPIVB_LAVISION_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* DaVis token stream (.im7 pack 1, IMX .set entries): decode npix uint16 values
 * from data[*off..n) with running value *prev; on return *off, *prev and
 * *written describe where it stopped.  Returns 0, 1 (input ended inside a token),
 * 2 (a 0x7f run past npix), 3 (running value outside 0..65535), -1 (bad
 * arguments).  Replaces _decode_tokens
 * (pivtools_core/image_handling/readers/davis_tokens.py:46-127). */
int pivb_davis_tokens_decode(const uint8_t *data, long long n, long long *off, long long *prev, uint16_t *out,
                             long long npix, long long *written);

/* One raw LZ4 block (.im7 pack 20, LZ4 .set entries) into exactly `expected`
 * bytes.  Returns 0, 1 (malformed block or output beyond `expected`), 2 (fewer
 * bytes than `expected`), -1 (bad arguments).  Replaces lz4_block_decompress
 * (im7_reader.py:270-291; python-lz4's lz4.block.decompress). */
int pivb_lz4_block_decode(const uint8_t *src, long long n, uint8_t *dst, long long expected);

/* One zlib stream (.im7 pack 2 blocks, Zlib .set entries) into exactly
 * `expected` bytes, ending at its last byte.  Returns 0, 1 (invalid stream),
 * 2 (more than `expected`), 3 (no end marker), 4 (fewer than `expected`),
 * 5 (bytes after the end marker), -1 (bad arguments): the bytes and codes of
 * zlib's inflate() driven to exactly `expected` bytes, from the library's own
 * Deflate decoder.  Replaces _read_zlib_block (im7_reader.py:569-594) and
 * _decompress_zlib (set_reader.py:1601-1633). */
int pivb_zlib_inflate_exact(const uint8_t *src, long long n, uint8_t *dst, long long expected);

/* At most `cap` bytes from the start of one zlib stream: the bytes produced, or
 * -1 for an invalid stream.  Replaces the first-block probe of _zlib_block_bytes
 * (im7_reader.py:534-566). */
long long pivb_zlib_inflate_prefix(const uint8_t *src, long long n, uint8_t *dst, long long cap);

/* A run of int32-size-prefixed zlib blocks (.im7 pack 2) in one buffer: skip
 * skip_before blocks, inflate the next n_blocks (each exactly block_bytes,
 * ending at its declared size) into dst on up to n_threads host threads, skip
 * skip_after blocks; *consumed = the bytes walked.  Returns 0; -1 bad arguments;
 * -2 a size prefix cut off, not positive or past the buffer (*err_block = its
 * index); 10 + the pivb_zlib_inflate_exact code of the first failing block
 * (*err_block = its index among the n_blocks).  Replaces the per-block loop of
 * _read_pixels_zlib (im7_reader.py:607-635). */
int pivb_zlib_blocks_decode(const uint8_t *buf, long long n, long long skip_before, long long n_blocks,
                            long long skip_after, uint8_t *dst, long long block_bytes, int n_threads,
                            long long *consumed, long long *err_block);

#ifdef __cplusplus
}
#endif
#endif
