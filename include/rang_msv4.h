/*
 * rang_msv4.h — the chunk codec of MSv4 (xradio) zarr stores, for the
 * reader that feeds the gridder (python: rang.msv4).
 *
 * The reference reads MSv4 processing sets in Python through xarray, zarr 3
 * and numcodecs (python/rang/msv4.py), and has its own Blosc-1 decoder for
 * its zarr ingest (core/src/blosc.rs, following c-blosc 1.21.6 `blosc_d`).
 * These entry points are this library's codec for the stores' visibility,
 * flag, weight and uvw arrays: Blosc-1 chunks (format version 2) with LZ4
 * blocks, byte shuffle, split streams and stored ("memcpyed") chunks; bit
 * shuffle and other codecs are refused with status 3. Host memory only; no
 * GPU. Status: 0 success, 1 invalid arguments or a malformed chunk, 3 a
 * chunk this codec does not decode.
 */
#ifndef RANG_MSV4_H
#define RANG_MSV4_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One LZ4 block into at most dstcap bytes; *written the decoded length. */
int32_t rang_b200_lz4_decode(const uint8_t* src, size_t srclen, uint8_t* dst, size_t dstcap, size_t* written);

/* One LZ4 block (a greedy encoder, for writing stores). */
int32_t rang_b200_lz4_encode(const uint8_t* src, size_t srclen, uint8_t* dst, size_t dstcap, size_t* written);

/* The header of a Blosc-1 chunk: decoded bytes, chunk bytes, block size,
 * type size and flags (any may be null); status 3 for a chunk whose codec or
 * filter `rang_b200_blosc_decode` refuses (the fields are still set). */
int32_t rang_b200_blosc_header(const uint8_t* src, size_t srclen, size_t* nbytes, size_t* cbytes, size_t* blocksize,
                               int32_t* typesize, int32_t* flags);

/* A whole Blosc-1 chunk into dst (dstcap >= its decoded bytes). */
int32_t rang_b200_blosc_decode(const uint8_t* src, size_t srclen, uint8_t* dst, size_t dstcap);

/* A Blosc-1 chunk of nbytes bytes with LZ4 blocks of `blocksize` bytes (0:
 * one block), byte shuffle of `typesize`-byte elements when shuffle is set,
 * split streams when split is set; stored uncompressed when that is smaller.
 * dstcap >= nbytes + 16 + 4 * blocks always suffices. */
int32_t rang_b200_blosc_encode(const uint8_t* src, size_t nbytes, int32_t typesize, int32_t shuffle, int32_t split,
                               size_t blocksize, uint8_t* dst, size_t dstcap, size_t* written);

/* n chunks on `threads` host threads; status[i] per chunk, the worst returned. */
int32_t rang_b200_blosc_decode_many(size_t n, const uint8_t* const* srcs, const size_t* srclens, uint8_t* const* dsts,
                                    const size_t* dstcaps, int32_t threads, int32_t* status);

#ifdef __cplusplus
}
#endif

#endif
