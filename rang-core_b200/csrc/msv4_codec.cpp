// Blosc-1 chunks with LZ4 blocks: the codec of the visibility, flag, weight
// and uvw arrays in MSv4 (xradio) zarr stores. Host code; C ABI in
// include/rang_msv4.h.
//
// Formats, from their published descriptions:
// * LZ4 block format: sequences of a token (high nibble literal count, low
//   nibble match length - 4, 15 meaning "continued by bytes summed until one
//   is not 255"), the literals, a 2-byte little-endian offset back into the
//   output and the match, which may overlap its own output; the last
//   sequence has literals only.
// * Blosc 1 chunk (c-blosc 1.x, format version 2): a 16-byte header
//   (version, compressor version, flags, type size, then little-endian
//   uncompressed bytes, block size and chunk bytes). Flags: 0x01 byte
//   shuffle, 0x02 stored uncompressed ("memcpyed", the data follows the
//   header), 0x04 bit shuffle, 0x10 blocks not split, bits 5-7 the codec
//   (1: LZ4). Unless memcpyed, the header is followed by one 32-bit start
//   offset per block; a block holds `nsplits` streams, each a 32-bit byte
//   count and the bytes, raw when the count equals the stream's decoded
//   size and LZ4 otherwise. A block is split into `typesize` streams when
//   splitting is allowed, typesize <= 16, the block holds at least 128
//   elements, and it is not the chunk's short last block; a byte-shuffled
//   block stores byte j of every element before byte j + 1.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "rang_msv4.h"

namespace {

constexpr size_t kHeader = 16;
constexpr uint8_t kShuffle = 0x01, kMemcpyed = 0x02, kBitShuffle = 0x04, kDontSplit = 0x10;
constexpr int kCodecLz4 = 1;
constexpr size_t kMinBuffer = 128, kMaxSplits = 16;
constexpr size_t kBad = ~size_t(0);

uint32_t le32(const uint8_t* p) { return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24; }
void put32(uint8_t* p, uint32_t v) {
  p[0] = (uint8_t)v;
  p[1] = (uint8_t)(v >> 8);
  p[2] = (uint8_t)(v >> 16);
  p[3] = (uint8_t)(v >> 24);
}

// LZ4 block decode into exactly `cap` bytes at most; returns the bytes
// written or kBad for a malformed block.
size_t lz4_decode(const uint8_t* src, size_t n, uint8_t* dst, size_t cap) {
  size_t ip = 0, op = 0;
  while (ip < n) {
    const unsigned token = src[ip++];
    size_t lit = token >> 4;
    if (lit == 15) {
      unsigned b;
      do {
        if (ip >= n) return kBad;
        b = src[ip++];
        lit += b;
      } while (b == 255);
    }
    if (lit > n - ip || lit > cap - op) return kBad;
    std::memcpy(dst + op, src + ip, lit);
    ip += lit;
    op += lit;
    if (ip == n) break;  // the last sequence: literals only
    if (n - ip < 2) return kBad;
    const size_t off = (size_t)src[ip] | (size_t)src[ip + 1] << 8;
    ip += 2;
    if (off == 0 || off > op) return kBad;
    size_t len = (token & 15u) + 4;
    if ((token & 15u) == 15u) {
      unsigned b;
      do {
        if (ip >= n) return kBad;
        b = src[ip++];
        len += b;
      } while (b == 255);
    }
    if (len > cap - op) return kBad;
    uint8_t* d = dst + op;
    const uint8_t* s = d - off;
    if (off >= len) {
      std::memcpy(d, s, len);
    } else {
      for (size_t i = 0; i < len; i++) d[i] = s[i];  // overlapping: byte order matters
    }
    op += len;
  }
  return op;
}

size_t put_length(uint8_t* dst, size_t op, size_t cap, size_t rem) {
  while (rem >= 255) {
    if (op >= cap) return kBad;
    dst[op++] = 255;
    rem -= 255;
  }
  if (op >= cap) return kBad;
  dst[op++] = (uint8_t)rem;
  return op;
}

// One sequence: literals src[a, a + lit), then (when len > 0) a match of
// `len` at `off`.
size_t put_sequence(uint8_t* dst, size_t op, size_t cap, const uint8_t* lits, size_t lit, size_t off, size_t len) {
  if (op >= cap) return kBad;
  const size_t tok_at = op++;
  uint8_t token = (uint8_t)(std::min<size_t>(lit, 15) << 4);
  if (lit >= 15 && (op = put_length(dst, op, cap, lit - 15)) == kBad) return kBad;
  if (lit > cap - op) return kBad;
  std::memcpy(dst + op, lits, lit);
  op += lit;
  if (len > 0) {
    if (cap - op < 2) return kBad;
    dst[op++] = (uint8_t)off;
    dst[op++] = (uint8_t)(off >> 8);
    token |= (uint8_t)std::min<size_t>(len - 4, 15);
    if (len - 4 >= 15 && (op = put_length(dst, op, cap, len - 4 - 15)) == kBad) return kBad;
  }
  dst[tok_at] = token;
  return op;
}

// A greedy LZ4 block encoder (4-byte hash of the current position, one
// candidate per hash): valid LZ4, not tuned for ratio.
size_t lz4_encode(const uint8_t* src, size_t n, uint8_t* dst, size_t cap) {
  size_t op = 0, anchor = 0;
  if (n >= 13) {
    std::vector<uint32_t> table(1u << 16, 0xffffffffu);
    const size_t limit = n - 12, match_end = n - 5;
    size_t ip = 0;
    while (ip < limit) {
      uint32_t v;
      std::memcpy(&v, src + ip, 4);
      const uint32_t h = (v * 2654435761u) >> 16;
      const uint32_t ref = table[h];
      table[h] = (uint32_t)ip;
      uint32_t w;
      if (ref != 0xffffffffu && ip - ref <= 65535 && (std::memcpy(&w, src + ref, 4), w == v)) {
        size_t len = 4;
        while (ip + len < match_end && src[ref + len] == src[ip + len]) len++;
        op = put_sequence(dst, op, cap, src + anchor, ip - anchor, ip - ref, len);
        if (op == kBad) return kBad;
        ip += len;
        anchor = ip;
      } else {
        ip++;
      }
    }
  }
  return put_sequence(dst, op, cap, src + anchor, n - anchor, 0, 0);
}

struct Header {
  uint8_t version, versionlz, flags;
  size_t typesize, nbytes, blocksize, cbytes;
  size_t nblocks() const { return blocksize ? (nbytes + blocksize - 1) / blocksize : 0; }
};

int parse(const uint8_t* src, size_t n, Header& h) {
  if (!src || n < kHeader) return 1;
  h.version = src[0];
  h.versionlz = src[1];
  h.flags = src[2];
  h.typesize = src[3];
  h.nbytes = le32(src + 4);
  h.blocksize = le32(src + 8);
  h.cbytes = le32(src + 12);
  if (h.cbytes > n || h.cbytes < kHeader || h.typesize == 0) return 1;
  if (h.nbytes > 0 && h.blocksize == 0) return 1;
  if (h.flags & kMemcpyed) return h.cbytes >= kHeader + h.nbytes ? 0 : 1;
  if (h.flags & kBitShuffle) return 3;
  if ((h.flags >> 5) != kCodecLz4) return 3;
  if (h.nblocks() > (h.cbytes - kHeader) / 4) return 1;
  return 0;
}

// Element i gathers its bytes from the ts byte planes; the writes run
// contiguously (the planes are read as ts sequential streams).
template <size_t TS>
void unshuffle_fixed(const uint8_t* src, uint8_t* dst, size_t ne) {
  for (size_t i = 0; i < ne; i++)
    for (size_t j = 0; j < TS; j++) dst[i * TS + j] = src[j * ne + i];
}

void unshuffle(const uint8_t* src, uint8_t* dst, size_t bytes, size_t ts) {
  const size_t ne = bytes / ts;
  switch (ts) {
    case 2: unshuffle_fixed<2>(src, dst, ne); break;
    case 4: unshuffle_fixed<4>(src, dst, ne); break;
    case 8: unshuffle_fixed<8>(src, dst, ne); break;
    case 16: unshuffle_fixed<16>(src, dst, ne); break;
    default:
      for (size_t i = 0; i < ne; i++)
        for (size_t j = 0; j < ts; j++) dst[i * ts + j] = src[j * ne + i];
  }
  std::memcpy(dst + ne * ts, src + ne * ts, bytes - ne * ts);
}

void shuffle(const uint8_t* src, uint8_t* dst, size_t bytes, size_t ts) {
  const size_t ne = bytes / ts;
  for (size_t j = 0; j < ts; j++)
    for (size_t i = 0; i < ne; i++) dst[j * ne + i] = src[i * ts + j];
  std::memcpy(dst + ne * ts, src + ne * ts, bytes - ne * ts);
}

size_t nsplits_for(const Header& h, size_t bsize, bool last) {
  const bool split = !(h.flags & kDontSplit) && h.typesize <= kMaxSplits && bsize / h.typesize >= kMinBuffer && !last;
  return split ? h.typesize : 1;
}

// Block j of a parsed, non-memcpyed chunk into dst + j * blocksize.
int decode_block(const Header& h, const uint8_t* src, size_t j, uint8_t* dst, std::vector<uint8_t>& scratch) {
  const size_t nb = h.nblocks();
  const size_t leftover = h.nbytes % h.blocksize;
  const bool last = j + 1 == nb && leftover > 0;
  const size_t bsize = last ? leftover : h.blocksize;
  const bool shuffled = (h.flags & kShuffle) && h.typesize > 1;
  size_t at = le32(src + kHeader + 4 * j);
  if (at < kHeader + 4 * nb || at > h.cbytes) return 1;
  const size_t ns = nsplits_for(h, bsize, last);
  const size_t neblock = bsize / ns;
  if (ns * neblock != bsize) return 1;
  if (shuffled && scratch.size() < bsize) scratch.resize(h.blocksize);
  uint8_t* out = shuffled ? scratch.data() : dst + j * h.blocksize;
  for (size_t k = 0; k < ns; k++) {
    if (h.cbytes - at < 4) return 1;
    const size_t cb = le32(src + at);
    at += 4;
    if (cb > h.cbytes - at) return 1;
    if (cb == neblock) {
      std::memcpy(out + k * neblock, src + at, neblock);
    } else if (lz4_decode(src + at, cb, out + k * neblock, neblock) != neblock) {
      return 1;
    }
    at += cb;
  }
  if (shuffled) unshuffle(scratch.data(), dst + j * h.blocksize, bsize, h.typesize);
  return 0;
}

int decode(const uint8_t* src, size_t n, uint8_t* dst, size_t cap) {
  Header h;
  int st = parse(src, n, h);
  if (st) return st;
  if (h.nbytes > cap) return 1;
  if (h.flags & kMemcpyed) {
    std::memcpy(dst, src + kHeader, h.nbytes);
    return 0;
  }
  std::vector<uint8_t> scratch;
  for (size_t j = 0; j < h.nblocks(); j++)
    if ((st = decode_block(h, src, j, dst, scratch))) return st;
  return 0;
}

int encode(const uint8_t* src, size_t nbytes, size_t ts, bool shuf, bool split, size_t blocksize, uint8_t* dst,
           size_t cap, size_t* written) {
  if (ts == 0 || ts > 255 || nbytes > 0x7fffffffu) return 1;
  if (blocksize == 0 || blocksize > nbytes) blocksize = std::max<size_t>(nbytes, 1);
  Header h{2, 1, (uint8_t)((kCodecLz4 << 5) | (shuf ? kShuffle : 0) | (split ? 0 : kDontSplit)), ts, nbytes,
           blocksize, 0};
  const size_t nb = h.nblocks();
  size_t op = kHeader + 4 * nb;
  bool stored = op > cap;
  std::vector<uint8_t> tmp(shuf ? blocksize : 0);
  for (size_t j = 0; j < nb && !stored; j++) {
    const bool last = j + 1 == nb && nbytes % blocksize > 0;
    const size_t bsize = last ? nbytes % blocksize : blocksize;
    const uint8_t* in = src + j * blocksize;
    if (shuf && ts > 1) {
      shuffle(in, tmp.data(), bsize, ts);
      in = tmp.data();
    }
    put32(dst + kHeader + 4 * j, (uint32_t)op);
    const size_t ns = nsplits_for(h, bsize, last), neblock = bsize / ns;
    for (size_t k = 0; k < ns && !stored; k++) {
      if (cap - op < 4 + neblock) {
        stored = true;
        break;
      }
      size_t cb = lz4_encode(in + k * neblock, neblock, dst + op + 4, neblock);
      if (cb == kBad || cb >= neblock) {  // incompressible stream: stored raw
        std::memcpy(dst + op + 4, in + k * neblock, neblock);
        cb = neblock;
      }
      put32(dst + op, (uint32_t)cb);
      op += 4 + cb;
    }
  }
  if (stored || op >= kHeader + nbytes) {  // the whole chunk stored uncompressed
    if (cap < kHeader + nbytes) return 1;
    h.flags = (uint8_t)((h.flags & ~kShuffle) | kMemcpyed);
    std::memcpy(dst + kHeader, src, nbytes);
    op = kHeader + nbytes;
  }
  dst[0] = h.version;
  dst[1] = h.versionlz;
  dst[2] = h.flags;
  dst[3] = (uint8_t)ts;
  put32(dst + 4, (uint32_t)nbytes);
  put32(dst + 8, (uint32_t)blocksize);
  put32(dst + 12, (uint32_t)op);
  *written = op;
  return 0;
}

}  // namespace

extern "C" {

int32_t rang_b200_lz4_decode(const uint8_t* src, size_t srclen, uint8_t* dst, size_t dstcap, size_t* written) {
  if ((!src && srclen) || (!dst && dstcap) || !written) return 1;
  const size_t n = lz4_decode(src, srclen, dst, dstcap);
  if (n == kBad) return 1;
  *written = n;
  return 0;
}

int32_t rang_b200_lz4_encode(const uint8_t* src, size_t srclen, uint8_t* dst, size_t dstcap, size_t* written) {
  if ((!src && srclen) || !dst || !written) return 1;
  const size_t n = lz4_encode(src, srclen, dst, dstcap);
  if (n == kBad) return 1;
  *written = n;
  return 0;
}

int32_t rang_b200_blosc_header(const uint8_t* src, size_t srclen, size_t* nbytes, size_t* cbytes, size_t* blocksize,
                               int32_t* typesize, int32_t* flags) {
  Header h;
  const int st = parse(src, srclen, h);
  if (st == 1) return 1;
  if (nbytes) *nbytes = h.nbytes;
  if (cbytes) *cbytes = h.cbytes;
  if (blocksize) *blocksize = h.blocksize;
  if (typesize) *typesize = (int32_t)h.typesize;
  if (flags) *flags = h.flags;
  return st;
}

int32_t rang_b200_blosc_decode(const uint8_t* src, size_t srclen, uint8_t* dst, size_t dstcap) {
  if (!dst && dstcap) return 1;
  return decode(src, srclen, dst, dstcap);
}

int32_t rang_b200_blosc_encode(const uint8_t* src, size_t nbytes, int32_t typesize, int32_t shuffle_bytes,
                               int32_t split, size_t blocksize, uint8_t* dst, size_t dstcap, size_t* written) {
  if ((!src && nbytes) || !dst || !written || typesize <= 0) return 1;
  return encode(src, nbytes, (size_t)typesize, shuffle_bytes != 0, split != 0, blocksize, dst, dstcap, written);
}

int32_t rang_b200_blosc_decode_many(size_t n, const uint8_t* const* srcs, const size_t* srclens, uint8_t* const* dsts,
                                    const size_t* dstcaps, int32_t threads, int32_t* status) {
  if (n && (!srcs || !srclens || !dsts || !dstcaps || !status)) return 1;
  // Tasks are (chunk, block) pairs, so that a few large chunks still use
  // every thread; a memcpyed chunk is one task.
  std::vector<Header> heads(n);
  std::vector<std::pair<size_t, size_t>> tasks;
  for (size_t i = 0; i < n; i++) {
    status[i] = parse(srcs[i], srclens[i], heads[i]);
    if (!status[i] && heads[i].nbytes > dstcaps[i]) status[i] = 1;
    if (status[i]) continue;
    const size_t nb = (heads[i].flags & kMemcpyed) ? 1 : heads[i].nblocks();
    for (size_t j = 0; j < nb; j++) tasks.emplace_back(i, j);
  }
  std::vector<std::atomic<int32_t>> fail(n);
  for (auto& f : fail) f = 0;
  std::atomic<size_t> next{0};
  auto work = [&] {
    std::vector<uint8_t> scratch;
    for (size_t t; (t = next.fetch_add(1)) < tasks.size();) {
      const size_t i = tasks[t].first, j = tasks[t].second;
      const Header& h = heads[i];
      int st = 0;
      if (h.flags & kMemcpyed)
        std::memcpy(dsts[i], srcs[i] + kHeader, h.nbytes);
      else
        st = decode_block(h, srcs[i], j, dsts[i], scratch);
      if (st) fail[i] = st;
    }
  };
  const size_t nt = std::max<size_t>(1, std::min<size_t>(threads > 0 ? (size_t)threads : 1, tasks.size()));
  std::vector<std::thread> pool;
  for (size_t t = 1; t < nt; t++) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
  int32_t worst = 0;
  for (size_t i = 0; i < n; i++) {
    if (!status[i]) status[i] = fail[i];
    worst = std::max(worst, status[i]);
  }
  return worst;
}

}  // extern "C"
