// md5.cpp — av1pf_frame_md5: the MD5 a conformance vector's .md5 file holds
// for a decoded frame (the reference's tests/common/mod.rs:101-119
// `frame_md5`), over the packed frame that av1pf_output writes. MD5 is the
// algorithm of RFC 1321, written here from the RFC's description. It runs on
// the host: MD5 chains every 64-byte block through the previous one, so one
// frame's hash is a single serial computation that a host core finishes
// long before a GPU thread would.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "av1pf.h"
#include "plan.h"

namespace {

// RFC 1321 section 3.4: T[i] = floor(2^32 * |sin(i + 1)|) and the per-round
// shift amounts.
struct Md5Tables {
  uint32_t t[64];
  Md5Tables() {
    for (int i = 0; i < 64; i++) t[i] = uint32_t(std::floor(std::fabs(std::sin(double(i + 1))) * 4294967296.0));
  }
};
const Md5Tables kMd5;
const int kShift[4][4] = {{7, 12, 17, 22}, {5, 9, 14, 20}, {4, 11, 16, 23}, {6, 10, 15, 21}};

inline uint32_t rotl(uint32_t x, int c) { return (x << c) | (x >> (32 - c)); }

class Md5 {
 public:
  void update(const uint8_t* p, size_t n) {
    len_ += n;
    if (fill_) {
      const size_t take = n < 64 - fill_ ? n : 64 - fill_;
      std::memcpy(buf_ + fill_, p, take);
      fill_ += take;
      p += take;
      n -= take;
      if (fill_ == 64) {
        block(buf_);
        fill_ = 0;
      }
    }
    for (; n >= 64; p += 64, n -= 64) block(p);
    if (n) {
      std::memcpy(buf_, p, n);
      fill_ = n;
    }
  }
  // RFC 1321 sections 3.1-3.2 and 3.5: pad with 0x80, zeros to 56 mod 64,
  // the message length in bits (64-bit little-endian); the digest is A B C D
  // little-endian.
  void finish(uint8_t out[16]) {
    const uint64_t bits = len_ * 8;
    const uint8_t one = 0x80, zero = 0;
    update(&one, 1);
    while (fill_ != 56) update(&zero, 1);
    uint8_t l[8];
    for (int i = 0; i < 8; i++) l[i] = uint8_t(bits >> (8 * i));
    update(l, 8);
    const uint32_t s[4] = {a_, b_, c_, d_};
    for (int i = 0; i < 4; i++)
      for (int k = 0; k < 4; k++) out[4 * i + k] = uint8_t(s[i] >> (8 * k));
  }

 private:
  // RFC 1321 section 3.4: the four rounds of 16 operations on one block.
  void block(const uint8_t* p) {
    uint32_t x[16];
    for (int i = 0; i < 16; i++)
      x[i] = uint32_t(p[4 * i]) | uint32_t(p[4 * i + 1]) << 8 | uint32_t(p[4 * i + 2]) << 16 |
             uint32_t(p[4 * i + 3]) << 24;
    uint32_t a = a_, b = b_, c = c_, d = d_;
    for (int i = 0; i < 64; i++) {
      uint32_t f;
      int g;
      if (i < 16) {
        f = (b & c) | (~b & d);
        g = i;
      } else if (i < 32) {
        f = (b & d) | (c & ~d);
        g = (5 * i + 1) & 15;
      } else if (i < 48) {
        f = b ^ c ^ d;
        g = (3 * i + 5) & 15;
      } else {
        f = c ^ (b | ~d);
        g = (7 * i) & 15;
      }
      const uint32_t nb = b + rotl(a + f + kMd5.t[i] + x[g], kShift[i >> 4][i & 3]);
      a = d;
      d = c;
      c = b;
      b = nb;
    }
    a_ += a;
    b_ += b;
    c_ += c;
    d_ += d;
  }
  uint32_t a_ = 0x67452301u, b_ = 0xefcdab89u, c_ = 0x98badcfeu, d_ = 0x10325476u;
  uint8_t buf_[64];
  size_t fill_ = 0;
  uint64_t len_ = 0;
};

}  // namespace

extern "C" {

int av1pf_md5(const uint8_t* data, size_t n, char md5_hex[33]) {
  if ((!data && n) || !md5_hex) return AV1PF_ERR_INVALID_INPUT;
  Md5 m;
  if (n) m.update(data, n);
  uint8_t dg[16];
  m.finish(dg);
  for (int i = 0; i < 16; i++) std::snprintf(md5_hex + 2 * i, 3, "%02x", dg[i]);
  return AV1PF_OK;
}

int av1pf_frame_md5(const av1pf_frame_info* info, const uint8_t* frame, char md5_hex[33]) {
  std::string why;
  if (!frame || !md5_hex || av1pf::validate_frame(info, nullptr, nullptr, &why) != AV1PF_OK)
    return AV1PF_ERR_INVALID_INPUT;
  Md5 m;
  m.update(frame, av1pf_frame_bytes(info));
  if (info->num_planes == 1) {
    // a monochrome frame is hashed with neutral chroma, as a 4:2:0 file
    // carries it
    const size_t cw = size_t(info->upscaled_width + 1) / 2, ch = size_t(info->frame_height + 1) / 2;
    const bool wide = info->bit_depth > 8;
    const uint32_t mid = 1u << (info->bit_depth - 1);
    std::vector<uint8_t> plane(cw * ch * (wide ? 2 : 1));
    for (size_t i = 0; i < cw * ch; i++) {
      if (wide) {
        plane[2 * i] = uint8_t(mid & 0xff);
        plane[2 * i + 1] = uint8_t(mid >> 8);
      } else {
        plane[i] = uint8_t(mid);
      }
    }
    m.update(plane.data(), plane.size());
    m.update(plane.data(), plane.size());
  }
  uint8_t dg[16];
  m.finish(dg);
  for (int i = 0; i < 16; i++) std::snprintf(md5_hex + 2 * i, 3, "%02x", dg[i]);
  return AV1PF_OK;
}

}  // extern "C"
