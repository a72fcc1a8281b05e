// SHA-256 (FIPS 180-4). The round constants are the first 32 bits of the fractional parts of the cube roots of the
// first 64 primes, the initial hash those of the square roots of the first 8, computed here in integer arithmetic.
// The compression function runs on the x86 SHA extensions (SHA256RNDS2 / MSG1 / MSG2, two rounds per instruction
// on the state split into ABEF and CDGH) when CPUID reports them, else in portable code.
#include "sha256.h"

#include <cpuid.h>
#include <immintrin.h>

#include <cstring>

namespace bs {
namespace {

struct Tables {
  uint32_t k[64], h0[8];
  Tables() {
    int primes[64], n = 0;
    for (int c = 2; n < 64; ++c) {
      bool prime = true;
      for (int d = 2; d * d <= c; ++d) prime = prime && c % d != 0;
      if (prime) primes[n++] = c;
    }
    // floor(root(p) 2^32) mod 2^32 from the integer root of p 2^96 (cube) or p 2^64 (square).
    for (int i = 0; i < 64; ++i) k[i] = static_cast<uint32_t>(iroot(static_cast<unsigned __int128>(primes[i]) << 96, 3));
    for (int i = 0; i < 8; ++i) h0[i] = static_cast<uint32_t>(iroot(static_cast<unsigned __int128>(primes[i]) << 64, 2));
  }
  static uint64_t iroot(unsigned __int128 v, int e) {
    uint64_t lo = 0, hi = uint64_t{1} << 40;
    while (hi - lo > 1) {
      const uint64_t m = lo + (hi - lo) / 2;
      unsigned __int128 p = m;
      for (int j = 1; j < e; ++j) p *= m;
      (p <= v ? lo : hi) = m;
    }
    return lo;
  }
};

const Tables& tables() {
  static const Tables t;
  return t;
}

bool have_sha_ni() {
  unsigned a = 0, b = 0, c = 0, d = 0;
  if (!__get_cpuid(1, &a, &b, &c, &d)) return false;
  const bool ssse3 = (c >> 9) & 1, sse41 = (c >> 19) & 1;
  if (!__get_cpuid_count(7, 0, &a, &b, &c, &d)) return false;
  return ssse3 && sse41 && ((b >> 29) & 1);
}

inline uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

void blocks_portable(uint32_t* h, const uint32_t* k, const uint8_t* p, size_t n) {
  for (; n > 0; --n, p += 64) {
    uint32_t w[64];
    for (int i = 0; i < 16; ++i) {
      w[i] = (uint32_t{p[4 * i]} << 24) | (uint32_t{p[4 * i + 1]} << 16) | (uint32_t{p[4 * i + 2]} << 8) | p[4 * i + 3];
    }
    for (int i = 16; i < 64; ++i) {
      const uint32_t s0 = rotr(w[i - 15], 7) ^ rotr(w[i - 15], 18) ^ (w[i - 15] >> 3);
      const uint32_t s1 = rotr(w[i - 2], 17) ^ rotr(w[i - 2], 19) ^ (w[i - 2] >> 10);
      w[i] = w[i - 16] + s0 + w[i - 7] + s1;
    }
    uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
    for (int i = 0; i < 64; ++i) {
      const uint32_t t1 = hh + (rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25)) + ((e & f) ^ (~e & g)) + k[i] + w[i];
      const uint32_t t2 = (rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
      hh = g;
      g = f;
      f = e;
      e = d + t1;
      d = c;
      c = b;
      b = a;
      a = t1 + t2;
    }
    h[0] += a;
    h[1] += b;
    h[2] += c;
    h[3] += d;
    h[4] += e;
    h[5] += f;
    h[6] += g;
    h[7] += hh;
  }
}

// The 64 rounds as 16 groups of 4: group g adds K[4g..4g+3] to its message words and runs two SHA256RNDS2; the
// schedule keeps the next words in four registers, m[(g + 1) % 4] finished by MSG2 in group g (3 <= g <= 14) and
// m[(g + 3) % 4] started by MSG1 (1 <= g <= 12).
__attribute__((target("sha,sse4.1,ssse3"))) void blocks_ni(uint32_t* h, const uint32_t* k, const uint8_t* p,
                                                           size_t n) {
  const __m128i swap = _mm_set_epi64x(0x0c0d0e0f08090a0bLL, 0x0405060700010203LL);
  __m128i t = _mm_shuffle_epi32(_mm_loadu_si128(reinterpret_cast<const __m128i*>(h)), 0xB1);      // C D A B
  __m128i s1 = _mm_shuffle_epi32(_mm_loadu_si128(reinterpret_cast<const __m128i*>(h + 4)), 0x1B);  // E F G H
  __m128i s0 = _mm_alignr_epi8(t, s1, 8);                                                           // A B E F
  s1 = _mm_blend_epi16(s1, t, 0xF0);                                                                // C D G H
  for (; n > 0; --n, p += 64) {
    const __m128i save0 = s0, save1 = s1;
    __m128i m[4];
#pragma GCC unroll 16
    for (int g = 0; g < 16; ++g) {
      if (g < 4) m[g] = _mm_shuffle_epi8(_mm_loadu_si128(reinterpret_cast<const __m128i*>(p + 16 * g)), swap);
      __m128i w = _mm_add_epi32(m[g & 3], _mm_loadu_si128(reinterpret_cast<const __m128i*>(k + 4 * g)));
      s1 = _mm_sha256rnds2_epu32(s1, s0, w);
      if (g >= 3 && g <= 14) {
        const __m128i x = _mm_alignr_epi8(m[g & 3], m[(g + 3) & 3], 4);
        m[(g + 1) & 3] = _mm_sha256msg2_epu32(_mm_add_epi32(m[(g + 1) & 3], x), m[g & 3]);
      }
      w = _mm_shuffle_epi32(w, 0x0E);
      s0 = _mm_sha256rnds2_epu32(s0, s1, w);
      if (g >= 1 && g <= 12) m[(g + 3) & 3] = _mm_sha256msg1_epu32(m[(g + 3) & 3], m[g & 3]);
    }
    s0 = _mm_add_epi32(s0, save0);
    s1 = _mm_add_epi32(s1, save1);
  }
  t = _mm_shuffle_epi32(s0, 0x1B);           // F E B A
  s1 = _mm_shuffle_epi32(s1, 0xB1);          // D C H G
  s0 = _mm_blend_epi16(t, s1, 0xF0);         // D C B A
  s1 = _mm_alignr_epi8(s1, t, 8);            // H G F E
  _mm_storeu_si128(reinterpret_cast<__m128i*>(h), s0);
  _mm_storeu_si128(reinterpret_cast<__m128i*>(h + 4), s1);
}

}  // namespace

Sha256::Sha256() { std::memcpy(h_, tables().h0, sizeof h_); }

void Sha256::blocks(const uint8_t* p, size_t n) {
  static const bool ni = have_sha_ni();
  if (ni) {
    blocks_ni(h_, tables().k, p, n);
  } else {
    blocks_portable(h_, tables().k, p, n);
  }
}

void Sha256::update(const void* data, size_t n) {
  const auto* p = static_cast<const uint8_t*>(data);
  bytes_ += n;
  if (fill_ > 0) {
    const size_t take = n < 64 - fill_ ? n : 64 - fill_;
    std::memcpy(buf_ + fill_, p, take);
    fill_ += take;
    p += take;
    n -= take;
    if (fill_ < 64) return;
    blocks(buf_, 1);
    fill_ = 0;
  }
  if (n >= 64) {
    blocks(p, n / 64);
    p += n / 64 * 64;
    n %= 64;
  }
  std::memcpy(buf_, p, n);
  fill_ = n;
}

std::string Sha256::hex() {
  const uint64_t bits = bytes_ * 8;
  uint8_t pad[72] = {0x80};
  const size_t zeros = (fill_ < 56 ? 56 - fill_ : 120 - fill_) - 1;
  for (int i = 0; i < 8; ++i) pad[1 + zeros + i] = static_cast<uint8_t>(bits >> (56 - 8 * i));
  update(pad, 1 + zeros + 8);
  static const char* digits = "0123456789abcdef";
  std::string out;
  for (int i = 0; i < 8; ++i) {
    for (int s = 28; s >= 0; s -= 4) out.push_back(digits[(h_[i] >> s) & 15]);
  }
  return out;
}

}  // namespace bs
