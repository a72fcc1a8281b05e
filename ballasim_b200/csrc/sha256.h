// SHA-256 (FIPS 180-4) of byte strings as lower-case hex: the event files' digests (the reference's config::Sha256,
// src/config/sha256.h). Host only; the blocks run on the x86 SHA extensions where the CPU has them.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

namespace bs {

class Sha256 {
 public:
  Sha256();
  void update(const void* data, size_t n);
  std::string hex();  // the padding, then the digest; once

 private:
  void blocks(const uint8_t* p, size_t n);
  uint32_t h_[8];
  uint8_t buf_[64];
  size_t fill_ = 0;
  uint64_t bytes_ = 0;
};

}  // namespace bs
