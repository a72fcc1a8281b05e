// Exhaustive check that bs::log_f (ballasim_b200/csrc/bs_math.cuh) is monotone non-decreasing over every positive
// float (denormals included), which the crossing search's exact node test relies on. Prints the number of drops.
#include <atomic>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include "bs_math.cuh"

int main() {
  const unsigned first = 1u, last = 0x7f800000u;  // (0, +inf)
  const unsigned n_threads = std::max(1u, std::thread::hardware_concurrency());
  std::atomic<long long> drops{0};
  std::vector<std::thread> pool;
  const unsigned chunk = (last - first) / n_threads + 1;
  for (unsigned k = 0; k < n_threads; ++k) {
    pool.emplace_back([&, k] {
      const unsigned a = first + k * chunk, b = std::min(last, a + chunk);
      if (a >= b) return;
      float x;
      unsigned u = a - 1 < first ? a : a - 1;  // overlap one value with the previous chunk
      std::memcpy(&x, &u, 4);
      float prev = bs::log_f(x);
      long long d = 0;
      for (++u; u < b; ++u) {
        std::memcpy(&x, &u, 4);
        const float y = bs::log_f(x);
        if (y < prev) ++d;
        prev = y;
      }
      drops += d;
    });
  }
  for (auto& t : pool) t.join();
  std::printf("%lld\n", drops.load());
  return 0;
}
