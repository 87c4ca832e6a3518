// Kokkos_Random.hpp — host stand-in for Kokkos::Random_XorShift64_Pool (the
// reference draws l-mer priorities from it; its unitigs do not depend on them).
// TEST INFRASTRUCTURE ONLY.
#pragma once
#include <cstdint>
#include <vector>

#include "Kokkos_Core.hpp"

namespace Kokkos {

struct Random_XorShift64 {
  uint64_t s;
  uint64_t urand64() {
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    return s;
  }
  uint32_t urand() { return static_cast<uint32_t>(urand64() >> 32); }
  int tid;
};

template <class D = Device<DefaultExecutionSpace, HostSpace>>
class Random_XorShift64_Pool {
 public:
  using generator_type = Random_XorShift64;
  Random_XorShift64_Pool() : Random_XorShift64_Pool(1) {}
  explicit Random_XorShift64_Pool(uint64_t seed) {
    if (const char* e = std::getenv("KSHIM_SEED")) seed = std::strtoull(e, nullptr, 10);
    states_ = std::make_shared<std::vector<uint64_t>>(shim_threads() + 1);
    for (std::size_t i = 0; i < states_->size(); ++i) {
      uint64_t z = seed + 0x9E3779B97F4A7C15ull * (i + 1);
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      (*states_)[i] = (z ^ (z >> 31)) | 1ull;
    }
  }
  generator_type get_state() const {
    const int t = shim_thread_id();
    return generator_type{(*states_)[t], t};
  }
  void free_state(const generator_type& g) const { (*states_)[g.tid] = g.s; }

 private:
  std::shared_ptr<std::vector<uint64_t>> states_;
};

}  // namespace Kokkos
