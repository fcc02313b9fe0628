// Test-infrastructure shim for Kokkos::Random_XorShift64_Pool.  Only the API is
// reproduced (get_state / free_state / drand); the generator is a project-written
// splitmix64-seeded xorshift64* stream per OpenMP thread, so its draws do NOT
// match real Kokkos.  RNG-dependent reference outputs are therefore compared in
// distribution, never draw for draw.
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "Kokkos_Core.hpp"

namespace Kokkos {

namespace shim_detail {
inline std::uint64_t splitmix64(std::uint64_t& x) {
    std::uint64_t z = (x += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
}  // namespace shim_detail

class ShimXorShiftState {
public:
    explicit ShimXorShiftState(std::uint64_t* slot) : slot_(slot), s_(*slot) {}
    std::uint64_t urand64() {
        s_ ^= s_ >> 12;
        s_ ^= s_ << 25;
        s_ ^= s_ >> 27;
        return s_ * 0x2545F4914F6CDD1DULL;
    }
    double drand() { return static_cast<double>(urand64() >> 11) * (1.0 / 9007199254740992.0); }
    double drand(double lo, double hi) { return lo + (hi - lo) * drand(); }
    std::uint64_t* slot_;
    std::uint64_t s_;
};

template <class Space = DefaultExecutionSpace>
class Random_XorShift64_Pool {
public:
    Random_XorShift64_Pool() : Random_XorShift64_Pool(0) {}
    explicit Random_XorShift64_Pool(std::uint64_t seed) {
        int threads = 1;
#ifdef _OPENMP
        threads = omp_get_max_threads();
#endif
        states_ = std::make_shared<std::vector<std::uint64_t>>(static_cast<std::size_t>(threads));
        std::uint64_t x = seed;
        for (auto& s : *states_) {
            s = shim_detail::splitmix64(x);
            if (s == 0) s = 0x9E3779B97F4A7C15ULL;
        }
    }
    ShimXorShiftState get_state() const {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        return ShimXorShiftState(&(*states_)[static_cast<std::size_t>(t) % states_->size()]);
    }
    void free_state(const ShimXorShiftState& state) const { *state.slot_ = state.s_; }

private:
    std::shared_ptr<std::vector<std::uint64_t>> states_;
};

}  // namespace Kokkos
