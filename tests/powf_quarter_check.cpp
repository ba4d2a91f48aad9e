// TEST INFRASTRUCTURE: checks vb::powf_quarter (the product's device function
// of vapor_b200/csrc/powf_quarter.cuh, compiled here for the host) against the
// C library's powf(x, 0.25f) bit for bit on every non-negative float, both
// zeros and infinity, split over the host's threads. Prints the number of
// differences; exits 1 on any.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include "../vapor_b200/csrc/powf_quarter.cuh"

int main() {
    std::atomic<unsigned long long> bad{0}, adjusted{0};
    const uint64_t end = uint64_t(0x7F800000u) + 1;
    const unsigned threads = std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < threads; ++t)
        pool.emplace_back([&, t] {
            unsigned long long my_bad = 0, my_adjusted = 0;
            for (uint64_t b = end * t / threads; b < end * (t + 1) / threads; ++b) {
                float x;
                const uint32_t bb = uint32_t(b);
                std::memcpy(&x, &bb, 4);
                const float want = std::pow(x, 0.25f), got = vb::powf_quarter(x);
                if (std::memcmp(&want, &got, 4)) {
                    if (my_bad < 3) std::printf("x=%a powf=%a got=%a\n", double(x), double(want), double(got));
                    ++my_bad;
                }
                if (got != float(std::sqrt(std::sqrt(double(x))))) ++my_adjusted;
            }
            bad += my_bad;
            adjusted += my_adjusted;
        });
    for (auto& th : pool) th.join();
    const float nz = -0.f, got = vb::powf_quarter(nz), want = std::pow(nz, 0.25f);
    if (std::memcmp(&want, &got, 4)) ++bad;
    std::printf("differences %llu, inputs away from the correctly rounded root %llu\n", bad.load(), adjusted.load());
    return bad ? 1 : 0;
}
