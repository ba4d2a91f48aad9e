// Generates powf_quarter_table.inc: where the C library's powf(x, 0.25f)
// differs from the correctly rounded x^(1/4), for every positive finite float.
//
// The C library's powf is not correctly rounded: it evaluates x^y in double
// and rounds that to float, so where the exact x^(1/4) lies very close to a
// midpoint between two floats it can land one ulp away from the correctly
// rounded value. Multiplying x by 16 multiplies x^(1/4) by exactly 2, and the
// library's result follows it almost everywhere, so the differences are
// listed once per class (unbiased exponent mod 4, 23-bit mantissa) from the
// four binades [2^-3, 2), and the few inputs elsewhere that break the period
// are listed exactly. powf_quarter.cuh applies the table to the correctly
// rounded value (double square root twice, rounded once to float).
//
// Build and run on the machine whose C library the reference uses:
//   g++ -O2 -ffp-contract=off -o gen vapor_b200/csrc/gen_powf_quarter.cpp
//   ./gen > vapor_b200/csrc/powf_quarter_table.inc
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

namespace {
float bits_to_float(uint32_t b) {
    float x;
    std::memcpy(&x, &b, 4);
    return x;
}
uint32_t float_to_bits(float x) {
    uint32_t b;
    std::memcpy(&b, &x, 4);
    return b;
}
float rounded_quarter(float x) { return float(std::sqrt(std::sqrt(double(x)))); }
// (unbiased exponent mod 4) << 23 | mantissa, for a positive finite x.
uint32_t period_class(uint32_t b) {
    int e = int(b >> 23);
    uint32_t m = b & 0x7FFFFFu;
    if (e == 0) {  // subnormal: normalise
        int shift = 0;
        while (!(m & 0x800000u)) {
            m <<= 1;
            ++shift;
        }
        m &= 0x7FFFFFu;
        e = 1 - shift;
    }
    return (uint32_t((e - 127) & 3) << 23) | m;
}
}  // namespace

int main() {
    std::vector<int8_t> step(size_t(4) << 23, 0);
    std::vector<uint32_t> periodic;
    for (uint32_t b = 124u << 23; b < 128u << 23; ++b) {
        const float x = bits_to_float(b), lib = std::pow(x, 0.25f), cr = rounded_quarter(x);
        if (lib == cr) continue;
        const int up = lib > cr ? 1 : 0;
        if (lib != std::nextafter(cr, up ? INFINITY : 0.f)) {
            std::fprintf(stderr, "difference of more than one ulp at %a\n", double(x));
            return 1;
        }
        step[period_class(b)] = int8_t(up ? 1 : -1);
    }
    for (uint32_t c = 0; c < (4u << 23); ++c)
        if (step[c]) periodic.push_back((c << 1) | (step[c] > 0 ? 1u : 0u));
    std::vector<uint32_t> exact_in, exact_out;
    for (uint32_t b = 1; b < 0x7F800000u; ++b) {
        const float x = bits_to_float(b), lib = std::pow(x, 0.25f), cr = rounded_quarter(x);
        const int8_t s = step[period_class(b)];
        const float predicted = s ? std::nextafter(cr, s > 0 ? INFINITY : 0.f) : cr;
        if (float_to_bits(predicted) != float_to_bits(lib)) {
            exact_in.push_back(b);
            exact_out.push_back(float_to_bits(lib));
        }
    }
    std::printf("// Generated by gen_powf_quarter.cpp from the C library's powf(x, 0.25f).\n");
    std::printf("// kQuarterPeriodic: (class << 1) | up, sorted; class = (exponent mod 4) << 23 | mantissa.\n");
    std::printf("// kQuarterExactIn / kQuarterExactOut: inputs outside the period and their results.\n");
    std::printf("VB_POWQ_TABLE uint32_t kQuarterPeriodic[%zu] = {\n", periodic.size());
    for (size_t i = 0; i < periodic.size(); ++i)
        std::printf("%s0x%07x,%s", i % 10 ? " " : "    ", periodic[i], i % 10 == 9 ? "\n" : "");
    std::printf("%s};\nconstexpr int kQuarterPeriodicCount = %zu;\n", periodic.size() % 10 ? "\n" : "",
                periodic.size());
    std::printf("VB_POWQ_TABLE uint32_t kQuarterExactIn[%zu] = {\n", exact_in.size());
    for (size_t i = 0; i < exact_in.size(); ++i)
        std::printf("%s0x%08x,%s", i % 8 ? " " : "    ", exact_in[i], i % 8 == 7 ? "\n" : "");
    std::printf("%s};\nVB_POWQ_TABLE uint32_t kQuarterExactOut[%zu] = {\n", exact_in.size() % 8 ? "\n" : "",
                exact_out.size());
    for (size_t i = 0; i < exact_out.size(); ++i)
        std::printf("%s0x%08x,%s", i % 8 ? " " : "    ", exact_out[i], i % 8 == 7 ? "\n" : "");
    std::printf("%s};\nconstexpr int kQuarterExactCount = %zu;\n", exact_out.size() % 8 ? "\n" : "",
                exact_in.size());
    return 0;
}
