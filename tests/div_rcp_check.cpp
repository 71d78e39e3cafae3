// Host check of sw2d::div_rcp (csrc/sp_math.cuh): the quotient from a shared reciprocal must have
// the bits of the IEEE division a / b for every input.  Built by tests/test_div_rcp.py with
// g++ -ffp-contract=off; prints "<case> <samples> <mismatches>" per input family.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "sp_math.cuh"

namespace {

uint64_t g_state = 0x9e3779b97f4a7c15ull;

uint64_t next_u64()  // splitmix64
{
    uint64_t z = (g_state += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

double from_bits(uint64_t u)
{
    double d;
    std::memcpy(&d, &u, sizeof d);
    return d;
}

uint64_t to_bits(double d)
{
    uint64_t u;
    std::memcpy(&u, &d, sizeof u);
    return u;
}

// a double with a random significand, the given unbiased exponent and a random sign
double with_exp(int e, bool random_sign = true)
{
    const uint64_t mant = next_u64() & 0xfffffffffffffull;
    const uint64_t sign = random_sign ? (next_u64() & 1ull) << 63 : 0ull;
    return from_bits(sign | ((uint64_t)(e + 1023) << 52) | mant);
}

int uniform_int(int lo, int hi) { return lo + (int)(next_u64() % (uint64_t)(hi - lo + 1)); }

double uniform(double lo, double hi) { return lo + (hi - lo) * ((next_u64() >> 11) * 0x1p-53); }

struct Count {
    long long n = 0, bad = 0;
};

void check(Count& c, double a, double b)
{
    const double y = 1.0 / b;
    const double got = sw2d::div_rcp(a, b, y);
    const double want = a / b;
    c.n++;
    const bool same = (std::isnan(got) && std::isnan(want)) || to_bits(got) == to_bits(want);
    if (!same) {
        if (c.bad < 5) std::fprintf(stderr, "mismatch a=%a b=%a got=%a want=%a\n", a, b, got, want);
        c.bad++;
    }
}

void report(const char* name, const Count& c) { std::printf("%s %lld %lld\n", name, c.n, c.bad); }

}  // namespace

int main()
{
    {  // random significands, wide exponent ranges
        Count c;
        for (int i = 0; i < 8000000; i++) check(c, with_exp(uniform_int(-800, 800)), with_exp(uniform_int(-59, 59), false));
        report("random_wide", c);
    }
    {  // the slope arithmetic: (zj - zc) dx over mesh distances, and sums of weights
        Count c;
        for (int i = 0; i < 8000000; i++) {
            const double dz = uniform(-5.0, 5.0) * std::pow(10.0, uniform_int(-12, 0));
            const double dx = uniform(-200.0, 200.0);
            const double dist = std::sqrt(dx * dx + uniform(0.0, 200.0) * uniform(0.0, 200.0)) + 1e-3;
            check(c, dz * dx, dist);
            check(c, dz * dx / dist, dist);
            check(c, uniform(-1.0, 1.0), uniform(1e-3, 1e4));
        }
        report("mesh_like", c);
    }
    {  // divisors with significands near 1 and near 2 (all ones), and powers of two
        Count c;
        for (int i = 0; i < 2000000; i++) {
            const uint64_t k = next_u64() & 0xffffull;
            const int e = uniform_int(-40, 40);
            const double b_hi = from_bits(((uint64_t)(e + 1023) << 52) | (0xfffffffffffffull - k));
            const double b_lo = from_bits(((uint64_t)(e + 1023) << 52) | k);
            const double a = with_exp(uniform_int(-500, 500));
            check(c, a, b_hi);
            check(c, a, b_lo);
            check(c, a, std::ldexp(1.0, e));
        }
        report("divisor_edges", c);
    }
    {  // quotients near the midpoint between two doubles (the hard rounding cases): a = RN(m b)
       // for m a midpoint of two neighbouring doubles, and its neighbours
        Count c;
        for (int i = 0; i < 4000000; i++) {
            const double q = with_exp(uniform_int(-300, 300));
            const double mid = q + (std::nextafter(q, 2.0 * q) - q) * 0.5;  // rounds to one side
            const double b = with_exp(uniform_int(-50, 50), false);
            const double a = mid * b;
            check(c, a, b);
            check(c, std::nextafter(a, 0.0), b);
            check(c, std::nextafter(a, 2.0 * a), b);
            check(c, q * b, b);
        }
        report("midpoints", c);
    }
    {  // special values: zeros of both signs, subnormal and huge numerators, infinities, NaN
        Count c;
        const double specials[] = {0.0, -0.0, 5e-324, -5e-324, 0x1p-1022, 0x1p-960, 0x1p-901, 0x1p-899, 0x1p+899,
                                   0x1p+901, 1.7976931348623157e308, -1.7976931348623157e308, INFINITY, -INFINITY,
                                   NAN, 1.0, -1.0, 3.0};
        for (double a : specials)
            for (int i = 0; i < 2000; i++) check(c, a, with_exp(uniform_int(-59, 59), false));
        report("specials", c);
    }
    return 0;
}
