// FP64 arithmetic, random streams and boundary maps shared by host and device code.
//
// Every FP64 operation on the decision path is spelled with an explicit IEEE
// round-to-nearest intrinsic on the device (__dadd_rn, __dmul_rn, __fma_rn, ...), so
// that nvcc never contracts a product and a sum into an FMA where the reference's Rust
// code rounds twice, and uses __fma_rn exactly where the reference calls f64::mul_add.
// The host side of this file is compiled with -ffp-contract=off for the same reason.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#ifdef __CUDACC__
#define HMC_HD __host__ __device__ __forceinline__
#else
#define HMC_HD inline
#endif

namespace hmc {

// ---- exact FP64 operations -------------------------------------------------------------
HMC_HD double dadd(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dadd_rn(a, b);
#else
    return a + b;
#endif
}
HMC_HD double dsub(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dsub_rn(a, b);
#else
    return a - b;
#endif
}
HMC_HD double dmul(double a, double b) {
#ifdef __CUDA_ARCH__
    return __dmul_rn(a, b);
#else
    return a * b;
#endif
}
HMC_HD double ddiv(double a, double b) {
#ifdef __CUDA_ARCH__
    return __ddiv_rn(a, b);
#else
    return a / b;
#endif
}
HMC_HD double dfma(double a, double b, double c) {
#ifdef __CUDA_ARCH__
    return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
HMC_HD double dsqrt(double a) {
#ifdef __CUDA_ARCH__
    return __dsqrt_rn(a);
#else
    return std::sqrt(a);
#endif
}
HMC_HD double as_double(uint64_t b) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double((long long)b);
#else
    double d;
    std::memcpy(&d, &b, 8);
    return d;
#endif
}
HMC_HD uint64_t as_bits(double d) {
#ifdef __CUDA_ARCH__
    return (uint64_t)__double_as_longlong(d);
#else
    uint64_t b;
    std::memcpy(&b, &d, 8);
    return b;
#endif
}

// ---- hoomd-rand SFC64 (sfc.rs:62-86) and Counter::make_rng (counter.rs:160-167) ----------
struct Sfc64 {
    uint64_t s0, s1, s2, ctr;
    HMC_HD uint64_t next_u64() {
        uint64_t out = s0 + s1 + ctr;
        s0 = s1 ^ (s1 >> 11);
        s1 = s2 + (s2 << 3);
        s2 = ((s2 << 24) | (s2 >> 40)) + out;
        ctr += 1;
        return out;
    }
    HMC_HD uint32_t next_u32() { return (uint32_t)next_u64(); }
};
HMC_HD Sfc64 make_rng(uint64_t step, uint32_t substep, uint32_t seed, uint64_t index) {
    Sfc64 r{step, ((uint64_t)substep << 32) | (uint64_t)seed, index, 0};
#pragma unroll
    for (int i = 0; i < 12; ++i) r.next_u64();
    return r;
}

// f64 in [0, 1): 53 high bits times 2^-53 (rand's StandardUniform for f64).
HMC_HD double uniform01(Sfc64& r) { return dmul((double)(r.next_u64() >> 11), 1.0 / 9007199254740992.0); }
// f64 in (0, 1): 52 bits as the mantissa of [1, 2) minus (1 - 2^-53) (rand's Open01).
HMC_HD double open01(Sfc64& r) {
    uint64_t b = r.next_u64() >> 12;
    return dsub(as_double(0x3FF0000000000000ULL | b), 1.0 - 1.0 / 9007199254740992.0);
}
// Integer in [0, range) by Canon's widening-multiply method with one refinement draw
// (rand's UniformInt<u32>::sample_single, used by IndexedRandom::choose).
HMC_HD uint32_t canon_range_u32(Sfc64& r, uint32_t range) {
    uint64_t m = (uint64_t)r.next_u32() * (uint64_t)range;
    uint32_t result = (uint32_t)(m >> 32);
    uint32_t lo = (uint32_t)m;
    if (lo > (uint32_t)(0u - range)) {
        uint64_t m2 = (uint64_t)r.next_u32() * (uint64_t)range;
        uint32_t hi2 = (uint32_t)(m2 >> 32);
        if ((uint32_t)(lo + hi2) < lo) result += 1;
    }
    return result;
}

// ---- standard normal: 256-layer ziggurat (Marsaglia & Tsang 2000, ZIGNOR form of
// Doornik 2005). Tables are computed on the host at context creation (see zig_tables)
// and read from global memory on the device.
constexpr int kZigLayers = 256;
constexpr double kZigR = 3.6541528853610088;
constexpr double kZigV = 0.00492867323399;

struct ZigTables {
    double x[kZigLayers + 1];
    double f[kZigLayers + 1];
};
inline void zig_tables(ZigTables& t) {
    auto pdf = [](double v) { return std::exp(-v * v / 2.0); };
    t.x[0] = kZigV / pdf(kZigR);
    t.x[1] = kZigR;
    for (int i = 2; i < kZigLayers; ++i) t.x[i] = std::sqrt(-2.0 * std::log(kZigV / t.x[i - 1] + pdf(t.x[i - 1])));
    t.x[kZigLayers] = 0.0;
    for (int i = 0; i <= kZigLayers; ++i) t.f[i] = pdf(t.x[i]);
}

HMC_HD double lib_exp(double v) {
#ifdef __CUDA_ARCH__
    return exp(v);
#else
    return std::exp(v);
#endif
}
HMC_HD double lib_log(double v) {
#ifdef __CUDA_ARCH__
    return log(v);
#else
    return std::log(v);
#endif
}

HMC_HD double standard_normal(Sfc64& r, const double* __restrict__ zx, const double* __restrict__ zf) {
    for (;;) {
        uint64_t bits = r.next_u64();
        int i = (int)(bits & 0xff);
        double u = dsub(as_double(0x4000000000000000ULL | (bits >> 12)), 3.0);
        double x = dmul(u, zx[i]);
        if (fabs(x) < zx[i + 1]) return x;
        if (i == 0) {
            double xt = 1.0, y = 0.0;
            while (dmul(-2.0, y) < dmul(xt, xt)) {
                double a = open01(r);
                double b = open01(r);
                xt = ddiv(lib_log(a), kZigR);
                y = lib_log(b);
            }
            return u < 0.0 ? dsub(xt, kZigR) : dsub(kZigR, xt);
        }
        double w = dadd(zf[i + 1], dmul(dsub(zf[i], zf[i + 1]), uniform01(r)));
        if (w < lib_exp(ddiv(dmul(-x, x), 2.0))) return x;
    }
}

// ---- deterministic cube root and half-angle sin/cos -------------------------------------
// Cube root without division: x = m 2^(3q + r) with m in [1, 2); y ~ m^(-1/3) from a
// quadratic Chebyshev fit refined by three Newton steps y += y (1 - m y^3) / 3; then
// cbrt(x) ~ m y^2 cbrt(2^r) 2^q, corrected once by a Newton step on the FMA-evaluated
// residual c^3 - m 2^r. Only correctly rounded operations (mul, fma), so host and device
// agree bit for bit; the result is within one ulp of the true cube root.
HMC_HD double portable_cbrt(double x) {
    if (x == 0.0 || !(fabs(x) <= 1.79769313486231570e308)) return x;
    const bool neg = x < 0.0;
    double ax = neg ? -x : x;
    int extra = 0;
    if (ax < 2.2250738585072014e-308) {
        ax = dmul(ax, 18014398509481984.0);
        extra = -18;
    }
    const uint64_t b = as_bits(ax);
    const int e = (int)((b >> 52) & 0x7ff) - 1023;
    const double m = as_double((b & 0x000FFFFFFFFFFFFFULL) | 0x3FF0000000000000ULL);
    const int q = (e >= 0) ? e / 3 : -((-e + 2) / 3);
    const int rr = e - 3 * q;
    double y = dfma(dfma(0.09303886055928341, m, -0.48224275792479104), m, 1.387389992245347);
    for (int it = 0; it < 3; ++it) {
        const double y3 = dmul(dmul(y, y), y);
        const double eps = dfma(-m, y3, 1.0);
        y = dfma(dmul(y, eps), 0.3333333333333333, y);
    }
    const double a = dmul(m, rr == 0 ? 1.0 : (rr == 1 ? 2.0 : 4.0));
    const double k = rr == 0 ? 1.0 : (rr == 1 ? 1.2599210498948732 : 1.5874010519681994);
    const double ik2 = rr == 0 ? 0.3333333333333333 : (rr == 1 ? 0.20998684164914552 : 0.13228342099734997);
    double c = dmul(dmul(dmul(m, y), y), k);
    const double c2 = dmul(c, c);
    const double c2lo = dfma(c, c, -c2);
    const double resid = dadd(dfma(c2, c, -a), dmul(c2lo, c));
    c = dsub(c, dmul(resid, dmul(dmul(y, y), ik2)));
    const double scale = as_double((uint64_t)(q + extra + 1023) << 52);
    const double res = dmul(c, scale);
    return neg ? -res : res;
}

// sin(h), cos(h) for 0 <= h <= pi/2: Taylor series in h^2 with FMA Horner steps.
HMC_HD void portable_sincos(double h, double* s, double* c) {
    const double SC[13] = {1.0,
                           -0.16666666666666666,
                           0.008333333333333333,
                           -0.0001984126984126984,
                           2.7557319223985893e-06,
                           -2.505210838544172e-08,
                           1.6059043836821613e-10,
                           -7.647163731819816e-13,
                           2.8114572543455206e-15,
                           -8.22063524662433e-18,
                           1.9572941063391263e-20,
                           -3.868170170630684e-23,
                           6.446950284384474e-26};
    const double CC[13] = {1.0,
                           -0.5,
                           0.041666666666666664,
                           -0.001388888888888889,
                           2.48015873015873e-05,
                           -2.755731922398589e-07,
                           2.08767569878681e-09,
                           -1.1470745597729725e-11,
                           4.779477332387385e-14,
                           -1.5619206968586225e-16,
                           4.110317623312165e-19,
                           -8.896791392450574e-22,
                           1.6117375710961184e-24};
    double h2 = dmul(h, h);
    double ps = SC[12], pc = CC[12];
#pragma unroll
    for (int k = 11; k >= 0; --k) {
        ps = dfma(ps, h2, SC[k]);
        pc = dfma(pc, h2, CC[k]);
    }
    *s = dmul(h, ps);
    *c = pc;
}

// x / d, correctly rounded, for a divisor d fixed per system with precomputed rd = RN(1/d).
// On the device: q = RN(q0 + r rd) with q0 = RN(x rd) and r = x - q0 d (exact by FMA), then
// q is accepted only if the exact residual x - q d proves |x/d - q| below half the spacing of
// doubles around q (a quarter ulp when q is a power of two); otherwise the IEEE division runs.
// The result therefore always equals x / d.
HMC_HD double div_fixed(double x, double d, double rd) {
#ifdef __CUDA_ARCH__
    const double q0 = __dmul_rn(x, rd);
    const double r0 = __fma_rn(-q0, d, x);
    const double q1 = __fma_rn(r0, rd, q0);
    const double r1 = __fma_rn(-q1, d, x);
    const uint64_t bits = (uint64_t)__double_as_longlong(q1);
    const uint32_t ex = (uint32_t)((bits >> 52) & 0x7ffu);
    if (ex > 60u && ex < 1990u) {
        const uint32_t hex = (bits & 0x000FFFFFFFFFFFFFULL) ? ex - 53u : ex - 54u;
        const double h = __longlong_as_double((long long)((uint64_t)hex << 52));
        if (fabs(r1) < __dmul_rn(h, fabs(d))) return q1;
    }
    return __ddiv_rn(x, d);
#else
    (void)rd;
    return x / d;
#endif
}

// ---- hoomd-vector arithmetic -------------------------------------------------------------
// InnerProduct::dot (cartesian.rs:293-296): mul_add fold from 0.0.
template <int N>
HMC_HD double dot(const double* a, const double* b) {
    double p = 0.0;
#pragma unroll
    for (int i = 0; i < N; ++i) p = dfma(a[i], b[i], p);
    return p;
}

// ---- Periodic<Hypercuboid>::wrap (boundary/periodic/cuboid.rs:91-103) ---------------------
template <int N>
HMC_HD void wrap(const double* L, double* x) {
#pragma unroll
    for (int a = 0; a < N; ++a) {
        double lam = ddiv(x[a], L[a]);
        lam = dsub(lam, round(lam));
        if (lam == 0.5) lam = -0.5;
        x[a] = dmul(lam, L[a]);
    }
}

// wrap with the division by the box length done by div_fixed (same result as wrap).
template <int N>
HMC_HD void wrap_inv(const double* L, const double* invL, double* x) {
#pragma unroll
    for (int a = 0; a < N; ++a) {
        double lam = div_fixed(x[a], L[a], invL[a]);
        lam = dsub(lam, round(lam));
        if (lam == 0.5) lam = -0.5;
        x[a] = dmul(lam, L[a]);
    }
}

}  // namespace hmc
