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

// ---- correctly rounded sin and cos ------------------------------------------------------
// Angle -> RotationMatrix (hoomd-vector angle.rs:120-150) calls f64::sin / f64::cos, i.e.
// the platform libm. Host and device use this deterministic method instead; it returns the
// correctly rounded values from correctly rounded +, -, *, fma only:
//  * Cody-Waite reduction x = k pi/2 + r, pi/2 split into 33 + 33 + 33 + 53 bits (products
//    k*C1..k*C3 exact for |k| < 2^20), r as a double-double (error-free transforms of
//    Dekker and Knuth);
//  * Taylor series of sin r and cos r, |r| <= pi/4, leading terms in double-double and the
//    rest in double (relative error below 2^-66); Ziv's rounding test against 2^-62; if it
//    fails, the whole series in double-double (error below 2^-95) decides.
// |x| >= 2^20 is outside the supported range (returns false).
struct DDouble {
    double h, l;
};
HMC_HD DDouble dd_two_sum(double a, double b) {
    const double s = dadd(a, b);
    const double bb = dsub(s, a);
    return {s, dadd(dsub(a, dsub(s, bb)), dsub(b, bb))};
}
HMC_HD DDouble dd_fast_sum(double a, double b) {  // |a| >= |b|
    const double s = dadd(a, b);
    return {s, dsub(b, dsub(s, a))};
}
HMC_HD DDouble dd_mul(DDouble a, DDouble b) {
    const double p = dmul(a.h, b.h);
    double e = dfma(a.h, b.h, -p);
    e = dfma(a.h, b.l, e);
    e = dfma(a.l, b.h, e);
    return dd_fast_sum(p, e);
}
HMC_HD DDouble dd_add(DDouble a, DDouble b) {
    const DDouble s = dd_two_sum(a.h, b.h);
    return dd_fast_sum(s.h, dadd(s.l, dadd(a.l, b.l)));
}
// (-1)^(k/2) / k!, k = 2..27, as double-doubles (the exact rationals rounded twice).
HMC_HD constexpr double inv_fact_hi(int k) {
    switch (k) {
        case 2: return -0x1.0000000000000p-1;
        case 3: return -0x1.5555555555555p-3;
        case 4: return 0x1.5555555555555p-5;
        case 5: return 0x1.1111111111111p-7;
        case 6: return -0x1.6c16c16c16c17p-10;
        case 7: return -0x1.a01a01a01a01ap-13;
        case 8: return 0x1.a01a01a01a01ap-16;
        case 9: return 0x1.71de3a556c734p-19;
        case 10: return -0x1.27e4fb7789f5cp-22;
        case 11: return -0x1.ae64567f544e4p-26;
        case 12: return 0x1.1eed8eff8d898p-29;
        case 13: return 0x1.6124613a86d09p-33;
        case 14: return -0x1.93974a8c07c9dp-37;
        case 15: return -0x1.ae7f3e733b81fp-41;
        case 16: return 0x1.ae7f3e733b81fp-45;
        case 17: return 0x1.952c77030ad4ap-49;
        case 18: return -0x1.6827863b97d97p-53;
        case 19: return -0x1.2f49b46814157p-57;
        case 20: return 0x1.e542ba4020225p-62;
        case 21: return 0x1.71b8ef6dcf572p-66;
        case 22: return -0x1.0ce396db7f853p-70;
        case 23: return -0x1.761b41316381ap-75;
        case 24: return 0x1.f2cf01972f578p-80;
        case 25: return 0x1.3f3ccdd165fa9p-84;
        case 26: return -0x1.88e85fc6a4e5ap-89;
        case 27: return -0x1.d1ab1c2dccea3p-94;
        default: return 0.0;
    }
}
HMC_HD constexpr double inv_fact_lo(int k) {
    switch (k) {
        case 2: return 0x0.0p+0;
        case 3: return -0x1.5555555555555p-57;
        case 4: return 0x1.5555555555555p-59;
        case 5: return 0x1.1111111111111p-63;
        case 6: return 0x1.f49f49f49f49fp-65;
        case 7: return -0x1.a01a01a01a01ap-73;
        case 8: return 0x1.a01a01a01a01ap-76;
        case 9: return -0x1.c154f8ddc6c00p-73;
        case 10: return -0x1.cbbc05b4fa99ap-76;
        case 11: return 0x1.c062e06d1f209p-80;
        case 12: return -0x1.2aec959e14c06p-83;
        case 13: return 0x1.f28e0cc748ebep-87;
        case 14: return -0x1.05d6f8a2efd1fp-92;
        case 15: return -0x1.1d8656b0ee8cbp-97;
        case 16: return 0x1.1d8656b0ee8cbp-101;
        case 17: return 0x1.ac981465ddc6cp-103;
        case 18: return -0x1.eec01221a8b0bp-107;
        case 19: return -0x1.2650f61dbdcb4p-112;
        case 20: return 0x1.ea72b4afe3c2fp-120;
        case 21: return -0x1.d043ae40c4647p-120;
        case 22: return 0x1.aebcdbd20331cp-124;
        case 23: return 0x1.3423c7d91404fp-130;
        case 24: return -0x1.9ada5fcc1ab14p-135;
        case 25: return -0x1.58ddadf344487p-139;
        case 26: return 0x1.71c37ebd16540p-143;
        case 27: return -0x1.054d0c78aea14p-149;
        default: return 0.0;
    }
}
// sum_j c_(FIRST + 2j) z^j, the first NDD coefficients in double-double, the rest in double.
template <int FIRST, int NDD>
HMC_HD DDouble taylor_series(DDouble z) {
    constexpr int LAST = (FIRST & 1) ? 27 : 26;
    constexpr int SPLIT = FIRST + 2 * NDD;
    double t = 0.0;
#pragma unroll
    for (int k = LAST; k >= SPLIT; k -= 2) t = dfma(t, z.h, inv_fact_hi(k));
    DDouble p{t, 0.0};
    if (SPLIT <= LAST) p = dd_mul(p, z);
#pragma unroll
    for (int k = SPLIT - 2; k >= FIRST; k -= 2) {
        p = dd_add(DDouble{inv_fact_hi(k), inv_fact_lo(k)}, p);
        if (k > FIRST) p = dd_mul(p, z);
    }
    return p;
}
HMC_HD double next_up_double(double x) {
    if (x == 0.0) return 4.9406564584124654e-324;
    const uint64_t b = as_bits(x);
    return as_double(x > 0.0 ? b + 1 : b - 1);
}
// Ziv's test: the exact value lies within err of v.h + v.l; true when it rounds to v.h.
HMC_HD bool rounds_to_head(DDouble v, double err) {
    const double up = dmul(dsub(next_up_double(v.h), v.h), 0.5);
    const double down = dmul(dsub(v.h, -next_up_double(-v.h)), 0.5);
    return dadd(v.l, err) < up && dsub(v.l, err) > -down;
}
template <int NDD>
HMC_HD void sincos_reduced(DDouble r, DDouble* s, DDouble* c) {
    const DDouble z = dd_mul(r, r);
    const DDouble ps = taylor_series<3, NDD>(z);
    const DDouble pc = taylor_series<2, NDD>(z);
    *s = dd_add(r, dd_mul(dd_mul(r, z), ps));
    *c = dd_add(DDouble{1.0, 0.0}, dd_mul(z, pc));
}
HMC_HD bool cr_sincos(double x, double* sn, double* cs) {
    const double ax = fabs(x);
    if (!(ax <= 1.79769313486231570e308)) {  // inf or nan
        *sn = *cs = dsub(x, x);
        return true;
    }
    if (ax < 0x1p-27) {
        *sn = x;
        *cs = 1.0;
        return true;
    }
    if (ax >= 0x1p20) return false;
    const double k = rint(dmul(x, 0x1.45f306dc9c883p-1));
    DDouble r{x, 0.0};
    if (k != 0.0) {
        const double t = dsub(x, dmul(k, 0x1.921fb54400000p+0));  // exact
        r = dd_two_sum(t, -dmul(k, 0x1.0b4611a600000p-34));
        r = dd_add(r, DDouble{-dmul(k, 0x1.3198a2e000000p-69), 0.0});
        const double p = dmul(k, 0x1.b839a252049c1p-104);
        r = dd_add(r, DDouble{-p, -dfma(k, 0x1.b839a252049c1p-104, -p)});
    }
    const int q = (int)(((long long)k) & 3);
    DDouble s, c;
    sincos_reduced<3>(r, &s, &c);
    if (!rounds_to_head(s, dmul(0x1p-62, fabs(s.h))) || !rounds_to_head(c, dmul(0x1p-62, fabs(c.h))))
        sincos_reduced<13>(r, &s, &c);
    const double sv = s.h, cv = c.h;
    switch (q) {
        case 0: *sn = sv; *cs = cv; break;
        case 1: *sn = cv; *cs = -sv; break;
        case 2: *sn = -sv; *cs = -cv; break;
        default: *sn = -cv; *cs = sv; break;
    }
    return true;
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
