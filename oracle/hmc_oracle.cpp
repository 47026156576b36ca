// CPU oracle for the hoomd-mc local-move sweep -- TEST INFRASTRUCTURE ONLY.
//
// A plain FP64 restatement of the reference's sweep path (glotzerlab/hoomd-rs
// v1.4.0). Each function names the reference file:line it follows. Used only by
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg; the shipped
// CUDA library never links or calls it.
//
// Build: see oracle/Makefile (g++ -O2 -ffp-contract=off, so products and sums
// round exactly where Rust rounds; std::fma appears exactly where the reference
// calls f64::mul_add).
//
// Random streams. SFC64 and Counter are pinned by the reference's known-answer
// tests (hoomd-rand/src/sfc.rs:158-214). The conversions on top of them come from
// the third-party crates rand 0.10.4 and rand_distr 0.6.0 (Cargo.lock), which are
// not vendored; they are restated here from their published algorithms:
//   * f64 in [0,1): the 53 high bits of a u64 times 2^-53;
//   * f64 in (0,1): 52 high bits as the mantissa of [1,2), minus (1 - 2^-53);
//   * integer in [0,n): Canon's widening-multiply method with one refinement draw;
//   * standard normal: the 256-layer ziggurat of Marsaglia & Tsang (2000) in the
//     ZIGNOR form of Doornik (2005), tables computed below from R and V.
// cbrt and the half-angle sin/cos use the deterministic algorithms in
// portable_cbrt / portable_sincos (Newton iteration, Taylor series) so that the
// CUDA library, which uses the same algorithms, proposes bit-identical moves.
#include "hmc_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <queue>
#include <vector>

namespace {

// ============================================================================
// hoomd-rand: SFC64 (sfc.rs:50-86) and Counter (counter.rs:160-167)
// ============================================================================
struct Sfc64 {
    uint64_t s0, s1, s2, ctr;
    // SFC64::initialize, sfc.rs:62-72: 12 discarded outputs.
    static Sfc64 initialize(uint64_t a, uint64_t b, uint64_t c, uint64_t counter) {
        Sfc64 r{a, b, c, counter};
        for (int i = 0; i < 12; ++i) r.next_u64();
        return r;
    }
    // SFC64::step, sfc.rs:74-86.
    uint64_t next_u64() {
        uint64_t out = s0 + s1 + ctr;
        s0 = s1 ^ (s1 >> 11);
        s1 = s2 + (s2 << 3);
        s2 = ((s2 << 24) | (s2 >> 40)) + out;
        ctr += 1;
        return out;
    }
    // try_next_u32, sfc.rs:99-101: truncation of the u64 output.
    uint32_t next_u32() { return (uint32_t)next_u64(); }
};

// Counter::make_rng, counter.rs:160-167.
Sfc64 make_rng(uint64_t step, uint32_t substep, uint32_t seed, uint64_t index) {
    return Sfc64::initialize(step, ((uint64_t)substep << 32) | (uint64_t)seed, index, 0);
}

double bits_to_double(uint64_t b) {
    double d;
    std::memcpy(&d, &b, 8);
    return d;
}
uint64_t double_to_bits(double d) {
    uint64_t b;
    std::memcpy(&b, &d, 8);
    return b;
}

// rand StandardUniform for f64: 53 random bits scaled by 2^-53, in [0, 1).
double uniform01(Sfc64& rng) { return (double)(rng.next_u64() >> 11) * (1.0 / 9007199254740992.0); }

// rand Open01 for f64: 52 bits as the mantissa of [1, 2) minus (1 - 2^-53), in (0, 1).
double open01(Sfc64& rng) {
    uint64_t bits = rng.next_u64() >> 12;
    return bits_to_double(0x3FF0000000000000ULL | bits) - (1.0 - 1.0 / 9007199254740992.0);
}

// Canon's method for an integer in [0, range) from 32-bit draws (rand's
// UniformInt::sample_single for u32; used by IndexedRandom::choose).
uint32_t canon_range_u32(Sfc64& rng, uint32_t range) {
    uint64_t m = (uint64_t)rng.next_u32() * (uint64_t)range;
    uint32_t result = (uint32_t)(m >> 32);
    uint32_t lo = (uint32_t)m;
    if (lo > (uint32_t)(0u - range)) {
        uint64_t m2 = (uint64_t)rng.next_u32() * (uint64_t)range;
        uint32_t new_hi = (uint32_t)(m2 >> 32);
        if ((uint32_t)(lo + new_hi) < lo) result += 1;
    }
    return result;
}

// ---- ziggurat standard normal (ZIGNOR, Doornik 2005) --------------------------------
constexpr int ZIG_LAYERS = 256;
constexpr double ZIG_R = 3.6541528853610088;
constexpr double ZIG_V = 0.00492867323399;

struct ZigTables {
    double x[ZIG_LAYERS + 1];
    double f[ZIG_LAYERS + 1];
    ZigTables() {
        auto pdf = [](double t) { return std::exp(-t * t / 2.0); };
        x[0] = ZIG_V / pdf(ZIG_R);
        x[1] = ZIG_R;
        for (int i = 2; i < ZIG_LAYERS; ++i) x[i] = std::sqrt(-2.0 * std::log(ZIG_V / x[i - 1] + pdf(x[i - 1])));
        x[ZIG_LAYERS] = 0.0;
        for (int i = 0; i <= ZIG_LAYERS; ++i) f[i] = pdf(x[i]);
    }
};
const ZigTables& zig() {
    static ZigTables t;
    return t;
}

double standard_normal(Sfc64& rng) {
    const ZigTables& t = zig();
    for (;;) {
        uint64_t bits = rng.next_u64();
        int i = (int)(bits & 0xff);
        // 52 high bits as the mantissa of [2, 4), minus 3: u in [-1, 1).
        double u = bits_to_double(0x4000000000000000ULL | (bits >> 12)) - 3.0;
        double x = u * t.x[i];
        if (std::fabs(x) < t.x[i + 1]) return x;
        if (i == 0) {
            // Tail beyond R (Marsaglia 1964).
            double xt = 1.0, y = 0.0;
            while (-2.0 * y < xt * xt) {
                double a = open01(rng);
                double b = open01(rng);
                xt = std::log(a) / ZIG_R;
                y = std::log(b);
            }
            return u < 0.0 ? xt - ZIG_R : ZIG_R - xt;
        }
        if (t.f[i + 1] + (t.f[i] - t.f[i + 1]) * uniform01(rng) < std::exp(-x * x / 2.0)) return x;
    }
}

// ---- deterministic cbrt and half-angle sin/cos --------------------------------------
// Cube root without division: x = m 2^(3q + r), m in [1, 2); y ~ m^(-1/3) from a quadratic
// Chebyshev fit and three Newton steps y += y (1 - m y^3) / 3; cbrt ~ m y^2 cbrt(2^r) 2^q,
// corrected by one Newton step on the FMA-evaluated residual. Only correctly rounded
// operations, so the CUDA library, which uses the same algorithm, agrees bit for bit.
double portable_cbrt(double x) {
    if (x == 0.0 || !std::isfinite(x)) return x;
    bool neg = x < 0.0;
    double ax = neg ? -x : x;
    int extra = 0;
    if (ax < 2.2250738585072014e-308) {  // subnormal: scale by 2^54
        ax = ax * 18014398509481984.0;
        extra = -18;
    }
    uint64_t b = double_to_bits(ax);
    int e = (int)((b >> 52) & 0x7ff) - 1023;
    double m = bits_to_double((b & 0x000FFFFFFFFFFFFFULL) | 0x3FF0000000000000ULL);
    int q = (e >= 0) ? e / 3 : -((-e + 2) / 3);
    int r = e - 3 * q;
    double y = std::fma(std::fma(0.09303886055928341, m, -0.48224275792479104), m, 1.387389992245347);
    for (int it = 0; it < 3; ++it) {
        double y3 = (y * y) * y;
        double eps = std::fma(-m, y3, 1.0);
        y = std::fma(y * eps, 0.3333333333333333, y);
    }
    double a = m * (r == 0 ? 1.0 : (r == 1 ? 2.0 : 4.0));
    double k = r == 0 ? 1.0 : (r == 1 ? 1.2599210498948732 : 1.5874010519681994);
    double ik2 = r == 0 ? 0.3333333333333333 : (r == 1 ? 0.20998684164914552 : 0.13228342099734997);
    double c = ((m * y) * y) * k;
    double c2 = c * c;
    double c2lo = std::fma(c, c, -c2);
    double resid = std::fma(c2, c, -a) + c2lo * c;
    c = c - resid * ((y * y) * ik2);
    double scale = bits_to_double((uint64_t)(q + extra + 1023) << 52);
    double res = c * scale;
    return neg ? -res : res;
}

// sin(h) and cos(h) for 0 <= h <= pi/2 by Taylor series in h^2 (Horner with fma).
void portable_sincos(double h, double* s, double* c) {
    static const double SC[13] = {1.0,
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
    static const double CC[13] = {1.0,
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
    double h2 = h * h;
    double ps = SC[12], pc = CC[12];
    for (int k = 11; k >= 0; --k) {
        ps = std::fma(ps, h2, SC[k]);
        pc = std::fma(pc, h2, CC[k]);
    }
    *s = h * ps;
    *c = pc;
}

// ---- correctly rounded sin and cos ----------------------------------------------
// The reference turns an Angle into a rotation with f64::sin / f64::cos (hoomd-vector
// angle.rs:120-150), i.e. the platform libm. The oracle and the device both use this
// deterministic method instead, which returns the correctly rounded values (what an exact
// libm returns) built only from correctly rounded +, -, *, fma:
//  * Cody-Waite reduction x = k pi/2 + r with pi/2 split into 33+33+33+53 bits (about 160
//    bits, the products k*C1..k*C3 exact for |k| < 2^20), r kept as a double-double;
//  * Taylor series of sin r and cos r, |r| <= pi/4: the leading terms in double-double,
//    the rest in double (relative error below 2^-66), then Ziv's rounding test against a
//    2^-62 bound; if the rounding is not decided, the whole series in double-double
//    (error below 2^-95) decides it. Ambiguous after that only when the exact value lies
//    within 2^-95 of a rounding boundary, where the double-double result is returned.
// Inputs with |x| >= 2^20 are outside the supported range (return 1).
struct DD {
    double h, l;
};
static inline DD dd_two_sum(double a, double b) {
    double s = a + b;
    double bb = s - a;
    return {s, (a - (s - bb)) + (b - bb)};
}
static inline DD dd_fast(double a, double b) {  // |a| >= |b|
    double s = a + b;
    return {s, b - (s - a)};
}
static inline DD dd_mul(DD a, DD b) {
    double p = a.h * b.h;
    double e = std::fma(a.h, b.h, -p);
    e = std::fma(a.h, b.l, e);
    e = std::fma(a.l, b.h, e);
    return dd_fast(p, e);
}
static inline DD dd_add(DD a, DD b) {
    DD s = dd_two_sum(a.h, b.h);
    return dd_fast(s.h, s.l + (a.l + b.l));
}
// (-1)^(k/2) / k! as double-doubles, k = 2..27 (exact rationals rounded twice).
static const double kInvFact[26][2] = {
    {-0x1.0000000000000p-1, 0x0.0p+0},
    {-0x1.5555555555555p-3, -0x1.5555555555555p-57},
    {0x1.5555555555555p-5, 0x1.5555555555555p-59},
    {0x1.1111111111111p-7, 0x1.1111111111111p-63},
    {-0x1.6c16c16c16c17p-10, 0x1.f49f49f49f49fp-65},
    {-0x1.a01a01a01a01ap-13, -0x1.a01a01a01a01ap-73},
    {0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-76},
    {0x1.71de3a556c734p-19, -0x1.c154f8ddc6c00p-73},
    {-0x1.27e4fb7789f5cp-22, -0x1.cbbc05b4fa99ap-76},
    {-0x1.ae64567f544e4p-26, 0x1.c062e06d1f209p-80},
    {0x1.1eed8eff8d898p-29, -0x1.2aec959e14c06p-83},
    {0x1.6124613a86d09p-33, 0x1.f28e0cc748ebep-87},
    {-0x1.93974a8c07c9dp-37, -0x1.05d6f8a2efd1fp-92},
    {-0x1.ae7f3e733b81fp-41, -0x1.1d8656b0ee8cbp-97},
    {0x1.ae7f3e733b81fp-45, 0x1.1d8656b0ee8cbp-101},
    {0x1.952c77030ad4ap-49, 0x1.ac981465ddc6cp-103},
    {-0x1.6827863b97d97p-53, -0x1.eec01221a8b0bp-107},
    {-0x1.2f49b46814157p-57, -0x1.2650f61dbdcb4p-112},
    {0x1.e542ba4020225p-62, 0x1.ea72b4afe3c2fp-120},
    {0x1.71b8ef6dcf572p-66, -0x1.d043ae40c4647p-120},
    {-0x1.0ce396db7f853p-70, 0x1.aebcdbd20331cp-124},
    {-0x1.761b41316381ap-75, 0x1.3423c7d91404fp-130},
    {0x1.f2cf01972f578p-80, -0x1.9ada5fcc1ab14p-135},
    {0x1.3f3ccdd165fa9p-84, -0x1.58ddadf344487p-139},
    {-0x1.88e85fc6a4e5ap-89, 0x1.71c37ebd16540p-143},
    {-0x1.d1ab1c2dccea3p-94, -0x1.054d0c78aea14p-149}};
static inline DD inv_fact(int k) { return {kInvFact[k - 2][0], kInvFact[k - 2][1]}; }

// sum_{j>=0} c_{first+2j} z^j with the first n_dd coefficients in double-double and the
// rest (up to k = 27) in double.
static DD series(int first, DD z, int n_dd) {
    int last = first;
    while (last + 2 <= 27) last += 2;
    int split = first + 2 * n_dd;  // first coefficient evaluated in double
    double t = 0.0;
    for (int k = last; k >= split; k -= 2) t = std::fma(t, z.h, kInvFact[k - 2][0]);
    DD p{t, 0.0};
    if (split <= last) p = dd_mul(p, z);
    for (int k = split - 2; k >= first; k -= 2) {
        p = dd_add(inv_fact(k), p);
        if (k > first) p = dd_mul(p, z);
    }
    return p;
}
static inline double next_up(double x) {
    uint64_t b = double_to_bits(x);
    if (x == 0.0) return 4.9406564584124654e-324;
    return bits_to_double(x > 0 ? b + 1 : b - 1);
}
static inline double next_down(double x) { return -next_up(-x); }
// Ziv's test: the exact value lies within err of h + l; returns true when it rounds to h.
static inline bool rounds_to_h(DD v, double err) {
    double up = (next_up(v.h) - v.h) * 0.5, down = (v.h - next_down(v.h)) * 0.5;
    return v.l + err < up && v.l - err > -down;
}
// sin r and cos r for r = rh + rl, |r| <= pi/4 (slightly above, after reduction).
static void sincos_reduced(DD r, int tier2, DD* s, DD* c) {
    DD z = dd_mul(r, r);
    int n = tier2 ? 13 : 3;
    DD ps = series(3, z, n);  // -1/6 + z/120 - ...
    DD pc = series(2, z, n);  // -1/2 + z/24 - ...
    *s = dd_add(r, dd_mul(dd_mul(r, z), ps));
    *c = dd_add(DD{1.0, 0.0}, dd_mul(z, pc));
}
int cr_sincos(double x, double* sn, double* cs) {
    if (!std::isfinite(x)) {
        *sn = *cs = x - x;
        return 0;
    }
    double ax = std::fabs(x);
    if (ax < 0x1p-27) {
        *sn = x;
        *cs = 1.0;
        return 0;
    }
    if (ax >= 0x1p20) {
        *sn = *cs = NAN;
        return 1;
    }
    double k = std::nearbyint(x * 0x1.45f306dc9c883p-1);
    DD r{x, 0.0};
    if (k != 0.0) {
        double t = x - k * 0x1.921fb54400000p+0;  // exact
        r = dd_two_sum(t, -(k * 0x1.0b4611a600000p-34));
        r = dd_add(r, DD{-(k * 0x1.3198a2e000000p-69), 0.0});
        double p = k * 0x1.b839a252049c1p-104;
        r = dd_add(r, DD{-p, -std::fma(k, 0x1.b839a252049c1p-104, -p)});
    }
    int q = (int)(((long long)k) & 3);
    DD s, c;
    sincos_reduced(r, 0, &s, &c);
    const double tol1 = 0x1p-62;
    if (!rounds_to_h(s, tol1 * std::fabs(s.h)) || !rounds_to_h(c, tol1 * std::fabs(c.h)))
        sincos_reduced(r, 1, &s, &c);
    double sv = s.h, cv = c.h;
    switch (q) {
        case 0: *sn = sv; *cs = cv; break;
        case 1: *sn = cv; *cs = -sv; break;
        case 2: *sn = -sv; *cs = -cv; break;
        default: *sn = -cv; *cs = sv; break;
    }
    return 0;
}

// ============================================================================
// hoomd-vector arithmetic with the reference's rounding
// ============================================================================
struct V3 {
    double v[3];
};
struct Quat {
    double s, x, y, z;
};

// InnerProduct::dot, cartesian.rs:293-296: fold with mul_add from 0.0.
double dot(const double* a, const double* b, int n) {
    double p = 0.0;
    for (int i = 0; i < n; ++i) p = std::fma(a[i], b[i], p);
    return p;
}
// Metric::distance_squared, cartesian.rs:339-342: fold of (x - y)^2 from 0.0.
double distance_squared(const double* a, const double* b, int n) {
    double p = 0.0;
    for (int i = 0; i < n; ++i) {
        double d = a[i] - b[i];
        p = p + d * d;
    }
    return p;
}
// Cross, cartesian.rs:604-610.
V3 cross(const double* a, const double* b) {
    return {{a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]}};
}
// Quaternion::mul, quaternion.rs:408-415.
Quat qmul(const Quat& a, const Quat& b) {
    double av[3] = {a.x, a.y, a.z}, bv[3] = {b.x, b.y, b.z};
    double sc = a.s * b.s - dot(av, bv, 3);
    V3 cr = cross(av, bv);
    double r[3];
    for (int i = 0; i < 3; ++i) r[i] = (bv[i] * a.s + av[i] * b.s) + cr.v[i];
    return {sc, r[0], r[1], r[2]};
}
Quat qconj(const Quat& a) { return {a.s, -a.x, -a.y, -a.z}; }
// Versor::rotate, quaternion.rs:740-747.
V3 versor_rotate(const Quat& q, const double* v) {
    double qv[3] = {q.x, q.y, q.z};
    double k1 = q.s * q.s - dot(qv, qv, 3);
    V3 c = cross(qv, v);
    double k2 = 2.0 * q.s;
    double k3 = 2.0 * dot(qv, v, 3);
    V3 r;
    for (int i = 0; i < 3; ++i) r.v[i] = (v[i] * k1 + c.v[i] * k2) + qv[i] * k3;
    return r;
}
struct Mat3 {
    double r[3][3];
};
// RotationMatrix::from(Versor), quaternion.rs:642-690.
Mat3 mat_from_versor(const Quat& q) {
    double a = q.s, b = q.x, c = q.y, d = q.z;
    Mat3 m;
    m.r[0][0] = a * a + b * b - c * c - d * d;
    m.r[0][1] = 2.0 * b * c - 2.0 * a * d;
    m.r[0][2] = 2.0 * b * d + 2.0 * a * c;
    m.r[1][0] = 2.0 * b * c + 2.0 * a * d;
    m.r[1][1] = a * a - b * b + c * c - d * d;
    m.r[1][2] = 2.0 * c * d - 2.0 * a * b;
    m.r[2][0] = 2.0 * b * d - 2.0 * a * c;
    m.r[2][1] = 2.0 * c * d + 2.0 * a * b;
    m.r[2][2] = a * a - b * b - c * c + d * d;
    return m;
}
// RotationMatrix::inverted, cartesian.rs:897-901 (transpose).
template <int N>
void mat_transpose(const double (&in)[N][N], double (&out)[N][N]) {
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) out[i][j] = in[j][i];
}
// Rotate for RotationMatrix, cartesian.rs:981-989: row.dot(v).
template <int N>
void mat_rotate(const double (&m)[N][N], const double* v, double* out) {
    for (int i = 0; i < N; ++i) out[i] = dot(m[i], v, N);
}

// ============================================================================
// hoomd-geometry: support mapping and XenoCollide
// ============================================================================
struct Polytope {
    int dim = 3;
    std::vector<double> verts;  // nv * dim
    int nv = 0;
    double bounding_radius = 0.0;
};
// ConvexPolytope::bounding_radius, convex_polytope.rs:199-207.
double polytope_bounding_radius(const double* verts, int nv, int dim) {
    double m = 0.0;
    for (int i = 0; i < nv; ++i) m = std::max(m, dot(verts + i * dim, verts + i * dim, dim));
    return std::sqrt(m);
}
// ConvexPolytope::support_mapping, convex_polytope.rs:222-244: argmax of
// (v0*n0 + v1*n1 [+ v2*n2]) with the first maximum winning.
void support(const Polytope& p, const double* n, double* out) {
    int argmax = 0;
    double max_val = -INFINITY;
    for (int i = 0; i < p.nv; ++i) {
        const double* v = p.verts.data() + i * p.dim;
        double x = -0.0;
        for (int m = 0; m < p.dim; ++m) x = x + v[m] * n[m];
        if (x > max_val) {
            argmax = i;
            max_val = x;
        }
    }
    for (int m = 0; m < p.dim; ++m) out[m] = p.verts[argmax * p.dim + m];
}

template <int N>
struct Minkowski {
    const Polytope* sa;
    const Polytope* sb;
    double vij[N];
    double q[N][N];
    double qinv[N][N];
    // composite_support_mapping, xenocollide.rs:318-328.
    void composite(const double* n, double* out) const {
        double t[N], sbn[N], rot[N], neg[N], san[N];
        mat_rotate<N>(qinv, n, t);
        support(*sb, t, sbn);
        mat_rotate<N>(q, sbn, rot);
        for (int i = 0; i < N; ++i) rot[i] = rot[i] + vij[i];
        for (int i = 0; i < N; ++i) neg[i] = -n[i];
        support(*sa, neg, san);
        for (int i = 0; i < N; ++i) out[i] = rot[i] - san[i];
    }
};

constexpr int XENO_MAX_ITER = 1024;  // xenocollide.rs:38

// collide for N = 3, xenocollide.rs:172-291 and :361-414.
bool collide3d(const Polytope& a, const Polytope& b, const double* vij, const Mat3& qij) {
    Minkowski<3> s;
    s.sa = &a;
    s.sb = &b;
    for (int i = 0; i < 3; ++i) s.vij[i] = vij[i];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) s.q[i][j] = qij.r[i][j];
    mat_transpose<3>(s.q, s.qinv);
    const double TOL = 2e-12;
    double v0[3] = {vij[0], vij[1], vij[2]};
    // discover_portal, :172-244
    if (std::fabs(v0[0]) < TOL && std::fabs(v0[1]) < TOL && std::fabs(v0[2]) < TOL) return true;
    double nv0[3] = {-v0[0], -v0[1], -v0[2]};
    double v1[3], v2[3], v3[3];
    s.composite(nv0, v1);
    if (dot(v1, v0, 3) > 0.0) return false;
    V3 n = cross(v1, v0);
    if (std::fabs(n.v[0]) < TOL && std::fabs(n.v[1]) < TOL && std::fabs(n.v[2]) < TOL) return true;
    s.composite(n.v, v2);
    if (dot(v2, n.v, 3) < 0.0) return false;
    auto plane = [&](const double* p1, const double* p2) {
        double d1[3] = {p1[0] - v0[0], p1[1] - v0[1], p1[2] - v0[2]};
        double d2[3] = {p2[0] - v0[0], p2[1] - v0[1], p2[2] - v0[2]};
        return cross(d1, d2);
    };
    n = plane(v1, v2);
    if (dot(n.v, v0, 3) > 0.0) {
        for (int i = 0; i < 3; ++i) std::swap(v1[i], v2[i]);
        for (int i = 0; i < 3; ++i) n.v[i] = -n.v[i];
    }
    int count = 0;
    for (;;) {
        count += 1;
        if (count >= XENO_MAX_ITER) return true;
        s.composite(n.v, v3);
        if (dot(v3, n.v, 3) <= 0.0) return false;
        V3 c13 = cross(v1, v3);
        if (dot(c13.v, v0, 3) < 0.0) {
            for (int i = 0; i < 3; ++i) v2[i] = v3[i];
            n = plane(v1, v2);
            continue;
        }
        V3 c32 = cross(v3, v2);
        if (dot(c32.v, v0, 3) < 0.0) {
            for (int i = 0; i < 3; ++i) v1[i] = v3[i];
            n = plane(v1, v2);
            continue;
        }
        break;
    }
    double portal[3][3];
    for (int i = 0; i < 3; ++i) {
        portal[0][i] = v1[i];
        portal[1][i] = v2[i];
        portal[2][i] = v3[i];
    }
    // refinement loop, :384-413
    count = 0;
    for (;;) {
        count += 1;
        // outward_normal, :162-170
        double e1[3], e2[3];
        for (int i = 0; i < 3; ++i) {
            e1[i] = portal[1][i] - portal[0][i];
            e2[i] = portal[2][i] - portal[0][i];
        }
        V3 nn = cross(e1, e2);
        double pm[3] = {portal[0][0] - v0[0], portal[0][1] - v0[1], portal[0][2] - v0[2]};
        if (dot(pm, nn.v, 3) < 0.0)
            for (int i = 0; i < 3; ++i) nn.v[i] = -nn.v[i];
        if (dot(portal[0], nn.v, 3) >= 0.0) return true;
        double vnew[3];
        s.composite(nn.v, vnew);
        if (dot(vnew, nn.v, 3) < 0.0) return false;
        // tolerance_check, :247-265
        double tol = TOL * std::sqrt(dot(nn.v, nn.v, 3));
        double dd[3] = {vnew[0] - portal[0][0], vnew[1] - portal[0][1], vnew[2] - portal[0][2]};
        if (std::fabs(dot(dd, nn.v, 3)) < tol) return false;
        if (std::fabs(dot(portal[0], nn.v, 3)) < tol) return true;
        // narrow_portal, :268-291
        V3 vp = cross(vnew, v0);
        bool t1 = dot(vp.v, portal[0], 3) > 0.0;
        bool t2 = dot(vp.v, portal[1], 3) > 0.0;
        bool t3 = dot(vp.v, portal[2], 3) > 0.0;
        int replace;
        if (t1 && t2)
            replace = 0;
        else if (t1 && !t2)
            replace = 2;
        else if (!t1 && t3)
            replace = 1;
        else
            replace = 0;
        for (int i = 0; i < 3; ++i) portal[replace][i] = vnew[i];
        if (count >= XENO_MAX_ITER) return true;
    }
}

// collide for N = 2, xenocollide.rs:92-154 and :361-414.
bool collide2d(const Polytope& a, const Polytope& b, const double* vij, const double (&qij)[2][2]) {
    Minkowski<2> s;
    s.sa = &a;
    s.sb = &b;
    for (int i = 0; i < 2; ++i) s.vij[i] = vij[i];
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) s.q[i][j] = qij[i][j];
    mat_transpose<2>(s.q, s.qinv);
    const double TOL = 1e-16;
    double v0[2] = {vij[0], vij[1]};
    auto perp = [](const double* v, double* o) {  // cartesian.rs:755
        o[0] = -v[1];
        o[1] = v[0];
    };
    double nv0[2] = {-v0[0], -v0[1]};
    double v1[2], v2[2];
    s.composite(nv0, v1);
    double d10[2] = {v1[0] - v0[0], v1[1] - v0[1]}, vp[2];
    perp(d10, vp);
    if (dot(v1, vp, 2) > 0.0) {
        vp[0] = -vp[0];
        vp[1] = -vp[1];
    }
    s.composite(vp, v2);
    double portal[2][2] = {{v1[0], v1[1]}, {v2[0], v2[1]}};
    int count = 0;
    for (;;) {
        count += 1;
        double e[2] = {portal[1][0] - portal[0][0], portal[1][1] - portal[0][1]}, nn[2];
        perp(e, nn);
        double pm[2] = {portal[0][0] - v0[0], portal[0][1] - v0[1]};
        if (dot(pm, nn, 2) < 0.0) {
            nn[0] = -nn[0];
            nn[1] = -nn[1];
        }
        if (dot(portal[0], nn, 2) >= 0.0) return true;
        double vnew[2];
        s.composite(nn, vnew);
        if (dot(vnew, nn, 2) < 0.0) return false;
        // tolerance_check 2-D, :127-138: d = w - project(w, e) with w = vnew - p0
        double w[2] = {vnew[0] - portal[0][0], vnew[1] - portal[0][1]};
        double ee[2] = {portal[1][0] - portal[0][0], portal[1][1] - portal[0][1]};
        // project: b * (a.dot(b)) / b.norm_squared(), lib.rs:686-688
        double k = dot(w, ee, 2);
        double nb = dot(ee, ee, 2);
        double pr[2] = {ee[0] * k / nb, ee[1] * k / nb};
        double d[2] = {w[0] - pr[0], w[1] - pr[1]};
        if (dot(d, d, 2) < TOL * dot(vnew, vnew, 2)) return true;
        // narrow_portal 2-D, :141-154
        double dvi[2] = {vnew[0] - v0[0], vnew[1] - v0[1]}, vpp[2];
        perp(dvi, vpp);
        double p0v[2] = {portal[0][0] - vnew[0], portal[0][1] - vnew[1]};
        if (dot(p0v, vpp, 2) < 0.0) {
            vpp[0] = -vpp[0];
            vpp[1] = -vpp[1];
        }
        if (dot(vnew, vpp, 2) < 0.0) {
            portal[1][0] = vnew[0];
            portal[1][1] = vnew[1];
        } else {
            portal[0][0] = vnew[0];
            portal[0][1] = vnew[1];
        }
        if (count >= XENO_MAX_ITER) return true;
    }
}

// Angle -> RotationMatrix<2>, angle.rs:130-138.
void mat2_from_angle(double theta, double (&m)[2][2]) {
    double s, c;
    cr_sincos(theta, &s, &c);
    m[0][0] = c;
    m[0][1] = -s;
    m[1][0] = s;
    m[1][1] = c;
}

// Convex::intersects_at_global 3-D, convex.rs:154-170, with pair_system_to_local
// (hoomd-vector/src/lib.rs:878-888).
bool convex_global_3d(const Polytope& p, const double* ri, const Quat& qi, const double* rj, const Quat& qj) {
    double rcut = p.bounding_radius + p.bounding_radius;
    if (distance_squared(ri, rj, 3) >= rcut * rcut) return false;
    double rab[3] = {rj[0] - ri[0], rj[1] - ri[1], rj[2] - ri[2]};
    Quat qa_inv = qconj(qi);
    V3 vij = versor_rotate(qa_inv, rab);
    Quat oij = qmul(qa_inv, qj);
    return collide3d(p, p, vij.v, mat_from_versor(oij));
}
// Convex::intersects_at_global 2-D, convex.rs:101-121 (Angle rotations,
// angle.rs:175-181 rotate, :212 inverted = -theta, :229 combine = sum).
bool convex_global_2d(const Polytope& p, const double* ri, double ti, const double* rj, double tj) {
    double rcut = p.bounding_radius + p.bounding_radius;
    if (distance_squared(ri, rj, 2) >= rcut * rcut) return false;
    double rab[2] = {rj[0] - ri[0], rj[1] - ri[1]};
    double inv = -ti;
    double s, c;
    cr_sincos(inv, &s, &c);
    double vij[2] = {rab[0] * c - rab[1] * s, rab[0] * s + rab[1] * c};
    double oij = inv + tj;
    double m[2][2];
    mat2_from_angle(oij, m);
    return collide2d(p, p, vij, m);
}

// ConvexSurfaceMesh2d separating-axis test (convex_surface_mesh_2d.rs:578-640): a and b
// hold counter-clockwise hull vertices; o_b rotates b into a's frame.
static void mat2_rotate(const double (&m)[2][2], const double* v, double* out) {  // rows dot v
    out[0] = dot(m[0], v, 2);
    out[1] = dot(m[1], v, 2);
}
// is_separating, :625-640: every vertex of a strictly outside the plane (p, n).
static bool is_separating(const Polytope& a, const double* p, const double* n) {
    double n_dot_p = dot(n, p, 2);
    for (int i = 0; i < a.nv; ++i)
        if (dot(n, &a.verts[2 * i], 2) - n_dot_p <= 0.0) return false;
    return true;
}
// b_edge_separates, :597-623.
static bool b_edge_separates(const Polytope& a, const Polytope& b, const double* v_ab, const double (&o_b)[2][2]) {
    int previous = b.nv - 1;
    for (int current = 0; current < b.nv; ++current) {
        const double* p = &b.verts[2 * current];
        double edge[2] = {p[0] - b.verts[2 * previous], p[1] - b.verts[2 * previous + 1]};
        double n[2] = {edge[1], -edge[0]};  // -edge.perpendicular(), perpendicular = (-y, x)
        double pa[2], na[2];
        mat2_rotate(o_b, p, pa);
        pa[0] = pa[0] + v_ab[0];
        pa[1] = pa[1] + v_ab[1];
        mat2_rotate(o_b, n, na);
        if (is_separating(a, pa, na)) return true;
        previous = current;
    }
    return false;
}
bool sat_intersects_at(const Polytope& a, const Polytope& b, const double* v_ij, const double (&o_j)[2][2]) {
    if (b_edge_separates(a, b, v_ij, o_j)) return false;
    double inv[2][2] = {{o_j[0][0], o_j[1][0]}, {o_j[0][1], o_j[1][1]}};
    double mv[2] = {-v_ij[0], -v_ij[1]}, v_ji[2];
    mat2_rotate(inv, mv, v_ji);
    return !b_edge_separates(b, a, v_ji, inv);
}
// IntersectsAtGlobal for ConvexSurfaceMesh2d, :514-536.
bool sat_global_2d(const Polytope& p, const double* ri, double ti, const double* rj, double tj) {
    double rcut = p.bounding_radius + p.bounding_radius;
    if (distance_squared(ri, rj, 2) >= rcut * rcut) return false;
    double rab[2] = {rj[0] - ri[0], rj[1] - ri[1]};
    double inv = -ti;
    double s, c;
    cr_sincos(inv, &s, &c);
    double vij[2] = {rab[0] * c - rab[1] * s, rab[0] * s + rab[1] * c};
    double m[2][2];
    mat2_from_angle(inv + tj, m);
    return sat_intersects_at(p, p, vij, m);
}

// IntersectsAt::approximate_separation_distance (hoomd-geometry/src/lib.rs:307-325) for two equal
// Convex polytopes in the local frame of the first: direction = v.to_unit() (lib.rs:632-639,
// norm = sqrt(fma dot)), else the default unit (last axis, cartesian.rs:313-318); d grows by
// `resolution` while Convex::intersects_at (convex.rs:87-99, :130-143) holds at v + direction * d:
// the bounding spheres |w|^2 <= (R + R)^2 (sphere.rs:262-264), then XenoCollide.
// SAT: ConvexSurfaceMesh2d, whose intersects_at (convex_surface_mesh_2d.rs:538-595) is the
// separating-axis test alone, without the bounding circles.
template <int N, class Q, bool SAT = false>
double approximate_separation(const Polytope& p, const double* v, const Q& q, double resolution) {
    double dir[N];
    const double norm = std::sqrt(dot(v, v, N));
    if (norm == 0.0) {
        for (int a = 0; a < N; ++a) dir[a] = a == N - 1 ? 1.0 : 0.0;
    } else {
        for (int a = 0; a < N; ++a) dir[a] = v[a] / norm;
    }
    const double rr = (p.bounding_radius + p.bounding_radius) * (p.bounding_radius + p.bounding_radius);
    double d = 0.0;
    for (;;) {
        double w[N];
        for (int a = 0; a < N; ++a) w[a] = v[a] + dir[a] * d;
        if (!SAT && !(dot(w, w, N) <= rr)) break;
        bool hit;
        if constexpr (N == 3)
            hit = collide3d(p, p, w, q);
        else if constexpr (SAT)
            hit = sat_intersects_at(p, p, w, q);
        else
            hit = collide2d(p, p, w, q);
        if (!hit) break;
        d = d + resolution;
    }
    return d;
}
// OverlapPenalty::energy (overlap_penalty.rs:109-115): inf below -d_max, (0.5 k) r^2 + eps below 0.
double overlap_penalty(double k, double dmax, double shoulder, double r) {
    if (r < -dmax) return INFINITY;
    if (r < 0.0) return 0.5 * k * (r * r) + shoulder;
    return 0.0;
}
// Anisotropic::site_pair_energy (anisotropic.rs:120-135) of ApproximateShapeOverlap<OverlapPenalty,
// Convex<ConvexPolyhedron>> (approximate_shape_overlap.rs:122-131): |r_j - r_i| >= r_cut -> 0, else
// pair_system_to_local (hoomd-vector/src/lib.rs:878-888) and OverlapPenalty(-separation).
double shape_penalty_3d(const Polytope& p, double rcut, double res, double k, double dmax, double shoulder,
                        const double* ri, const Quat& qi, const double* rj, const Quat& qj) {
    if (std::sqrt(distance_squared(ri, rj, 3)) >= rcut) return 0.0;
    double rab[3] = {rj[0] - ri[0], rj[1] - ri[1], rj[2] - ri[2]};
    const Quat qa_inv = qconj(qi);
    const V3 vij = versor_rotate(qa_inv, rab);
    const Quat oij = qmul(qa_inv, qj);
    const Mat3 m = mat_from_versor(oij);
    return overlap_penalty(k, dmax, shoulder, -approximate_separation<3>(p, vij.v, m, res));
}
// The same for Convex<ConvexPolygon> (SAT: ConvexSurfaceMesh2d) with Angle orientations
// (angle.rs:175-181, :212, :229).
template <bool SAT = false>
double shape_penalty_2d(const Polytope& p, double rcut, double res, double k, double dmax, double shoulder,
                        const double* ri, double ti, const double* rj, double tj) {
    if (std::sqrt(distance_squared(ri, rj, 2)) >= rcut) return 0.0;
    double rab[2] = {rj[0] - ri[0], rj[1] - ri[1]};
    const double inv = -ti;
    double s, c;
    cr_sincos(inv, &s, &c);
    double vij[2] = {rab[0] * c - rab[1] * s, rab[0] * s + rab[1] * c};
    double m[2][2];
    mat2_from_angle(inv + tj, m);
    return overlap_penalty(k, dmax, shoulder, -approximate_separation<2, double[2][2], SAT>(p, vij, m, res));
}

// ============================================================================
// hoomd-interaction: pair energies
// ============================================================================
// powi with repeated squaring (the multiply order LLVM uses for powi).
double powi(double a, int b) {
    double r = 1.0;
    for (;;) {
        if (b & 1) r = r * a;
        b /= 2;
        if (b == 0) break;
        a = a * a;
    }
    return r;
}
// LennardJones::energy, lennard_jones.rs:107-111.
double lj_energy(double eps, double sigma, double r) {
    double sr = sigma / r;
    return 4.0 * eps * (powi(sr, 12) - powi(sr, 6));
}
// Isotropic<Shifted<LJ>>::site_pair_energy, isotropic.rs:147-156 + shifted.rs:92-94.
double shifted_lj_pair(double eps, double sigma, double rcut, double rshift, double r2) {
    if (r2 >= rcut * rcut) return 0.0;
    double r = std::sqrt(r2);
    return lj_energy(eps, sigma, r) - lj_energy(eps, sigma, rshift);
}

// The univariate energies Isotropic accepts (hoomd-interaction/src/univariate/*.rs), each with
// the reference's order of operations, and the wrappers around them.
enum { UV_LENNARD_JONES = 0, UV_WEEKS_CHANDLER_ANDERSON = 1, UV_HARMONIC = 2, UV_HARMONIC_REPULSION = 3,
       UV_BOXCAR = 4, UV_OVERLAP_PENALTY = 5, UV_LENNARD_JONES_GAUSS = 6 };
enum { UVW_NONE = 0, UVW_SHIFTED = 1, UVW_EXPANDED = 2, UVW_XPLOR = 3 };
struct Univariate {
    int kind = UV_LENNARD_JONES, wrap = UVW_NONE;
    double p[4] = {0, 0, 0, 0};  // the univariate's parameters
    double w[2] = {0, 0};        // Shifted: r_shift; Expanded: delta; Xplor: r_cut, r_smooth
    double rcut = 1.0;           // Isotropic::r_cut
    double f(double r) const {
        switch (kind) {
            case UV_LENNARD_JONES:  // lennard_jones.rs:107-111
                return lj_energy(p[0], p[1], r);
            case UV_WEEKS_CHANDLER_ANDERSON:  // weeks_chandler_anderson.rs: r < 2^(1/6) sigma (p[2] = 2^(1/6))
                return r < p[2] * p[1] ? lj_energy(p[0], p[1], r) + p[0] : 0.0;
            case UV_HARMONIC:  // harmonic.rs: 0.5 k (r - r_0) (r - r_0)
                return 0.5 * p[0] * (r - p[1]) * (r - p[1]);
            case UV_HARMONIC_REPULSION:  // harmonic_repulsion.rs: 0.5 a / r_cut (r - r_cut)^2 below r_cut
                return r < p[1] ? 0.5 * p[0] / p[1] * ((r - p[1]) * (r - p[1])) : 0.0;
            case UV_BOXCAR:  // boxcar.rs: epsilon on [left, right)
                return r < p[1] ? 0.0 : (r < p[2] ? p[0] : 0.0);
            case UV_LENNARD_JONES_GAUSS: {  // lennard_jones_gauss.rs: {eps, sigma^2, r_0, scale}
                const double r_inv = p[3] / r;
                const double arg = -((r / p[3] - p[2]) * (r / p[3] - p[2])) / (2.0 * p[1]);
                return powi(r_inv, 12) - 2.0 * powi(r_inv, 6) - p[0] * std::exp(arg);
            }
            default:  // overlap_penalty.rs:109-115
                if (r < -p[1]) return INFINITY;
                if (r < 0.0) return 0.5 * p[0] * (r * r) + p[2];
                return 0.0;
        }
    }
    // Xplor::s (xplor.rs): 1 below r_smooth, 0 beyond r_cut, the smoothing polynomial between.
    double xplor_s(double r) const {
        if (r < w[1]) return 1.0;
        if (r > w[0]) return 0.0;
        const double r_sq = r * r, rc_sq = w[0] * w[0], rs_sq = w[1] * w[1];
        const double a = rc_sq - r_sq, d = rc_sq - rs_sq;
        return a * a * (rc_sq + 2.0 * r_sq - 3.0 * rs_sq) / (d * d * d);
    }
    double energy(double r) const {
        switch (wrap) {
            case UVW_SHIFTED:  // shifted.rs:92-94
                return f(r) - f(w[0]);
            case UVW_EXPANDED:  // expanded.rs:64-66
                return f(r - w[0]);
            case UVW_XPLOR:
                return xplor_s(r) * f(r);
            default:
                return f(r);
        }
    }
    // Isotropic::site_pair_energy (isotropic.rs:147-156)
    double pair(double r2) const {
        if (r2 >= rcut * rcut) return 0.0;
        return energy(std::sqrt(r2));
    }
};

// ============================================================================
// hoomd-microstate: periodic hypercuboid boundary
// ============================================================================
// Periodic<Hypercuboid>::wrap, boundary/periodic/cuboid.rs:91-103.
void wrap(int dim, const double* L, double* x) {
    for (int a = 0; a < dim; ++a) {
        double lam = x[a] / L[a];
        lam = lam - std::round(lam);
        if (lam == 0.5) lam = -0.5;
        x[a] = lam * L[a];
    }
}
// generate_ghosts_in_range, cuboid.rs:109-161. Returns ghost count.
int ghosts(int dim, const double* L, double range, const double* x, double (*out)[3]) {
    unsigned mask = 0;
    double tr[3] = {0.0, 0.0, 0.0};
    for (int i = 0; i < dim; ++i) {
        double half = L[i] / 2.0;
        if (x[i] < -half || x[i] >= half) return 0;
        if (x[i] > half - range) {
            mask |= 1u << i;
            tr[i] = -L[i];
        } else if (x[i] < -half + range) {
            mask |= 1u << i;
            tr[i] = L[i];
        }
    }
    int n = 0;
    unsigned subset = mask;
    while (subset != 0) {
        for (int i = 0; i < dim; ++i) {
            out[n][i] = x[i];
            if (subset & (1u << i)) out[n][i] += tr[i];
        }
        ++n;
        subset = (subset - 1) & mask;
    }
    return n;
}

// ============================================================================
// hoomd-mc: HypercuboidCheckerboard (hypercuboid.rs)
// ============================================================================
struct Checkerboard {
    int dim = 0;
    double origin[3] = {0, 0, 0};
    double width[3] = {1, 1, 1};
    uint64_t shape[3] = {2, 2, 2};
    bool periodic = true;
};
// compute_dimensions, hypercuboid.rs:188-228. Returns false if the range is too large.
bool compute_dimensions(int dim, const double* L, double range, bool periodic, double* width, uint64_t* shape) {
    uint64_t inside[3];
    for (int i = 0; i < dim; ++i) {
        double f = std::floor(L[i] / range);
        if (!(f >= 2.0)) return false;
        inside[i] = (uint64_t)f;
    }
    for (int i = 0; i < dim; ++i) {
        if (periodic && inside[i] % 2 != 0) inside[i] -= 1;
        if (!periodic && inside[i] % 2 == 0) inside[i] -= 1;
    }
    for (int i = 0; i < dim; ++i) {
        width[i] = L[i] / (double)inside[i];
        shape[i] = periodic ? inside[i] : inside[i] + 1;
    }
    return true;
}
// multi_index_to_index, hypercuboid.rs:152-162 (last axis fastest).
uint64_t multi_to_index(int dim, const uint64_t* m, const uint64_t* shape) {
    uint64_t idx = 0, w = 1;
    for (int i = dim - 1; i >= 0; --i) {
        idx += m[i] * w;
        w *= shape[i];
    }
    return idx;
}
void index_to_multi(int dim, uint64_t idx, const uint64_t* shape, uint64_t* m) {
    for (int i = dim - 1; i >= 0; --i) {
        m[i] = idx % shape[i];
        idx /= shape[i];
    }
}
// point_to_space_index, hypercuboid.rs:85-128. Returns -1 for None.
int64_t point_to_space(const Checkerboard& cb, const double* x) {
    uint64_t m[3];
    for (int i = 0; i < cb.dim; ++i) {
        double p = x[i] - cb.origin[i];
        double f = std::floor(p / cb.width[i]);
        if (!(f >= 0.0)) return -1;  // negative index (also rejects NaN)
        if (f > 9.2e18) return -1;
        uint64_t idx = (uint64_t)(int64_t)f;
        if (cb.periodic) {
            if (idx == cb.shape[i]) idx = 0;
            if (idx > cb.shape[i]) return -1;
        } else if (idx >= cb.shape[i]) {
            return -1;
        }
        m[i] = idx;
    }
    return (int64_t)multi_to_index(cb.dim, m, cb.shape);
}
// construct_space_indices_by_color, hypercuboid.rs:231-256.
std::vector<std::vector<uint64_t>> colors(int dim, const uint64_t* shape) {
    uint64_t half[3], total = 1;
    for (int i = 0; i < dim; ++i) {
        half[i] = shape[i] / 2;
        total *= half[i];
    }
    std::vector<uint64_t> base(total);
    for (uint64_t idx = 0; idx < total; ++idx) {
        uint64_t hm[3], m[3];
        index_to_multi(dim, idx, half, hm);
        for (int i = 0; i < dim; ++i) m[i] = 2 * hm[i];
        base[idx] = multi_to_index(dim, m, shape);
    }
    int ncol = 1 << dim;
    uint64_t two[3] = {2, 2, 2};
    std::vector<std::vector<uint64_t>> out(ncol);
    for (int c = 0; c < ncol; ++c) {
        uint64_t off[3];
        index_to_multi(dim, (uint64_t)c, two, off);
        uint64_t delta = multi_to_index(dim, off, shape);
        out[c].resize(total);
        for (uint64_t k = 0; k < total; ++k) out[c][k] = base[k] + delta;
    }
    return out;
}
// HypercuboidCheckerboard::update with the ParallelSweep RNG, parallel_sweep.rs:176-201 and
// hypercuboid.rs:315-341: three (two) uniforms for the origin shift.
bool checkerboard_for_counter(int dim, const double* L, double range, uint64_t step, uint32_t substep,
                              uint32_t seed, Checkerboard& cb) {
    cb.dim = dim;
    cb.periodic = true;
    if (!compute_dimensions(dim, L, range, true, cb.width, cb.shape)) return false;
    Sfc64 rng = make_rng(step, substep, seed, UINT64_MAX);
    double off[3];
    for (int i = 0; i < dim; ++i) off[i] = uniform01(rng);
    for (int i = 0; i < dim; ++i) cb.origin[i] = -L[i] / 2.0 - off[i] * cb.width[i];
    return true;
}

// ============================================================================
// hoomd-mc trial moves
// ============================================================================
// Ball::sample, hoomd-vector/src/distribution.rs:41-69.
void ball_sample(Sfc64& rng, int dim, double r, double* out) {
    if (dim == 2) {
        for (;;) {
            double c0 = uniform01(rng);
            double c1 = uniform01(rng);
            double v[2] = {(c0 * 2.0 - 1.0) * r, (c1 * 2.0 - 1.0) * r};
            if (dot(v, v, 2) < r * r) {
                out[0] = v[0];
                out[1] = v[1];
                return;
            }
        }
    }
    double p[3];
    for (int i = 0; i < 3; ++i) p[i] = standard_normal(rng);
    double norm = std::sqrt(dot(p, p, 3));
    double u = uniform01(rng);
    double scale = r / norm * portable_cbrt(u);
    for (int i = 0; i < 3; ++i) out[i] = p[i] * scale;
}
// VersorDisplacement::sample, rotate/versor.rs:40-71 (Karney 2007).
Quat versor_displacement(Sfc64& rng, double sigma) {
    for (;;) {
        double s[3];
        for (int i = 0; i < 3; ++i) s[i] = 0.0 + sigma * standard_normal(rng);
        double theta = std::sqrt(dot(s, s, 3));
        if (theta > M_PI) continue;
        double half = 0.5 * theta;
        double sh, ch;
        portable_sincos(half, &sh, &ch);
        double vf = sh / theta;
        if (!std::isfinite(vf)) vf = 0.5;
        return {ch, s[0] * vf, s[1] * vf, s[2] * vf};
    }
}

// ============================================================================
// The microstate with a periodic neighbour grid
// ============================================================================
struct Grid {
    int dim = 3;
    uint64_t nc[3] = {1, 1, 1};
    double L[3] = {1, 1, 1};
    std::vector<std::vector<uint32_t>> cells;
    std::vector<uint64_t> cell_of;
    uint64_t cell_index(const double* x) const {
        uint64_t m[3] = {0, 0, 0};
        for (int a = 0; a < dim; ++a) {
            double f = (x[a] + L[a] / 2.0) / L[a];
            f = f - std::floor(f);
            double c = std::floor(f * (double)nc[a]);
            uint64_t ci = (c >= 0.0) ? (uint64_t)c : 0;
            if (ci >= nc[a]) ci = nc[a] - 1;
            m[a] = ci;
        }
        uint64_t idx = 0;
        for (int a = 0; a < dim; ++a) idx = idx * nc[a] + m[a];
        return idx;
    }
};

}  // namespace

struct oracle_system {
    int dim = 3;
    double L[3] = {1, 1, 1};
    uint64_t n = 0;
    std::vector<double> body;    // n * 3 (body positions B)
    std::vector<double> site;    // n * 3 (site positions S = wrap(B))
    std::vector<double> orient;  // n * 4 (versor) or n (angle)
    uint64_t step = 0;
    uint32_t substep = 0;
    uint32_t seed = 0;
    int interaction = ORACLE_HARD_SPHERE;
    double diameter = 1.0;
    Polytope poly;
    double eps = 1, sigma = 1, rcut = 2.5, rshift = 2.5;
    double boundary_range = 1.0;
    double body_range = 1.0;
    double search_range = 1.0;
    Grid grid;
    // tagged container (microstate.rs:60-123): tags by index, freed tags reused smallest first
    std::vector<uint64_t> tag;
    uint64_t tag_bound = 0;
    std::priority_queue<uint64_t, std::vector<uint64_t>, std::greater<uint64_t>> free_tags;
    uint64_t take_tag() {
        if (free_tags.empty()) return tag_bound++;
        const uint64_t t = free_tags.top();
        free_tags.pop();
        return t;
    }
    // Microstate::add_body: body = wrap(x), site = wrap(body), appended with orientation o
    // (oriented bodies; the site's orientation is the body's).
    void append_body(const double* x, const double* o) {
        for (int k = 0; k < ori_len(); ++k) orient.push_back(o[k]);
        append_body(x);
    }
    // Microstate::add_body for a point body: body = wrap(x), site = wrap(body), appended.
    void append_body(const double* x) {
        double b[3] = {x[0], x[1], x[2]};
        wrap(dim, L, b);
        double sv[3] = {b[0], b[1], b[2]};
        wrap(dim, L, sv);
        for (int a = 0; a < 3; ++a) body.push_back(b[a]);
        for (int a = 0; a < 3; ++a) site.push_back(sv[a]);
        const uint64_t i = n++;
        const uint64_t c = grid.cell_index(sv);
        grid.cell_of.push_back(c);
        grid.cells[c].push_back((uint32_t)i);
        tag.push_back(take_tag());
    }
    // Microstate::remove_body (microstate.rs:917-943) for a point body: swap_remove.
    void remove_body(uint64_t idx) {
        const uint64_t last = n - 1;
        auto drop = [&](uint64_t c, uint64_t v) {
            auto& cell = grid.cells[c];
            for (size_t k = 0; k < cell.size(); ++k)
                if (cell[k] == v) {
                    cell[k] = cell.back();
                    cell.pop_back();
                    return;
                }
        };
        drop(grid.cell_of[idx], idx);
        free_tags.push(tag[idx]);
        if (idx != last) {
            auto& cell = grid.cells[grid.cell_of[last]];
            for (auto& v : cell)
                if (v == last) v = (uint32_t)idx;
            for (int a = 0; a < 3; ++a) {
                body[3 * idx + a] = body[3 * last + a];
                site[3 * idx + a] = site[3 * last + a];
            }
            grid.cell_of[idx] = grid.cell_of[last];
            tag[idx] = tag[last];
        }
        body.resize(3 * last);
        site.resize(3 * last);
        grid.cell_of.resize(last);
        tag.resize(last);
        n = last;
    }

    bool shape_penalty() const {
        return interaction == ORACLE_CONVEX_POLYHEDRON_PENALTY || interaction == ORACLE_CONVEX_POLYGON_PENALTY ||
               interaction == ORACLE_SURFACE_MESH_2D_PENALTY;
    }
    bool hard() const {
        return interaction != ORACLE_LENNARD_JONES && interaction != ORACLE_OVERLAP_PENALTY &&
               interaction != ORACLE_ISOTROPIC && !shape_penalty();
    }
    double pk = 10000.0, pdmax = 0.2, pshoulder = 100.0;  // OverlapPenalty
    double presolution = 0.01, prcut = 1.0;              // ApproximateShapeOverlap, Anisotropic r_cut
    Univariate uv;                                       // ORACLE_ISOTROPIC
    bool oriented() const {
        return interaction == ORACLE_HARD_CONVEX_POLYGON || interaction == ORACLE_HARD_CONVEX_POLYHEDRON ||
               interaction == ORACLE_HARD_CONVEX_SURFACE_MESH_2D || shape_penalty();
    }

    void build_grid() {
        grid.dim = dim;
        for (int a = 0; a < dim; ++a) {
            grid.L[a] = L[a];
            double f = std::floor(L[a] / (search_range * (1.0 + 1e-9)));
            grid.nc[a] = f >= 1.0 ? (uint64_t)f : 1;
        }
        uint64_t total = 1;
        for (int a = 0; a < dim; ++a) total *= grid.nc[a];
        grid.cells.assign(total, {});
        grid.cell_of.assign(n, 0);
        for (uint64_t i = 0; i < n; ++i) {
            uint64_t c = grid.cell_index(&site[3 * i]);
            grid.cell_of[i] = c;
            grid.cells[c].push_back((uint32_t)i);
        }
    }
    void grid_move(uint64_t i) {
        uint64_t c = grid.cell_index(&site[3 * i]);
        uint64_t old = grid.cell_of[i];
        if (c == old) return;
        auto& v = grid.cells[old];
        for (size_t k = 0; k < v.size(); ++k)
            if (v[k] == i) {
                v[k] = v.back();
                v.pop_back();
                break;
            }
        grid.cells[c].push_back((uint32_t)i);
        grid.cell_of[i] = c;
    }
    // Candidate bodies near x (deduplicated periodic 3^d stencil), sorted by tag.
    void candidates(const double* x, std::vector<uint32_t>& out) const {
        out.clear();
        uint64_t c = grid.cell_index(x);
        uint64_t m[3] = {0, 0, 0};
        uint64_t rem = c;
        for (int a = dim - 1; a >= 0; --a) {
            m[a] = rem % grid.nc[a];
            rem /= grid.nc[a];
        }
        std::vector<uint64_t> axis_cells[3];
        for (int a = 0; a < dim; ++a) {
            if (grid.nc[a] < 3) {
                for (uint64_t k = 0; k < grid.nc[a]; ++k) axis_cells[a].push_back(k);
            } else {
                for (int o = -1; o <= 1; ++o)
                    axis_cells[a].push_back((m[a] + grid.nc[a] + (uint64_t)(int64_t)o) % grid.nc[a]);
            }
        }
        if (dim == 2) {
            for (uint64_t c0 : axis_cells[0])
                for (uint64_t c1 : axis_cells[1])
                    for (uint32_t j : grid.cells[c0 * grid.nc[1] + c1]) out.push_back(j);
        } else {
            for (uint64_t c0 : axis_cells[0])
                for (uint64_t c1 : axis_cells[1])
                    for (uint64_t c2 : axis_cells[2])
                        for (uint32_t j : grid.cells[(c0 * grid.nc[1] + c1) * grid.nc[2] + c2]) out.push_back(j);
        }
        std::sort(out.begin(), out.end());
    }

    // Pair energy between a trial site (x, o) and site j's image at y:
    // HardSphere hard_shape.rs:143-153; HardShape :79-94; Isotropic<Shifted<LJ>>.
    double pair(const double* x, const double* o, const double* y, uint64_t j) const {
        switch (interaction) {
            case ORACLE_HARD_SPHERE:
                return distance_squared(x, y, dim) < diameter * diameter ? INFINITY : 0.0;
            case ORACLE_HARD_CONVEX_POLYHEDRON: {
                Quat qi{o[0], o[1], o[2], o[3]};
                const double* oj = &orient[4 * j];
                Quat qj{oj[0], oj[1], oj[2], oj[3]};
                return convex_global_3d(poly, x, qi, y, qj) ? INFINITY : 0.0;
            }
            case ORACLE_HARD_CONVEX_POLYGON:
                return convex_global_2d(poly, x, o[0], y, orient[j]) ? INFINITY : 0.0;
            case ORACLE_HARD_CONVEX_SURFACE_MESH_2D:
                return sat_global_2d(poly, x, o[0], y, orient[j]) ? INFINITY : 0.0;
            case ORACLE_CONVEX_POLYHEDRON_PENALTY: {
                const double* oj = &orient[4 * j];
                return shape_penalty_3d(poly, prcut, presolution, pk, pdmax, pshoulder, x, Quat{o[0], o[1], o[2], o[3]},
                                        y, Quat{oj[0], oj[1], oj[2], oj[3]});
            }
            case ORACLE_CONVEX_POLYGON_PENALTY:
                return shape_penalty_2d(poly, prcut, presolution, pk, pdmax, pshoulder, x, o[0], y, orient[j]);
            case ORACLE_SURFACE_MESH_2D_PENALTY:
                return shape_penalty_2d<true>(poly, prcut, presolution, pk, pdmax, pshoulder, x, o[0], y, orient[j]);
            case ORACLE_ISOTROPIC:
                return uv.pair(distance_squared(x, y, dim));
            case ORACLE_OVERLAP_PENALTY: {
                // Isotropic::site_pair_energy (isotropic.rs:147-156) of Expanded { delta: diameter,
                // OverlapPenalty } (expanded.rs:64-66, overlap_penalty.rs:109-115), r_cut = diameter
                const double r2 = distance_squared(x, y, dim);
                if (r2 >= diameter * diameter) return 0.0;
                const double r = std::sqrt(r2) - diameter;
                if (r < -pdmax) return INFINITY;
                if (r < 0.0) return 0.5 * pk * (r * r) + pshoulder;
                return 0.0;
            }
            default:
                return shifted_lj_pair(eps, sigma, rcut, rshift, distance_squared(x, y, dim));
        }
    }

    // filtered_site_energy over the primary and the ghosts of every candidate,
    // excluding `self_body` (pairwise_cutoff.rs:355-385).
    double site_energy(const double* x, const double* o, uint64_t self_body, std::vector<uint32_t>& cand) const {
        candidates(x, cand);
        double energy = 0.0;
        double img[7][3];
        for (uint32_t j : cand) {
            if (j == self_body) continue;
            const double* sj = &site[3 * j];
            double one = pair(x, o, sj, j);
            if (one == INFINITY) return one;
            energy += one;
            int ng = ghosts(dim, L, boundary_range, sj, img);
            for (int g = 0; g < ng; ++g) {
                one = pair(x, o, img[g], j);
                if (one == INFINITY) return one;
                energy += one;
            }
        }
        return energy;
    }

    // PairwiseCutoff::delta_energy_one, pairwise_cutoff.rs:919-941, for a body whose trial
    // properties are (pos, ori) as passed to delta_energy_one (site = wrap(pos)).
    double delta_energy_one(uint64_t b, const double* pos, const double* ori) const {
        std::vector<uint32_t> cand;
        double t[3] = {pos[0], pos[1], dim == 3 ? pos[2] : 0.0};
        wrap(dim, L, t);
        double ef = site_energy(t, ori, b, cand);
        if (ef == INFINITY) return ef;
        double ei = 0.0;
        if (!hard()) ei = site_energy(&site[3 * b], ori_of(b), b, cand);
        return ef - ei;
    }
    const double* ori_of(uint64_t b) const {
        if (!oriented()) return nullptr;
        return dim == 3 ? &orient[4 * b] : &orient[b];
    }
    int ori_len() const { return oriented() ? (dim == 3 ? 4 : 1) : 0; }

    // Microstate::update_body_properties, microstate.rs:985-1056: body = wrap(props),
    // site = wrap(body).
    void update_body(uint64_t b, const double* pos, const double* ori) {
        double p[3] = {pos[0], pos[1], dim == 3 ? pos[2] : 0.0};
        wrap(dim, L, p);
        for (int a = 0; a < 3; ++a) body[3 * b + a] = p[a];
        wrap(dim, L, p);
        for (int a = 0; a < 3; ++a) site[3 * b + a] = p[a];
        for (int k = 0; k < ori_len(); ++k) orient[(size_t)ori_len() * b + k] = ori[k];
        grid_move(b);
    }

    // LocalTrial::propose for Translate<Cartesian> (translate/cartesian.rs:40-51),
    // Rotate<Versor> (rotate/versor.rs:112-123), Rotate<Angle> (rotate/angle.rs:46-55).
    void propose(Sfc64& rng, int move, double maximum, uint64_t b, double* pos, double* ori) const {
        for (int a = 0; a < 3; ++a) pos[a] = body[3 * b + a];
        for (int k = 0; k < ori_len(); ++k) ori[k] = orient[(size_t)ori_len() * b + k];
        if (move == ORACLE_TRANSLATE) {
            double d[3] = {0, 0, 0};
            ball_sample(rng, dim, maximum, d);
            for (int a = 0; a < dim; ++a) pos[a] = pos[a] + d[a];
        } else if (dim == 3) {
            Quat dq = versor_displacement(rng, maximum);
            Quat q = qmul(dq, Quat{ori[0], ori[1], ori[2], ori[3]});
            ori[0] = q.s;
            ori[1] = q.x;
            ori[2] = q.y;
            ori[3] = q.z;
        } else {
            // Uniform(-a, a): low + (high - low) * U with 52-bit U in [0, 1).
            uint64_t bits = rng.next_u64() >> 12;
            double u = bits_to_double(0x3FF0000000000000ULL | bits) - 1.0;
            ori[0] = ori[0] + (u * (maximum - (-maximum)) + (-maximum));
        }
    }
};

extern "C" {

void oracle_sfc64_outputs(uint64_t a, uint64_t b, uint64_t c, uint64_t counter, uint64_t n_skip, uint64_t n,
                          uint64_t* out) {
    Sfc64 r = Sfc64::initialize(a, b, c, counter);
    for (uint64_t i = 0; i < n_skip; ++i) r.next_u64();
    for (uint64_t i = 0; i < n; ++i) out[i] = r.next_u64();
}
// SeedableRng::seed_from_u64, sfc.rs:119-122.
void oracle_sfc64_seed_from_u64(uint64_t state, uint64_t n_skip, uint64_t n, uint64_t* out) {
    oracle_sfc64_outputs(state, 0, 0, 1, n_skip, n, out);
}
void oracle_counter_outputs(uint64_t step, uint32_t substep, uint32_t seed, uint64_t index, uint64_t n,
                            uint64_t* out) {
    Sfc64 r = make_rng(step, substep, seed, index);
    for (uint64_t i = 0; i < n; ++i) out[i] = r.next_u64();
}
void oracle_counter_uniforms(uint64_t step, uint32_t substep, uint32_t seed, uint64_t index, uint64_t n,
                             double* out) {
    Sfc64 r = make_rng(step, substep, seed, index);
    for (uint64_t i = 0; i < n; ++i) out[i] = uniform01(r);
}
void oracle_counter_normals(uint64_t step, uint32_t substep, uint32_t seed, uint64_t index, uint64_t n,
                            double* out) {
    Sfc64 r = make_rng(step, substep, seed, index);
    for (uint64_t i = 0; i < n; ++i) out[i] = standard_normal(r);
}
void oracle_counter_ball(uint64_t step, uint32_t substep, uint32_t seed, uint64_t index, uint32_t dim,
                         double radius, uint64_t n, double* out) {
    Sfc64 r = make_rng(step, substep, seed, index);
    for (uint64_t i = 0; i < n; ++i) ball_sample(r, (int)dim, radius, out + i * dim);
}
uint32_t oracle_counter_choose(uint64_t step, uint32_t substep, uint32_t seed, uint64_t index, uint32_t len) {
    Sfc64 r = make_rng(step, substep, seed, index);
    return canon_range_u32(r, len);
}
double oracle_cbrt(double x) { return portable_cbrt(x); }
void oracle_sincos_half(double theta, double* s, double* c) { portable_sincos(theta, s, c); }
int oracle_cr_sincos(double x, double* s, double* c) { return cr_sincos(x, s, c); }
void oracle_ziggurat_tables(double* x_out, double* f_out) {
    for (int i = 0; i <= ZIG_LAYERS; ++i) {
        x_out[i] = zig().x[i];
        f_out[i] = zig().f[i];
    }
}

void oracle_wrap(uint32_t dim, const double* L, double* point) { wrap((int)dim, L, point); }
void oracle_set_penalty(oracle_system* s, double k, double maximum_allowed_overlap, double epsilon_shoulder) {
    s->pk = k;
    s->pdmax = maximum_allowed_overlap;
    s->pshoulder = epsilon_shoulder;
}
static Polytope make_poly(const double* verts, uint32_t nv, int dim);
void oracle_set_isotropic(oracle_system* s, uint32_t kind, const double* params, uint32_t wrap,
                          const double* wrap_params, double r_cut) {
    Univariate& u = s->uv;
    u.kind = (int)kind;
    u.wrap = (int)wrap;
    for (int k = 0; k < 4; ++k) u.p[k] = params[k];
    for (int k = 0; k < 2; ++k) u.w[k] = wrap_params[k];
    if (kind == UV_WEEKS_CHANDLER_ANDERSON) u.p[2] = std::pow(2.0, 1.0 / 6.0);
    u.rcut = r_cut;
    s->search_range = r_cut;
    s->build_grid();
}
double oracle_univariate_energy(uint32_t kind, const double* params, uint32_t wrap, const double* wrap_params,
                                double r) {
    Univariate u;
    u.kind = (int)kind;
    u.wrap = (int)wrap;
    for (int k = 0; k < 4; ++k) u.p[k] = params[k];
    for (int k = 0; k < 2; ++k) u.w[k] = wrap_params[k];
    if (kind == UV_WEEKS_CHANDLER_ANDERSON) u.p[2] = std::pow(2.0, 1.0 / 6.0);
    return u.energy(r);
}
void oracle_set_shape_overlap(oracle_system* s, double resolution, double r_cut) {
    s->presolution = resolution;
    s->prcut = r_cut;
    s->search_range = r_cut;
    s->build_grid();
}
double oracle_approximate_separation(uint32_t dim, const double* vertices, uint32_t n_vertices, const double* v_ij,
                                     const double* o_ij, double resolution, uint32_t sat) {
    const Polytope p = make_poly(vertices, n_vertices, (int)dim);
    if (dim == 3) return approximate_separation<3>(p, v_ij, mat_from_versor(Quat{o_ij[0], o_ij[1], o_ij[2], o_ij[3]}),
                                                   resolution);
    double m[2][2];
    mat2_from_angle(o_ij[0], m);
    if (sat) return approximate_separation<2, double[2][2], true>(p, v_ij, m, resolution);
    return approximate_separation<2>(p, v_ij, m, resolution);
}
uint64_t oracle_n_bodies(const oracle_system* s) { return s->n; }
void oracle_get_box(const oracle_system* s, double* edge_lengths) {
    for (int a = 0; a < s->dim; ++a) edge_lengths[a] = s->L[a];
}

// Microstate::clone_with_boundary (microstate.rs:1529-1565) with Hypercuboid::map_point
// (cuboid.rs:553-565): inside check in the old box, scale by L'/L, clamp to
// [-L'/2, next_down(L'/2)], then update_body_properties (body = wrap, site = wrap(body)).
int oracle_set_box(oracle_system* s, const double* edge_lengths) {
    std::vector<double> body = s->body;
    for (uint64_t i = 0; i < s->n; ++i) {
        double* x = &body[3 * i];
        for (int a = 0; a < s->dim; ++a)
            if (!(-s->L[a] / 2.0 <= x[a] && x[a] < s->L[a] / 2.0)) return -1;
        for (int a = 0; a < s->dim; ++a) {
            const double scale = edge_lengths[a] / s->L[a];
            double y = scale * x[a];
            const double lo = -edge_lengths[a] / 2.0, hi = std::nextafter(edge_lengths[a] / 2.0, -INFINITY);
            if (y < lo) y = lo;
            if (y > hi) y = hi;
            x[a] = y;
        }
    }
    for (int a = 0; a < s->dim; ++a) s->L[a] = edge_lengths[a];
    for (uint64_t i = 0; i < s->n; ++i) {
        double p[3] = {body[3 * i], body[3 * i + 1], body[3 * i + 2]};
        wrap(s->dim, s->L, p);
        for (int a = 0; a < 3; ++a) s->body[3 * i + a] = p[a];
        wrap(s->dim, s->L, p);
        for (int a = 0; a < 3; ++a) s->site[3 * i + a] = p[a];
    }
    s->build_grid();
    return 0;
}

// StandardUniform orientations: Versor from four standard normals, scalar first, divided by
// sqrt(|v|^2 + s^2) (quaternion.rs:863-885); Angle from Uniform::new(0, 2 pi) (angle.rs:268-285).
static void uniform_orientation(Sfc64& rng, int dim, double* o) {
    if (dim == 3) {
        const double sc = standard_normal(rng);
        double v[3];
        for (int a = 0; a < 3; ++a) v[a] = standard_normal(rng);
        const double norm = std::sqrt(dot(v, v, 3) + sc * sc);
        o[0] = sc / norm;
        for (int a = 0; a < 3; ++a) o[1 + a] = v[a] / norm;
    } else {
        const double two_pi = 2.0 * 3.141592653589793;
        const uint64_t bits = rng.next_u64() >> 12;
        const double u = bits_to_double(0x3FF0000000000000ULL | bits) - 1.0;
        o[0] = u * (two_pi - 0.0) + 0.0;
    }
}

void oracle_quick_insert(oracle_system* s, uint64_t target, uint64_t allowed_overlaps, uint64_t* inserted,
                         uint32_t* complete, uint64_t* accepted, uint64_t* rejected) {
    *accepted = 0;
    *rejected = 0;
    if (*complete) return;
    const double energy = oracle_total_energy(s);
    if (energy <= 0.0 && *inserted >= target) {
        *complete = 1;
        return;
    }
    if (energy <= 0.0) {
        Sfc64 rng = make_rng(s->step, s->substep, s->seed, 0);
        uint64_t overlapping = 0;
        std::vector<uint32_t> cand;
        for (uint64_t attempt = 0; attempt < target; ++attempt) {
            // UniformIn::sample: per axis Uniform::new(-L/2, L/2).sample(rng) (cuboid.rs:568-596)
            double x[3] = {0.0, 0.0, 0.0};
            for (int a = 0; a < s->dim; ++a) {
                const double low = -s->L[a] / 2.0, high = s->L[a] / 2.0;
                const uint64_t bits = rng.next_u64() >> 12;
                const double u = bits_to_double(0x3FF0000000000000ULL | bits) - 1.0;
                x[a] = u * (high - low) + low;
            }
            // oriented bodies: then a uniform random orientation (uniform_in.rs:158-176)
            double o[4] = {1.0, 0.0, 0.0, 0.0};
            if (s->oriented()) uniform_orientation(rng, s->dim, o);
            // delta_energy_insert: the site is wrap(transform(body, site)) (pairwise_cutoff.rs:420-450)
            double t[3] = {x[0], x[1], x[2]};
            wrap(s->dim, s->L, t);
            const double de = s->site_energy(t, s->oriented() ? o : nullptr, UINT64_MAX, cand);
            if (std::isfinite(de)) {
                if (s->oriented())
                    s->append_body(x, o);
                else
                    s->append_body(x);
                *accepted += 1;
                *inserted += 1;
                if (de > 0.0) overlapping += 1;
                if (*inserted == target || overlapping >= allowed_overlaps) break;
            } else {
                *rejected += 1;
            }
        }
    }
    s->substep += 1;
}

// GrandCanonical::apply (grand_canonical.rs:49-110) for point bodies, one trial.
void oracle_grand_canonical(oracle_system* s, double temperature, double fugacity, uint64_t* counts) {
    const uint64_t n = s->n;
    double volume = s->L[0];
    for (int a = 1; a < s->dim; ++a) volume = volume * s->L[a];
    Sfc64 rng = make_rng(s->step, s->substep, s->seed, 0);
    if (n == 0 && fugacity <= 0.0) {
        s->substep += 1;
        return;
    }
    const bool insert = (int32_t)(uint32_t)rng.next_u64() < 0;  // rand bool: sign of next_u32
    std::vector<uint32_t> cand;
    if (insert) {
        double x[3] = {0.0, 0.0, 0.0};
        for (int a = 0; a < s->dim; ++a) {
            const double low = -s->L[a] / 2.0, high = s->L[a] / 2.0;
            const uint64_t bits = rng.next_u64() >> 12;
            const double u = bits_to_double(0x3FF0000000000000ULL | bits) - 1.0;
            x[a] = u * (high - low) + low;
        }
        double t[3] = {x[0], x[1], x[2]};
        wrap(s->dim, s->L, t);
        const double de = s->site_energy(t, nullptr, UINT64_MAX, cand);
        if (std::isfinite(de)) {
            const double p = (volume * fugacity * std::exp(-de / temperature)) / ((double)n + 1.0);
            if (p > uniform01(rng)) {
                s->append_body(x);
                counts[0] += 1;
            } else {
                counts[1] += 1;
            }
        } else {
            counts[1] += 1;
        }
    } else if (n > 0) {
        const uint64_t idx = canon_range_u32(rng, (uint32_t)n);
        const double ei = s->hard() ? 0.0 : s->site_energy(&s->site[3 * idx], nullptr, idx, cand);
        const double de = -ei;
        const double p = fugacity <= 0.0 ? 1.0 : ((double)n * std::exp(-de / temperature)) / (volume * fugacity);
        if (p > uniform01(rng)) {
            s->remove_body(idx);
            counts[2] += 1;
        } else {
            counts[3] += 1;
        }
    }
    s->substep += 1;
}

int oracle_quick_compress(oracle_system* s, double target_volume, double maximum_energy_per_site,
                          double maximum_delta, uint32_t* state, uint32_t* is_final, double* boundary) {
    Sfc64 rng = make_rng(s->step, s->substep, s->seed, 0);
    s->substep += 1;
    double L[3] = {s->L[0], s->L[1], s->L[2]};
    auto same = [&]() {
        for (int a = 0; a < s->dim; ++a)
            if (boundary[a] != L[a]) return false;
        return true;
    };
    auto wait_on = [&](bool fin, const double* b) {
        *state = 1;
        *is_final = fin ? 1u : 0u;
        for (int a = 0; a < 3; ++a) boundary[a] = a < s->dim ? b[a] : 0.0;
    };
    switch (*state) {
        case 0:
            wait_on(false, L);
            break;
        case 3:
            if (!same()) wait_on(false, L);
            break;
        case 2: {
            const uint64_t bits = rng.next_u64() >> 12;
            const double u = bits_to_double(0x3FF0000000000000ULL | bits) - 1.0;
            const double delta = u * (maximum_delta - 0.0) + 0.0;
            double volume = L[0];
            for (int a = 1; a < s->dim; ++a) volume = volume * L[a];
            const double trial_volume = target_volume > volume ? std::min(volume * (1.0 + delta), target_volume)
                                                               : std::max(volume * (1.0 - delta), target_volume);
            const double v = std::pow(trial_volume / volume, 1.0 / (double)s->dim);
            double Ln[3] = {L[0], L[1], L[2]};
            for (int a = 0; a < s->dim; ++a) Ln[a] = L[a] * v;
            const double e0 = oracle_total_energy(s);
            oracle_system saved = *s;
            if (oracle_set_box(s, Ln) != 0) return -1;
            const double e1 = oracle_total_energy(s);
            if (e1 - e0 > maximum_energy_per_site * (double)s->n) {
                *s = saved;
            } else {
                wait_on(trial_volume == target_volume, Ln);
            }
            break;
        }
        case 1:
            if (oracle_total_energy(s) <= 0.0) {
                if (*is_final && same()) {
                    *state = 3;
                    for (int a = 0; a < 3; ++a) boundary[a] = a < s->dim ? L[a] : 0.0;
                } else {
                    *state = 2;
                }
            }
            break;
    }
    return 0;
}
// AppendMicrostate::append_microstate (hoomd-microstate/src/append.rs:46-113) for single-site
// bodies: each site is wrap(body.transform(site_local)) with the site at the body origin and the
// identity orientation (microstate.rs:995-1010; Transform for Point: position + site position,
// for OrientedPoint: position + rotate(site position), orientation.combine(site orientation),
// property/oriented_point.rs:108-113), written in tag order as FP32 (Rust `as f32`). 2-D
// orientations are written as Versor::from_axis_angle(z, theta) (append.rs:91-104,
// quaternion.rs:560-567). pos: n x 3 floats; ori: n x 4 floats (oriented shapes only).
void oracle_gsd_frame(const oracle_system* s, float* pos, float* ori) {
    const double zero[3] = {0.0, 0.0, 0.0};
    std::vector<uint64_t> order(s->n);  // iter_sites_tag_order
    for (uint64_t i = 0; i < s->n; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) { return s->tag[a] < s->tag[b]; });
    for (uint64_t row = 0; row < s->n; ++row) {
        const uint64_t i = order[row];
        double p[3] = {0.0, 0.0, 0.0};
        const double* b = &s->body[3 * i];
        if (!s->oriented()) {
            for (int a = 0; a < s->dim; ++a) p[a] = b[a] + zero[a];
        } else if (s->dim == 3) {
            const double* o = &s->orient[4 * i];
            const Quat q{o[0], o[1], o[2], o[3]};
            const V3 r = versor_rotate(q, zero);
            for (int a = 0; a < 3; ++a) p[a] = b[a] + r.v[a];
            const Quat site = qmul(q, Quat{1.0, 0.0, 0.0, 0.0});
            ori[4 * row + 0] = (float)site.s;
            ori[4 * row + 1] = (float)site.x;
            ori[4 * row + 2] = (float)site.y;
            ori[4 * row + 3] = (float)site.z;
        } else {
            const double theta = s->orient[i];
            double sn, cs;
            cr_sincos(theta, &sn, &cs);  // Angle::rotate (angle.rs:175-182)
            const double r[2] = {zero[0] * cs - zero[1] * sn, zero[0] * sn + zero[1] * cs};
            for (int a = 0; a < 2; ++a) p[a] = b[a] + r[a];
            const double t = theta + 0.0;  // Angle::combine with the site's angle 0
            double hs, hc;
            cr_sincos(t / 2.0, &hs, &hc);
            ori[4 * row + 0] = (float)hc;
            ori[4 * row + 1] = (float)(0.0 * hs);
            ori[4 * row + 2] = (float)(0.0 * hs);
            ori[4 * row + 3] = (float)(1.0 * hs);
        }
        wrap(s->dim, s->L, p);
        pos[3 * row + 0] = (float)p[0];
        pos[3 * row + 1] = (float)p[1];
        pos[3 * row + 2] = s->dim == 3 ? (float)p[2] : 0.0f;
    }
}
uint32_t oracle_generate_ghosts(uint32_t dim, const double* L, double range, const double* point,
                                double* out) {
    double g[7][3];
    int n = ghosts((int)dim, L, range, point, g);
    for (int k = 0; k < n; ++k)
        for (uint32_t a = 0; a < dim; ++a) out[k * dim + a] = g[k][a];
    return (uint32_t)n;
}
int oracle_checkerboard_dimensions(uint32_t dim, const double* L, double range, int periodic, double* width,
                                   uint64_t* shape) {
    return compute_dimensions((int)dim, L, range, periodic != 0, width, shape) ? 0 : 1;
}
int64_t oracle_point_to_space_index(uint32_t dim, const double* origin, const double* width,
                                    const uint64_t* shape, int periodic, const double* point) {
    Checkerboard cb;
    cb.dim = (int)dim;
    cb.periodic = periodic != 0;
    for (uint32_t i = 0; i < dim; ++i) {
        cb.origin[i] = origin[i];
        cb.width[i] = width[i];
        cb.shape[i] = shape[i];
    }
    return point_to_space(cb, point);
}
void oracle_space_indices_by_color(uint32_t dim, const uint64_t* shape, uint64_t* out) {
    auto c = colors((int)dim, shape);
    size_t k = 0;
    for (auto& v : c)
        for (uint64_t x : v) out[k++] = x;
}
int oracle_checkerboard_for_counter(uint32_t dim, const double* L, double range, uint64_t step, uint32_t substep,
                                    uint32_t seed, double* origin, double* width, uint64_t* shape) {
    Checkerboard cb;
    if (!checkerboard_for_counter((int)dim, L, range, step, substep, seed, cb)) return 1;
    for (uint32_t i = 0; i < dim; ++i) {
        origin[i] = cb.origin[i];
        width[i] = cb.width[i];
        shape[i] = cb.shape[i];
    }
    return 0;
}

static Polytope make_poly(const double* verts, uint32_t nv, int dim) {
    Polytope p;
    p.dim = dim;
    p.nv = (int)nv;
    p.verts.assign(verts, verts + nv * dim);
    p.bounding_radius = polytope_bounding_radius(verts, (int)nv, dim);
    return p;
}
// Convex::intersects_at 3-D, convex.rs:125-137 (bounding-sphere check with <=).
int oracle_convex_intersects_at_3d(const double* va, uint32_t na, const double* vb, uint32_t nb, const double* vij,
                                   const double* qij) {
    Polytope a = make_poly(va, na, 3), b = make_poly(vb, nb, 3);
    double rs = a.bounding_radius + b.bounding_radius;
    if (!(dot(vij, vij, 3) <= rs * rs)) return 0;
    return collide3d(a, b, vij, mat_from_versor(Quat{qij[0], qij[1], qij[2], qij[3]})) ? 1 : 0;
}
int oracle_convex_intersects_at_2d(const double* va, uint32_t na, const double* vb, uint32_t nb, const double* vij,
                                   double theta) {
    Polytope a = make_poly(va, na, 2), b = make_poly(vb, nb, 2);
    double rs = a.bounding_radius + b.bounding_radius;
    if (!(dot(vij, vij, 2) <= rs * rs)) return 0;
    double m[2][2];
    mat2_from_angle(theta, m);
    return collide2d(a, b, vij, m) ? 1 : 0;
}
int oracle_surface_mesh_intersects_at_2d(const double* va, uint32_t na, const double* vb, uint32_t nb,
                                         const double* vij, double theta) {
    Polytope a = make_poly(va, na, 2), b = make_poly(vb, nb, 2);
    double m[2][2];
    mat2_from_angle(theta, m);
    return sat_intersects_at(a, b, vij, m) ? 1 : 0;
}
int oracle_convex_intersects_at_global_3d(const double* verts, uint32_t nv, const double* ri, const double* qi,
                                          const double* rj, const double* qj) {
    Polytope p = make_poly(verts, nv, 3);
    return convex_global_3d(p, ri, Quat{qi[0], qi[1], qi[2], qi[3]}, rj, Quat{qj[0], qj[1], qj[2], qj[3]}) ? 1 : 0;
}
// Versor::from_axis_angle, quaternion.rs:560-567 (library cos/sin, as the reference).
void oracle_versor_from_axis_angle(const double* axis, double angle, double* q) {
    q[0] = std::cos(angle / 2.0);
    double s = std::sin(angle / 2.0);
    q[1] = axis[0] * s;
    q[2] = axis[1] * s;
    q[3] = axis[2] * s;
}
void oracle_versor_combine(const double* a, const double* b, double* out) {
    Quat r = qmul(Quat{a[0], a[1], a[2], a[3]}, Quat{b[0], b[1], b[2], b[3]});
    out[0] = r.s;
    out[1] = r.x;
    out[2] = r.y;
    out[3] = r.z;
}
void oracle_versor_rotate(const double* q, const double* v, double* out) {
    V3 r = versor_rotate(Quat{q[0], q[1], q[2], q[3]}, v);
    for (int i = 0; i < 3; ++i) out[i] = r.v[i];
}
double oracle_lj_energy(double eps, double sigma, double r) { return lj_energy(eps, sigma, r); }
double oracle_shifted_lj_pair(double eps, double sigma, double rcut, double rshift, double r2) {
    return shifted_lj_pair(eps, sigma, rcut, rshift, r2);
}

oracle_system* oracle_system_create(uint32_t dim, const double* L, uint64_t n, const double* positions,
                                    const double* orientations, uint64_t step, uint32_t substep, uint32_t seed,
                                    uint32_t interaction, double diameter, const double* vertices,
                                    uint32_t n_vertices, double eps, double sigma, double rcut, double rshift,
                                    double boundary_range) {
    oracle_system* s = new oracle_system();
    s->dim = (int)dim;
    for (uint32_t a = 0; a < dim; ++a) s->L[a] = L[a];
    s->n = n;
    s->step = step;
    s->substep = substep;
    s->seed = seed;
    s->interaction = (int)interaction;
    s->diameter = diameter;
    s->eps = eps;
    s->sigma = sigma;
    s->rcut = rcut;
    s->rshift = rshift;
    s->boundary_range = boundary_range;
    if (s->oriented()) s->poly = make_poly(vertices, n_vertices, (int)dim);
    switch (interaction) {
        case ORACLE_HARD_SPHERE:
            s->search_range = diameter;
            break;
        case ORACLE_LENNARD_JONES:
            s->search_range = rcut;
            break;
        case ORACLE_OVERLAP_PENALTY:
            s->search_range = diameter;
            break;
        case ORACLE_ISOTROPIC:  // r_cut, set again by oracle_set_isotropic
            s->search_range = boundary_range;
            break;
        default:
            s->search_range = s->poly.bounding_radius * 2.0;
            s->prcut = s->search_range;
    }
    s->body.assign(3 * n, 0.0);
    s->site.assign(3 * n, 0.0);
    s->tag.resize(n);
    for (uint64_t i = 0; i < n; ++i) s->tag[i] = i;
    s->tag_bound = n;
    int ol = s->ori_len();
    s->orient.assign((size_t)ol * n, 0.0);
    // Microstate::add_body, microstate.rs:777-835: body = wrap(input), site = wrap(body).
    for (uint64_t i = 0; i < n; ++i) {
        double p[3] = {0, 0, 0};
        for (uint32_t a = 0; a < dim; ++a) p[a] = positions[i * dim + a];
        wrap((int)dim, s->L, p);
        for (int a = 0; a < 3; ++a) s->body[3 * i + a] = p[a];
        wrap((int)dim, s->L, p);
        for (int a = 0; a < 3; ++a) s->site[3 * i + a] = p[a];
        for (int k = 0; k < ol; ++k) s->orient[(size_t)ol * i + k] = orientations ? orientations[(size_t)ol * i + k] : (k == 0 && ol == 4 ? 1.0 : 0.0);
    }
    s->build_grid();
    return s;
}
void oracle_system_destroy(oracle_system* s) { delete s; }
void oracle_get_state(const oracle_system* s, double* positions, double* orientations, uint64_t* step,
                      uint32_t* substep) {
    for (uint64_t i = 0; i < s->n; ++i)
        for (int a = 0; a < s->dim; ++a) positions[i * s->dim + a] = s->body[3 * i + a];
    if (orientations)
        for (size_t k = 0; k < s->orient.size(); ++k) orientations[k] = s->orient[k];
    if (step) *step = s->step;
    if (substep) *substep = s->substep;
}
void oracle_set_counter(oracle_system* s, uint64_t step, uint32_t substep) {
    s->step = step;
    s->substep = substep;
}
// Microstate::increment_step, microstate.rs:412-415.
void oracle_increment_step(oracle_system* s) {
    s->step += 1;
    s->substep = 0;
}

// ParallelSweep::apply (parallel_sweep.rs:390-421). The trials of one colour pass only read
// the pre-colour state, so `threads` workers evaluate contiguous slices of the colour's
// space list (the reference does this with rayon); the accepted moves are then applied in
// space-list order, so the cell lists, and with them every later sum, do not depend on the
// thread count.
static int parallel_sweep_impl(oracle_system* s, uint32_t move, double maximum, double kt, double range,
                               unsigned threads, uint64_t* accepted, uint64_t* rejected) {
    // update_checkerboard, parallel_sweep.rs:176-201
    Checkerboard cb;
    if (!checkerboard_for_counter(s->dim, s->L, range, s->step, s->substep, s->seed, cb)) return 1;
    uint64_t nspaces = 1;
    for (int a = 0; a < s->dim; ++a) nspaces *= cb.shape[a];
    std::vector<std::vector<uint32_t>> spaces(nspaces);
    for (uint64_t i = 0; i < s->n; ++i) {
        int64_t sp = point_to_space(cb, &s->body[3 * i]);
        if (sp < 0) return 2;  // the reference panics ("body should be inside the checkerboard")
        spaces[(size_t)sp].push_back((uint32_t)i);
    }
    auto by_color = colors(s->dim, cb.shape);
    uint64_t acc = 0, rej = 0;
    struct Trial {
        uint64_t body;
        double pos[3];
        double ori[4];
        int outcome;  // 0 empty space, 1 rejected, 2 accepted
    };
    std::vector<Trial> trials;
    int ol = s->ori_len();
    if (threads == 0) threads = 1;
    // generate_trial_moves, :209-279 (every trial sees the pre-colour state)
    auto generate = [&](const std::vector<uint64_t>& space_indices, size_t lo, size_t hi) {
        for (size_t k = lo; k < hi; ++k) {
            uint64_t sp = space_indices[k];
            Trial& t = trials[k];
            t.outcome = 0;
            const auto& members = spaces[sp];
            Sfc64 rng = make_rng(s->step, s->substep, s->seed, sp);
            if (members.empty()) continue;  // EmptySpace: not counted (:299)
            uint32_t pick = canon_range_u32(rng, (uint32_t)members.size());
            uint64_t b = members[pick];
            t.body = b;
            for (int q = 0; q < 4; ++q) t.ori[q] = 0.0;
            s->propose(rng, (int)move, maximum, b, t.pos, t.ori);
            wrap(s->dim, s->L, t.pos);
            t.outcome = 1;
            if (point_to_space(cb, t.pos) != (int64_t)sp) continue;
            double dh = s->delta_energy_one(b, t.pos, t.ori);
            if (dh != INFINITY && (dh <= 0.0 || uniform01(rng) < std::exp(-dh / kt))) t.outcome = 2;
        }
    };
    // apply, :390-421
    while (acc + rej < s->n) {
        for (auto& space_indices : by_color) {
            size_t m = space_indices.size();
            trials.resize(m);
            if (threads == 1 || m < 4 * (size_t)threads) {
                generate(space_indices, 0, m);
            } else {
                std::vector<std::thread> pool;
                size_t chunk = (m + threads - 1) / threads;
                for (unsigned w = 0; w < threads; ++w) {
                    size_t lo = std::min(m, w * chunk), hi = std::min(m, lo + chunk);
                    pool.emplace_back(generate, std::cref(space_indices), lo, hi);
                }
                for (auto& th : pool) th.join();
            }
            // update_bodies, :283-314
            for (auto& t : trials) {
                if (t.outcome == 2) {
                    s->update_body(t.body, t.pos, ol ? t.ori : nullptr);
                    acc += 1;
                } else if (t.outcome == 1) {
                    rej += 1;
                }
            }
        }
        s->substep += 1;
    }
    *accepted = acc;
    *rejected = rej;
    return 0;
}

int oracle_parallel_sweep(oracle_system* s, uint32_t move, double maximum, double kt, double range,
                          uint64_t* accepted, uint64_t* rejected) {
    return parallel_sweep_impl(s, move, maximum, kt, range, 1, accepted, rejected);
}

int oracle_parallel_sweep_threads(oracle_system* s, uint32_t move, double maximum, double kt, double range,
                                  uint32_t threads, uint64_t* accepted, uint64_t* rejected) {
    return parallel_sweep_impl(s, move, maximum, kt, range, threads, accepted, rejected);
}

int oracle_serial_sweep(oracle_system* s, uint32_t move, double maximum, double kt, uint64_t* accepted,
                        uint64_t* rejected) {
    return oracle_serial_sweep_filter(s, move, maximum, kt, nullptr, accepted, rejected);
}

int oracle_serial_sweep_filter(oracle_system* s, uint32_t move, double maximum, double kt, const uint8_t* mask,
                               uint64_t* accepted, uint64_t* rejected) {
    // Sweep::apply_with_filter, sweep.rs:159-224; a body the filter excludes draws nothing
    Sfc64 rng = make_rng(s->step, s->substep, s->seed, 0);
    uint64_t acc = 0, rej = 0;
    int ol = s->ori_len();
    for (uint64_t b = 0; b < s->n; ++b) {
        if (mask && !mask[b]) continue;
        double pos[3] = {0, 0, 0}, ori[4] = {0, 0, 0, 0};
        s->propose(rng, (int)move, maximum, b, pos, ori);
        wrap(s->dim, s->L, pos);
        double dh = s->delta_energy_one(b, pos, ori);
        if (dh != INFINITY && (dh <= 0.0 || uniform01(rng) < std::exp(-dh / kt))) {
            s->update_body(b, pos, ol ? ori : nullptr);
            acc += 1;
        } else {
            rej += 1;
        }
    }
    s->substep += 1;
    *accepted = acc;
    *rejected = rej;
    return 0;
}

// Tune::tune_with_options (tune_local.rs:21-89) with one counter stream per sample:
// sample j of round t uses Counter(step, substep, seed).index(2^63 | t << 32 | j), draws the
// body index, the move and the Metropolis uniform; the state is not modified.
double oracle_tune(const oracle_system* s, uint32_t move, double maximum, double kt, double target, uint32_t samples,
                   uint32_t steps) {
    int ol = s->ori_len();
    for (uint32_t t = 0; t < steps; ++t) {
        uint64_t acc = 0;
        for (uint32_t j = 0; j < samples; ++j) {
            Sfc64 rng = make_rng(s->step, s->substep, s->seed, (1ull << 63) | ((uint64_t)t << 32) | (uint64_t)j);
            uint64_t b = canon_range_u32(rng, (uint32_t)s->n);
            double pos[3] = {0, 0, 0}, ori[4] = {0, 0, 0, 0};
            s->propose(rng, (int)move, maximum, b, pos, ori);
            wrap(s->dim, s->L, pos);
            double u = uniform01(rng);
            double dh = s->delta_energy_one(b, pos, ol ? ori : nullptr);
            if (dh != INFINITY && (dh <= 0.0 || u < std::exp(-dh / kt))) acc += 1;
        }
        double ratio = (double)acc / (double)samples;
        maximum *= (ratio + 1.5) / (target + 1.5);
    }
    return maximum;
}

// The trial-move samplers for a body at the origin with the identity orientation, sample i from
// Counter(step, substep, seed).index(i): kind 0 Translate (ball_sample, distribution.rs:41-69),
// kind 1 Rotate (3-D Rotate<Versor>, rotate/versor.rs:40-71, 112-123; 2-D Rotate<Angle>,
// rotate/angle.rs:46-55), kind 2 one StandardNormal.
void oracle_sample_moves(uint32_t dim, uint32_t kind, double maximum, uint64_t step, uint32_t substep, uint32_t seed,
                         uint64_t n, double* out) {
    for (uint64_t i = 0; i < n; ++i) {
        Sfc64 rng = make_rng(step, substep, seed, i);
        if (kind == 2) {
            out[i] = standard_normal(rng);
        } else if (kind == 0) {
            double d[3] = {0, 0, 0};
            ball_sample(rng, (int)dim, maximum, d);
            for (uint32_t a = 0; a < dim; ++a) out[i * dim + a] = d[a];
        } else if (dim == 3) {
            Quat q = qmul(versor_displacement(rng, maximum), Quat{1.0, 0.0, 0.0, 0.0});
            out[i * 4 + 0] = q.s;
            out[i * 4 + 1] = q.x;
            out[i * 4 + 2] = q.y;
            out[i * 4 + 3] = q.z;
        } else {
            uint64_t bits = rng.next_u64() >> 12;
            double u = bits_to_double(0x3FF0000000000000ULL | bits) - 1.0;
            out[i] = 0.0 + (u * (maximum - (-maximum)) + (-maximum));
        }
    }
}

// tune_local_trial (hoomd-mc/src/tune_local.rs:42-88) as the reference runs it: one stream
// Counter(step, substep, seed).make_rng() (index 0) for every sample of every step, in order:
// random_range(0..n) for the body, propose, wrap, delta_energy_one, and the uniform only when
// 0 < dH < infinity. Each step scales the maximum by (a + 1.5) / (t + 1.5) (tune_by_scaling,
// lib.rs:514-524); Rotate<Versor> clamps it at pi/2 (rotate/versor.rs:128-135), Rotate<Angle>
// at pi (rotate/angle.rs:62-68), Translate not at all (translate.rs:90-92).
double oracle_tune_stream(const oracle_system* s, uint32_t move, double maximum, double kt, double target,
                          uint32_t samples, uint32_t steps) {
    const int ol = s->ori_len();
    Sfc64 rng = make_rng(s->step, s->substep, s->seed, 0);
    const double pi = 3.141592653589793;
    const double cap = move == ORACLE_TRANSLATE ? 0.0 : (s->dim == 3 ? pi / 2.0 : pi);
    for (uint32_t t = 0; t < steps; ++t) {
        uint64_t acc = 0;
        for (uint32_t j = 0; j < samples; ++j) {
            uint64_t b = canon_range_u32(rng, (uint32_t)s->n);
            double pos[3] = {0, 0, 0}, ori[4] = {0, 0, 0, 0};
            s->propose(rng, (int)move, maximum, b, pos, ori);
            wrap(s->dim, s->L, pos);
            double dh = s->delta_energy_one(b, pos, ol ? ori : nullptr);
            if (dh != INFINITY && (dh <= 0.0 || uniform01(rng) < std::exp(-dh / kt))) acc += 1;
        }
        double ratio = (double)acc / (double)samples;
        maximum *= (ratio + 1.5) / (target + 1.5);
        if (cap > 0.0 && maximum > cap) maximum = cap;
    }
    return maximum;
}

// Pair histograms by minimum-image distance (no reference counterpart: the equilibrium
// estimators of the device library, restated here as their checker). Pairs i < j; per axis
// d = t - s - L rint((t - s)/L); SDF bins x = 1 - sigma/r in [0, x_max), g(r) bins r in
// [0, r_max), bin = floor(v * n_bins / limit) (clamped to the last bin).
static void pair_histogram(const oracle_system* s, bool sdf, double sigma, double limit, uint32_t n_bins,
                           uint64_t* counts) {
    for (uint32_t b = 0; b < n_bins; ++b) counts[b] = 0;
    const double inv = (double)n_bins / limit;
    for (uint64_t i = 0; i < s->n; ++i) {
        for (uint64_t j = i + 1; j < s->n; ++j) {
            double p = 0.0;
            for (int a = 0; a < s->dim; ++a) {
                double d = s->site[3 * i + a] - s->site[3 * j + a];
                double k = std::nearbyint(d / s->L[a]);
                d = d - k * s->L[a];
                p = p + d * d;
            }
            double r = std::sqrt(p), v;
            if (sdf) {
                if (!(r > sigma)) continue;
                v = 1.0 - sigma / r;
            } else {
                v = r;
            }
            if (v < limit) {
                double f = std::floor(v * inv);
                uint32_t bin = f < (double)n_bins ? (uint32_t)f : n_bins - 1;
                counts[bin] += 1;
            }
        }
    }
}

void oracle_sdf(const oracle_system* s, double x_max, uint32_t n_bins, uint64_t* counts) {
    pair_histogram(s, true, s->diameter, x_max, n_bins, counts);
}
void oracle_gr(const oracle_system* s, double r_max, uint32_t n_bins, uint64_t* counts) {
    pair_histogram(s, false, 0.0, r_max, n_bins, counts);
}

uint64_t oracle_overlap_count(const oracle_system* s) {
    // total_energy, pairwise_cutoff.rs:720-745: pairs of sites (and ghosts) with tag_i < tag_j.
    std::vector<uint32_t> cand;
    double img[7][3];
    uint64_t count = 0;
    for (uint64_t i = 0; i < s->n; ++i) {
        const double* x = &s->site[3 * i];
        s->candidates(x, cand);
        for (uint32_t j : cand) {
            if (j <= i) continue;
            const double* sj = &s->site[3 * j];
            bool hit = s->pair(x, s->ori_of(i), sj, j) == INFINITY;
            int ng = ghosts(s->dim, s->L, s->boundary_range, sj, img);
            for (int g = 0; g < ng && !hit; ++g) hit = s->pair(x, s->ori_of(i), img[g], j) == INFINITY;
            if (hit) count += 1;
        }
    }
    return count;
}
double oracle_total_energy(const oracle_system* s) {
    std::vector<uint32_t> cand;
    double img[7][3];
    double total = 0.0;
    for (uint64_t i = 0; i < s->n; ++i) {
        const double* x = &s->site[3 * i];
        s->candidates(x, cand);
        for (uint32_t j : cand) {
            if (j <= i) continue;
            const double* sj = &s->site[3 * j];
            total += s->pair(x, s->ori_of(i), sj, j);
            int ng = ghosts(s->dim, s->L, s->boundary_range, sj, img);
            for (int g = 0; g < ng; ++g) total += s->pair(x, s->ori_of(i), img[g], j);
        }
    }
    return total;
}
double oracle_delta_energy_one(const oracle_system* s, uint64_t b, const double* position,
                               const double* orientation) {
    double p[3] = {position[0], position[1], s->dim == 3 ? position[2] : 0.0};
    return s->delta_energy_one(b, p, orientation);
}
// Each move is independent of the others (the state is read only), so the moves are split over
// the host's threads; the results do not depend on the split.
void oracle_eval_moves(const oracle_system* s, uint64_t n, const uint64_t* bodies, const double* positions,
                       const double* orientations, const double* u, double kt, uint8_t* decisions,
                       double* delta_h) {
    const int ol = s->ori_len();
    auto run = [&](uint64_t lo, uint64_t hi) {
        for (uint64_t k = lo; k < hi; ++k) {
            double p[3] = {0, 0, 0};
            for (int a = 0; a < s->dim; ++a) p[a] = positions[k * s->dim + a];
            const double* o = ol ? orientations + (size_t)ol * k : nullptr;
            double dh = s->delta_energy_one(bodies[k], p, o);
            delta_h[k] = dh;
            bool ok = dh != INFINITY && (dh <= 0.0 || u[k] < std::exp(-dh / kt));
            decisions[k] = ok ? 1 : 0;
        }
    };
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const uint64_t threads = n < 4096 ? 1 : std::min<uint64_t>(hw, (n + 4095) / 4096);
    if (threads == 1) {
        run(0, n);
        return;
    }
    std::vector<std::thread> pool;
    const uint64_t chunk = (n + threads - 1) / threads;
    for (uint64_t w = 0; w < threads; ++w) {
        const uint64_t lo = std::min(n, w * chunk), hi = std::min(n, lo + chunk);
        pool.emplace_back(run, lo, hi);
    }
    for (auto& th : pool) th.join();
}

}  // extern "C"
