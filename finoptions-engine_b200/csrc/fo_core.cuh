// fo_core.cuh - arithmetic shared by every B200 LSM kernel (device code; the pure functions are
// also callable from host code).
//
// Bit-level conventions follow the reference CPU engine:
//   * Philox4x32-10 keyed by the seed, counter [block_lo, block_hi, path, domain]
//     (crates/finoptions-sim/src/random/philox.rs:9-114);
//   * bounded ZIGNOR standard normals over 256 layers (random/normal.rs:33-109);
//   * the exact GBM step S' = S * exp(fma(sigma*sqrt(dt), Z, log_drift)) with zero absorbing
//     (crates/finoptions-sim/src/step.rs:89-95).
// The library is compiled with --fmad=false: a multiply-add is fused only where the source calls
// fma(), exactly where the reference calls mul_add.
#pragma once

#include <stdint.h>

#include "zignor_tables.h"

#if defined(__CUDACC__)
#define FO_HD __host__ __device__ __forceinline__
#define FO_D __device__ __forceinline__
#define FO_HD_NOINLINE static __host__ __device__ __noinline__
#else
#define FO_HD inline
#define FO_D inline
#define FO_HD_NOINLINE static inline
#endif

#if !defined(__CUDACC__)
#include <cmath>
#endif

namespace fo {

// ----------------------------------------------------------------------------------------------
// Philox4x32-10 and the path-local stream.
// ----------------------------------------------------------------------------------------------

constexpr uint32_t kPhiloxM0 = 0xd2511f53u;
constexpr uint32_t kPhiloxM1 = 0xcd9e8d57u;
constexpr uint32_t kPhiloxW0 = 0x9e3779b9u;
constexpr uint32_t kPhiloxW1 = 0xbb67ae85u;

// Ten rounds; round r uses key + r * (W0, W1). Output words are the Random123 ordering.
FO_HD void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
                         uint32_t out[4]) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        // One widening multiply gives both halves of each product.
        const uint64_t p0 = uint64_t(kPhiloxM0) * c0, p1 = uint64_t(kPhiloxM1) * c2;
        const uint32_t hi0 = uint32_t(p0 >> 32), lo0 = uint32_t(p0);
        const uint32_t hi1 = uint32_t(p1 >> 32), lo1 = uint32_t(p1);
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += kPhiloxW0;
        k1 += kPhiloxW1;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

// Words are consumed as u64 pairs (low word first); one Philox block yields two. The next words
// wait in a small FIFO (b0 first, up to three). Before every odd-numbered normal (the 1st, 3rd,
// ...) the stream appends a block while at most one word is queued: the fast path of the sampler
// takes exactly one word per normal, so in the common case every lane of a warp generates its
// block at the same normal, even after rejections have shifted lanes against each other within
// their blocks. A block is also generated whenever a word is wanted from an empty FIFO (only after
// a rejection). Blocks are generated in counter order and words leave in order, so a path's word
// sequence does not depend on when its blocks are generated.
struct PathStream {
    uint32_t k0, k1, domain, path;
    uint64_t next_block;
    uint64_t b0, b1, b2;
    uint32_t count;      // queued words
    uint32_t remaining;  // normals left in the budget
    uint32_t drawn;      // normals begun

    FO_HD void init(uint64_t seed, uint32_t domain_, uint32_t path_, uint32_t budget) {
        k0 = uint32_t(seed);
        k1 = uint32_t(seed >> 32);
        domain = domain_;
        path = path_;
        next_block = 0;
        b0 = b1 = b2 = 0;
        count = 0;
        remaining = budget;
        drawn = 0;
    }
    // Appends one block; requires count <= 1.
    FO_HD void append_block() {
        uint32_t w[4];
        philox4x32_10(uint32_t(next_block), uint32_t(next_block >> 32), path, domain, k0, k1, w);
        next_block += 1;
        const uint64_t n0 = uint64_t(w[0]) | (uint64_t(w[1]) << 32);
        const uint64_t n1 = uint64_t(w[2]) | (uint64_t(w[3]) << 32);
        if (count == 0) {
            b0 = n0;
            b1 = n1;
        } else {
            b1 = n0;
            b2 = n1;
        }
        count += 2;
    }
    FO_HD uint64_t next_u64() {
        if (count == 0) append_block();
        const uint64_t v = b0;
        b0 = b1;
        b1 = b2;
        count -= 1;
        return v;
    }
    FO_HD bool begin_normal() {
        if (remaining == 0) return false;
        remaining -= 1;
        if ((drawn & 1u) == 0 && count <= 1) append_block();
        drawn += 1;
        return true;
    }
};

// ----------------------------------------------------------------------------------------------
// ZIGNOR standard normals. Tables live in shared memory on the device (257 + 257 doubles).
// ----------------------------------------------------------------------------------------------

enum NormalStatus : int { kNormalOk = 0, kNormalBudget = 1, kNormalRejection = 2 };

constexpr int kMaxRejectionIterations = 1048576;
constexpr uint64_t kFractionMask = (uint64_t(1) << 52) - 1;
constexpr uint64_t kExponent0 = uint64_t(1023) << 52;
constexpr uint64_t kExponent1 = uint64_t(1024) << 52;

FO_HD double bits_to_double(uint64_t b) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)b);
#else
    double d;
    __builtin_memcpy(&d, &b, sizeof(d));
    return d;
#endif
}

FO_HD uint64_t double_to_bits(double d) {
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(d);
#else
    uint64_t b;
    __builtin_memcpy(&b, &d, sizeof(b));
    return b;
#endif
}

FO_HD double zig_symmetric_unit(uint64_t bits) {
    return bits_to_double(((bits >> 12) & kFractionMask) | kExponent1) - 3.0;
}

FO_HD double fo_exp(double x) {
#if defined(__CUDA_ARCH__)
    return ::exp(x);
#else
    return std::exp(x);
#endif
}
FO_HD double fo_log(double x) {
#if defined(__CUDA_ARCH__)
    return ::log(x);
#else
    return std::log(x);
#endif
}
FO_HD double fo_sqrt(double x) {
#if defined(__CUDA_ARCH__)
    return ::sqrt(x);
#else
    return std::sqrt(x);
#endif
}
FO_HD double fo_fma(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
    return ::fma(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
FO_HD double fo_fabs(double x) {
#if defined(__CUDA_ARCH__)
    return ::fabs(x);
#else
    return std::fabs(x);
#endif
}
FO_HD bool fo_isfinite(double x) {
#if defined(__CUDA_ARCH__)
    return ::isfinite(x);
#else
    return std::isfinite(x);
#endif
}

// Tail beyond R (random/normal.rs:50-63), out of line: reached by about one normal in 4000.
template <typename Tables>
#if defined(__CUDACC__)
__host__ __device__ __noinline__
#else
inline
#endif
int zig_sample_tail(PathStream& s, const Tables& t, double unit, double* out) {
    const double r = t.r();
    for (int jt = 0; jt < kMaxRejectionIterations; ++jt) {
        const double ox = bits_to_double(((s.next_u64() >> 12) & kFractionMask) | kExponent0) -
                          (1.0 - 1.1102230246251565e-16);
        const double x = fo_log(ox) / r;
        const double oy = bits_to_double(((s.next_u64() >> 12) & kFractionMask) | kExponent0) -
                          (1.0 - 1.1102230246251565e-16);
        const double y = fo_log(oy);
        if (-2.0 * y >= x * x) {
            *out = unit < 0.0 ? x - r : r - x;
            return kNormalOk;
        }
    }
    return kNormalRejection;
}

// The rejection loop (random/normal.rs:66-91) from its second pass on, or from the tail, out of line:
// few normals get here (the tail layer, or a wedge rejection followed by a fast rejection).
template <typename Tables>
#if defined(__CUDACC__)
__host__ __device__ __noinline__
#else
inline
#endif
int zig_sample_rest(PathStream& s, const Tables& t, int index, double unit, double value, double* out) {
    for (int it = 0; it < kMaxRejectionIterations - 1; ++it) {
        if (index == 0) return zig_sample_tail(s, t, unit, out);
        const double u = double(s.next_u64() >> 11) * (1.0 / 9007199254740992.0);
        const double ordinate = t.f(index + 1) + (t.f(index) - t.f(index + 1)) * u;
        if (ordinate < fo_exp(-0.5 * value * value)) {
            *out = value;
            return kNormalOk;
        }
        const uint64_t bits = s.next_u64();
        index = int(bits & 0xff);
        unit = zig_symmetric_unit(bits);
        value = unit * t.x(index);
        if (fo_fabs(value) < t.x(index + 1)) {
            *out = value;
            return kNormalOk;
        }
    }
    return kNormalRejection;
}

// One standard normal (random/normal.rs:96-109). The fast test accepts 98.5% of draws; the first wedge
// test and its redraw are straight-line code, so a warp whose lanes reject at the same normal
// runs them once; the tail and any further rejection run out of line on a copy of the stream.
template <typename Tables>
FO_HD int zig_sample(PathStream& s, const Tables& t, double* out) {
    if (!s.begin_normal()) return kNormalBudget;
    uint64_t bits = s.next_u64();
    int index = int(bits & 0xff);
    double unit = zig_symmetric_unit(bits);
    double value = unit * t.x(index);
    if (fo_fabs(value) < t.x(index + 1)) {
        *out = value;
        return kNormalOk;
    }
    if (index != 0) {
        const double u = double(s.next_u64() >> 11) * (1.0 / 9007199254740992.0);
        const double ordinate = t.f(index + 1) + (t.f(index) - t.f(index + 1)) * u;
        if (ordinate < fo_exp(-0.5 * value * value)) {
            *out = value;
            return kNormalOk;
        }
        bits = s.next_u64();
        index = int(bits & 0xff);
        unit = zig_symmetric_unit(bits);
        value = unit * t.x(index);
        if (fo_fabs(value) < t.x(index + 1)) {
            *out = value;
            return kNormalOk;
        }
    }
    PathStream copy = s;
    const int status = zig_sample_rest(copy, t, index, unit, value, out);
    s = copy;
    return status;
}

// ----------------------------------------------------------------------------------------------
// Division by a divisor used many times (the strike, a fitted scale): the reciprocal y = 1/b is
// formed once and each quotient takes Markstein's correction step (P. Markstein, "Computation of
// elementary functions on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990;
// M. Cornea, J. Harrison, P. Tang, "Scientific Computing on Itanium-based Systems", 2002):
//   q0 = a * y,   r = a - b * q0 (exact in one fma),   q = q0 + r * y (one fma).
// The residual of q0 is exact and the corrected quotient lies within a tiny fraction of an ulp of
// a / b before its final rounding, so q is the correctly rounded quotient except when a / b falls
// within about 2^-51 ulp of a rounding boundary. Operands outside [2^-960, 2^960] divide.
// ----------------------------------------------------------------------------------------------

struct Divisor {
    double b;
    double inv;  // 1 / b, or 0 when b is outside the corrected range
};

FO_HD Divisor make_divisor(double b) {
    const double m = fo_fabs(b);
    return Divisor{b, (m > 0x1p-960 && m < 0x1p960) ? 1.0 / b : 0.0};
}

FO_HD double divide(double a, const Divisor& d) {
    const double m = fo_fabs(a);
    if (d.inv == 0.0 || !(m > 0x1p-960 && m < 0x1p960)) return a / d.b;
    const double q0 = a * d.inv;
    const double r = fo_fma(-d.b, q0, a);
    return fo_fma(r, d.inv, q0);
}

// ----------------------------------------------------------------------------------------------
// GBM step and cash-dividend policies.
// ----------------------------------------------------------------------------------------------

FO_HD double gbm_advance(double spot, double diffusion, double log_drift, double normal) {
    if (spot == 0.0) return 0.0;
    return spot * fo_exp(fo_fma(diffusion, normal, log_drift));
}

// Liquidator (policy 0): max(S - D, 0); Survivor (policy 1): S > D ? S - D : S.
// crates/finoptions-core/src/dividend.rs:59-80.
FO_HD double apply_cash_dividend(int policy, double amount, double spot) {
    if (policy == 0) {
        const double d = spot - amount;
        return d > 0.0 ? d : 0.0;
    }
    return spot > amount ? spot - amount : spot;
}

// ----------------------------------------------------------------------------------------------
// Double-double arithmetic (Dekker 1971; Knuth's TwoSum). Valid only without FMA contraction.
// ----------------------------------------------------------------------------------------------

struct dd {
    double hi, lo;
};

FO_HD dd dd_make(double a) { return dd{a, 0.0}; }

FO_HD dd two_sum(double a, double b) {
    const double s = a + b;
    const double bb = s - a;
    const double e = (a - (s - bb)) + (b - bb);
    return dd{s, e};
}

FO_HD dd fast_two_sum(double a, double b) {
    const double s = a + b;
    const double e = b - (s - a);
    return dd{s, e};
}

FO_HD dd two_prod(double a, double b) {
    const double p = a * b;
    return dd{p, fo_fma(a, b, -p)};
}

FO_HD dd dd_add(dd x, dd y) {
    dd s = two_sum(x.hi, y.hi);
    dd t = two_sum(x.lo, y.lo);
    s.lo += t.hi;
    s = fast_two_sum(s.hi, s.lo);
    s.lo += t.lo;
    return fast_two_sum(s.hi, s.lo);
}

FO_HD dd dd_neg(dd x) { return dd{-x.hi, -x.lo}; }
FO_HD dd dd_sub(dd x, dd y) { return dd_add(x, dd_neg(y)); }

FO_HD dd dd_mul(dd x, dd y) {
    dd p = two_prod(x.hi, y.hi);
    p.lo += x.hi * y.lo + x.lo * y.hi;
    return fast_two_sum(p.hi, p.lo);
}

FO_HD dd dd_mul_d(dd x, double y) {
    dd p = two_prod(x.hi, y);
    p.lo += x.lo * y;
    return fast_two_sum(p.hi, p.lo);
}

FO_HD dd dd_div(dd x, dd y) {
    const double q1 = x.hi / y.hi;
    dd r = dd_sub(x, dd_mul_d(y, q1));
    const double q2 = r.hi / y.hi;
    r = dd_sub(r, dd_mul_d(y, q2));
    const double q3 = r.hi / y.hi;
    dd q = fast_two_sum(q1, q2);
    return dd_add(q, dd_make(q3));
}

FO_HD dd dd_sqrt(dd x) {
    if (x.hi <= 0.0) return dd{fo_sqrt(x.hi), 0.0};
    const double s = fo_sqrt(x.hi);
    const dd r = dd_sub(x, two_prod(s, s));
    return fast_two_sum(s, r.hi / (2.0 * s));
}

FO_HD double dd_round(dd x) { return x.hi + x.lo; }

// ----------------------------------------------------------------------------------------------
// Continuation regression from in-the-money moments.
//
// The reference fits degree-d OLS on standardised moneyness z = (x - mean) / scale with a
// Stieltjes (empirical three-term) recurrence: d + 1 sequential passes produce, per basis degree
// j, norm_j = sum p_j^2, projection_j = sum y p_j and sum z p_j^2, from which
// alpha_j = sum z p_j^2 / norm_j, beta_j = norm_j / norm_{j-1}, c_j = projection_j / norm_j
// (crates/finoptions-lsm/src/regression.rs:432-523). The kernels instead reduce, in ONE pass over
// the in-the-money paths, the power sums T_k = sum t^k (k <= 2d) and U_k = sum y t^k (k <= d) of
// t = x - pivot. Everything below is then exact functional algebra on those sums, carried out in
// double-double: the mean and population scale, the moments of z about the rounded mean, and the
// recurrence sigma_{j,l} = <p_j, z^l> with the ROUNDED alpha_j and beta_j the reference uses to
// build its next basis vector (Chebyshev's algorithm on ordinary moments). The results agree with
// the sequential reference to its own rounding level.
// ----------------------------------------------------------------------------------------------

constexpr int kMaxDegree = 4;
constexpr int kMaxColumns = kMaxDegree + 1;
constexpr int kPowerSums = 2 * kMaxDegree + 1;  // T_0..T_8
constexpr int kResponseSums = kMaxColumns;      // U_0..U_4
constexpr int kMomentSlots = kPowerSums + kResponseSums;  // 14 accumulated sums (T_0 = count)

enum FitStatus : int {
    kFitOk = 0,
    kFitDegeneratePredictor = 1,
    kFitRankDeficient = 2,
    kFitNonFinite = 3,
};

struct alignas(16) FitModel {  // 16-byte aligned: pairs of fields load together
    double mean, scale;
    double inv_scale;  // 1 / scale for the prediction's corrected division (see Divisor)
    double alpha[kMaxDegree];
    double beta[kMaxDegree];
    double coef[kMaxColumns];
    double norm[kMaxColumns];
    int status;      // FitStatus
    int aux;         // rank for kFitRankDeficient, basis degree for kFitNonFinite
    double aux_value;  // scale for kFitDegeneratePredictor
};

// Binomial coefficients C(k, j) for k, j <= 8 (exact in binary64; zero above the diagonal). The
// binomial shift reads them as constants instead of forming them by a chain of divisions; device
// code reads the __constant__ copy.
static constexpr double kBinomialHost[9][9] = {{1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, {1.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, {1.0, 2.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, {1.0, 3.0, 3.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0}, {1.0, 4.0, 6.0, 4.0, 1.0, 0.0, 0.0, 0.0, 0.0}, {1.0, 5.0, 10.0, 10.0, 5.0, 1.0, 0.0, 0.0, 0.0}, {1.0, 6.0, 15.0, 20.0, 15.0, 6.0, 1.0, 0.0, 0.0}, {1.0, 7.0, 21.0, 35.0, 35.0, 21.0, 7.0, 1.0, 0.0}, {1.0, 8.0, 28.0, 56.0, 70.0, 56.0, 28.0, 8.0, 1.0}};
#ifdef __CUDACC__
static __constant__ double kBinomialDevice[9][9] = {{1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, {1.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, {1.0, 2.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, {1.0, 3.0, 3.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0}, {1.0, 4.0, 6.0, 4.0, 1.0, 0.0, 0.0, 0.0, 0.0}, {1.0, 5.0, 10.0, 10.0, 5.0, 1.0, 0.0, 0.0, 0.0}, {1.0, 6.0, 15.0, 20.0, 15.0, 6.0, 1.0, 0.0, 0.0}, {1.0, 7.0, 21.0, 35.0, 35.0, 21.0, 7.0, 1.0, 0.0}, {1.0, 8.0, 28.0, 56.0, 70.0, 56.0, 28.0, 8.0, 1.0}};
#endif
#ifdef __CUDA_ARCH__
#define FO_BINOMIAL kBinomialDevice
#else
#define FO_BINOMIAL kBinomialHost
#endif

// sums[k] for k in 0..8 are T_k (T_0 = count), sums[9 + k] for k in 0..4 are U_k.
FO_HD_NOINLINE void fit_from_moments(const dd* sums, double pivot, uint64_t count, int degree, double rank_tolerance,
                            FitModel* m) {
    for (int j = 0; j < kMaxDegree; ++j) {
        m->alpha[j] = 0.0;
        m->beta[j] = 0.0;
    }
    for (int j = 0; j < kMaxColumns; ++j) {
        m->coef[j] = 0.0;
        m->norm[j] = 0.0;
    }
    m->status = kFitOk;
    m->aux = 0;
    m->aux_value = 0.0;
    const double n = double(count);
    dd mom[kPowerSums];   // moments of z: m_k = sum z^k
    dd resp[kResponseSums];  // r_k = sum y z^k
    if (degree == 0) {
        m->mean = 0.0;
        m->scale = 1.0;
        m->inv_scale = make_divisor(m->scale).inv;
        mom[0] = dd_make(n);
        for (int k = 1; k < kPowerSums; ++k) mom[k] = dd_make(0.0);
        resp[0] = sums[kPowerSums + 0];
        for (int k = 1; k < kResponseSums; ++k) resp[k] = dd_make(0.0);
    } else {
        const dd T0 = dd_make(n);
        const dd mean_offset = dd_div(sums[1], T0);
        const dd mean = dd_add(dd_make(pivot), mean_offset);
        // M2 = T2 - T1^2 / n  (sum of squared deviations)
        const dd m2 = dd_sub(sums[2], dd_mul(sums[1], mean_offset));
        const dd var = dd_div(m2, T0);
        const dd sd = dd_sqrt(var);
        const double mean_d = dd_round(mean);
        const double scale_d = dd_round(sd);
        m->mean = mean_d;
        m->scale = scale_d;
        m->inv_scale = make_divisor(m->scale).inv;
        if (!fo_isfinite(mean_d) || !fo_isfinite(scale_d) || !(scale_d > 0.0)) {
            m->status = kFitDegeneratePredictor;
            m->aux_value = scale_d;
            return;
        }
        // delta = pivot - mean_d exactly; moments of (x - mean_d) by the binomial theorem.
        const dd delta = two_sum(pivot, -mean_d);
        dd dpow[kPowerSums];
        dpow[0] = dd_make(1.0);
        for (int k = 1; k < kPowerSums; ++k) dpow[k] = dd_mul(dpow[k - 1], delta);
        const int top = 2 * degree;
        const dd inv_scale = dd_div(dd_make(1.0), dd_make(scale_d));
        dd spow = dd_make(1.0);
        for (int k = 0; k <= top; ++k) {
            dd acc = dd_make(0.0);
            for (int j = k; j >= 0; --j) {
                // term: C(k, j) * delta^(k - j) * T_j
                const dd tj = j == 0 ? T0 : sums[j];
                acc = dd_add(acc, dd_mul_d(dd_mul(dpow[k - j], tj), FO_BINOMIAL[k][j]));
            }
            mom[k] = dd_mul(acc, spow);
            if (k <= degree) {
                dd racc = dd_make(0.0);
                for (int j = k; j >= 0; --j)
                    racc = dd_add(racc, dd_mul_d(dd_mul(dpow[k - j], sums[kPowerSums + j]), FO_BINOMIAL[k][j]));
                resp[k] = dd_mul(racc, spow);
            }
            spow = dd_mul(spow, inv_scale);
        }
        for (int k = top + 1; k < kPowerSums; ++k) mom[k] = dd_make(0.0);
        for (int k = degree + 1; k < kResponseSums; ++k) resp[k] = dd_make(0.0);
    }
    // Stieltjes recurrence on moment functionals. a_cur / a_prev: monomial coefficients of p_j,
    // p_{j-1}; sig_cur[l] = <p_j, z^l>, sig_prev[l] = <p_{j-1}, z^l>.
    dd a_prev[kMaxColumns + 1], a_cur[kMaxColumns + 1];
    dd sig_prev[kPowerSums + 1], sig_cur[kPowerSums + 1];
    for (int i = 0; i <= kMaxColumns; ++i) {
        a_prev[i] = dd_make(0.0);
        a_cur[i] = dd_make(0.0);
    }
    a_cur[0] = dd_make(1.0);
    for (int l = 0; l <= kPowerSums; ++l) {
        sig_prev[l] = dd_make(0.0);
        sig_cur[l] = l < kPowerSums ? mom[l] : dd_make(0.0);
    }
    double previous_norm = 1.0;
    for (int j = 0; j <= degree; ++j) {
        dd norm = dd_make(0.0), proj = dd_make(0.0), wp = dd_make(0.0);
        for (int a = 0; a <= j; ++a) {
            norm = dd_add(norm, dd_mul(a_cur[a], sig_cur[a]));
            wp = dd_add(wp, dd_mul(a_cur[a], sig_cur[a + 1]));
            proj = dd_add(proj, dd_mul(a_cur[a], resp[a]));
        }
        const double norm_d = dd_round(norm);
        const double proj_d = dd_round(proj);
        const double wp_d = dd_round(wp);
        if (!fo_isfinite(norm_d) || !fo_isfinite(proj_d) || !fo_isfinite(wp_d)) {
            m->status = kFitNonFinite;
            m->aux = j;
            return;
        }
        if (norm_d <= 0.0 || fo_sqrt(norm_d / n) <= rank_tolerance) {
            m->status = kFitRankDeficient;
            m->aux = j;
            return;
        }
        m->norm[j] = norm_d;
        m->coef[j] = proj_d / norm_d;
        if (!fo_isfinite(m->coef[j])) {
            m->status = kFitNonFinite;
            m->aux = j;
            return;
        }
        if (j < degree) {
            const double alpha = wp_d / norm_d;
            const double beta = j == 0 ? 0.0 : norm_d / previous_norm;
            if (!fo_isfinite(alpha) || !fo_isfinite(beta)) {
                m->status = kFitNonFinite;
                m->aux = j;
                return;
            }
            m->alpha[j] = alpha;
            m->beta[j] = beta;
            // p_{j+1} = (z - alpha) p_j - beta p_{j-1}
            dd a_next[kMaxColumns + 1];
            for (int i = 0; i <= kMaxColumns; ++i) {
                dd v = i > 0 ? a_cur[i - 1] : dd_make(0.0);
                v = dd_sub(v, dd_mul_d(a_cur[i], alpha));
                v = dd_sub(v, dd_mul_d(a_prev[i], beta));
                a_next[i] = v;
            }
            dd sig_next[kPowerSums + 1];
            for (int l = 0; l <= kPowerSums; ++l) {
                dd v = l + 1 <= kPowerSums ? sig_cur[l + 1] : dd_make(0.0);
                v = dd_sub(v, dd_mul_d(sig_cur[l], alpha));
                v = dd_sub(v, dd_mul_d(sig_prev[l], beta));
                sig_next[l] = v;
            }
            for (int i = 0; i <= kMaxColumns; ++i) {
                a_prev[i] = a_cur[i];
                a_cur[i] = a_next[i];
            }
            for (int l = 0; l <= kPowerSums; ++l) {
                sig_prev[l] = sig_cur[l];
                sig_cur[l] = sig_next[l];
            }
            previous_norm = norm_d;
        }
    }
}

// The same solve in binary64 after rounding the reduced sums. When the pivot lies within one
// standard deviation of the in-the-money mean, the binomial shift and the recurrence lose no more
// than the reference's own summation rounding (measured against the sequential reference fit:
// the same 3e-13 worst relative prediction difference as the double-double solve), at a fraction
// of the latency. Specialised per degree so every array stays in registers. Returns false,
// without writing, when the pivot is too far for this path.
template <int D>
FO_HD bool fit_near_pivot(const dd* sums, double pivot, uint64_t count, double rank_tolerance, FitModel* m) {
    const double n = double(count);
    double mean = 0.0, scale = 1.0;
    if (D != 0) {
        const double t1 = sums[1].hi + sums[1].lo;
        const double offset = t1 / n;
        const double t2 = sums[2].hi + sums[2].lo;
        const double var = (t2 - t1 * offset) / n;
        if (!(var > 0.0) || !(offset * offset <= var)) return false;
        mean = pivot + offset;
        scale = fo_sqrt(var);
    }
#pragma unroll
    for (int j = 0; j < kMaxDegree; ++j) {
        m->alpha[j] = 0.0;
        m->beta[j] = 0.0;
    }
#pragma unroll
    for (int j = 0; j < kMaxColumns; ++j) {
        m->coef[j] = 0.0;
        m->norm[j] = 0.0;
    }
    m->status = kFitOk;
    m->aux = 0;
    m->aux_value = 0.0;
    m->mean = mean;
    m->scale = scale;
    m->inv_scale = make_divisor(m->scale).inv;
    if (!fo_isfinite(mean) || !fo_isfinite(scale) || !(scale > 0.0)) {
        m->status = kFitDegeneratePredictor;
        m->aux_value = scale;
        return true;
    }
    constexpr int K = 2 * D + 2;  // moments 0..2D+1 (the last stays zero)
    double mom[K], resp[D + 1];
    if (D == 0) {
        mom[0] = n;
        mom[1] = 0.0;
        resp[0] = sums[kPowerSums].hi + sums[kPowerSums].lo;
    } else {
        const double delta = pivot - mean;
        double T[2 * D + 1], U[D + 1], dpow[2 * D + 1];
        T[0] = n;
#pragma unroll
        for (int k = 1; k <= 2 * D; ++k) T[k] = sums[k].hi + sums[k].lo;
#pragma unroll
        for (int k = 0; k <= D; ++k) U[k] = sums[kPowerSums + k].hi + sums[kPowerSums + k].lo;
        dpow[0] = 1.0;
#pragma unroll
        for (int k = 1; k <= 2 * D; ++k) dpow[k] = dpow[k - 1] * delta;
        const double inv_scale = 1.0 / scale;
        double spow = 1.0;
#pragma unroll
        for (int k = 0; k <= 2 * D; ++k) {
            double acc = 0.0;
#pragma unroll
            for (int j = k; j >= 0; --j) acc += FO_BINOMIAL[k][j] * dpow[k - j] * T[j];
            mom[k] = acc * spow;
            if (k <= D) {
                double racc = 0.0;
#pragma unroll
                for (int j = k; j >= 0; --j) racc += FO_BINOMIAL[k][j] * dpow[k - j] * U[j];
                resp[k] = racc * spow;
            }
            spow *= inv_scale;
        }
        mom[K - 1] = 0.0;
    }
    double a_prev[D + 2], a_cur[D + 2], sig_prev[K], sig_cur[K];
#pragma unroll
    for (int i = 0; i < D + 2; ++i) {
        a_prev[i] = 0.0;
        a_cur[i] = 0.0;
    }
    a_cur[0] = 1.0;
#pragma unroll
    for (int l = 0; l < K; ++l) {
        sig_prev[l] = 0.0;
        sig_cur[l] = mom[l];
    }
    double previous_norm = 1.0;
#pragma unroll
    for (int j = 0; j <= D; ++j) {
        double norm = 0.0, proj = 0.0, wp = 0.0;
#pragma unroll
        for (int a = 0; a <= j; ++a) {
            norm += a_cur[a] * sig_cur[a];
            wp += a_cur[a] * sig_cur[a + 1];
            proj += a_cur[a] * resp[a];
        }
        if (!fo_isfinite(norm) || !fo_isfinite(proj) || !fo_isfinite(wp)) {
            m->status = kFitNonFinite;
            m->aux = j;
            return true;
        }
        if (norm <= 0.0 || fo_sqrt(norm / n) <= rank_tolerance) {
            m->status = kFitRankDeficient;
            m->aux = j;
            return true;
        }
        m->norm[j] = norm;
        m->coef[j] = proj / norm;
        if (!fo_isfinite(m->coef[j])) {
            m->status = kFitNonFinite;
            m->aux = j;
            return true;
        }
        if (j < D) {
            const double alpha = wp / norm;
            const double beta = j == 0 ? 0.0 : norm / previous_norm;
            if (!fo_isfinite(alpha) || !fo_isfinite(beta)) {
                m->status = kFitNonFinite;
                m->aux = j;
                return true;
            }
            m->alpha[j] = alpha;
            m->beta[j] = beta;
            double a_next[D + 2], sig_next[K];
#pragma unroll
            for (int i = 0; i < D + 2; ++i)
                a_next[i] = (i > 0 ? a_cur[i - 1] : 0.0) - alpha * a_cur[i] - beta * a_prev[i];
#pragma unroll
            for (int l = 0; l < K; ++l)
                sig_next[l] = (l + 1 < K ? sig_cur[l + 1] : 0.0) - alpha * sig_cur[l] - beta * sig_prev[l];
#pragma unroll
            for (int i = 0; i < D + 2; ++i) {
                a_prev[i] = a_cur[i];
                a_cur[i] = a_next[i];
            }
#pragma unroll
            for (int l = 0; l < K; ++l) {
                sig_prev[l] = sig_cur[l];
                sig_cur[l] = sig_next[l];
            }
            previous_norm = norm;
        }
    }
    return true;
}

// Whether a row's power sums about `pivot` must be taken again about the row's own mean. Each
// term t^k = (x - pivot)^k is rounded on its own, and the binomial shift to the mean multiplies
// those roundings by about ((|mean - pivot| + sd) / sd)^(2d): a pivot more than one standard
// deviation from the mean (a small in-the-money population whose mean moved far from the previous
// row's) loses the digits the fit needs. *mean_out receives the mean rounded to binary64, the new
// pivot; about it the offset is a rounding error and the near-pivot solve applies.
FO_HD bool pivot_too_far(const dd* sums, double pivot, uint64_t count, double* mean_out) {
    const double n = double(count);
    const double t1 = sums[1].hi + sums[1].lo;
    const double offset = t1 / n;
    const double var = (sums[2].hi + sums[2].lo - t1 * offset) / n;
    *mean_out = pivot + offset;
    return var > 0.0 && offset * offset > var && fo_isfinite(*mean_out);
}

FO_HD_NOINLINE void fit_continuation(const dd* sums, double pivot, uint64_t count, int degree,
                                     double rank_tolerance, FitModel* m) {
    bool done = false;
    switch (degree) {
        case 0: done = fit_near_pivot<0>(sums, pivot, count, rank_tolerance, m); break;
        case 1: done = fit_near_pivot<1>(sums, pivot, count, rank_tolerance, m); break;
        case 2: done = fit_near_pivot<2>(sums, pivot, count, rank_tolerance, m); break;
        case 3: done = fit_near_pivot<3>(sums, pivot, count, rank_tolerance, m); break;
        default: done = fit_near_pivot<4>(sums, pivot, count, rank_tolerance, m); break;
    }
    if (!done) fit_from_moments(sums, pivot, count, degree, rank_tolerance, m);
}

// The largest q >= 0 whose correctly rounded square root is at most `tol` (host side, for tol in
// (0, 1)). The square root is monotone, so the solve's rank test fo_sqrt(norm / n) <= tol takes
// the same decision as norm / n <= rank_limit(tol), without a square root on the device.
inline double rank_limit(double tol) {
    const auto step = [](double v, int64_t by) {
        int64_t bits;
        __builtin_memcpy(&bits, &v, sizeof bits);
        bits += by;
        __builtin_memcpy(&v, &bits, sizeof v);
        return v;
    };
    double q = tol * tol;  // within an ulp or two of the limit
    for (int i = 0; i < 64 && fo_sqrt(step(q, 1)) <= tol; ++i) q = step(q, 1);
    for (int i = 0; i < 64 && q > 0.0 && fo_sqrt(q) > tol; ++i) q = step(q, -1);
    return q;
}

// PolynomialModel::predict_for (regression.rs:197-224). Returns false for a non-finite result.
// Model is FitModel or any type with the same mean / scale / alpha / beta / coef fields.
template <typename Model>
FO_HD bool predict_continuation(const Model& m, int degree, double predictor, double* out) {
    if (!fo_isfinite(predictor)) return false;
    const double z = degree == 0 ? 0.0 : divide(predictor - m.mean, Divisor{m.scale, m.inv_scale});
    double prediction = m.coef[0];
    double previous = 0.0, current = 1.0;
    for (int j = 0; j < degree; ++j) {
        const double next = fo_fma(z - m.alpha[j], current, -m.beta[j] * previous);
        prediction = fo_fma(m.coef[j + 1], next, prediction);
        previous = current;
        current = next;
    }
    if (!fo_isfinite(prediction)) return false;
    *out = prediction;
    return true;
}

// predict_continuation for a degree fixed at compile time: the same operations in the same order,
// with the basis recurrence unrolled (kernels that evaluate a fitted policy on every path are
// instantiated per degree).
template <int D, typename Model>
FO_HD bool predict_continuation_d(const Model& m, double predictor, double* out) {
    if (!fo_isfinite(predictor)) return false;
    const double z = D == 0 ? 0.0 : divide(predictor - m.mean, Divisor{m.scale, m.inv_scale});
    double prediction = m.coef[0];
    double previous = 0.0, current = 1.0;
#pragma unroll
    for (int j = 0; j < D; ++j) {
        const double next = fo_fma(z - m.alpha[j], current, -m.beta[j] * previous);
        prediction = fo_fma(m.coef[j + 1], next, prediction);
        previous = current;
        current = next;
    }
    if (!fo_isfinite(prediction)) return false;
    *out = prediction;
    return true;
}

#ifdef __CUDACC__
// predict_continuation_d for a model in shared memory that the pass reads at every path: the same
// operations in the same order, with the fields read through a volatile reference so the compiler
// loads them per path (broadcast shared-memory loads) instead of holding the 14 of them in
// registers across the pass; the registers go to resident CTAs instead.
template <int D>
__device__ __forceinline__ bool predict_continuation_shared(const FitModel* model, double predictor, double* out) {
    const volatile FitModel& m = *model;
    if (!fo_isfinite(predictor)) return false;
    const double z = D == 0 ? 0.0 : divide(predictor - m.mean, Divisor{m.scale, m.inv_scale});
    double prediction = m.coef[0];
    double previous = 0.0, current = 1.0;
#pragma unroll
    for (int j = 0; j < D; ++j) {
        const double next = fo_fma(z - m.alpha[j], current, -m.beta[j] * previous);
        prediction = fo_fma(m.coef[j + 1], next, prediction);
        previous = current;
        current = next;
    }
    if (!fo_isfinite(prediction)) return false;
    *out = prediction;
    return true;
}
#endif

// ----------------------------------------------------------------------------------------------
// Rank and two-norm condition diagnostic: one-sided Jacobi SVD of the <= 5x5 upper-triangular
// transform from monomials to the orthonormal basis (regression.rs:540-577, 711-850).
// ----------------------------------------------------------------------------------------------

enum DiagnoseStatus : int {
    kDiagOk = 0,
    kDiagNonFinite = 1,
    kDiagNotConverged = 2,
    kDiagRankDeficient = 3,
    kDiagConditionExceeded = 4,
};

FO_HD double fo_hypot(double a, double b) {
#if defined(__CUDA_ARCH__)
    return ::hypot(a, b);
#else
    return std::hypot(a, b);
#endif
}

// Returns DiagnoseStatus; writes rank, condition, and aux (basis degree for non-finite).
FO_HD_NOINLINE int diagnose_design(const FitModel& model, int degree, double rank_tolerance, double condition_limit,
                          int* rank_out, double* condition_out, int* aux) {
    const int columns = degree + 1;
    double t[kMaxColumns * kMaxColumns];
    for (int i = 0; i < kMaxColumns * kMaxColumns; ++i) t[i] = 0.0;
    double previous[kMaxColumns], current[kMaxColumns];
    for (int i = 0; i < kMaxColumns; ++i) {
        previous[i] = 0.0;
        current[i] = 0.0;
    }
    current[0] = 1.0;
    for (int j = 0; j <= degree; ++j) {
        const double inverse_norm = 1.0 / fo_sqrt(model.norm[j]);
        if (!fo_isfinite(inverse_norm)) {
            *aux = j;
            return kDiagNonFinite;
        }
        for (int k = 0; k <= j; ++k) t[j * kMaxColumns + k] = current[k] * inverse_norm;
        if (j == degree) break;
        double next[kMaxColumns];
        for (int i = 0; i < kMaxColumns; ++i) next[i] = 0.0;
        for (int k = 0; k <= j; ++k) {
            next[k + 1] += current[k];
            next[k] -= model.alpha[j] * current[k];
            next[k] -= model.beta[j] * previous[k];
        }
        for (int i = 0; i < kMaxColumns; ++i) {
            if (!fo_isfinite(next[i])) {
                *aux = j + 1;
                return kDiagNonFinite;
            }
        }
        for (int i = 0; i < kMaxColumns; ++i) {
            previous[i] = current[i];
            current[i] = next[i];
        }
    }
    const double tolerance = 16.0 * 2.220446049250313e-16;
    bool converged = false;
    for (int sweep = 0; sweep < 32; ++sweep) {
        converged = true;
        for (int left = 0; left + 1 < columns; ++left) {
            for (int right = left + 1; right < columns; ++right) {
                double ln = 0.0, rn = 0.0, cross = 0.0;
                for (int row = 0; row < columns; ++row) {
                    const double lv = t[left * kMaxColumns + row];
                    const double rv = t[right * kMaxColumns + row];
                    ln = fo_fma(lv, lv, ln);
                    rn = fo_fma(rv, rv, rn);
                    cross = fo_fma(lv, rv, cross);
                }
                if (!fo_isfinite(ln) || !fo_isfinite(rn) || !fo_isfinite(cross) || ln <= 0.0 || rn <= 0.0) {
                    *aux = right;
                    return kDiagNonFinite;
                }
                if (fo_fabs(cross) <= tolerance * fo_sqrt(ln * rn)) continue;
                converged = false;
                const double zeta = (rn - ln) / (2.0 * cross);
                double tangent = 1.0;
                if (zeta != 0.0) tangent = (zeta > 0.0 ? 1.0 : -1.0) / (fo_fabs(zeta) + fo_hypot(zeta, 1.0));
                const double cosine = 1.0 / fo_sqrt(fo_fma(tangent, tangent, 1.0));
                const double sine = cosine * tangent;
                for (int row = 0; row < columns; ++row) {
                    const int li = left * kMaxColumns + row, ri = right * kMaxColumns + row;
                    const double lv = t[li], rv = t[ri];
                    t[li] = fo_fma(cosine, lv, -sine * rv);
                    t[ri] = fo_fma(sine, lv, cosine * rv);
                }
            }
        }
        if (converged) break;
    }
    if (!converged) {
        *aux = columns;
        return kDiagNotConverged;
    }
    double sv[kMaxColumns];
    for (int c = 0; c < kMaxColumns; ++c) sv[c] = 0.0;
    for (int c = 0; c < columns; ++c) {
        double sq = 0.0;
        for (int row = 0; row < columns; ++row) {
            const double v = t[c * kMaxColumns + row];
            sq += v * v;
        }
        sv[c] = fo_sqrt(sq);
    }
    // descending insertion sort
    for (int i = 1; i < columns; ++i) {
        const double v = sv[i];
        int k = i - 1;
        while (k >= 0 && sv[k] < v) {
            sv[k + 1] = sv[k];
            --k;
        }
        sv[k + 1] = v;
    }
    const double largest = sv[0];
    const double threshold = rank_tolerance * largest;
    int rank = 0;
    for (int c = 0; c < columns; ++c) rank += sv[c] > threshold ? 1 : 0;
    *rank_out = rank;
    if (rank < columns) return kDiagRankDeficient;
    const double condition = largest / sv[columns - 1];
    *condition_out = condition;
    if (!fo_isfinite(condition)) {
        *aux = degree;
        return kDiagNonFinite;
    }
    if (condition > condition_limit) return kDiagConditionExceeded;
    return kDiagOk;
}

}  // namespace fo
