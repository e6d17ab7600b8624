// numtypes.hpp -- number types for the CPU oracle (test infrastructure only).
//
// f16: IEEE binary16 with Julia's Float16 semantics: every +,-,*,/ and sqrt
//      is evaluated in Float32 and rounded once to Float16 (round to nearest,
//      ties to even), conversions from Float32/Float64 round directly.
// Dual: forward-mode dual number (value, derivative) used to take directional
//      derivatives of the restated time loop.  ForwardDiff.Dual cannot be
//      used with the reference (its entry points require T<:AbstractFloat),
//      so this type stands in.  sqrt'(0) is taken as 0, the derivative of the
//      |x|x forms (quadratic drag, Smagorinsky) at rest.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>

namespace swo {

// ---------------------------------------------------------------- binary16
inline uint16_t f32_to_f16_bits(float f) {
    uint32_t x;
    std::memcpy(&x, &f, 4);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t ax = x & 0x7fffffffu;
    if (ax >= 0x7f800000u) {  // inf or nan
        if (ax > 0x7f800000u) return (uint16_t)(sign | 0x7e00u | ((ax >> 13) & 0x3ffu));
        return (uint16_t)(sign | 0x7c00u);
    }
    if (ax >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u);  // rounds to inf
    if (ax < 0x38800000u) {                                      // subnormal half
        if (ax < 0x33000000u) return (uint16_t)sign;             // < half of min subnormal
        uint32_t m = (ax & 0x7fffffu) | 0x800000u;
        int e = (int)(ax >> 23);                                 // 102..112
        int shift = 126 - e;                                     // bits to drop: 14..24
        uint32_t r = m >> shift;
        uint32_t rem = m & ((1u << shift) - 1u);
        uint32_t half = 1u << (shift - 1);
        if (rem > half || (rem == half && (r & 1u))) r++;
        return (uint16_t)(sign | r);
    }
    uint32_t e = (ax >> 23) - 112u;
    uint32_t m = ax & 0x7fffffu;
    uint32_t r = (e << 10) | (m >> 13);
    uint32_t rem = m & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (r & 1u))) r++;
    return (uint16_t)(sign | r);
}

inline uint16_t f64_to_f16_bits(double d) {
    // exact two-step: round to the nearest float with sticky bit preserved,
    // i.e. round-to-odd into float, then round-to-nearest into half
    if (std::isnan(d) || std::isinf(d)) return f32_to_f16_bits((float)d);
    float f = (float)d;                       // RNE
    double back = (double)f;
    if (back != d) {                          // make the float round-to-odd
        uint32_t x;
        std::memcpy(&x, &f, 4);
        if ((x & 1u) == 0) {
            // move one ulp toward d so the last bit is odd (sticky)
            float g = std::nextafter(f, (d > back) ? INFINITY : -INFINITY);
            uint32_t y;
            std::memcpy(&y, &g, 4);
            if (y & 1u) f = g;
        }
    }
    return f32_to_f16_bits(f);
}

inline float f16_bits_to_f32(uint16_t h) {
    uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    uint32_t e = (h >> 10) & 0x1fu;
    uint32_t m = h & 0x3ffu;
    uint32_t x;
    if (e == 0) {
        if (m == 0) {
            x = sign;
        } else {
            int k = 0;
            while (!(m & 0x400u)) { m <<= 1; k++; }
            m &= 0x3ffu;
            x = sign | ((uint32_t)(113 - k) << 23) | (m << 13);
        }
    } else if (e == 31) {
        x = sign | 0x7f800000u | (m << 13);
    } else {
        x = sign | ((e + 112u) << 23) | (m << 13);
    }
    float f;
    std::memcpy(&f, &x, 4);
    return f;
}

struct f16 {
    uint16_t b = 0;
    f16() = default;
    explicit f16(float x) : b(f32_to_f16_bits(x)) {}
    explicit f16(double x) : b(f64_to_f16_bits(x)) {}
    explicit f16(int x) : b(f64_to_f16_bits((double)x)) {}
    explicit operator float() const { return f16_bits_to_f32(b); }
    explicit operator double() const { return (double)f16_bits_to_f32(b); }
    static f16 from_bits(uint16_t v) { f16 h; h.b = v; return h; }
};
inline f16 operator+(f16 a, f16 b) { return f16((float)a + (float)b); }
inline f16 operator-(f16 a, f16 b) { return f16((float)a - (float)b); }
inline f16 operator*(f16 a, f16 b) { return f16((float)a * (float)b); }
inline f16 operator/(f16 a, f16 b) { return f16((float)a / (float)b); }
inline f16 operator-(f16 a) { return f16::from_bits((uint16_t)(a.b ^ 0x8000u)); }
inline f16& operator+=(f16& a, f16 b) { a = a + b; return a; }
inline bool operator<(f16 a, f16 b) { return (float)a < (float)b; }
inline bool operator>(f16 a, f16 b) { return (float)a > (float)b; }
inline bool operator==(f16 a, f16 b) { return (float)a == (float)b; }

// ---------------------------------------------------------------- Dual
struct Dual {
    double v = 0.0, d = 0.0;
    Dual() = default;
    Dual(double v_, double d_) : v(v_), d(d_) {}
    explicit Dual(double x) : v(x), d(0.0) {}
    explicit Dual(float x) : v((double)x), d(0.0) {}
    explicit Dual(int x) : v((double)x), d(0.0) {}
    explicit operator double() const { return v; }
    explicit operator float() const { return (float)v; }
};
inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
inline Dual operator/(Dual a, Dual b) {
    double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
inline Dual operator-(Dual a) { return {-a.v, -a.d}; }
inline Dual& operator+=(Dual& a, Dual b) { a = a + b; return a; }
inline bool operator<(Dual a, Dual b) { return a.v < b.v; }
inline bool operator>(Dual a, Dual b) { return a.v > b.v; }
inline bool operator==(Dual a, Dual b) { return a.v == b.v; }

// ---------------------------------------------------------------- helpers
template <class T> struct is_dual : std::false_type {};
template <> struct is_dual<Dual> : std::true_type {};

template <class T> inline T sqrt_(T x) { return std::sqrt(x); }
template <> inline f16 sqrt_<f16>(f16 x) { return f16(std::sqrt((float)x)); }
template <> inline Dual sqrt_<Dual>(Dual x) {
    double s = std::sqrt(x.v);
    return {s, (s > 0.0) ? x.d / (2.0 * s) : 0.0};
}

template <class T> inline double val(T x) { return (double)x; }
template <> inline double val<Dual>(Dual x) { return x.v; }

template <class T> inline bool isnan_(T x) { return std::isnan(val(x)); }

// conversion between number types (Julia's T(x))
template <class To, class From> inline To cvt(From x) {
    if constexpr (std::is_same_v<To, From>) return x;
    else if constexpr (is_dual<To>::value && is_dual<From>::value) return x;
    else if constexpr (is_dual<From>::value) return To(x.v);
    else if constexpr (std::is_same_v<From, f16>) return To((float)x);
    else return To(x);
}

// Julia's Int(floor(x)) for the tracer's departure indices
template <class T> inline int64_t ifloor(T x) { return (int64_t)std::floor(val(x)); }

}  // namespace swo
