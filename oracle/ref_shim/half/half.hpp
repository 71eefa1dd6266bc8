// Minimal stand-in for the half-ieee754 header ("half/half.hpp") that noa includes.
//
// ORACLE TEST INFRASTRUCTURE. This header exists only so that the reference's own CPU sources can be
// compiled into oracle/_ref (the parity checker). It provides `half_float::half` as a thin wrapper over
// the compiler's `_Float16`, plus the handful of free functions noa's `f16` type forwards to
// (noa/base/Half.hpp). The Fourier-projection path never computes in half precision, so these only need
// to compile and be reasonable; they are not used by any parity case.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>

namespace half_float {
    class half {
    public:
        constexpr half() noexcept = default;
        constexpr half(const half&) noexcept = default;
        constexpr half& operator=(const half&) noexcept = default;

        // Conversion from any arithmetic type (the reference only converts through half_cast).
        template<typename T, std::enable_if_t<std::is_arithmetic_v<T>, int> = 0>
        explicit constexpr half(T v) noexcept : m_v(static_cast<_Float16>(v)) {}

        constexpr operator float() const noexcept { return static_cast<float>(m_v); }

        constexpr half& operator+=(half o) noexcept { m_v += o.m_v; return *this; }
        constexpr half& operator-=(half o) noexcept { m_v -= o.m_v; return *this; }
        constexpr half& operator*=(half o) noexcept { m_v *= o.m_v; return *this; }
        constexpr half& operator/=(half o) noexcept { m_v /= o.m_v; return *this; }
        constexpr half& operator++() noexcept { m_v += static_cast<_Float16>(1); return *this; }
        constexpr half& operator--() noexcept { m_v -= static_cast<_Float16>(1); return *this; }
        constexpr half operator++(int) noexcept { half t = *this; ++*this; return t; }
        constexpr half operator--(int) noexcept { half t = *this; --*this; return t; }

        friend constexpr half operator+(half a, half b) noexcept { return from_f16(a.m_v + b.m_v); }
        friend constexpr half operator-(half a, half b) noexcept { return from_f16(a.m_v - b.m_v); }
        friend constexpr half operator*(half a, half b) noexcept { return from_f16(a.m_v * b.m_v); }
        friend constexpr half operator/(half a, half b) noexcept { return from_f16(a.m_v / b.m_v); }
        friend constexpr half operator-(half a) noexcept { return from_f16(-a.m_v); }
        friend constexpr half operator+(half a) noexcept { return a; }
        friend constexpr bool operator==(half a, half b) noexcept { return a.m_v == b.m_v; }
        friend constexpr bool operator!=(half a, half b) noexcept { return a.m_v != b.m_v; }
        friend constexpr bool operator<(half a, half b) noexcept { return a.m_v < b.m_v; }
        friend constexpr bool operator>(half a, half b) noexcept { return a.m_v > b.m_v; }
        friend constexpr bool operator<=(half a, half b) noexcept { return a.m_v <= b.m_v; }
        friend constexpr bool operator>=(half a, half b) noexcept { return a.m_v >= b.m_v; }

        static constexpr half from_f16(_Float16 v) noexcept { half h; h.m_v = v; return h; }
        constexpr _Float16 raw() const noexcept { return m_v; }

    private:
        _Float16 m_v{};
    };
    static_assert(sizeof(half) == 2 && std::is_standard_layout_v<half>);

    // Bit reinterpretation usable in constant expressions.
    constexpr half reinterpret_as_half(std::uint16_t bits) noexcept {
        return half::from_f16(__builtin_bit_cast(_Float16, bits));
    }

    template<typename T, typename U>
    constexpr T half_cast(U value) noexcept {
        if constexpr (std::is_same_v<T, half>) {
            if constexpr (std::is_same_v<U, half>)
                return value;
            else
                return half::from_f16(static_cast<_Float16>(value));
        } else {
            return static_cast<T>(static_cast<float>(value));
        }
    }

    namespace detail {
        inline half h(float v) noexcept { return half::from_f16(static_cast<_Float16>(v)); }
    }

#define NOA_B200_HALF_UNARY(name, expr) \
    inline half name(half x) noexcept { const float a = static_cast<float>(x); return detail::h(expr); }
    NOA_B200_HALF_UNARY(abs, std::fabs(a))
    NOA_B200_HALF_UNARY(cos, std::cos(a))
    NOA_B200_HALF_UNARY(sin, std::sin(a))
    NOA_B200_HALF_UNARY(tan, std::tan(a))
    NOA_B200_HALF_UNARY(cosh, std::cosh(a))
    NOA_B200_HALF_UNARY(sinh, std::sinh(a))
    NOA_B200_HALF_UNARY(tanh, std::tanh(a))
    NOA_B200_HALF_UNARY(acos, std::acos(a))
    NOA_B200_HALF_UNARY(asin, std::asin(a))
    NOA_B200_HALF_UNARY(atan, std::atan(a))
    NOA_B200_HALF_UNARY(acosh, std::acosh(a))
    NOA_B200_HALF_UNARY(asinh, std::asinh(a))
    NOA_B200_HALF_UNARY(atanh, std::atanh(a))
    NOA_B200_HALF_UNARY(exp, std::exp(a))
    NOA_B200_HALF_UNARY(log, std::log(a))
    NOA_B200_HALF_UNARY(log10, std::log10(a))
    NOA_B200_HALF_UNARY(log1p, std::log1p(a))
    NOA_B200_HALF_UNARY(sqrt, std::sqrt(a))
    NOA_B200_HALF_UNARY(rsqrt, 1.0f / std::sqrt(a))
    NOA_B200_HALF_UNARY(round, std::round(a))
    NOA_B200_HALF_UNARY(rint, std::rint(a))
    NOA_B200_HALF_UNARY(ceil, std::ceil(a))
    NOA_B200_HALF_UNARY(floor, std::floor(a))
    NOA_B200_HALF_UNARY(trunc, std::trunc(a))
#undef NOA_B200_HALF_UNARY

    inline half atan2(half y, half x) noexcept { return detail::h(std::atan2(float(y), float(x))); }
    inline half pow(half x, half e) noexcept { return detail::h(std::pow(float(x), float(e))); }
    inline half fma(half x, half y, half z) noexcept { return detail::h(std::fma(float(x), float(y), float(z))); }
    inline half fmin(half x, half y) noexcept { return detail::h(std::fmin(float(x), float(y))); }
    inline half fmax(half x, half y) noexcept { return detail::h(std::fmax(float(x), float(y))); }
    inline bool isnan(half x) noexcept { return std::isnan(float(x)); }
    inline bool isinf(half x) noexcept { return std::isinf(float(x)); }
    inline void sincos(half x, half* s, half* c) noexcept {
        *s = detail::h(std::sin(float(x)));
        *c = detail::h(std::cos(float(x)));
    }
}
