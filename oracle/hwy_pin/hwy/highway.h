// Pinned stand-in for the subset of the Highway SIMD API that the reference
// CPU core uses (src/core/distance_highway.hpp, src/linalg/kernels_highway.hpp).
//
// TEST INFRASTRUCTURE ONLY.  This header is part of the oracle: it lets the
// reference's own C++ sources compile here without the Highway library, and it
// fixes the floating-point order that Highway leaves to the compile target.
// Nothing in the product includes it.
//
// Semantics (written from the documented meaning of each op, one vector =
// 256 bits, which is what an AVX2 build of the reference uses):
//   * float vectors have 8 lanes, double vectors 4 lanes;
//   * Add/Sub/Mul are lane-wise IEEE operations, each rounded once;
//   * MulAdd(a, b, c) is lane-wise fused a*b+c (one rounding), as on every
//     FMA-capable target;
//   * ReduceSum folds halves: lanes [i] + [i + n/2] first, then again on the
//     lower half, until one lane is left.  For 8 floats that is
//     ((v0+v4)+(v2+v6)) + ((v1+v5)+(v3+v7)).
// The GPU plain path reproduces exactly this order.
#pragma once

#include <cmath>
#include <cstddef>

#define HWY_NAMESPACE N_PIN256

namespace hwy {
namespace HWY_NAMESPACE {

template <typename T> struct ScalableTag {
    static constexpr std::size_t kLanes = 32 / sizeof(T);
};

template <typename T> struct Vec {
    T lane[32 / sizeof(T)];
};

template <typename T>
constexpr std::size_t Lanes(ScalableTag<T>) noexcept {
    return ScalableTag<T>::kLanes;
}

template <typename T> inline Vec<T> Zero(ScalableTag<T>) noexcept {
    Vec<T> out;
    for (std::size_t i = 0; i < ScalableTag<T>::kLanes; ++i) {
        out.lane[i] = T(0);
    }
    return out;
}

template <typename T> inline Vec<T> Set(ScalableTag<T>, T value) noexcept {
    Vec<T> out;
    for (std::size_t i = 0; i < ScalableTag<T>::kLanes; ++i) {
        out.lane[i] = value;
    }
    return out;
}

template <typename T>
inline Vec<T> LoadU(ScalableTag<T>, const T* source) noexcept {
    Vec<T> out;
    for (std::size_t i = 0; i < ScalableTag<T>::kLanes; ++i) {
        out.lane[i] = source[i];
    }
    return out;
}

template <typename T>
inline void StoreU(Vec<T> value, ScalableTag<T>, T* destination) noexcept {
    for (std::size_t i = 0; i < ScalableTag<T>::kLanes; ++i) {
        destination[i] = value.lane[i];
    }
}

template <typename T> inline Vec<T> Add(Vec<T> a, Vec<T> b) noexcept {
    for (std::size_t i = 0; i < sizeof(a.lane) / sizeof(T); ++i) {
        a.lane[i] = a.lane[i] + b.lane[i];
    }
    return a;
}

template <typename T> inline Vec<T> Sub(Vec<T> a, Vec<T> b) noexcept {
    for (std::size_t i = 0; i < sizeof(a.lane) / sizeof(T); ++i) {
        a.lane[i] = a.lane[i] - b.lane[i];
    }
    return a;
}

template <typename T> inline Vec<T> Mul(Vec<T> a, Vec<T> b) noexcept {
    for (std::size_t i = 0; i < sizeof(a.lane) / sizeof(T); ++i) {
        a.lane[i] = a.lane[i] * b.lane[i];
    }
    return a;
}

template <typename T>
inline Vec<T> MulAdd(Vec<T> a, Vec<T> b, Vec<T> c) noexcept {
    for (std::size_t i = 0; i < sizeof(a.lane) / sizeof(T); ++i) {
        c.lane[i] = std::fma(a.lane[i], b.lane[i], c.lane[i]);
    }
    return c;
}

template <typename T> inline T ReduceSum(ScalableTag<T>, Vec<T> v) noexcept {
    for (std::size_t half = ScalableTag<T>::kLanes / 2; half > 0; half /= 2) {
        for (std::size_t i = 0; i < half; ++i) {
            v.lane[i] = v.lane[i] + v.lane[i + half];
        }
    }
    return v.lane[0];
}

} // namespace HWY_NAMESPACE
} // namespace hwy
