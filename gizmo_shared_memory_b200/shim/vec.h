// Small vector / symmetric-tensor types for the shmem:: shim, with the interface callers of the
// reference's tree use (math_types/vec3.h, math_types/symmetric_tensor2.h via shmem/vec.h):
// aggregate storage, operator[], and for the tensor the (i, j) indexing over the storage order
// xx, yy, zz, xy, yz, xz -- the order is part of the interface, since callers read tensors
// element by element.
#pragma once
#include <cmath>

template <typename T>
struct Vec3 {
    T data[3];
    T& operator[](int i) noexcept { return data[i]; }
    const T& operator[](int i) const noexcept { return data[i]; }
    Vec3& operator+=(const Vec3& o) noexcept {
        for (int k = 0; k < 3; ++k) data[k] += o.data[k];
        return *this;
    }
    Vec3& operator-=(const Vec3& o) noexcept {
        for (int k = 0; k < 3; ++k) data[k] -= o.data[k];
        return *this;
    }
    Vec3& operator*=(T s) noexcept {
        for (int k = 0; k < 3; ++k) data[k] *= s;
        return *this;
    }
    T norm_sq() const noexcept { return data[0] * data[0] + data[1] * data[1] + data[2] * data[2]; }
    T norm() const noexcept { return std::sqrt(norm_sq()); }
};
template <typename T> inline Vec3<T> operator+(Vec3<T> a, const Vec3<T>& b) noexcept { return a += b; }
template <typename T> inline Vec3<T> operator-(Vec3<T> a, const Vec3<T>& b) noexcept { return a -= b; }
template <typename T> inline Vec3<T> operator*(Vec3<T> a, T s) noexcept { return a *= s; }
template <typename T> inline Vec3<T> operator*(T s, Vec3<T> a) noexcept { return a *= s; }

template <typename T>
struct SymmetricTensor2 {
    T data[6];  // xx, yy, zz, xy, yz, xz
    static constexpr int slot(int i, int j) noexcept {
        return i == j ? i : ((i + j == 1) ? 3 : ((i + j == 3) ? 4 : 5));
    }
    struct Row {
        SymmetricTensor2& t;
        int i;
        T& operator[](int j) noexcept { return t.data[slot(i, j)]; }
    };
    struct ConstRow {
        const SymmetricTensor2& t;
        int i;
        const T& operator[](int j) const noexcept { return t.data[slot(i, j)]; }
    };
    Row operator[](int i) noexcept { return {*this, i}; }
    ConstRow operator[](int i) const noexcept { return {*this, i}; }
    T trace() const noexcept { return data[0] + data[1] + data[2]; }
};

namespace shmem {
using Vec3d = Vec3<double>;
using SymTensor3d = SymmetricTensor2<double>;

// Minimum-image separation for periodic boxes (box <= 0: non-periodic), as callers of the tree use it.
static inline double min_image(double s, double box) {
    if (box > 0) {
        if (s > 0.5 * box) s -= box;
        else if (s < -0.5 * box) s += box;
    }
    return s;
}
}  // namespace shmem
