// ORACLE — test infrastructure only.  CPU restatement of agent-ray's math
// layer (glam Vec3A/Mat4 semantics as used by the reference crate).  Only the
// tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it.
//
// PARITY UNPINNED: the reference is Rust with no tests or golden vectors and
// cannot be built here (no cargo/rustc, no crates).  glam's SSE2 code paths are
// restated from their published arithmetic order (products, then a left-to-
// right sum; no FMA contraction: build with -ffp-contract=off).
#pragma once
#include <cmath>
#include <cstdint>
#include <cfloat>
#include <limits>

#include "../agent-ray_b200/csrc/ar_trig.h"

namespace oracle {

// Sine and cosine of a sampling angle.  The FP32 oracle takes them from
// ar_trig.h, the single-precision routine the kernels use too, so the GPU and
// the oracle draw bit-identical directions (libm's sinf/cosf, which the Rust
// reference's f32::sin/cos reach, differ from it by at most about 1e-7 in
// absolute terms); the FP64 oracle uses the double-precision library.
inline void sin_cos(float phi, float& s, float& c) { ar_trig::sincos(phi, &s, &c); }
inline void sin_cos(double phi, double& s, double& c) {
    s = std::sin(phi);
    c = std::cos(phi);
}

template <class T> struct V2 { T x, y; };

template <class T>
struct V3 {
    T x, y, z;
    V3() : x(0), y(0), z(0) {}
    V3(T a, T b, T c) : x(a), y(b), z(c) {}
    T operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    template <class U>
    explicit V3(const V3<U>& o) : x(T(o.x)), y(T(o.y)), z(T(o.z)) {}
};

template <class T> inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> inline V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> inline V3<T> operator*(V3<T> a, V3<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T> inline V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> inline V3<T> operator/(V3<T> a, V3<T> b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
template <class T> inline V3<T>& operator+=(V3<T>& a, V3<T> b) { a = a + b; return a; }
template <class T> inline V3<T>& operator*=(V3<T>& a, V3<T> b) { a = a * b; return a; }
template <class T> inline V3<T>& operator/=(V3<T>& a, T s) { a = a / s; return a; }
template <class T> inline bool operator==(V3<T> a, V3<T> b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

// glam dot3: (x*x' + y*y') + z*z'
template <class T> inline T dot(V3<T> a, V3<T> b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
template <class T> inline V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> inline T length_squared(V3<T> a) { return dot(a, a); }
template <class T> inline T length(V3<T> a) { return std::sqrt(dot(a, a)); }
// glam normalize = self * (1 / length)
template <class T> inline V3<T> normalize(V3<T> a) { return a * (T(1) / length(a)); }
template <class T> inline V3<T> vabs(V3<T> a) { return {std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)}; }

// SSE minps/maxps semantics (second operand on NaN), used by AABB code.
template <class T> inline T sse_min(T a, T b) { return a < b ? a : b; }
template <class T> inline T sse_max(T a, T b) { return a > b ? a : b; }
template <class T> inline V3<T> vmin(V3<T> a, V3<T> b) { return {sse_min(a.x, b.x), sse_min(a.y, b.y), sse_min(a.z, b.z)}; }
template <class T> inline V3<T> vmax(V3<T> a, V3<T> b) { return {sse_max(a.x, b.x), sse_max(a.y, b.y), sse_max(a.z, b.z)}; }
// glam Vec3A::max_element / min_element (SSE2 shuffle reduction order)
template <class T> inline T max_element(V3<T> v) { return sse_max(sse_max(v.x, v.z), sse_max(v.y, v.z)); }
template <class T> inline T min_element(V3<T> v) { return sse_min(sse_min(v.x, v.z), sse_min(v.y, v.z)); }
// Rust f32::max / f32::min (IEEE maxNum: a NaN operand is ignored)
template <class T> inline T rmax(T a, T b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (a > b ? a : b)); }
template <class T> inline T rmin(T a, T b) { return std::isnan(a) ? b : (std::isnan(b) ? a : (a < b ? a : b)); }
// Rust f32::signum: +1 for +0.0 and positives, -1 for -0.0 and negatives
template <class T> inline T signum(T a) { return std::isnan(a) ? a : std::copysign(T(1), a); }

template <class T> inline T pi() { return T(3.14159265358979323846); }
template <> inline float pi<float>() { return 3.14159265358979323846f; }
template <class T> inline T frac_1_pi() { return T(0.318309886183790671538); }
template <> inline float frac_1_pi<float>() { return 0.318309886183790671538f; }
template <class T> inline T tmax_value() { return std::numeric_limits<T>::max(); }
// f32::MAX is used by the reference for "unbounded" rays even in the f64 oracle.
template <class T> inline T ray_unbounded() { return T(FLT_MAX); }

// 4x4 column-major matrix (glam::Mat4).  Columns c[0..3].
template <class T>
struct Mat4 {
    V3<T> c[4];   // xyz of each column; the bottom row is (0,0,0,1) for affine transforms
    // glam transform_point3a: ((c0*x + c1*y) + c2*z) + c3
    V3<T> transform_point(V3<T> p) const {
        V3<T> r = c[0] * p.x;
        r = c[1] * p.y + r;
        r = c[2] * p.z + r;
        return c[3] + r;
    }
    V3<T> transform_vector(V3<T> v) const {
        V3<T> r = c[0] * v.x;
        r = c[1] * v.y + r;
        return c[2] * v.z + r;
    }
};

// glam::Mat3 (columns).  mul_vec3: (c0*x + c1*y) + c2*z
template <class T>
struct Mat3 {
    V3<T> c[3];
    V3<T> mul(V3<T> v) const {
        V3<T> r = c[0] * v.x;
        r = r + c[1] * v.y;
        return r + c[2] * v.z;
    }
};

// Mat3::from_mat4(m).inverse().transpose() as glam computes it:
// inverse = from_cols(y×z, z×x, x×y)/det transposed; the trailing transpose
// cancels, leaving columns (y×z, z×x, x×y) * (1/det).
template <class T>
inline Mat3<T> normal_matrix(const Mat4<T>& m) {
    V3<T> x = m.c[0], y = m.c[1], z = m.c[2];
    V3<T> t0 = cross(y, z), t1 = cross(z, x), t2 = cross(x, y);
    T det = dot(z, t2);
    T inv_det = T(1) / det;
    Mat3<T> r;
    r.c[0] = t0 * inv_det;
    r.c[1] = t1 * inv_det;
    r.c[2] = t2 * inv_det;
    return r;
}

// General 4x4 inverse in double (cofactor expansion), used only when the scene
// description does not carry the inverse.  glam's own Mat4::inverse is not
// restated (its rounding is unpinned); callers that need bit parity pass it.
inline void invert4x4_colmajor(const float* m, float* out) {
    double a[16];
    for (int i = 0; i < 16; ++i) a[i] = m[i];
    double inv[16];
    inv[0] = a[5] * a[10] * a[15] - a[5] * a[11] * a[14] - a[9] * a[6] * a[15] + a[9] * a[7] * a[14] + a[13] * a[6] * a[11] - a[13] * a[7] * a[10];
    inv[4] = -a[4] * a[10] * a[15] + a[4] * a[11] * a[14] + a[8] * a[6] * a[15] - a[8] * a[7] * a[14] - a[12] * a[6] * a[11] + a[12] * a[7] * a[10];
    inv[8] = a[4] * a[9] * a[15] - a[4] * a[11] * a[13] - a[8] * a[5] * a[15] + a[8] * a[7] * a[13] + a[12] * a[5] * a[11] - a[12] * a[7] * a[9];
    inv[12] = -a[4] * a[9] * a[14] + a[4] * a[10] * a[13] + a[8] * a[5] * a[14] - a[8] * a[6] * a[13] - a[12] * a[5] * a[10] + a[12] * a[6] * a[9];
    inv[1] = -a[1] * a[10] * a[15] + a[1] * a[11] * a[14] + a[9] * a[2] * a[15] - a[9] * a[3] * a[14] - a[13] * a[2] * a[11] + a[13] * a[3] * a[10];
    inv[5] = a[0] * a[10] * a[15] - a[0] * a[11] * a[14] - a[8] * a[2] * a[15] + a[8] * a[3] * a[14] + a[12] * a[2] * a[11] - a[12] * a[3] * a[10];
    inv[9] = -a[0] * a[9] * a[15] + a[0] * a[11] * a[13] + a[8] * a[1] * a[15] - a[8] * a[3] * a[13] - a[12] * a[1] * a[11] + a[12] * a[3] * a[9];
    inv[13] = a[0] * a[9] * a[14] - a[0] * a[10] * a[13] - a[8] * a[1] * a[14] + a[8] * a[2] * a[13] + a[12] * a[1] * a[10] - a[12] * a[2] * a[9];
    inv[2] = a[1] * a[6] * a[15] - a[1] * a[7] * a[14] - a[5] * a[2] * a[15] + a[5] * a[3] * a[14] + a[13] * a[2] * a[7] - a[13] * a[3] * a[6];
    inv[6] = -a[0] * a[6] * a[15] + a[0] * a[7] * a[14] + a[4] * a[2] * a[15] - a[4] * a[3] * a[14] - a[12] * a[2] * a[7] + a[12] * a[3] * a[6];
    inv[10] = a[0] * a[5] * a[15] - a[0] * a[7] * a[13] - a[4] * a[1] * a[15] + a[4] * a[3] * a[13] + a[12] * a[1] * a[7] - a[12] * a[3] * a[5];
    inv[14] = -a[0] * a[5] * a[14] + a[0] * a[6] * a[13] + a[4] * a[1] * a[14] - a[4] * a[2] * a[13] - a[12] * a[1] * a[6] + a[12] * a[2] * a[5];
    inv[3] = -a[1] * a[6] * a[11] + a[1] * a[7] * a[10] + a[5] * a[2] * a[11] - a[5] * a[3] * a[10] - a[9] * a[2] * a[7] + a[9] * a[3] * a[6];
    inv[7] = a[0] * a[6] * a[11] - a[0] * a[7] * a[10] - a[4] * a[2] * a[11] + a[4] * a[3] * a[10] + a[8] * a[2] * a[7] - a[8] * a[3] * a[6];
    inv[11] = -a[0] * a[5] * a[11] + a[0] * a[7] * a[9] + a[4] * a[1] * a[11] - a[4] * a[3] * a[9] - a[8] * a[1] * a[7] + a[8] * a[3] * a[5];
    inv[15] = a[0] * a[5] * a[10] - a[0] * a[6] * a[9] - a[4] * a[1] * a[10] + a[4] * a[2] * a[9] + a[8] * a[1] * a[6] - a[8] * a[2] * a[5];
    double det = a[0] * inv[0] + a[1] * inv[4] + a[2] * inv[8] + a[3] * inv[12];
    double id = 1.0 / det;
    for (int i = 0; i < 16; ++i) out[i] = float(inv[i] * id);
}

}  // namespace oracle
