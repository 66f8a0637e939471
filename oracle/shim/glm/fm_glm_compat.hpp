// Test infrastructure for the oracle build only (never linked into the product).
//
// The reference declares `thirdparty/glm` as a git submodule that is empty in this
// checkout, and no glm installation exists on the machine.  This header supplies the
// subset of glm's API that the reference engine uses (vec2/3/4, mat4, dot, cross,
// length, normalize, sqrt, inverse, transpose, lookAt (left-handed), rotate,
// translate, scale), written from the underlying mathematics.
//
// Rounding conventions (chosen to follow glm's documented evaluation order where it is
// observable; the glm release the reference was built against is unknown, so any
// glm-dependent rounding is unpinned):
//   dot(a, b)        = (a.x*b.x + a.y*b.y) + a.z*b.z      (left to right)
//   length(v)        = sqrt(dot(v, v))
//   normalize(v)     = v * (1 / sqrt(dot(v, v)))
//   mat4 * vec4      = (c0*v.x + c1*v.y) + (c2*v.z + c3*v.w)   (column-major)
//   mat4 * mat4      = column j: ((c0*b.x + c1*b.y) + c2*b.z) + c3*b.w
// Identity and translation-only transforms are exact under any of these orders, which
// is why the hit-ID parity tests restrict themselves to such transforms.
#ifndef FM_ORACLE_GLM_COMPAT_HPP
#define FM_ORACLE_GLM_COMPAT_HPP

#include <cmath>
#include <cstddef>
#include <type_traits>

namespace glm {

template <int L, typename T> struct vec;

template <typename T> struct vec<2, T> {
    T x, y;
    vec() = default;
    explicit vec(T s) : x(s), y(s) {}
    vec(T a, T b) : x(a), y(b) {}
    // glm converts longer vectors to shorter ones implicitly, keeping the leading
    // components; the reference relies on this (e.g. bsdf.h:88 passes a vec3 sample).
    vec(const vec<3, T>& v);
    vec(const vec<4, T>& v);
    T& operator[](int i) { return i == 0 ? x : y; }
    const T& operator[](int i) const { return i == 0 ? x : y; }
};

template <typename T> struct vec<3, T> {
    T x, y, z;
    vec() = default;
    explicit vec(T s) : x(s), y(s), z(s) {}
    vec(T a, T b, T c) : x(a), y(b), z(c) {}
    vec(const vec<4, T>& v);
    T& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    const T& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

template <typename T> struct vec<4, T> {
    T x, y, z, w;
    vec() = default;
    explicit vec(T s) : x(s), y(s), z(s), w(s) {}
    vec(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
    vec(const vec<3, T>& v, T d) : x(v.x), y(v.y), z(v.z), w(d) {}
    T& operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    const T& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
};

template <typename T>
vec<3, T>::vec(const vec<4, T>& v) : x(v.x), y(v.y), z(v.z) {}
template <typename T>
vec<2, T>::vec(const vec<3, T>& v) : x(v.x), y(v.y) {}
template <typename T>
vec<2, T>::vec(const vec<4, T>& v) : x(v.x), y(v.y) {}

// ---- component-wise arithmetic -------------------------------------------------
#define FM_GLM_BINOP(OP)                                                                   \
    template <int L, typename T> vec<L, T> operator OP(const vec<L, T>& a, const vec<L, T>& b) \
    { vec<L, T> r; for (int i = 0; i < L; ++i) r[i] = a[i] OP b[i]; return r; }            \
    template <int L, typename T> vec<L, T> operator OP(const vec<L, T>& a, T s)            \
    { vec<L, T> r; for (int i = 0; i < L; ++i) r[i] = a[i] OP s; return r; }               \
    template <int L, typename T> vec<L, T> operator OP(T s, const vec<L, T>& a)            \
    { vec<L, T> r; for (int i = 0; i < L; ++i) r[i] = s OP a[i]; return r; }               \
    template <int L, typename T, typename U,                                               \
              typename = std::enable_if_t<std::is_arithmetic<U>::value>>                   \
    vec<L, T>& operator OP##=(vec<L, T>& a, U s)                                           \
    { for (int i = 0; i < L; ++i) a[i] = a[i] OP static_cast<T>(s); return a; }            \
    template <int L, typename T> vec<L, T>& operator OP##=(vec<L, T>& a, const vec<L, T>& b) \
    { for (int i = 0; i < L; ++i) a[i] = a[i] OP b[i]; return a; }

FM_GLM_BINOP(+)
FM_GLM_BINOP(-)
FM_GLM_BINOP(*)
FM_GLM_BINOP(/)
#undef FM_GLM_BINOP

template <int L, typename T> vec<L, T> operator-(const vec<L, T>& a)
{ vec<L, T> r; for (int i = 0; i < L; ++i) r[i] = -a[i]; return r; }

template <int L, typename T> bool operator==(const vec<L, T>& a, const vec<L, T>& b)
{ for (int i = 0; i < L; ++i) if (!(a[i] == b[i])) return false; return true; }

// ---- geometric functions -------------------------------------------------------
template <typename T> T dot(const vec<2, T>& a, const vec<2, T>& b) { return a.x * b.x + a.y * b.y; }
template <typename T> T dot(const vec<3, T>& a, const vec<3, T>& b)
{ return (a.x * b.x + a.y * b.y) + a.z * b.z; }
template <typename T> T dot(const vec<4, T>& a, const vec<4, T>& b)
{ return (a.x * b.x + a.y * b.y) + (a.z * b.z + a.w * b.w); }

template <typename T> vec<3, T> cross(const vec<3, T>& a, const vec<3, T>& b)
{ return vec<3, T>(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y); }

template <int L, typename T> T length(const vec<L, T>& v) { return std::sqrt(dot(v, v)); }

template <int L, typename T> vec<L, T> normalize(const vec<L, T>& v)
{ const T inv = static_cast<T>(1) / std::sqrt(dot(v, v)); return v * inv; }

template <int L, typename T> vec<L, T> sqrt(const vec<L, T>& v)
{ vec<L, T> r; for (int i = 0; i < L; ++i) r[i] = std::sqrt(v[i]); return r; }

// ---- 4x4 column-major matrices -------------------------------------------------
template <int C, int R, typename T> struct mat;

template <typename T> struct mat<4, 4, T> {
    vec<4, T> c[4];
    mat() = default;
    explicit mat(T d)
    {
        for (int j = 0; j < 4; ++j)
            for (int i = 0; i < 4; ++i) c[j][i] = (i == j) ? d : static_cast<T>(0);
    }
    vec<4, T>& operator[](int j) { return c[j]; }
    const vec<4, T>& operator[](int j) const { return c[j]; }
};

template <typename T> vec<4, T> operator*(const mat<4, 4, T>& m, const vec<4, T>& v)
{
    const vec<4, T> a = m[0] * v.x + m[1] * v.y;
    const vec<4, T> b = m[2] * v.z + m[3] * v.w;
    return a + b;
}

template <typename T> mat<4, 4, T> operator*(const mat<4, 4, T>& a, const mat<4, 4, T>& b)
{
    mat<4, 4, T> r;
    for (int j = 0; j < 4; ++j)
        r[j] = ((a[0] * b[j].x + a[1] * b[j].y) + a[2] * b[j].z) + a[3] * b[j].w;
    return r;
}

template <typename T> mat<4, 4, T> operator*(const mat<4, 4, T>& a, T s)
{ mat<4, 4, T> r; for (int j = 0; j < 4; ++j) r[j] = a[j] * s; return r; }

template <typename T> mat<4, 4, T> transpose(const mat<4, 4, T>& m)
{
    mat<4, 4, T> r;
    for (int j = 0; j < 4; ++j)
        for (int i = 0; i < 4; ++i) r[j][i] = m[i][j];
    return r;
}

// General inverse by the adjugate: inv = adj(M) / det(M), with the cofactors built
// from the 2x2 minors of the first two and last two rows (Laplace expansion).
template <typename T> mat<4, 4, T> inverse(const mat<4, 4, T>& m)
{
    // a[r][c] = element at row r, column c
    T a[4][4];
    for (int r = 0; r < 4; ++r)
        for (int cc = 0; cc < 4; ++cc) a[r][cc] = m[cc][r];
    // 2x2 minors of rows 0,1 and rows 2,3
    const T s0 = a[0][0] * a[1][1] - a[1][0] * a[0][1];
    const T s1 = a[0][0] * a[1][2] - a[1][0] * a[0][2];
    const T s2 = a[0][0] * a[1][3] - a[1][0] * a[0][3];
    const T s3 = a[0][1] * a[1][2] - a[1][1] * a[0][2];
    const T s4 = a[0][1] * a[1][3] - a[1][1] * a[0][3];
    const T s5 = a[0][2] * a[1][3] - a[1][2] * a[0][3];
    const T c5 = a[2][2] * a[3][3] - a[3][2] * a[2][3];
    const T c4 = a[2][1] * a[3][3] - a[3][1] * a[2][3];
    const T c3 = a[2][1] * a[3][2] - a[3][1] * a[2][2];
    const T c2 = a[2][0] * a[3][3] - a[3][0] * a[2][3];
    const T c1 = a[2][0] * a[3][2] - a[3][0] * a[2][2];
    const T c0 = a[2][0] * a[3][1] - a[3][0] * a[2][1];
    const T det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
    const T id = static_cast<T>(1) / det;
    T b[4][4];
    b[0][0] = ( a[1][1] * c5 - a[1][2] * c4 + a[1][3] * c3) * id;
    b[0][1] = (-a[0][1] * c5 + a[0][2] * c4 - a[0][3] * c3) * id;
    b[0][2] = ( a[3][1] * s5 - a[3][2] * s4 + a[3][3] * s3) * id;
    b[0][3] = (-a[2][1] * s5 + a[2][2] * s4 - a[2][3] * s3) * id;
    b[1][0] = (-a[1][0] * c5 + a[1][2] * c2 - a[1][3] * c1) * id;
    b[1][1] = ( a[0][0] * c5 - a[0][2] * c2 + a[0][3] * c1) * id;
    b[1][2] = (-a[3][0] * s5 + a[3][2] * s2 - a[3][3] * s1) * id;
    b[1][3] = ( a[2][0] * s5 - a[2][2] * s2 + a[2][3] * s1) * id;
    b[2][0] = ( a[1][0] * c4 - a[1][1] * c2 + a[1][3] * c0) * id;
    b[2][1] = (-a[0][0] * c4 + a[0][1] * c2 - a[0][3] * c0) * id;
    b[2][2] = ( a[3][0] * s4 - a[3][1] * s2 + a[3][3] * s0) * id;
    b[2][3] = (-a[2][0] * s4 + a[2][1] * s2 - a[2][3] * s0) * id;
    b[3][0] = (-a[1][0] * c3 + a[1][1] * c1 - a[1][2] * c0) * id;
    b[3][1] = ( a[0][0] * c3 - a[0][1] * c1 + a[0][2] * c0) * id;
    b[3][2] = (-a[3][0] * s3 + a[3][1] * s1 - a[3][2] * s0) * id;
    b[3][3] = ( a[2][0] * s3 - a[2][1] * s1 + a[2][2] * s0) * id;
    mat<4, 4, T> r;
    for (int rr = 0; rr < 4; ++rr)
        for (int cc = 0; cc < 4; ++cc) r[cc][rr] = b[rr][cc];
    return r;
}

// translate(m, v): m * T(v)
template <typename T> mat<4, 4, T> translate(const mat<4, 4, T>& m, const vec<3, T>& v)
{
    mat<4, 4, T> r = m;
    r[3] = ((m[0] * v.x + m[1] * v.y) + m[2] * v.z) + m[3];
    return r;
}

// scale(m, v): m * S(v)
template <typename T> mat<4, 4, T> scale(const mat<4, 4, T>& m, const vec<3, T>& v)
{
    mat<4, 4, T> r;
    r[0] = m[0] * v.x;
    r[1] = m[1] * v.y;
    r[2] = m[2] * v.z;
    r[3] = m[3];
    return r;
}

// rotate(m, angle, axis): m * R where R is the Rodrigues rotation about the normalized
// axis a by `angle` radians: R = cos*I + (1-cos)*a*a^T + sin*[a]_x.
template <typename T> mat<4, 4, T> rotate(const mat<4, 4, T>& m, T angle, const vec<3, T>& axis_in)
{
    const T c = std::cos(angle);
    const T s = std::sin(angle);
    const vec<3, T> a = normalize(axis_in);
    const vec<3, T> k = (static_cast<T>(1) - c) * a;
    // R stored column-major: R[col][row]
    T R[3][3];
    R[0][0] = c + k.x * a.x;        R[0][1] = k.x * a.y + s * a.z;  R[0][2] = k.x * a.z - s * a.y;
    R[1][0] = k.y * a.x - s * a.z;  R[1][1] = c + k.y * a.y;        R[1][2] = k.y * a.z + s * a.x;
    R[2][0] = k.z * a.x + s * a.y;  R[2][1] = k.z * a.y - s * a.x;  R[2][2] = c + k.z * a.z;
    mat<4, 4, T> r;
    for (int j = 0; j < 3; ++j)
        r[j] = (m[0] * R[j][0] + m[1] * R[j][1]) + m[2] * R[j][2];
    r[3] = m[3];
    return r;
}

template <typename T> mat<4, 4, T> rotate(T angle, const vec<3, T>& axis)
{ return rotate(mat<4, 4, T>(static_cast<T>(1)), angle, axis); }

// Left-handed view matrix (the reference defines GLM_FORCE_LEFT_HANDED): the camera
// looks down +z of its local frame, x = normalize(cross(up, forward)), y = cross(f, x).
template <typename T> mat<4, 4, T> lookAt(const vec<3, T>& eye, const vec<3, T>& center, const vec<3, T>& up)
{
    const vec<3, T> f = normalize(center - eye);
    const vec<3, T> s = normalize(cross(up, f));
    const vec<3, T> u = cross(f, s);
    mat<4, 4, T> r(static_cast<T>(1));
    r[0][0] = s.x; r[1][0] = s.y; r[2][0] = s.z;
    r[0][1] = u.x; r[1][1] = u.y; r[2][1] = u.z;
    r[0][2] = f.x; r[1][2] = f.y; r[2][2] = f.z;
    r[3][0] = -dot(s, eye);
    r[3][1] = -dot(u, eye);
    r[3][2] = -dot(f, eye);
    return r;
}

using vec2 = vec<2, float>;
using vec3 = vec<3, float>;
using vec4 = vec<4, float>;
using dvec2 = vec<2, double>;
using dvec3 = vec<3, double>;
using dvec4 = vec<4, double>;
using mat4 = mat<4, 4, float>;
using dmat4 = mat<4, 4, double>;

}  // namespace glm

#endif
