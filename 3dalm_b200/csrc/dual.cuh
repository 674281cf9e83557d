// Forward-mode dual numbers with N directions, host and device.  Used by
// the actuator-line adjoint to differentiate one blade point's force model
// (a few dozen operations on scalars) with respect to its turbine's
// parameters and the sampled velocity.
#pragma once

#include <cmath>

#ifndef DALM_HD
#define DALM_HD __host__ __device__ __forceinline__
#endif

namespace dalm {
namespace adj {

// plain doubles, so the same generic code compiles for both
DALM_HD double sin(double x) { return ::sin(x); }
DALM_HD double cos(double x) { return ::cos(x); }
DALM_HD double atan(double x) { return ::atan(x); }
DALM_HD double fabs(double x) { return ::fabs(x); }

template <int N>
struct Dual {
    double v;
    double d[N];
    DALM_HD Dual() : v(0) {
        for (int i = 0; i < N; i++) d[i] = 0;
    }
    DALM_HD Dual(double x) : v(x) {
        for (int i = 0; i < N; i++) d[i] = 0;
    }
    // value x with derivative s in direction `dir`
    DALM_HD static Dual seed(double x, int dir, double s = 1.0) {
        Dual r(x);
        r.d[dir] = s;
        return r;
    }
};

DALM_HD double value(double x) { return x; }
template <int N>
DALM_HD double value(const Dual<N> &x) { return x.v; }

template <int N>
DALM_HD Dual<N> operator-(const Dual<N> &a) {
    Dual<N> r;
    r.v = -a.v;
    for (int i = 0; i < N; i++) r.d[i] = -a.d[i];
    return r;
}
template <int N>
DALM_HD Dual<N> operator+(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r;
    r.v = a.v + b.v;
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N>
DALM_HD Dual<N> operator-(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r;
    r.v = a.v - b.v;
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N>
DALM_HD Dual<N> operator*(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r;
    r.v = a.v * b.v;
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N>
DALM_HD Dual<N> operator/(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r;
    r.v = a.v / b.v;
    for (int i = 0; i < N; i++) r.d[i] = (a.d[i] - r.v * b.d[i]) / b.v;
    return r;
}
template <int N>
DALM_HD Dual<N> operator+(const Dual<N> &a, double b) {
    Dual<N> r = a;
    r.v = a.v + b;
    return r;
}
template <int N>
DALM_HD Dual<N> operator+(double a, const Dual<N> &b) {
    Dual<N> r = b;
    r.v = a + b.v;
    return r;
}
template <int N>
DALM_HD Dual<N> operator-(const Dual<N> &a, double b) {
    Dual<N> r = a;
    r.v = a.v - b;
    return r;
}
template <int N>
DALM_HD Dual<N> operator-(double a, const Dual<N> &b) {
    Dual<N> r;
    r.v = a - b.v;
    for (int i = 0; i < N; i++) r.d[i] = -b.d[i];
    return r;
}
template <int N>
DALM_HD Dual<N> operator*(const Dual<N> &a, double b) {
    Dual<N> r;
    r.v = a.v * b;
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * b;
    return r;
}
template <int N>
DALM_HD Dual<N> operator*(double a, const Dual<N> &b) {
    Dual<N> r;
    r.v = a * b.v;
    for (int i = 0; i < N; i++) r.d[i] = a * b.d[i];
    return r;
}
template <int N>
DALM_HD Dual<N> operator/(const Dual<N> &a, double b) {
    Dual<N> r;
    r.v = a.v / b;
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] / b;
    return r;
}
template <int N>
DALM_HD Dual<N> operator/(double a, const Dual<N> &b) {
    Dual<N> r;
    r.v = a / b.v;
    for (int i = 0; i < N; i++) r.d[i] = -r.v * b.d[i] / b.v;
    return r;
}

template <int N>
DALM_HD Dual<N> sin(const Dual<N> &a) {
    Dual<N> r;
    r.v = ::sin(a.v);
    double c = ::cos(a.v);
    for (int i = 0; i < N; i++) r.d[i] = c * a.d[i];
    return r;
}
template <int N>
DALM_HD Dual<N> cos(const Dual<N> &a) {
    Dual<N> r;
    r.v = ::cos(a.v);
    double s = -::sin(a.v);
    for (int i = 0; i < N; i++) r.d[i] = s * a.d[i];
    return r;
}
template <int N>
DALM_HD Dual<N> atan(const Dual<N> &a) {
    Dual<N> r;
    r.v = ::atan(a.v);
    double k = 1. / (1. + a.v * a.v);
    for (int i = 0; i < N; i++) r.d[i] = k * a.d[i];
    return r;
}
// derivative of the branch taken (sign of the value; 0 at 0)
template <int N>
DALM_HD Dual<N> fabs(const Dual<N> &a) {
    Dual<N> r;
    r.v = ::fabs(a.v);
    double s = (double)((a.v > 0.) - (a.v < 0.));
    for (int i = 0; i < N; i++) r.d[i] = s * a.d[i];
    return r;
}

}  // namespace adj
}  // namespace dalm
