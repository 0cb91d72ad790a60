// Test infrastructure -- NOT part of the product path.
//
// Host stand-in for goss_b200/csrc/goss_device_math.cuh, found first on the
// include path when oracle/tangent/tangent_grl1.cpp compiles a generated
// model's device.cuh with g++.  It turns the CUDA qualifiers into plain C++
// and supplies the scalar functions the generated code calls (gexp, glog,
// gpow, ...) for double and for Dual<D>, a forward-mode dual number carrying
// D tangent directions.  Instantiating the generated `linearized<T>` with
// T = Dual<D> gives the exact FP64 directional derivatives of the linearised
// right-hand side, independent of the reverse-mode sweep the adjoint kernels
// use (goss_b200/codegen/ad.py).
#ifndef GOSS_DEVICE_MATH_CUH
#define GOSS_DEVICE_MATH_CUH

#include <cmath>

#ifndef __device__
#define __device__
#endif
#ifndef __host__
#define __host__
#endif
#ifndef __forceinline__
#define __forceinline__ inline
#endif

namespace goss_b200 { namespace models {

using std::ceil;
using std::exp;
using std::fabs;
using std::floor;
using std::log;
using std::pow;
using std::sqrt;

template <int D>
struct Dual {
    double v;
    double d[D];
    Dual() : v(0.0) { for (int k = 0; k < D; ++k) d[k] = 0.0; }
    explicit Dual(double x) : v(x) { for (int k = 0; k < D; ++k) d[k] = 0.0; }
    // value f, derivative scale g: result.d = g * a.d
    static Dual chain(double f, double g, const Dual& a)
    {
        Dual r(f);
        for (int k = 0; k < D; ++k) r.d[k] = g * a.d[k];
        return r;
    }
    bool has_tangent() const
    {
        for (int k = 0; k < D; ++k)
            if (d[k] != 0.0) return true;
        return false;
    }
};

template <int D> inline Dual<D> operator+(const Dual<D>& a) { return a; }
template <int D> inline Dual<D> operator-(const Dual<D>& a) { return Dual<D>::chain(-a.v, -1.0, a); }

template <int D> inline Dual<D> operator+(const Dual<D>& a, const Dual<D>& b)
{
    Dual<D> r(a.v + b.v);
    for (int k = 0; k < D; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
template <int D> inline Dual<D> operator-(const Dual<D>& a, const Dual<D>& b)
{
    Dual<D> r(a.v - b.v);
    for (int k = 0; k < D; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
template <int D> inline Dual<D> operator*(const Dual<D>& a, const Dual<D>& b)
{
    Dual<D> r(a.v * b.v);
    for (int k = 0; k < D; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <int D> inline Dual<D> operator/(const Dual<D>& a, const Dual<D>& b)
{
    const double q = a.v / b.v;
    Dual<D> r(q);
    for (int k = 0; k < D; ++k) r.d[k] = (a.d[k] - q * b.d[k]) / b.v;
    return r;
}
template <int D> inline Dual<D> operator+(const Dual<D>& a, double b) { return a + Dual<D>(b); }
template <int D> inline Dual<D> operator+(double a, const Dual<D>& b) { return Dual<D>(a) + b; }
template <int D> inline Dual<D> operator-(const Dual<D>& a, double b) { return a - Dual<D>(b); }
template <int D> inline Dual<D> operator-(double a, const Dual<D>& b) { return Dual<D>(a) - b; }
template <int D> inline Dual<D> operator*(const Dual<D>& a, double b) { return a * Dual<D>(b); }
template <int D> inline Dual<D> operator*(double a, const Dual<D>& b) { return Dual<D>(a) * b; }
template <int D> inline Dual<D> operator/(const Dual<D>& a, double b) { return a / Dual<D>(b); }
template <int D> inline Dual<D> operator/(double a, const Dual<D>& b) { return Dual<D>(a) / b; }

// comparisons (conditionals and the GRL1 threshold) see values only
#define GOSS_DUAL_CMP(op)                                                                         \
    template <int D> inline bool operator op(const Dual<D>& a, const Dual<D>& b) { return a.v op b.v; } \
    template <int D> inline bool operator op(const Dual<D>& a, double b) { return a.v op b; }         \
    template <int D> inline bool operator op(double a, const Dual<D>& b) { return a op b.v; }
GOSS_DUAL_CMP(<)
GOSS_DUAL_CMP(<=)
GOSS_DUAL_CMP(>)
GOSS_DUAL_CMP(>=)
GOSS_DUAL_CMP(==)
GOSS_DUAL_CMP(!=)
#undef GOSS_DUAL_CMP

inline double gexp(double x) { return exp(x); }
inline double gexp2(double x) { return std::exp2(x); }
inline double glog(double x) { return log(x); }
inline double gsqrt(double x) { return sqrt(x); }
inline double gfabs(double x) { return fabs(x); }
inline double gfloor(double x) { return floor(x); }
inline double gceil(double x) { return ceil(x); }
inline double gpow(double x, double y) { return pow(x, y); }
inline double gfmax(double x, double y) { return std::fmax(x, y); }
inline double gfmin(double x, double y) { return std::fmin(x, y); }
inline double gsin(double x) { return std::sin(x); }
inline double gcos(double x) { return std::cos(x); }
inline double gtan(double x) { return std::tan(x); }
inline double gtanh(double x) { return std::tanh(x); }

template <int D> inline Dual<D> gexp(const Dual<D>& a) { const double e = exp(a.v); return Dual<D>::chain(e, e, a); }
template <int D> inline Dual<D> gexp2(const Dual<D>& a)
{
    const double e = std::exp2(a.v);
    return Dual<D>::chain(e, e * 0.6931471805599453, a);  // d 2^x = 2^x ln 2 dx
}
template <int D> inline Dual<D> glog(const Dual<D>& a) { return Dual<D>::chain(log(a.v), 1.0 / a.v, a); }
template <int D> inline Dual<D> gsqrt(const Dual<D>& a)
{
    const double s = sqrt(a.v);
    return Dual<D>::chain(s, 0.5 / s, a);
}
template <int D> inline Dual<D> gfabs(const Dual<D>& a) { return Dual<D>::chain(fabs(a.v), a.v < 0 ? -1.0 : 1.0, a); }
template <int D> inline Dual<D> gfloor(const Dual<D>& a) { return Dual<D>(floor(a.v)); }
template <int D> inline Dual<D> gceil(const Dual<D>& a) { return Dual<D>(ceil(a.v)); }
template <int D> inline Dual<D> gsin(const Dual<D>& a) { return Dual<D>::chain(std::sin(a.v), std::cos(a.v), a); }
template <int D> inline Dual<D> gcos(const Dual<D>& a) { return Dual<D>::chain(std::cos(a.v), -std::sin(a.v), a); }
template <int D> inline Dual<D> gtan(const Dual<D>& a)
{
    const double t = std::tan(a.v);
    return Dual<D>::chain(t, 1.0 + t * t, a);
}
template <int D> inline Dual<D> gtanh(const Dual<D>& a)
{
    const double t = std::tanh(a.v);
    return Dual<D>::chain(t, 1.0 - t * t, a);
}
// d(x^y) = y x^(y-1) dx + x^y log(x) dy; the log term only when y varies
template <int D> inline Dual<D> gpow(const Dual<D>& x, const Dual<D>& y)
{
    const double p = pow(x.v, y.v);
    Dual<D> r(p);
    const double gx = y.v * pow(x.v, y.v - 1.0);
    const bool vary_y = y.has_tangent();
    const double gy = vary_y ? p * log(x.v) : 0.0;
    for (int k = 0; k < D; ++k) r.d[k] = gx * x.d[k] + (vary_y ? gy * y.d[k] : 0.0);
    return r;
}
template <int D> inline Dual<D> gpow(const Dual<D>& x, double y) { return gpow(x, Dual<D>(y)); }
template <int D> inline Dual<D> gpow(double x, const Dual<D>& y) { return gpow(Dual<D>(x), y); }
// fmax/fmin pick one argument; ties take the first (its derivative)
template <int D> inline Dual<D> gfmax(const Dual<D>& a, const Dual<D>& b) { return b.v > a.v ? b : a; }
template <int D> inline Dual<D> gfmin(const Dual<D>& a, const Dual<D>& b) { return b.v < a.v ? b : a; }

}}  // namespace goss_b200::models

#endif
