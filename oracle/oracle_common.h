/* TEST INFRASTRUCTURE ONLY -- the CPU oracle for the sysmat generator.
 * Nothing in the product includes, links or calls this code; tests/, the
 * smoke check and bench.py's CPU baseline use it as the checker.
 *
 * Number types the oracle is instantiated with:
 *   float   the reference's arithmetic replicated operation by operation
 *           (IEEE single, no fused multiply-add, double where the reference
 *           promotes), so its results equal the reference code's bit for bit;
 *   double  the same algorithm in IEEE double (the reference source with
 *           `float` read as `double`);
 *   Dual    every value is carried in both precisions; every comparison, and
 *           therefore every hit/miss decision, is taken on the single-precision
 *           half exactly as the reference kernel takes it, while the reported
 *           magnitudes come from the double half.  This separates arithmetic
 *           error from decision flips at box and hole edges.
 */
#ifndef SYSMAT_ORACLE_COMMON_H
#define SYSMAT_ORACLE_COMMON_H

#include <cmath>
#include <cstdint>

namespace oracle {

struct Dual {
    float f;
    double d;
    Dual() : f(0.0f), d(0.0) {}
    Dual(float v) : f(v), d((double)v) {}                 /* constants: the float literal, widened */
    Dual(float vf, double vd) : f(vf), d(vd) {}
    static Dual from_int(long long v) { return Dual((float)v, (double)v); }
};

inline Dual operator+(Dual a, Dual b) { return Dual(a.f + b.f, a.d + b.d); }
inline Dual operator-(Dual a, Dual b) { return Dual(a.f - b.f, a.d - b.d); }
inline Dual operator*(Dual a, Dual b) { return Dual(a.f * b.f, a.d * b.d); }
inline Dual operator/(Dual a, Dual b) { return Dual(a.f / b.f, a.d / b.d); }
inline Dual operator-(Dual a) { return Dual(-a.f, -a.d); }
inline Dual& operator+=(Dual& a, Dual b) { a = a + b; return a; }
inline Dual& operator*=(Dual& a, Dual b) { a = a * b; return a; }
inline bool operator<(Dual a, Dual b) { return a.f < b.f; }
inline bool operator<=(Dual a, Dual b) { return a.f <= b.f; }
inline bool operator>(Dual a, Dual b) { return a.f > b.f; }
inline bool operator>=(Dual a, Dual b) { return a.f >= b.f; }

/* Elementary functions: float uses the single-precision libm entry points
 * (as the reference's float overloads do), double the double ones. */
inline float  m_sqrt(float x) { return std::sqrt(x); }
inline double m_sqrt(double x) { return std::sqrt(x); }
inline Dual   m_sqrt(Dual x) { return Dual(std::sqrt(x.f), std::sqrt(x.d > 0.0 ? x.d : 0.0)); }
inline float  m_exp(float x) { return std::exp(x); }
inline double m_exp(double x) { return std::exp(x); }
inline Dual   m_exp(Dual x) { return Dual(std::exp(x.f), std::exp(x.d)); }
inline float  m_fabs(float x) { return std::fabs(x); }
inline double m_fabs(double x) { return std::fabs(x); }
inline Dual   m_fabs(Dual x) { return Dual(std::fabs(x.f), std::fabs(x.d)); }
inline float  m_cos(float x) { return std::cos(x); }
inline double m_cos(double x) { return std::cos(x); }
inline Dual   m_cos(Dual x) { return Dual(std::cos(x.f), std::cos(x.d)); }
inline float  m_sin(float x) { return std::sin(x); }
inline double m_sin(double x) { return std::sin(x); }
inline Dual   m_sin(Dual x) { return Dual(std::sin(x.f), std::sin(x.d)); }
inline float  m_acos(float x) { return std::acos(x); }
inline double m_acos(double x) { return std::acos(x); }
inline Dual   m_acos(Dual x) { return Dual(std::acos(x.f), std::acos(x.d > 1.0 ? 1.0 : (x.d < -1.0 ? -1.0 : x.d))); }
inline float  m_asin(float x) { return std::asin(x); }
inline double m_asin(double x) { return std::asin(x); }
inline Dual   m_asin(Dual x) { return Dual(std::asin(x.f), std::asin(x.d > 1.0 ? 1.0 : x.d)); }
inline float  m_erf(float x) { return std::erf(x); }
inline double m_erf(double x) { return std::erf(x); }
inline Dual   m_erf(Dual x) { return Dual(std::erf(x.f), std::erf(x.d)); }
inline float  m_floor(float x) { return std::floor(x); }

/* The magnitude a result contributes to a sum of doubles. */
inline double mag(float x) { return (double)x; }
inline double mag(double x) { return x; }
inline double mag(Dual x) { return x.d; }

/* Reference's max/min macros ((a>=b)?a:b) / ((a<=b)?a:b). */
template <class N> inline N ref_max(N a, N b) { return (a >= b) ? a : b; }
template <class N> inline N ref_min(N a, N b) { return (a <= b) ? a : b; }

/* A value of type N read from a float32 table. */
template <class N> inline N tab(const float* t, long long i) { return N(t[i]); }

/* An integer (loop index) converted the way the reference converts it to
 * float: the conversion always happens in single precision first in the
 * reference source ((float)NumX, (float)(NumX + 0.5f)). */
template <class N> inline N from_float(float v) { return N(v); }

/* Expression `A / (4 * M_PI * dsq) * P / S` with A, dsq, P, S of the
 * reference's float type, evaluated in double as C++ promotes it
 * (PESysMatGen.cu:624-636), then stored into the float result. */
inline float solid_face(float a, float dsq, float p, float s) {
    return (float)((double)a / (4 * M_PI * (double)dsq) * (double)p / (double)s);
}
inline double solid_face(double a, double dsq, double p, double s) {
    return a / (4 * M_PI * dsq) * p / s;
}
inline Dual solid_face(Dual a, Dual dsq, Dual p, Dual s) {
    return Dual(solid_face(a.f, dsq.f, p.f, s.f), solid_face(a.d, dsq.d, p.d, s.d));
}

}  /* namespace oracle */

#endif
