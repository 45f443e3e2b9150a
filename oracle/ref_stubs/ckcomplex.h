// Minimal stand-in for Charm++'s ckcomplex.h so the reference's PINY physics
// files compile for the oracle (oracle/_ref).  Project-written: a double
// complex with the member names and operators those files use.
#ifndef OA_REF_STUB_CKCOMPLEX_H
#define OA_REF_STUB_CKCOMPLEX_H
#include <cmath>
struct complex {
  double re, im;
  complex() : re(0.0), im(0.0) {}
  complex(double r) : re(r), im(0.0) {}
  complex(double r, double i) : re(r), im(i) {}
  double getMagSqr() const { return re * re + im * im; }
  complex conj() const { return complex(re, -im); }
  complex operator+(const complex& a) const { return complex(re + a.re, im + a.im); }
  complex operator-(const complex& a) const { return complex(re - a.re, im - a.im); }
  complex operator-() const { return complex(-re, -im); }
  complex operator*(const complex& a) const { return complex(re * a.re - im * a.im, re * a.im + im * a.re); }
  complex operator*(double s) const { return complex(re * s, im * s); }
  complex operator/(double s) const { return complex(re / s, im / s); }
  complex& operator+=(const complex& a) { re += a.re; im += a.im; return *this; }
  complex& operator-=(const complex& a) { re -= a.re; im -= a.im; return *this; }
  complex& operator*=(const complex& a) { double r = re * a.re - im * a.im; im = re * a.im + im * a.re; re = r; return *this; }
  complex& operator*=(double s) { re *= s; im *= s; return *this; }
  complex& operator=(double s) { re = s; im = 0.0; return *this; }
};
inline complex operator*(double s, const complex& a) { return complex(a.re * s, a.im * s); }
typedef complex ckcomplex;
#endif
