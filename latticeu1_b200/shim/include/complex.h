// complexd / complexs for the drop-in API: the subset of the reference's
// _complex<Real> (reference include/complex.h:76-505) that driver code uses:
// arithmetic, real()/imag() as lvalues, abs(), abs2(), conj, and '<<'
// printing "re<TAB>im" (reference include/complex.h:367-371).
#ifndef U1_SHIM_COMPLEX_H
#define U1_SHIM_COMPLEX_H
#include <cmath>
#include <ostream>

template <class Real>
class _complex {
  Real re_, im_;

 public:
  _complex(Real r = Real(0), Real i = Real(0)) : re_(r), im_(i) {}
  Real &real() { return re_; }
  Real real() const { return re_; }
  Real &imag() { return im_; }
  Real imag() const { return im_; }
  Real abs() const { return std::sqrt(re_ * re_ + im_ * im_); }
  Real abs2() const { return re_ * re_ + im_ * im_; }
  Real arg() const { return std::atan2(im_, re_); }
  _complex operator+(const _complex &b) const { return _complex(re_ + b.re_, im_ + b.im_); }
  _complex operator-(const _complex &b) const { return _complex(re_ - b.re_, im_ - b.im_); }
  _complex operator-() const { return _complex(-re_, -im_); }
  _complex operator*(const _complex &b) const { return _complex(re_ * b.re_ - im_ * b.im_, re_ * b.im_ + im_ * b.re_); }
  _complex operator/(const _complex &b) const {
    const Real d = b.abs2();
    return _complex((re_ * b.re_ + im_ * b.im_) / d, (im_ * b.re_ - re_ * b.im_) / d);
  }
  _complex operator+(Real b) const { return _complex(re_ + b, im_); }
  _complex operator-(Real b) const { return _complex(re_ - b, im_); }
  _complex operator*(Real b) const { return _complex(re_ * b, im_ * b); }
  _complex operator/(Real b) const { return _complex(re_ / b, im_ / b); }
  _complex &operator+=(const _complex &b) { re_ += b.re_; im_ += b.im_; return *this; }
  _complex &operator-=(const _complex &b) { re_ -= b.re_; im_ -= b.im_; return *this; }
  _complex &operator*=(const _complex &b) { return *this = *this * b; }
  _complex &operator/=(const _complex &b) { return *this = *this / b; }
  _complex &operator+=(Real b) { re_ += b; return *this; }
  _complex &operator-=(Real b) { re_ -= b; return *this; }
  _complex &operator*=(Real b) { re_ *= b; im_ *= b; return *this; }
  _complex &operator/=(Real b) { re_ /= b; im_ /= b; return *this; }
  bool operator==(const _complex &b) const { return re_ == b.re_ && im_ == b.im_; }
  bool operator!=(const _complex &b) const { return !(*this == b); }
  friend _complex operator+(Real a, const _complex &z) { return _complex(a + z.re_, z.im_); }
  friend _complex operator-(Real a, const _complex &z) { return _complex(a - z.re_, -z.im_); }
  friend _complex operator*(Real a, const _complex &z) { return _complex(a * z.re_, a * z.im_); }
  friend _complex operator/(Real a, const _complex &z) { return _complex(a, Real(0)) / z; }
  friend _complex conj(const _complex &z) { return _complex(z.re_, -z.im_); }
  friend Real abs(const _complex &z) { return z.abs(); }
  friend Real abs2(const _complex &z) { return z.abs2(); }
  friend std::ostream &operator<<(std::ostream &out, _complex z) { return out << z.re_ << '\t' << z.im_; }
};

typedef _complex<float> complexs;
typedef _complex<double> complexd;

inline complexd make_complexd(double a, double b) { return complexd(a, b); }
inline complexs make_complexs(float a, float b) { return complexs(a, b); }

#endif
