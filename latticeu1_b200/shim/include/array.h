// Array<T> of the reference's API (reference include/array.h:19-181).
// Host arrays are plain buffers.  A Device Array<double> of
// Volume()*Dirs() elements is the gauge field: it owns a C ABI lattice
// (u1_lattice, float2 links) created cold with the current
// SetupLatticeParameters geometry; getPtr() is not available for it, use
// Copy-in/out through importAngles/exportAngles (reference angle layout).
#ifndef U1_SHIM_ARRAY_H
#define U1_SHIM_ARRAY_H
#include <cstddef>
#include <cstring>
#include <iostream>
#include <stdexcept>
#include <vector>

#include "complex.h"
#include "enum.h"
#include "parameters.h"

struct u1_lattice;

namespace U1 {

u1_lattice *shim_new_lattice();
void shim_free_lattice(u1_lattice *lat);
void shim_lattice_import(u1_lattice *lat, const double *host_angles);
void shim_lattice_export(u1_lattice *lat, double *host_angles);

template <class Real>
class Array {
 public:
  Array() : location_(Host) {}
  explicit Array(ReadMode location) : location_(location) {}
  Array(ReadMode location, size_t size) : location_(location), size_(size) {
    if (location_ == Host) {
      host_.assign(size_, Real());
    } else {
      bind_device();
    }
  }
  ~Array() {
    if (lattice_) shim_free_lattice(lattice_);
  }
  Array(const Array &) = delete;
  Array &operator=(const Array &) = delete;

  Real *getPtr() {
    if (location_ == Device) throw std::runtime_error("Array<Device>::getPtr: the gauge field lives in the C ABI lattice");
    return host_.data();
  }
  size_t Size() const { return size_; }
  ReadMode Location() const { return location_; }
  Real &operator()(int i) { return host_[i]; }
  Real &operator[](int i) { return host_[i]; }
  Real &at(int i) { return host_.at(i); }
  Real at(int i) const { return host_.at(i); }
  void Clear() {
    if (location_ == Host) std::fill(host_.begin(), host_.end(), Real());
    else if (lattice_) {
      std::vector<double> zero(size_, 0.0);
      shim_lattice_import(lattice_, zero.data());
    }
  }
  // Copy contents of another array (host<->host, device gauge field <-> device gauge field,
  // host angles -> device gauge field and back), as the reference's Array::Copy.
  void Copy(Array *in);
  void Backup() { backup_ = snapshot(); }
  void Restore() { restore(backup_); }
  u1_lattice *lattice() const { return lattice_; }

  friend std::ostream &operator<<(std::ostream &out, Array<Real> *M) {
    for (size_t i = 0; i < M->size_; ++i) out << i << '\t' << M->host_[i] << std::endl;
    return out;
  }

 private:
  ReadMode location_;
  size_t size_ = 0;
  std::vector<Real> host_;
  std::vector<Real> backup_;
  u1_lattice *lattice_ = nullptr;

  void bind_device();
  std::vector<Real> snapshot();
  void restore(const std::vector<Real> &v);
};

template <class Real>
inline void Array<Real>::bind_device() {
  throw std::runtime_error("Array<Device>: only the Array<double> gauge field lives on the device");
}
template <>
inline void Array<double>::bind_device() {
  if (size_ != (size_t)Volume() * Dirs())
    throw std::runtime_error("Array<double>(Device, n): n must be Volume()*Dirs() (the gauge field)");
  lattice_ = shim_new_lattice();
}

template <class Real>
inline std::vector<Real> Array<Real>::snapshot() {
  return host_;
}
template <>
inline std::vector<double> Array<double>::snapshot() {
  if (location_ == Host) return host_;
  std::vector<double> v(size_);
  shim_lattice_export(lattice_, v.data());
  return v;
}
template <class Real>
inline void Array<Real>::restore(const std::vector<Real> &v) {
  host_ = v;
}
template <>
inline void Array<double>::restore(const std::vector<double> &v) {
  if (location_ == Host) host_ = v;
  else shim_lattice_import(lattice_, v.data());
}

template <class Real>
inline void Array<Real>::Copy(Array *in) {
  size_ = in->size_;
  host_ = in->host_;
}
template <>
inline void Array<double>::Copy(Array *in) {
  std::vector<double> v = in->snapshot();
  if (location_ == Device) {
    if (!lattice_) {
      size_ = v.size();
      bind_device();
    }
    shim_lattice_import(lattice_, v.data());
  } else {
    size_ = v.size();
    host_ = v;
  }
}

}  // namespace U1
#endif
