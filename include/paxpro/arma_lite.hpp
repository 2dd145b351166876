// arma_lite.hpp -- the subset of Armadillo's column-major containers that the
// PaxPro solver API exposes (arma::cx_vec, cx_mat, cx_cube, vec, mat).
//
// The reference's Solver getters return Armadillo objects
// (include/solver.hpp:33-45).  Armadillo is not a dependency of this build, so
// this header provides containers with the same names, memory layout
// (column-major, contiguous) and the members user code of the solver API
// touches: n_rows, n_cols, n_slices, n_elem, memptr(), element access,
// set_size, zeros, fill.  Define PAXPRO_B200_USE_ARMADILLO to use the real
// library instead.
#pragma once
#ifdef PAXPRO_B200_USE_ARMADILLO
#include <armadillo>
#else
#include <complex>
#include <cstddef>
#include <stdexcept>
#include <vector>

namespace arma {

typedef std::size_t uword;

template <typename T> class Cube;

template <typename T> class Mat {
 public:
  uword n_rows = 0, n_cols = 0, n_elem = 0;
  Mat() = default;
  Mat(uword r, uword c) { set_size(r, c); }
  Mat(uword r, uword c, const T &v) { set_size(r, c); fill(v); }
  void set_size(uword r, uword c) {
    n_rows = r;
    n_cols = c;
    n_elem = r * c;
    data_.assign(n_elem, T());
  }
  void zeros() { fill(T()); }
  void zeros(uword r, uword c) { set_size(r, c); }
  void fill(const T &v) { data_.assign(n_elem, v); }
  T *memptr() { return data_.data(); }
  const T *memptr() const { return data_.data(); }
  T &operator()(uword i, uword j) { return data_[j * n_rows + i]; }
  const T &operator()(uword i, uword j) const { return data_[j * n_rows + i]; }
  T &operator()(uword i) { return data_[i]; }
  const T &operator()(uword i) const { return data_[i]; }
  T &operator[](uword i) { return data_[i]; }
  const T &operator[](uword i) const { return data_[i]; }
  bool is_square() const { return n_rows == n_cols; }

 protected:
  std::vector<T> data_;
};

template <typename T> class Col : public Mat<T> {
 public:
  Col() = default;
  explicit Col(uword n) { this->set_size(n, 1); }
  Col(uword n, const T &v) { this->set_size(n, 1); this->fill(v); }
  void set_size(uword n) { Mat<T>::set_size(n, 1); }
  void set_size(uword r, uword c) { Mat<T>::set_size(r, c); }
};

template <typename T> class Cube {
 public:
  uword n_rows = 0, n_cols = 0, n_slices = 0, n_elem = 0;
  Cube() = default;
  Cube(uword r, uword c, uword s) { set_size(r, c, s); }
  void set_size(uword r, uword c, uword s) {
    n_rows = r;
    n_cols = c;
    n_slices = s;
    n_elem = r * c * s;
    data_.assign(n_elem, T());
  }
  T *memptr() { return data_.data(); }
  const T *memptr() const { return data_.data(); }
  T *slice_memptr(uword s) { return data_.data() + s * n_rows * n_cols; }
  T &operator()(uword i, uword j, uword k) { return data_[(k * n_cols + j) * n_rows + i]; }
  const T &operator()(uword i, uword j, uword k) const {
    return data_[(k * n_cols + j) * n_rows + i];
  }

 private:
  std::vector<T> data_;
};

typedef Col<std::complex<double>> cx_vec;
typedef Mat<std::complex<double>> cx_mat;
typedef Cube<std::complex<double>> cx_cube;
typedef Col<double> vec;
typedef Mat<double> mat;

}  // namespace arma
#endif
