// Minimal stand-in for the parts of Armadillo's Mat<T> that the C++ adapter
// (include/stpgpu_stp.hpp) and its test use: column-major storage,
// memptr(), n_rows, n_cols, n_elem, set_size(), reset(), element access.
// Armadillo itself is not installed here; this is test scaffolding only.
#pragma once

#include <complex>
#include <cstddef>
#include <vector>

namespace arma {

using uword = std::size_t;

template <typename T>
class Mat {
public:
    Mat() = default;
    Mat(uword r, uword c) { set_size(r, c); }
    void set_size(uword r, uword c)
    {
        n_rows = r;
        n_cols = c;
        n_elem = r * c;
        data_.assign(n_elem, T());
    }
    void reset() { set_size(0, 0); }
    T* memptr() { return data_.empty() ? nullptr : data_.data(); }
    const T* memptr() const { return data_.empty() ? nullptr : data_.data(); }
    T& operator()(uword r, uword c) { return data_[c * n_rows + r]; }
    const T& operator()(uword r, uword c) const { return data_[c * n_rows + r]; }
    T& operator[](uword i) { return data_[i]; }
    bool is_empty() const { return n_elem == 0; }

    uword n_rows = 0;
    uword n_cols = 0;
    uword n_elem = 0;

private:
    std::vector<T> data_;
};

template <typename T>
class Col : public Mat<T> {
};

using mat = Mat<double>;
using cx_mat = Mat<std::complex<double>>;
using uvec = Col<uword>;
using ivec = Col<long long>;

} // namespace arma
