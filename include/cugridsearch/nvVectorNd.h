/*
 * nvVectorNd.h -- nv_ext::Vec<T, D>, the fixed-size vector that carries a grid point into
 * every cost functor (reference: include/nvVectorNd.h:114-340).  Only the part of the
 * interface the grid search and its callers use: construction from a scalar or an array,
 * indexing, size(), pointer conversion and element-wise arithmetic.
 */
#ifndef CUGRIDSEARCH_NVVECTORND_H
#define CUGRIDSEARCH_NVVECTORND_H

#ifndef CUDAFUNCTION
#define CUDAFUNCTION __host__ __device__
#endif

#include <cmath>

namespace nv_ext {

template <class T, unsigned int D>
class Vec {
public:
    typedef T value_type;

    CUDAFUNCTION int size() const { return (int)D; }

    // every element set to t (default: T())
    CUDAFUNCTION Vec(const T &t = T()) {
        for (unsigned int i = 0; i < D; i++) _array[i] = t;
    }

    // D elements read from tp
    CUDAFUNCTION Vec(const T *tp) {
        for (unsigned int i = 0; i < D; i++) _array[i] = tp[i];
    }

    CUDAFUNCTION T &operator[](int i) { return _array[i]; }
    CUDAFUNCTION const T &operator[](int i) const { return _array[i]; }

    CUDAFUNCTION operator T *() { return _array; }
    CUDAFUNCTION operator const T *() const { return _array; }

    CUDAFUNCTION Vec &operator+=(const Vec &r) {
        for (unsigned int i = 0; i < D; i++) _array[i] += r._array[i];
        return *this;
    }
    CUDAFUNCTION Vec &operator-=(const Vec &r) {
        for (unsigned int i = 0; i < D; i++) _array[i] -= r._array[i];
        return *this;
    }
    CUDAFUNCTION Vec &operator*=(T d) {
        for (unsigned int i = 0; i < D; i++) _array[i] *= d;
        return *this;
    }
    CUDAFUNCTION Vec &operator/=(T d) {
        for (unsigned int i = 0; i < D; i++) _array[i] /= d;
        return *this;
    }
    friend CUDAFUNCTION Vec operator+(Vec l, const Vec &r) { return l += r; }
    friend CUDAFUNCTION Vec operator-(Vec l, const Vec &r) { return l -= r; }
    friend CUDAFUNCTION Vec operator*(Vec l, T d) { return l *= d; }
    friend CUDAFUNCTION Vec operator/(Vec l, T d) { return l /= d; }
    friend CUDAFUNCTION Vec operator-(Vec v) {
        for (unsigned int i = 0; i < D; i++) v._array[i] = -v._array[i];
        return v;
    }
    friend CUDAFUNCTION T dot(const Vec &a, const Vec &b) {
        T s = T();
        for (unsigned int i = 0; i < D; i++) s += a._array[i] * b._array[i];
        return s;
    }
    friend CUDAFUNCTION T length(const Vec &a) { return sqrt(dot(a, a)); }

protected:
    T _array[D];
};

}  // namespace nv_ext

#endif  // CUGRIDSEARCH_NVVECTORND_H
