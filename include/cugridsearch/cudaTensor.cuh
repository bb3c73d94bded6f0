/*
 * cudaTensor.cuh -- drop-in CudaTensor / CudaMatrix / CudaImage / CudaVector for the B200
 * grid search (reference: include/cudaTensor.cuh:106-630).
 *
 * Same layout contract as the reference: a tensor is a view of caller-owned device memory
 * (the caller cudaMallocs data() of bytesSize() bytes), axis 0 varies fastest, and the
 * objects are passed to kernels by value.  CudaImage<T, C>(height, width) has dims
 * {C, W, H}: element (y, x, c) lives at c + C * (x + W * y) (HWC row-major).
 *
 * Differences from the reference, all at its undefined-behaviour edges:
 *   - valueAt_bilinear reads a tap whose flat index is past the end of the image as 0
 *     (the reference reads beyond the buffer when a sample lands in (H-1, H) on the last
 *     row, include/cudaTensor.cuh:561-566);
 *   - find_extrema runs the library's argmin (lowest value, lowest index on ties; NaN and
 *     +inf never win unless nothing else exists, in which case element 0 is returned, as
 *     the reference's strict '<' scan does) instead of an iota upload plus block reduction;
 *   - errors throw cgs_compat::Error (or exit under CGS_COMPAT_EXIT) instead of exiting.
 */
#ifndef CUGRIDSEARCH_CUDATENSOR_CUH
#define CUGRIDSEARCH_CUDATENSOR_CUH

#ifndef CUDAFUNCTION
#define CUDAFUNCTION __host__ __device__
#endif

#include <cuda_runtime.h>

#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <iostream>
#include <string>
#include <type_traits>
#include <vector>

#include "cgsCompat.cuh"
#include "nvVectorNd.h"

#ifndef OUTSIDE_IMAGE_VALUE
#define OUTSIDE_IMAGE_VALUE 0
#endif

// Per-channel behaviour of CudaImage::filter (include/cudaTensor.cuh:64-68).
enum CHANNEL_ACTION { FILTER, COPY, ZERO };

template <typename precision, unsigned int D>
struct CudaTensor;

namespace cgs_compat {

template <typename P>
__global__ void fill_kernel(P *data, uint32_t n, P value) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) data[i] = value;
}

// Argmin for element types other than float (the float case goes through cgs_argmin_f32):
// one block scans the array, each thread its indices in increasing order with a strict
// '<', then the block keeps the lower value, the lower index among equals.  NaN never
// beats a number; an array of NaN gives index 0.
template <typename P>
__device__ __forceinline__ bool argmin_better(P v, int32_t i, P w, int32_t j) {
    if (j < 0) return i >= 0;
    if (i < 0) return false;
    if (v < w) return true;
    if (w < v) return false;
    const bool vn = !(v == v), wn = !(w == w);
    if (vn != wn) return wn;  // a number beats NaN
    return i < j;
}

template <typename P>
__global__ void argmin_kernel(const P *data, uint32_t n, P *best_value, int32_t *best_index) {
    __shared__ P sv[1024];
    __shared__ int32_t si[1024];
    P v = P();
    int32_t k = -1;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
        if (argmin_better(data[i], (int32_t)i, v, k)) {
            v = data[i];
            k = (int32_t)i;
        }
    sv[threadIdx.x] = v;
    si[threadIdx.x] = k;
    __syncthreads();
    for (unsigned s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s && argmin_better(sv[threadIdx.x + s], si[threadIdx.x + s], sv[threadIdx.x], si[threadIdx.x])) {
            sv[threadIdx.x] = sv[threadIdx.x + s];
            si[threadIdx.x] = si[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *best_value = si[0] >= 0 ? sv[0] : P();
        *best_index = si[0] >= 0 ? si[0] : 0;
    }
}

// Strided host<->device copy: count elements of elem_size bytes, dst_stride / src_stride in
// elements (the reference's cudaMemcpyStrided, include/cudaTensor.cuh:88-104).
inline void memcpy_strided(void *dst, int dst_stride, const void *src, int src_stride, int count, int elem_size,
                           cudaMemcpyKind kind) {
    check_cuda(cudaMemcpy2D(dst, (size_t)dst_stride * elem_size, src, (size_t)src_stride * elem_size, elem_size,
                            count, kind),
               "cudaMemcpyStrided");
}

}  // namespace cgs_compat

template <typename precision, unsigned int D>
struct __align__(16) CudaTensor {
    precision *_data;
    int32_t _dims[D];
    int32_t _dimensional_increments[D];
    int32_t _total_size;

    CUDAFUNCTION CudaTensor() : _data(nullptr), _total_size(0) {
        for (unsigned int d = 0; d < D; d++) {
            _dims[d] = 0;
            _dimensional_increments[d] = 0;
        }
    }

    // dims[0] varies fastest; no memory is allocated (the caller cudaMallocs data()).
    template <typename T>
    CUDAFUNCTION CudaTensor(const T (&dims)[D]) : _data(nullptr) {
        _total_size = 1;
        int32_t inc = 1;
        for (unsigned int d = 0; d < D; d++) {
            _dims[d] = (int32_t)dims[d];
            _dimensional_increments[d] = inc;
            inc *= _dims[d];
            _total_size *= _dims[d];
        }
    }

    CUDAFUNCTION precision *&data() { return _data; }

    __device__ precision &operator[](int index) { return _data[index]; }

    // size() = number of elements; size(d) = extent of axis d
    CUDAFUNCTION uint32_t size(const int dim = -1) const {
        if (dim == -1) return (uint32_t)_total_size;
        return dim < (int)D ? (uint32_t)_dims[dim] : 0u;
    }

    uint32_t bytesSize() const { return size() * (uint32_t)sizeof(precision); }

    // Flat index of an axis index.  With float axis indices each step is the reference's
    // int += int * float (the product and sum in float, truncated back to int).
    template <typename T>
    CUDAFUNCTION int toIndex1d(const T (&axis_index)[D]) const {
        int e = axis_index[0];
        for (unsigned int a = 1; a < D; a++) e += _dimensional_increments[a] * axis_index[a];
        return e;
    }

    CUDAFUNCTION void toIndexNd(uint32_t index1d, uint32_t (&indexNd)[D]) const {
        for (int a = (int)D - 1; a >= 0; a--) {
            indexNd[a] = index1d / (uint32_t)_dimensional_increments[a];
            index1d -= indexNd[a] * (uint32_t)_dimensional_increments[a];
        }
    }

    CUDAFUNCTION precision &at(const uint32_t (&pt)[D]) const { return _data[toIndex1d(pt)]; }

    void fill(precision value) {
        unsigned blocks, threads;
        cgs_compat::launch_shape(size(), blocks, threads);
        cgs_compat::fill_kernel<precision><<<blocks, threads>>>(_data, size(), value);
        cgs_compat::check_launch("CudaTensor::fill");
    }

    void setValuesFromVector(const std::vector<precision> &vals) const {
        const size_t n = vals.size() < size() ? vals.size() : size();
        cgs_compat::check_cuda(cudaMemcpy(_data, vals.data(), n * sizeof(precision), cudaMemcpyHostToDevice),
                               "CudaTensor::setValuesFromVector");
    }

    std::vector<precision> toVector() const {
        std::vector<precision> out(size());
        cgs_compat::check_cuda(cudaMemcpy(out.data(), _data, bytesSize(), cudaMemcpyDeviceToHost), "CudaTensor::toVector");
        return out;
    }

    // Lowest value and its flat index (lowest index among equal values).
    void find_extrema(precision &extrema_value, int32_t &extrema_index1d) {
        if (size() == 0) cgs_compat::fail("CudaTensor::find_extrema: empty tensor", CGS_ERROR_INVALID_VALUE);
        if constexpr (std::is_same<precision, float>::value) {
            cgs_argmin *d_res = nullptr;
            cgs_compat::check_cuda(cudaMalloc(&d_res, sizeof(cgs_argmin)), "CudaTensor::find_extrema");
            cgs_argmin res{};
            const cgs_status st = cgs_argmin_f32(_data, size(), d_res, nullptr);
            cudaError_t e = cudaSuccess;
            if (st == CGS_SUCCESS) e = cudaMemcpy(&res, d_res, sizeof(res), cudaMemcpyDeviceToHost);
            cudaFree(d_res);
            cgs_compat::check(st, "CudaTensor::find_extrema");
            cgs_compat::check_cuda(e, "CudaTensor::find_extrema");
            if (res.valid) {
                extrema_value = res.cost;
                extrema_index1d = (int32_t)res.index;
            } else {  // nothing finite: the reference's scan keeps element 0
                cgs_compat::check_cuda(cudaMemcpy(&extrema_value, _data, sizeof(float), cudaMemcpyDeviceToHost),
                                       "CudaTensor::find_extrema");
                extrema_index1d = 0;
            }
        } else {
            precision *d_v = nullptr;
            int32_t *d_i = nullptr;
            cgs_compat::check_cuda(cudaMalloc(&d_v, sizeof(precision)), "CudaTensor::find_extrema");
            cgs_compat::check_cuda(cudaMalloc(&d_i, sizeof(int32_t)), "CudaTensor::find_extrema");
            cgs_compat::argmin_kernel<precision><<<1, 1024>>>(_data, size(), d_v, d_i);
            cudaError_t e = cudaPeekAtLastError();
            if (e == cudaSuccess) e = cudaMemcpy(&extrema_value, d_v, sizeof(precision), cudaMemcpyDeviceToHost);
            if (e == cudaSuccess) e = cudaMemcpy(&extrema_index1d, d_i, sizeof(int32_t), cudaMemcpyDeviceToHost);
            cudaFree(d_v);
            cudaFree(d_i);
            cgs_compat::check_cuda(e, "CudaTensor::find_extrema");
        }
#ifdef CGS_COMPAT_VERBOSE
        printf("\n Grid MIN value has idx: %d  value: %f\n", extrema_index1d, (double)extrema_value);
#endif
    }

    void display(const std::string &name = "") const {
        const std::vector<precision> v = toVector();
        std::cout << name << " = [";
        for (size_t i = 0; i < v.size(); i++) std::cout << (i ? ", " : "") << v[i];
        std::cout << "]" << std::endl;
    }
};

template <typename precision>
struct CudaMatrix : public CudaTensor<precision, 2> {
    CUDAFUNCTION CudaMatrix(uint32_t rows, uint32_t columns) : CudaTensor<precision, 2>({columns, rows}) {}

    CUDAFUNCTION int32_t width() const { return (int32_t)this->size(0); }
    CUDAFUNCTION int32_t height() const { return (int32_t)this->size(1); }

    template <typename T>
    CUDAFUNCTION int toIndex(T y, T x) const {
        return CudaTensor<precision, 2>::toIndex1d({x, y});
    }

    template <typename T>
    CUDAFUNCTION precision &at(T row_index, T column_index) const {
        return this->_data[toIndex(row_index, column_index)];
    }

    void display(const std::string &name = "") const {
        const std::vector<precision> v = this->toVector();
        std::cout << name << " = [" << std::endl;
        for (int r = 0; r < height(); r++) {
            for (int c = 0; c < width(); c++) std::cout << (c ? ", " : "  ") << v[(size_t)r * width() + c];
            std::cout << (r + 1 < height() ? ";" : "") << std::endl;
        }
        std::cout << "]" << std::endl;
    }

    void setDiagonal(const precision value) {
        std::vector<precision> values(height(), value);
        cgs_compat::memcpy_strided(this->data(), width() + 1, values.data(), 1, height(), sizeof(precision),
                                   cudaMemcpyHostToDevice);
    }

    void setColumnFromVector(int column_index, const std::vector<precision> &values) {
        assert(column_index < width() && (int)values.size() == height());
        cgs_compat::memcpy_strided(this->data() + column_index, width(), values.data(), 1, height(),
                                   sizeof(precision), cudaMemcpyHostToDevice);
    }

    void setRowFromVector(int row_index, const std::vector<precision> &values) {
        assert(row_index < height() && (int)values.size() == width());
        cgs_compat::check_cuda(cudaMemcpy(this->data() + (size_t)row_index * width(), values.data(),
                                          (size_t)width() * sizeof(precision), cudaMemcpyHostToDevice),
                               "CudaMatrix::setRowFromVector");
    }

    void setIdentity() {
        std::vector<precision> values(this->size(), precision(0));
        for (int i = 0; i < width() && i < height(); i++) values[(size_t)i * width() + i] = precision(1);
        this->setValuesFromVector(values);
    }
};

template <typename precision, uint32_t CHANNELS = 1>
struct CudaImage : public CudaTensor<precision, 3> {
    CUDAFUNCTION CudaImage(uint32_t _height, uint32_t _width) : CudaTensor<precision, 3>({CHANNELS, _width, _height}) {}

    CUDAFUNCTION int32_t channels() const { return (int32_t)this->size(0); }
    CUDAFUNCTION int32_t width() const { return (int32_t)this->size(1); }
    CUDAFUNCTION int32_t height() const { return (int32_t)this->size(2); }

    template <typename T>
    CUDAFUNCTION int toIndex(T y, T x, T c = 0) const {
        return CudaTensor<precision, 3>::toIndex1d({c, x, y});
    }

    template <typename T>
    CUDAFUNCTION precision &at(T row_index, T column_index, T channel_index = 0) const {
        return this->_data[toIndex(row_index, column_index, channel_index)];
    }

    // float coordinates against the integer extent (include/cudaTensor.cuh:548-550)
    CUDAFUNCTION bool inImage(float y, float x) const {
        return x >= 0 && y >= 0 && x < this->width() && y < this->height();
    }

    CUDAFUNCTION float valueAt(float y, float x, float c = 0) const { return valueAt_bilinear(y, x, c); }

    CUDAFUNCTION precision valueAt_nearest_neighbor(float y, float x, float c = 0) const {
        return inImage(y, x) ? this->_data[toIndex(y, x, c)] : (precision)OUTSIDE_IMAGE_VALUE;
    }

    // Bilinear sample with the reference's taps (floor / ceil of each coordinate, so a
    // sample in (W-1, W) reads column 0 of the next row through the flat index) and its
    // interpolation order: (1-a)p + aq along x on both rows, then along y.
    CUDAFUNCTION float valueAt_bilinear(float y, float x, float c = 0) const {
        if (!inImage(y, x)) return (float)OUTSIDE_IMAGE_VALUE;
        const float y0 = floor(y), x0 = floor(x), y1 = ceil(y), x1 = ceil(x);
        const float tlc = tap(toIndex(y0, x0, c));
        const float trc = tap(toIndex(y0, x1, c));
        const float blc = tap(toIndex(y1, x0, c));
        const float brc = tap(toIndex(y1, x1, c));
        const float ax = x - x0;
        const float ay = y - y0;
        const float top = (1.0f - ax) * tlc + ax * trc;
        const float bottom = (1.0f - ax) * blc + ax * brc;
        return (1.0f - ay) * top + ay * bottom;
    }

private:
    CUDAFUNCTION float tap(int flat) const {
        return (flat >= 0 && flat < this->_total_size) ? (float)this->_data[flat] : 0.0f;
    }
};

template <typename precision>
struct CudaVector : public CudaMatrix<precision> {
    CUDAFUNCTION CudaVector(uint32_t _dim) : CudaMatrix<precision>(_dim, 1) {}

    template <typename T>
    CUDAFUNCTION int toIndex(T row_index) const {
        return (int)row_index;
    }

    CUDAFUNCTION precision &at(int row_index) const { return this->_data[row_index]; }
};

#endif  // CUGRIDSEARCH_CUDATENSOR_CUH
