/*
 * cudaGridSearch.cuh -- drop-in CudaGrid / CudaGridSearcher for the B200 grid search
 * (reference: src/gpu/cudaGridSearch.cuh:74-853).
 *
 * Source compatibility: code written against the reference's templates compiles against
 * these headers unchanged -- the grid is a 4 x D matrix {start, end, resolution, count} in
 * caller-allocated device memory (cudaMalloc(&grid.data(), grid.bytesSize())), the result
 * is a caller-allocated CudaTensor<float, D> (axis 0 fastest), and a cost functor is passed
 * as a device function pointer fetched with cudaMemcpyFromSymbol from a __device__
 * variable.  Every searcher call blocks until the work is done, as the reference's do.
 *
 * What runs.  The searcher compares the functor pointer with the device addresses of the
 * library's known functors instantiated for the same types (a table built once per
 * instantiation and device by a small kernel in the caller's own module, where the caller's
 * __device__ pointer was initialised, so the addresses are comparable):
 *   - a functor the library has a fused kernel for (the reference functors of
 *     cudaErrorFunctions.cuh / cudaErrorFunction_mi.cuh, calcZNCC, calcMI, calcMIBins) runs
 *     through cgs_search: one persistent sm_100a launch evaluates every grid point, writes
 *     the cost tensor and reduces the argmin (available from last_argmin());
 *   - the block-cooperative functors (cudaErrorFunctionsStreams.cuh,
 *     cudaErrorFunction_miStreams.cuh), and known functors for pixel types or channel
 *     counts the library has no kernel for, run their own body in a kernel that calls it
 *     directly, one thread per grid point;
 *   - any other pointer (a caller's own functor) runs in a kernel that calls it through
 *     the pointer, one thread per grid point -- the reference's execution model, with the
 *     bound check fixed (the reference writes result[n], cudaGridSearch.cuh:295).
 * Nothing runs on the CPU.
 *
 * search_by_value_stream and search_by_value_block keep their signatures; their launch
 * geometry arguments (stream count, cores, threads per block) do not apply to the
 * kernels above and are ignored.
 */
#ifndef CUGRIDSEARCH_CUDAGRIDSEARCH_CUH
#define CUGRIDSEARCH_CUDAGRIDSEARCH_CUH

#ifndef CUDAFUNCTION
#define CUDAFUNCTION __host__ __device__
#endif

#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <iostream>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "cgsCompat.cuh"
#include "cudaErrorFunction_mi.cuh"
#include "cudaErrorFunction_miStreams.cuh"
#include "cudaErrorFunctions.cuh"
#include "cudaErrorFunctionsStreams.cuh"
#include "cudaImageFunctions.cuh"
#include "cudaTensor.cuh"
#include "nvVectorNd.h"

#define ROW_IDX_START 0
#define ROW_IDX_END 1
#define ROW_IDX_RESOLUTION 2
#define ROW_IDX_SAMPLE_COUNT 3
#ifndef BLOCK_DIM
#define BLOCK_DIM 512
#endif
#ifndef MAX_THREADS_PER_BLOCK
#define MAX_THREADS_PER_BLOCK 1024
#endif

template <typename precision, unsigned int D>
struct CudaGrid;

namespace cgs_compat {

template <typename precision, unsigned int D>
__global__ void grid_point_kernel(CudaGrid<precision, D> grid, int index, precision *out);

// updateProcess (cudaGridSearch.cuh:235-272) for grids the C ABI does not describe
// (precision other than float, or more than 8 axes); float grids with D <= 8 use
// cgs_grid_update.  A step below 1e-7 * count collapses the axis to one sample; an
// explicitly changed axis truncates its extent to an integer.
template <typename precision>
inline void grid_update_generic(precision *start, precision *end, precision *res, precision *count, int D,
                                int changed_axis) {
    auto one = [&](int a, bool changed) {
        if (std::abs(end[a] - start[a]) < 1.0e-7 * count[a]) count[a] = 1;
        if (count[a] == 1)
            res[a] = 2 * (end[a] - start[a]);
        else if (changed)
            res[a] = (int)(end[a] - start[a]) / (count[a] - 1);
        else
            res[a] = (end[a] - start[a]) / (count[a] - 1);
    };
    if (changed_axis >= 0 && changed_axis < D)
        one(changed_axis, true);
    else
        for (int a = 0; a < D; a++) one(a, false);
}

}  // namespace cgs_compat

template <typename precision, unsigned int D>
struct CudaGrid : private CudaMatrix<precision> {
    CudaGrid() : CudaMatrix<precision>(4, D) {}

    void getAxisSampleCounts(precision *axis_sample_counts) {
        cgs_compat::check_cuda(
            cudaMemcpy(axis_sample_counts, axis_sample_count(), D * sizeof(precision), cudaMemcpyDeviceToHost),
            "CudaGrid::getAxisSampleCounts");
    }

    // Product of the axis counts, accumulated as the reference does (int32 * count, truncated).
    uint32_t numElements() {
        precision counts[D];
        getAxisSampleCounts(counts);
        int32_t total = 1;
        for (unsigned int a = 0; a < D; a++) total = total * counts[a];
        return (uint32_t)total;
    }

    // Recomputes resolution (and collapsed counts) from start, end and count.
    void update(int changed_axis = -1) {
        std::vector<precision> m = hostMatrix();
        precision *start = m.data() + ROW_IDX_START * D, *end = m.data() + ROW_IDX_END * D;
        precision *res = m.data() + ROW_IDX_RESOLUTION * D, *count = m.data() + ROW_IDX_SAMPLE_COUNT * D;
        if constexpr (std::is_same<precision, float>::value && D <= 8) {
            cgs_grid g = toCgsGrid(m);
            cgs_compat::check(cgs_grid_update(&g, changed_axis), "CudaGrid::update");
            for (unsigned int a = 0; a < D; a++) {
                res[a] = g.resolution[a];
                count[a] = g.count[a];
            }
        } else {
            cgs_compat::grid_update_generic<precision>(start, end, res, count, (int)D, changed_axis);
        }
        this->setValuesFromVector(m);
    }

    precision *&data() { return this->CudaMatrix<precision>::data(); }
    uint32_t bytesSize() const { return this->CudaMatrix<precision>::bytesSize(); }

    CUDAFUNCTION precision *start_point(int axis_index = 0) { return this->_data + ROW_IDX_START * D + axis_index; }
    CUDAFUNCTION precision *end_point(int axis_index = 0) { return this->_data + ROW_IDX_END * D + axis_index; }
    CUDAFUNCTION precision *axis_sample_count(int axis_index = 0) {
        return this->_data + ROW_IDX_SAMPLE_COUNT * D + axis_index;
    }
    CUDAFUNCTION precision *resolution(int axis_index = 0) { return this->_data + ROW_IDX_RESOLUTION * D + axis_index; }

    // Nearest grid index of a point (cudaGridSearch.cuh:125-148, including its rounding of
    // the offset before the division by the resolution).
    template <typename T>
    __device__ uint32_t gridPointToIndex(T *grid_point) {
        int32_t inc = 1;
        int code = 0;
        for (unsigned int a = 0; a < D; a++) {
            const int32_t idx = round(grid_point[a] - start_point()[a]) / resolution()[a];
            code += inc * idx;
            inc *= axis_sample_count()[a];
        }
        return code;
    }

    // Grid point of a flat index (axis 0 fastest): integer decode with the reference's
    // float-product increments, then start + i * resolution as one fused multiply-add,
    // the rounding the reference's device code gets (cudaGridSearch.cuh:160-187).
    template <typename T>
    __device__ void indexToGridPoint(T index, precision *device_grid_point) {
        int32_t inc[D];
        inc[0] = 1;
        for (unsigned int a = 1; a < D; a++) inc[a] = axis_sample_count()[a - 1] * inc[a - 1];
        int32_t rem = (int32_t)index;
        for (int a = (int)D - 1; a >= 0; a--) {
            const int32_t i = rem / inc[a];
            rem -= i * inc[a];
            if constexpr (std::is_same<precision, float>::value)
                device_grid_point[a] = fmaf((float)i, resolution()[a], start_point()[a]);
            else if constexpr (std::is_same<precision, double>::value)
                device_grid_point[a] = fma((double)i, resolution()[a], start_point()[a]);
            else
                device_grid_point[a] = start_point()[a] + i * resolution()[a];
        }
    }

    __host__ void getGridPoint(precision (&grid_point)[D], int index) {
        if constexpr (std::is_same<precision, float>::value && D <= 8) {
            const cgs_grid g = toCgsGrid(hostMatrix());
            float out[8];
            cgs_compat::check(cgs_grid_point(&g, index, out), "CudaGrid::getGridPoint");
            for (unsigned int a = 0; a < D; a++) grid_point[a] = out[a];
        } else {
            precision *d = nullptr;
            cgs_compat::check_cuda(cudaMalloc(&d, D * sizeof(precision)), "CudaGrid::getGridPoint");
            cgs_compat::grid_point_kernel<precision, D><<<1, 1>>>(*this, index, d);
            cudaError_t e = cudaPeekAtLastError();
            if (e == cudaSuccess) e = cudaMemcpy(grid_point, d, D * sizeof(precision), cudaMemcpyDeviceToHost);
            cudaFree(d);
            cgs_compat::check_cuda(e, "CudaGrid::getGridPoint");
        }
    }

    template <typename T>
    void setStartPoint(std::vector<T> start_point) {
        setRow(ROW_IDX_START, start_point);
        update();
    }

    template <typename T>
    void setEndPoint(std::vector<T> end_point) {
        setRow(ROW_IDX_END, end_point);
        update();
    }

    template <typename T>
    void setNumSamples(std::vector<T> num_samples) {
        setRow(ROW_IDX_SAMPLE_COUNT, num_samples);
        update();
    }

    int getDimension() { return (int)D; }

    void display(const std::string &name = "") const { this->CudaMatrix<precision>::display(name); }

    void setValuesFromVector(const std::vector<precision> vals) const {
        this->CudaMatrix<precision>::setValuesFromVector(vals);
    }

    // The 4 x D matrix on the host, rows {start, end, resolution, count}.
    std::vector<precision> hostMatrix() const { return this->toVector(); }

    // The grid as the C ABI's descriptor (float grids with at most 8 axes).
    cgs_grid cgsGrid() const { return toCgsGrid(hostMatrix()); }

private:
    template <typename T>
    void setRow(int row, const std::vector<T> &v) {
        std::vector<precision> r(D);
        for (unsigned int a = 0; a < D; a++) r[a] = a < v.size() ? (precision)v[a] : precision(0);
        this->CudaMatrix<precision>::setRowFromVector(row, r);
    }

    static cgs_grid toCgsGrid(const std::vector<precision> &m) {
        cgs_grid g{};
        g.dims = (int32_t)D;
        for (unsigned int a = 0; a < D && a < 8; a++) {
            g.start[a] = (float)m[ROW_IDX_START * D + a];
            g.end[a] = (float)m[ROW_IDX_END * D + a];
            g.resolution[a] = (float)m[ROW_IDX_RESOLUTION * D + a];
            g.count[a] = (float)m[ROW_IDX_SAMPLE_COUNT * D + a];
        }
        return g;
    }
};

// Cost-functor pointer types (cudaGridSearch.cuh:283-285, 484-485).
template <typename func_precision, typename grid_precision, unsigned int D, typename... Types>
using func_byvalue_t = func_precision (*)(nv_ext::Vec<grid_precision, D> &gridpt, Types... arg_vals);

template <typename func_precision, typename grid_precision, unsigned int D, typename... Types>
using func_byreference_t = func_precision (*)(nv_ext::Vec<grid_precision, D> &gridpt, Types *...arg_ptrs);

namespace cgs_compat {

template <typename precision, unsigned int D>
__global__ void grid_point_kernel(CudaGrid<precision, D> grid, int index, precision *out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) grid.indexToGridPoint(index, out);
}

// Pixel type code of the C ABI, -1 when the library has no kernels for T.
template <typename T>
constexpr int pixel_code() {
    return std::is_same<T, float>::value      ? CGS_PIXEL_F32
           : std::is_same<T, uint8_t>::value  ? CGS_PIXEL_U8
           : std::is_same<T, double>::value   ? CGS_PIXEL_F64
           : std::is_same<T, uint16_t>::value ? CGS_PIXEL_U16
                                              : -1;
}

template <typename P, uint32_t C>
inline cgs_image describe(CudaImage<P, C> &img) {
    cgs_image d{};
    d.data = img.data();
    d.height = img.height();
    d.width = img.width();
    d.channels = (int32_t)C;
    d.pixel = pixel_code<P>();
    return d;
}

template <typename F, typename G, unsigned int D, typename P>
__global__ void by_reference_address_kernel(uintptr_t *out) {
    typedef F (*Fn)(nv_ext::Vec<G, D> &, CudaImage<P> *, CudaImage<P> *);
    constexpr Fn sad = &sumOfAbsoluteDifferences<F, G, D, 1, P>;
    *out = reinterpret_cast<uintptr_t>(sad);
}

// One thread per grid point (grid-stride), the functor called through its pointer; the
// result element is 0 + value, as the reference stores it.
template <typename F, typename G, unsigned int D, typename... Types>
__global__ void by_value_kernel(CudaGrid<G, D> grid, F *result, uint32_t n, func_byvalue_t<F, G, D, Types...> op,
                                Types... args) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        G pt[D];
        grid.indexToGridPoint(i, pt);
        nv_ext::Vec<G, D> v(pt);
        F r = 0;
        r += (*op)(v, args...);
        result[i] = r;
    }
}

template <typename F, typename G, unsigned int D, typename... Types>
__global__ void by_reference_kernel(CudaGrid<G, D> grid, F *result, uint32_t n,
                                    func_byreference_t<F, G, D, Types...> op, Types *...ptrs) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        G pt[D];
        grid.indexToGridPoint(i, pt);
        nv_ext::Vec<G, D> v(pt);
        F r = 0;
        r += (*op)(v, ptrs...);
        result[i] = r;
    }
}

// The same with the functor known at compile time, so its stack frame is sized statically.
template <typename F, typename G, unsigned int D, typename P, uint32_t C,
          F (*FN)(nv_ext::Vec<G, D> &, CudaImage<P, C>, CudaImage<P, C>)>
__global__ void direct_kernel(CudaGrid<G, D> grid, F *result, uint32_t n, CudaImage<P, C> mov, CudaImage<P, C> fix) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        G pt[D];
        grid.indexToGridPoint(i, pt);
        nv_ext::Vec<G, D> v(pt);
        F r = 0;
        r += FN(v, mov, fix);
        result[i] = r;
    }
}

inline void launch_points(uint32_t n, unsigned &blocks, unsigned &threads) {
    threads = 128;
    const uint64_t want = ((uint64_t)n + threads - 1) / threads;
    blocks = (unsigned)(want == 0 ? 1 : (want < 148u * 64u ? want : 148u * 64u));
}

// A known functor: its device address, the library cost it maps to (-1: none), MI bins,
// and the launcher of its direct-call kernel.
template <typename F, typename G, unsigned int D, typename P, uint32_t C>
struct KnownFunctor {
    uintptr_t addr;
    int cost;
    int mi_bins;
    void (*launch)(CudaGrid<G, D> &, F *, uint32_t, CudaImage<P, C> &, CudaImage<P, C> &);
};

template <typename F, typename G, unsigned int D, typename P, uint32_t C,
          F (*FN)(nv_ext::Vec<G, D> &, CudaImage<P, C>, CudaImage<P, C>)>
void launch_direct(CudaGrid<G, D> &grid, F *result, uint32_t n, CudaImage<P, C> &mov, CudaImage<P, C> &fix) {
    unsigned blocks, threads;
    launch_points(n, blocks, threads);
    direct_kernel<F, G, D, P, C, FN><<<blocks, threads>>>(grid, result, n, mov, fix);
}

// The functor list, in one order for the address kernel and the host table.
template <typename F, typename G, unsigned int D, typename P, uint32_t C>
struct FunctorList {
    typedef F (*Fn)(nv_ext::Vec<G, D> &, CudaImage<P, C>, CudaImage<P, C>);
    typedef KnownFunctor<F, G, D, P, C> Entry;

    // The launcher is named in both compilation passes: the device pass instantiates
    // direct_kernel<..., FN> only through it, and a launcher whose kernel has no device code
    // fails at launch with "invalid device function".  On the device the pointer is never used.
    template <Fn FN>
    static CUDAFUNCTION Entry make(int cost, int bins) {
        return Entry{reinterpret_cast<uintptr_t>(FN), cost, bins, &launch_direct<F, G, D, P, C, FN>};
    }

    // Fills out (capacity 32); returns the count.  Device side: only addr is meaningful.
    static CUDAFUNCTION int fill(Entry *out) {
        int k = 0;
        if constexpr (std::is_same<F, float>::value && std::is_same<G, float>::value) {
            constexpr uint8_t D8 = (uint8_t)D, C8 = (uint8_t)C;
            if constexpr (D == 8) {
                out[k++] = make<&averageAbsoluteDifference<F, G, D, C, P>>(CGS_COST_SAD_AVG, 0);
                out[k++] = make<&calcSQD<F, G, D, C, P>>(CGS_COST_SQD_REF, 0);
                out[k++] = make<&calcNCC<F, G, D, C, P>>(CGS_COST_NCC_REF, 0);
                out[k++] = make<&calcSQDAlt<F, G, D, C, P>>(CGS_COST_SQD_ALT, 0);
                out[k++] = make<&calcNCCAlt<F, G, D, C, P>>(CGS_COST_NCC_ALT, 0);
                out[k++] = make<&calcMIAlt<F, G, D8, C8, P>>(CGS_COST_MI_ALT, 64);
                out[k++] = make<&calcZNCC<F, G, D, C, P>>(CGS_COST_ZNCC, 0);
                out[k++] = make<&calcMI<F, G, D8, C8, P>>(CGS_COST_MI, 32);
                out[k++] = make<&calcMIBins<F, G, D8, C8, P, 2>>(CGS_COST_MI, 2);
                out[k++] = make<&calcMIBins<F, G, D8, C8, P, 4>>(CGS_COST_MI, 4);
                out[k++] = make<&calcMIBins<F, G, D8, C8, P, 8>>(CGS_COST_MI, 8);
                out[k++] = make<&calcMIBins<F, G, D8, C8, P, 16>>(CGS_COST_MI, 16);
                out[k++] = make<&calcMIBins<F, G, D8, C8, P, 32>>(CGS_COST_MI, 32);
                out[k++] = make<&calcMIBins<F, G, D8, C8, P, 64>>(CGS_COST_MI, 64);
                out[k++] = make<&calcNCCstream<F, G, D, C, P>>(-1, 0);
                out[k++] = make<&calcNCCstreamAlt<F, G, D, C, P>>(-1, 0);
                out[k++] = make<&calcSQDstream<F, G, D, C, P>>(-1, 0);
                out[k++] = make<&calcMIstreamAlt<F, G, D, C, P>>(-1, 0);
                out[k++] = make<&calcMIstream<F, G, D, C, P>>(-1, 0);
            }
            if constexpr (D >= 2) out[k++] = make<&averageAbsoluteDifference_stream<F, G, D, C, P>>(-1, 0);
            if constexpr (C == 1 && D == 8) out[k++] = make<&averageAbsoluteDifferenceH<F, G, D, 1, P>>(CGS_COST_SAD_AVG_H, 0);
            if constexpr (C == 1 && D >= 2) {
                constexpr Fn sad = &sumOfAbsoluteDifferences<F, G, D, 1, P>;
                out[k++] = make<sad>(CGS_COST_SAD_SUM_T, 0);
            }
        }
        return k;
    }
};

template <typename F, typename G, unsigned int D, typename P, uint32_t C>
__global__ void functor_address_kernel(uintptr_t *addr, int *count) {
    KnownFunctor<F, G, D, P, C> e[32];
    const int n = FunctorList<F, G, D, P, C>::fill(e);
    for (int i = 0; i < n; i++) addr[i] = e[i].addr;
    *count = n;
}

// The known-functor table of one instantiation on the current device, built on first use.
template <typename F, typename G, unsigned int D, typename P, uint32_t C>
const std::vector<KnownFunctor<F, G, D, P, C>> &known_functors() {
    typedef KnownFunctor<F, G, D, P, C> Entry;
    static std::mutex mu;
    static std::map<int, std::vector<Entry>> tables;
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "functor table");
    std::lock_guard<std::mutex> lock(mu);
    auto it = tables.find(dev);
    if (it != tables.end()) return it->second;
    Entry host[32];
    const int n = FunctorList<F, G, D, P, C>::fill(host);
    std::vector<Entry> table(host, host + n);
    if (n > 0) {
        uintptr_t *d_addr = nullptr;
        int *d_n = nullptr;
        check_cuda(cudaMalloc(&d_addr, 32 * sizeof(uintptr_t)), "functor table");
        cudaError_t e = cudaMalloc(&d_n, sizeof(int));
        uintptr_t addr[32];
        int dn = 0;
        if (e == cudaSuccess) {
            functor_address_kernel<F, G, D, P, C><<<1, 1>>>(d_addr, d_n);
            e = cudaPeekAtLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpy(addr, d_addr, 32 * sizeof(uintptr_t), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(&dn, d_n, sizeof(int), cudaMemcpyDeviceToHost);
        cudaFree(d_addr);
        cudaFree(d_n);
        check_cuda(e, "functor table");
        if (dn != n) fail("functor table: device and host lists differ", CGS_ERROR_CUDA);
        for (int i = 0; i < n; i++) table[i].addr = addr[i];
    }
    return tables.emplace(dev, std::move(table)).first->second;
}

// CudaImage<P, C>, CudaImage<P, C> -- the argument pack of every image functor.
template <typename... Types>
struct ImagePair : std::false_type {};
template <typename P, uint32_t C>
struct ImagePair<CudaImage<P, C>, CudaImage<P, C>> : std::true_type {
    typedef P pix;
    static constexpr uint32_t channels = C;
};

}  // namespace cgs_compat

template <typename func_precision, typename grid_precision, unsigned int D>
struct CudaGridSearcher {
    CudaGrid<grid_precision, D> *_grid;
    CudaTensor<func_precision, D> *_result;

    CudaGridSearcher(CudaGrid<grid_precision, D> &grid, CudaTensor<func_precision, D> &result)
        : _grid(&grid), _result(&result) {
        _options.cost = 0;
        _options.mi_bins = 0;
        _options.overlap_gate = 0.0f;
        _options.points_per_warp = 0;
        _options.warps_per_block = 0;
        _options.flags = 0;
    }

    // Search options of the fused path (overlap gate of calcZNCC / calcMI, sampling flags,
    // tuning).  The cost and MI bins come from the functor.
    cgs_options &options() { return _options; }

    // Argmin of the last search that ran on the fused kernel (valid = 0 otherwise).
    const cgs_argmin &last_argmin() const { return _last; }

    // Which path the last search took: "fused", "direct" or "pointer".
    const char *last_path() const { return _path; }

    template <typename... Types>
    void search(func_byvalue_t<func_precision, grid_precision, D, Types...> errorFunction, Types &...arg_vals) {
        search_by_value(errorFunction, arg_vals...);
    }

    template <typename... Types>
    void search_by_value(func_byvalue_t<func_precision, grid_precision, D, Types...> errorFunction,
                         Types &...arg_vals) {
        const uint32_t n = begin();
        const auto t0 = std::chrono::system_clock::now();
        run_by_value(errorFunction, n, arg_vals...);
        end(t0);
    }

    // The stream count and core count of the reference's per-grid-point launches
    // (cudaGridSearch.cuh:562-649) do not apply; the search runs as search_by_value.
    template <typename... Types>
    void search_by_value_stream(func_byvalue_t<func_precision, grid_precision, D, Types...> errorFunction,
                                int STREAM_BLOCK_DIM, int numCores, Types &...arg_vals) {
        (void)STREAM_BLOCK_DIM;
        (void)numCores;
        search_by_value(errorFunction, arg_vals...);
    }

    // One block per grid point in the reference (cudaGridSearch.cuh:796-827); here as
    // search_by_value.
    template <typename... Types>
    void search_by_value_block(func_byvalue_t<func_precision, grid_precision, D, Types...> errorFunction,
                               int numThreads, Types &...arg_vals) {
        (void)numThreads;
        search_by_value(errorFunction, arg_vals...);
    }

    // Functors taking DEVICE pointers to their arguments (cudaGridSearch.cuh:831-853).
    template <typename... Types>
    void search_by_reference(func_byreference_t<func_precision, grid_precision, D, Types...> errorFunction,
                             Types *...arg_ptrs) {
        const uint32_t n = begin();
        const auto t0 = std::chrono::system_clock::now();
        run_by_reference(errorFunction, n, arg_ptrs...);
        end(t0);
    }

    template <typename... Types>
    void search_by_reference_stream(func_byreference_t<func_precision, grid_precision, D, Types...> errorFunction,
                                    int STREAM_BLOCK_DIM, int numCores, Types *...arg_ptrs) {
        (void)STREAM_BLOCK_DIM;
        (void)numCores;
        search_by_reference(errorFunction, arg_ptrs...);
    }

    // Fisher-information style covariance around the grid minimum of the last search's
    // cost tensor (cudaGridSearch.cuh:316-419, 768-794), added into covar_matrix (host,
    // D x D row-major, as the reference indexes it; the reference's buffer is (D+1) x (D+1)
    // of which it updates the first D x D elements).  Runs on the device (cgs_covariance).
    template <typename... Types>
    void covariance_by_value(grid_precision *covar_matrix);

private:
    cgs_options _options;
    cgs_argmin _last{};
    const char *_path = "";
    std::shared_ptr<cgs_argmin> _d_argmin;

    uint32_t begin() {
        const uint32_t n = _grid->numElements();
#ifdef CGS_COMPAT_VERBOSE
        std::cout << "CudaGrid has " << n << " search samples." << std::endl;
#endif
        _last = cgs_argmin{};
        _last.index = -1;
        return n;
    }

    void end(std::chrono::time_point<std::chrono::system_clock> t0) {
        const std::chrono::duration<double> dt = std::chrono::system_clock::now() - t0;
#ifdef CGS_COMPAT_VERBOSE
        printf("Time Taken: %f\n", dt.count());
#endif
        (void)dt;
    }

    cgs_argmin *device_argmin() {
        if (!_d_argmin) {
            cgs_argmin *p = nullptr;
            cgs_compat::check_cuda(cudaMalloc(&p, sizeof(cgs_argmin)), "CudaGridSearcher");
            _d_argmin.reset(p, [](cgs_argmin *q) { cudaFree(q); });
        }
        return _d_argmin.get();
    }

    void check_result_size(uint32_t n) {
        if (_result->size() < n)
            cgs_compat::fail("CudaGridSearcher: the result tensor holds fewer elements than the grid",
                             CGS_ERROR_INVALID_VALUE);
    }

    // The fused kernel; false when the library reports the request unsupported.
    template <typename P, uint32_t C>
    bool run_fused(int cost, int bins, CudaImage<P, C> &mov, CudaImage<P, C> &fix) {
        if constexpr (!std::is_same<func_precision, float>::value || !std::is_same<grid_precision, float>::value ||
                      D > 8 || cgs_compat::pixel_code<P>() < 0) {
            return false;
        } else {
            const cgs_grid g = _grid->cgsGrid();
            const cgs_image m = cgs_compat::describe(mov), f = cgs_compat::describe(fix);
            cgs_options o = _options;
            o.cost = cost;
            o.mi_bins = cost == CGS_COST_MI ? bins : 0;
            cgs_argmin *d = device_argmin();
            const cgs_status st = cgs_search(&m, &f, &g, &o, _result->data(), d, nullptr);
            if (st == CGS_ERROR_UNSUPPORTED) return false;
            cgs_compat::check(st, "CudaGridSearcher (fused search)");
            cgs_compat::check_cuda(cudaMemcpy(&_last, d, sizeof(_last), cudaMemcpyDeviceToHost),
                                   "CudaGridSearcher (fused search)");
            if (_last.status != CGS_SUCCESS)
                cgs_compat::fail("CudaGridSearcher: the search kernel reported an error (status " +
                                     std::to_string(_last.status) + ")",
                                 (cgs_status)_last.status);
            _path = "fused";
            return true;
        }
    }

    template <typename... Types>
    void run_by_value(func_byvalue_t<func_precision, grid_precision, D, Types...> fn, uint32_t n, Types &...args) {
        check_result_size(n);
        if constexpr (cgs_compat::ImagePair<Types...>::value) {
            typedef typename cgs_compat::ImagePair<Types...>::pix P;
            constexpr uint32_t C = cgs_compat::ImagePair<Types...>::channels;
            const auto &table = cgs_compat::known_functors<func_precision, grid_precision, D, P, C>();
            const uintptr_t a = reinterpret_cast<uintptr_t>(fn);
            for (const auto &e : table) {
                if (e.addr != a) continue;
                CudaImage<P, C> *im[2] = {&args...};
                if (e.cost >= 0 && run_fused(e.cost, e.mi_bins, *im[0], *im[1])) return;
                e.launch(*_grid, _result->data(), n, *im[0], *im[1]);
                cgs_compat::check_launch("CudaGridSearcher (direct kernel)");
                _path = "direct";
                return;
            }
        }
        unsigned blocks, threads;
        cgs_compat::launch_points(n, blocks, threads);
        cgs_compat::by_value_kernel<func_precision, grid_precision, D, Types...>
            <<<blocks, threads>>>(*_grid, _result->data(), n, fn, args...);
        cgs_compat::check_launch("CudaGridSearcher (functor pointer kernel)");
        _path = "pointer";
    }

    template <typename... Types>
    void run_by_reference(func_byreference_t<func_precision, grid_precision, D, Types...> fn, uint32_t n,
                          Types *...ptrs) {
        check_result_size(n);
        if constexpr (cgs_compat::ImagePair<Types...>::value) {
            typedef typename cgs_compat::ImagePair<Types...>::pix P;
            constexpr uint32_t C = cgs_compat::ImagePair<Types...>::channels;
            if constexpr (C == 1 && D >= 2 && std::is_same<func_precision, float>::value &&
                          std::is_same<grid_precision, float>::value) {
                static std::mutex mu;
                static std::map<int, uintptr_t> addr;
                int dev = 0;
                cgs_compat::check_cuda(cudaGetDevice(&dev), "functor table");
                uintptr_t known = 0;
                {
                    std::lock_guard<std::mutex> lock(mu);
                    auto it = addr.find(dev);
                    if (it == addr.end()) {
                        uintptr_t *d = nullptr;
                        cgs_compat::check_cuda(cudaMalloc(&d, sizeof(uintptr_t)), "functor table");
                        cgs_compat::by_reference_address_kernel<func_precision, grid_precision, D, P><<<1, 1>>>(d);
                        cudaError_t e = cudaPeekAtLastError();
                        if (e == cudaSuccess) e = cudaMemcpy(&known, d, sizeof(known), cudaMemcpyDeviceToHost);
                        cudaFree(d);
                        cgs_compat::check_cuda(e, "functor table");
                        addr[dev] = known;
                    } else {
                        known = it->second;
                    }
                }
                if (reinterpret_cast<uintptr_t>(fn) == known) {
                    // the by-reference SAD: the image descriptors live in device memory
                    CudaImage<P, 1> *dp[2] = {ptrs...};
                    CudaImage<P, 1> m(0, 0), f(0, 0);
                    cgs_compat::check_cuda(cudaMemcpy(&m, dp[0], sizeof(m), cudaMemcpyDeviceToHost),
                                           "CudaGridSearcher (by reference)");
                    cgs_compat::check_cuda(cudaMemcpy(&f, dp[1], sizeof(f), cudaMemcpyDeviceToHost),
                                           "CudaGridSearcher (by reference)");
                    if (run_fused(CGS_COST_SAD_SUM_T_REF, 0, m, f)) return;
                }
            }
        }
        unsigned blocks, threads;
        cgs_compat::launch_points(n, blocks, threads);
        cgs_compat::by_reference_kernel<func_precision, grid_precision, D, Types...>
            <<<blocks, threads>>>(*_grid, _result->data(), n, fn, ptrs...);
        cgs_compat::check_launch("CudaGridSearcher (functor pointer kernel)");
        _path = "pointer";
    }

};

template <typename func_precision, typename grid_precision, unsigned int D>
template <typename... Types>
void CudaGridSearcher<func_precision, grid_precision, D>::covariance_by_value(grid_precision *covar_matrix) {
    static_assert(std::is_same<func_precision, float>::value && std::is_same<grid_precision, float>::value && D <= 8,
                  "covariance_by_value: float costs on a float grid of at most 8 axes");
    const uint32_t n = begin();
    check_result_size(n);
    const auto t0 = std::chrono::system_clock::now();
    const cgs_grid g = _grid->cgsGrid();
    double *d = nullptr;
    cgs_compat::check_cuda(cudaMalloc(&d, D * D * sizeof(double)), "covariance_by_value");
    cgs_status st = cgs_covariance(&g, _result->data(), n, d, nullptr);
    double h[D * D];
    cudaError_t e = cudaSuccess;
    if (st == CGS_SUCCESS) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    cgs_compat::check(st, "covariance_by_value");
    cgs_compat::check_cuda(e, "covariance_by_value");
    for (unsigned int i = 0; i < D * D; i++) covar_matrix[i] += (grid_precision)h[i];
    end(t0);
}

#endif  // CUGRIDSEARCH_CUDAGRIDSEARCH_CUH
