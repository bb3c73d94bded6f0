// dropin_main.cu -- a program written against the reference's template API, built against
// the drop-in headers (include/cugridsearch/) and the library; the GPU tests run it and
// check its outputs against the oracle.
//
//   dropin_main <in_dir> <out_dir>
//
// <in_dir>/cases.txt holds one case per line:
//   name functor pixel channels dims mh mw fh fw method start[dims] end[dims] count[dims]
// with the images in <in_dir>/<name>_mov.bin and <name>_fix.bin (raw, HWC row-major).
// pixel: f32 | f64 | u8 | i16 (i16 has no library kernel: known functors run their body).
// method: value | stream | block | ref (by-reference, device pointers to the images) | cov
// (search by value, then covariance_by_value).
// Writes <out_dir>/<name>_costs.bin (float32 per grid point) and <out_dir>/<name>.txt:
//   path index value point[dims] [covar[dims*dims] for cov]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "cugridsearch/cudaGridSearch.cuh"

// ---- device pointers to the functors, as a reference user declares them
#define FN8(P, C) func_byvalue_t<float, float, 8, CudaImage<P, C>, CudaImage<P, C>>
typedef FN8(float, 1) f32c1_t;
typedef FN8(uint8_t, 3) u8c3_t;
typedef FN8(int16_t, 1) i16c1_t;
typedef func_byvalue_t<float, float, 2, CudaImage<double, 1>, CudaImage<double, 1>> f64t_t;
typedef func_byreference_t<float, float, 2, CudaImage<double, 1>, CudaImage<double, 1>> f64r_t;

// A caller's own functor: runs through the function-pointer kernel.
template <typename P, uint32_t C>
__device__ float user_ncc(nv_ext::Vec<float, 8> &p, CudaImage<P, C> m, CudaImage<P, C> f) {
    return 0.5f * calcNCC<float, float, 8, C, P>(p, m, f);
}

__device__ f32c1_t d_f32_ncc = calcNCC<float, float, 8, 1, float>;
__device__ f32c1_t d_f32_sqd = calcSQD<float, float, 8, 1, float>;
__device__ f32c1_t d_f32_sad = averageAbsoluteDifference<float, float, 8, 1, float>;
__device__ f32c1_t d_f32_sadh = averageAbsoluteDifferenceH<float, float, 8, 1, float>;
__device__ f32c1_t d_f32_ncca = calcNCCAlt<float, float, 8, 1, float>;
__device__ f32c1_t d_f32_sqda = calcSQDAlt<float, float, 8, 1, float>;
__device__ f32c1_t d_f32_mia = calcMIAlt<float, float, 8, 1, float>;
__device__ f32c1_t d_f32_zncc = calcZNCC<float, float, 8, 1, float>;
__device__ f32c1_t d_f32_mi = calcMI<float, float, 8, 1, float>;
__device__ f32c1_t d_f32_mi16 = calcMIBins<float, float, 8, 1, float, 16>;
__device__ f32c1_t d_f32_nccs = calcNCCstream<float, float, 8, 1, float>;
__device__ f32c1_t d_f32_sqds = calcSQDstream<float, float, 8, 1, float>;
__device__ f32c1_t d_f32_nccsa = calcNCCstreamAlt<float, float, 8, 1, float>;
__device__ f32c1_t d_f32_mis = calcMIstream<float, float, 8, 1, float>;
__device__ f32c1_t d_f32_misa = calcMIstreamAlt<float, float, 8, 1, float>;
__device__ f32c1_t d_f32_user = user_ncc<float, 1>;
__device__ u8c3_t d_u8_ncc = calcNCC<float, float, 8, 3, uint8_t>;
__device__ u8c3_t d_u8_mia = calcMIAlt<float, float, 8, 3, uint8_t>;
__device__ u8c3_t d_u8_mi = calcMI<float, float, 8, 3, uint8_t>;
__device__ i16c1_t d_i16_ncc = calcNCC<float, float, 8, 1, int16_t>;
__device__ f64t_t d_f64_sadt = sumOfAbsoluteDifferences<float, float, 2, 1, double>;
__device__ f64t_t d_f64_sads = averageAbsoluteDifference_stream<float, float, 2, 1, double>;
__device__ f64r_t d_f64_sadr = sumOfAbsoluteDifferences<float, float, 2, 1, double>;

struct Case {
    std::string name, functor, pixel, method;
    int channels, dims, mh, mw, fh, fw;
    std::vector<float> start, end, count;
};

static std::vector<char> read_file(const std::string &path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        fprintf(stderr, "cannot read %s\n", path.c_str());
        exit(2);
    }
    return std::vector<char>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

template <typename P, uint32_t C>
static CudaImage<P, C> upload(const std::string &path, int h, int w) {
    CudaImage<P, C> im(h, w);
    const std::vector<char> raw = read_file(path);
    if (raw.size() != im.bytesSize()) {
        fprintf(stderr, "%s: %zu bytes, expected %u\n", path.c_str(), raw.size(), im.bytesSize());
        exit(2);
    }
    cgs_compat::check_cuda(cudaMalloc(&im.data(), im.bytesSize()), "cudaMalloc");
    cgs_compat::check_cuda(cudaMemcpy(im.data(), raw.data(), raw.size(), cudaMemcpyHostToDevice), "cudaMemcpy");
    return im;
}

template <typename T>
static T fetch(const T &symbol) {
    T h;
    cgs_compat::check_cuda(cudaMemcpyFromSymbol(&h, symbol, sizeof(T)), "cudaMemcpyFromSymbol");
    return h;
}

// Runs one case on a grid of D axes with functor pointer fn (by value) and writes outputs.
template <unsigned int D, typename P, uint32_t C, typename Fn>
static void run(const Case &cs, Fn fn, const std::string &in, const std::string &out) {
    CudaImage<P, C> mov = upload<P, C>(in + "/" + cs.name + "_mov.bin", cs.mh, cs.mw);
    CudaImage<P, C> fix = upload<P, C>(in + "/" + cs.name + "_fix.bin", cs.fh, cs.fw);
    CudaGrid<float, D> grid;
    cgs_compat::check_cuda(cudaMalloc(&grid.data(), grid.bytesSize()), "cudaMalloc");
    grid.setStartPoint(cs.start);
    grid.setEndPoint(cs.end);
    grid.setNumSamples(cs.count);
    float counts[D];
    grid.getAxisSampleCounts(counts);
    CudaTensor<float, D> values(counts);
    cgs_compat::check_cuda(cudaMalloc(&values._data, values.bytesSize()), "cudaMalloc");
    values.fill(0);
    CudaGridSearcher<float, float, D> searcher(grid, values);
    std::vector<float> covar(D * D, 0.0f);
    if constexpr (std::is_same<Fn, func_byvalue_t<float, float, D, CudaImage<P, C>, CudaImage<P, C>>>::value) {
        if (cs.method == "stream")
            searcher.search_by_value_stream(fn, 10000, 1, mov, fix);
        else if (cs.method == "block")
            searcher.search_by_value_block(fn, 64, mov, fix);
        else
            searcher.search_by_value(fn, mov, fix);
        if (cs.method == "cov") searcher.covariance_by_value(covar.data());
    } else {
        CudaImage<P, C> *dm = nullptr, *df = nullptr;
        cgs_compat::check_cuda(cudaMalloc(&dm, sizeof(mov)), "cudaMalloc");
        cgs_compat::check_cuda(cudaMalloc(&df, sizeof(fix)), "cudaMalloc");
        cgs_compat::check_cuda(cudaMemcpy(dm, &mov, sizeof(mov), cudaMemcpyHostToDevice), "cudaMemcpy");
        cgs_compat::check_cuda(cudaMemcpy(df, &fix, sizeof(fix), cudaMemcpyHostToDevice), "cudaMemcpy");
        searcher.search_by_reference_stream(fn, 10000, 1, dm, df);
        cudaFree(dm);
        cudaFree(df);
    }
    float best;
    int32_t index;
    values.find_extrema(best, index);
    float point[D];
    grid.getGridPoint(point, index);
    const uint32_t n = grid.numElements();
    std::vector<float> host(n);
    cgs_compat::check_cuda(cudaMemcpy(host.data(), values.data(), n * sizeof(float), cudaMemcpyDeviceToHost),
                           "cudaMemcpy");
    std::ofstream(out + "/" + cs.name + "_costs.bin", std::ios::binary)
        .write(reinterpret_cast<const char *>(host.data()), n * sizeof(float));
    std::ofstream txt(out + "/" + cs.name + ".txt");
    txt.precision(9);
    txt << searcher.last_path() << " " << index << " " << best;
    for (unsigned int a = 0; a < D; a++) txt << " " << point[a];
    if (cs.method == "cov")
        for (float v : covar) txt << " " << v;
    txt << "\n";
    cudaFree(mov.data());
    cudaFree(fix.data());
    cudaFree(grid.data());
    cudaFree(values.data());
}

int main(int argc, char **argv) {
    if (argc != 3) {
        fprintf(stderr, "usage: dropin_main <in_dir> <out_dir>\n");
        return 2;
    }
    const std::string in = argv[1], out = argv[2];
    std::ifstream list(in + "/cases.txt");
    std::string line;
    int done = 0;
    std::string current;
    try {
        while (std::getline(list, line)) {
            if (line.empty() || line[0] == '#') continue;
            std::istringstream ss(line);
            Case cs;
            ss >> cs.name >> cs.functor >> cs.pixel >> cs.channels >> cs.dims >> cs.mh >> cs.mw >> cs.fh >> cs.fw >>
                cs.method;
            cs.start.resize(cs.dims);
            cs.end.resize(cs.dims);
            cs.count.resize(cs.dims);
            for (auto &v : cs.start) ss >> v;
            for (auto &v : cs.end) ss >> v;
            for (auto &v : cs.count) ss >> v;
            const std::string key = cs.pixel + ":" + std::to_string(cs.channels) + ":" + cs.functor;
            current = cs.name;
            if (key == "f32:1:ncc") run<8, float, 1>(cs, fetch(d_f32_ncc), in, out);
            else if (key == "f32:1:sqd") run<8, float, 1>(cs, fetch(d_f32_sqd), in, out);
            else if (key == "f32:1:sad") run<8, float, 1>(cs, fetch(d_f32_sad), in, out);
            else if (key == "f32:1:sadh") run<8, float, 1>(cs, fetch(d_f32_sadh), in, out);
            else if (key == "f32:1:ncc_alt") run<8, float, 1>(cs, fetch(d_f32_ncca), in, out);
            else if (key == "f32:1:sqd_alt") run<8, float, 1>(cs, fetch(d_f32_sqda), in, out);
            else if (key == "f32:1:mi_alt") run<8, float, 1>(cs, fetch(d_f32_mia), in, out);
            else if (key == "f32:1:zncc") run<8, float, 1>(cs, fetch(d_f32_zncc), in, out);
            else if (key == "f32:1:mi") run<8, float, 1>(cs, fetch(d_f32_mi), in, out);
            else if (key == "f32:1:mi16") run<8, float, 1>(cs, fetch(d_f32_mi16), in, out);
            else if (key == "f32:1:ncc_stream") run<8, float, 1>(cs, fetch(d_f32_nccs), in, out);
            else if (key == "f32:1:sqd_stream") run<8, float, 1>(cs, fetch(d_f32_sqds), in, out);
            else if (key == "f32:1:ncc_stream_alt") run<8, float, 1>(cs, fetch(d_f32_nccsa), in, out);
            else if (key == "f32:1:mi_stream") run<8, float, 1>(cs, fetch(d_f32_mis), in, out);
            else if (key == "f32:1:mi_stream_alt") run<8, float, 1>(cs, fetch(d_f32_misa), in, out);
            else if (key == "f32:1:user_ncc") run<8, float, 1>(cs, fetch(d_f32_user), in, out);
            else if (key == "u8:3:ncc") run<8, uint8_t, 3>(cs, fetch(d_u8_ncc), in, out);
            else if (key == "u8:3:mi_alt") run<8, uint8_t, 3>(cs, fetch(d_u8_mia), in, out);
            else if (key == "u8:3:mi") run<8, uint8_t, 3>(cs, fetch(d_u8_mi), in, out);
            else if (key == "i16:1:ncc") run<8, int16_t, 1>(cs, fetch(d_i16_ncc), in, out);
            else if (key == "f64:1:sad_t" && cs.method == "ref") run<2, double, 1>(cs, fetch(d_f64_sadr), in, out);
            else if (key == "f64:1:sad_t") run<2, double, 1>(cs, fetch(d_f64_sadt), in, out);
            else if (key == "f64:1:sad_stream") run<2, double, 1>(cs, fetch(d_f64_sads), in, out);
            else {
                fprintf(stderr, "unknown case %s\n", key.c_str());
                return 2;
            }
            done++;
        }
    } catch (const cgs_compat::Error &e) {
        fprintf(stderr, "error in case %s: %s\n", current.c_str(), e.what());
        return 1;
    }
    printf("%d cases\n", done);
    return 0;
}
