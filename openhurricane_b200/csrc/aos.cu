// Record-per-cell (array-of-structures) buffers of the reference's CUDA
// calls <-> the species-major fields of this library's kernels.
//
// The reference's GPU path hands the device one record per cell:
//   integration   [T, Y_0 .. Y_{nsp-1}, rho]   (nsp + 2 doubles;
//                 calcChemODEsArray, chemistrySource/src/CUDAChemistrySourceODEs.cu:823-858,
//                 packed by CUDAChemistrySource.cpp:377-385)
//   source terms  [Y_0 .. Y_{nsp-1}, rho, T]   (nsp + 2 doubles; getYiRhoT,
//                 CUDAChemistrySource.cpp:73-81) -> RRi[cell * nsp + i]
//                 (laminarSpeciesSolverCUDA.cpp:326-330)
// Both sides are plain matrix transposes between [ncells][rec] records and
// [rec][ncells] rows. Each block moves tiles of 32 cells through shared
// memory, so that the record side is read or written as one contiguous run
// of 32 * rec doubles and the row side as 256-byte runs of one field; the
// shared tile has an odd row pitch (rec | 1 doubles) so that a warp reading
// one field of 32 cells touches distinct banks. HBM-bound byte work: each
// element is read once and written once.
#include <cuda_runtime.h>

#include <string>

#include "../../include/hurchem_b200.h"
#include "rtc_base.cuh"
#include "variants.h"

namespace hc {

namespace {

constexpr int kAosTile = 32;      // cells per tile
constexpr int kAosThreads = 256;

__global__ void __launch_bounds__(kAosThreads)
records_to_rows_kernel(int64_t n, int rec, const double *__restrict__ recs,
                       double *__restrict__ rows) {
    extern __shared__ double tile[];
    const int pitch = rec | 1;
    for (int64_t c0 = (int64_t)blockIdx.x * kAosTile; c0 < n;
         c0 += (int64_t)gridDim.x * kAosTile) {
        const int cnt = (int)((n - c0) < kAosTile ? (n - c0) : kAosTile);
        const double *src = recs + c0 * rec;
        for (int k = threadIdx.x; k < cnt * rec; k += blockDim.x) {
            const int c = k / rec, j = k - c * rec;
            tile[c * pitch + j] = src[k];
        }
        __syncthreads();
        for (int k = threadIdx.x; k < cnt * rec; k += blockDim.x) {
            const int j = k / cnt, c = k - j * cnt;
            rows[(int64_t)j * n + c0 + c] = tile[c * pitch + j];
        }
        __syncthreads();
    }
}

// rows [rec][n] -> records [n][rec], writing the first `ncols` fields of each
// record (the rest keep their contents). With W given, fields 1..nsp are
// mass fractions converted to concentrations on the way,
// c_i = Y_i * rho / W_i with rho in row nsp + 1.
__global__ void __launch_bounds__(kAosThreads)
rows_to_records_kernel(int64_t n, int rec, int ncols, const double *__restrict__ rows,
                       double *__restrict__ recs, const double *__restrict__ W, int nsp) {
    extern __shared__ double tile[];
    const int pitch = rec | 1;
    for (int64_t c0 = (int64_t)blockIdx.x * kAosTile; c0 < n;
         c0 += (int64_t)gridDim.x * kAosTile) {
        const int cnt = (int)((n - c0) < kAosTile ? (n - c0) : kAosTile);
        for (int k = threadIdx.x; k < cnt * rec; k += blockDim.x) {
            const int j = k / cnt, c = k - j * cnt;
            double v = rows[(int64_t)j * n + c0 + c];
            if (W && j >= 1 && j <= nsp) v = v * rows[(int64_t)(nsp + 1) * n + c0 + c] / W[j - 1];
            tile[c * pitch + j] = v;
        }
        __syncthreads();
        double *dst = recs + c0 * rec;
        for (int k = threadIdx.x; k < cnt * rec; k += blockDim.x) {
            const int c = k / rec, j = k - c * rec;
            if (j < ncols) dst[k] = tile[c * pitch + j];
        }
        __syncthreads();
    }
}

// p = rho Ru T sum_i Y_i / W_i (ideal gas, mixture gas constant from the
// mass fractions), evaluated as ((rho * Ru) * T) * s with s summed in
// species order.
__global__ void ideal_gas_p_kernel(int64_t n, int nsp, const double *__restrict__ W,
                                   const double *__restrict__ T, const double *__restrict__ rho,
                                   const double *__restrict__ Y, double *__restrict__ p) {
    for (int64_t cell = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; cell < n;
         cell += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int i = 0; i < nsp; ++i) s += Y[(int64_t)i * n + cell] / W[i];
        p[cell] = rho[cell] * kRu * T[cell] * s;
    }
}

__global__ void scaled_copy_kernel(int64_t n, const double *__restrict__ src, double factor,
                                   double *__restrict__ dst) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = src[i] * factor;
}

unsigned tiles_grid(int64_t n) {
    const int64_t tiles = (n + kAosTile - 1) / kAosTile;
    const int64_t cap = 148 * 16;
    return (unsigned)(tiles < cap ? tiles : cap);
}

int launched(const char *what, std::string &err) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        err = std::string(what) + ": " + cudaGetErrorString(e);
        return HC_E_CUDA;
    }
    return HC_OK;
}

}  // namespace

int launch_records_to_rows(int64_t n, int rec, const double *recs, double *rows,
                           cudaStream_t st, std::string &err) {
    if (n <= 0) return HC_OK;
    if (rec < 1 || rec > kAosMaxRec) {
        err = "record width out of range";
        return HC_E_INVALID;
    }
    const size_t smem = sizeof(double) * kAosTile * (size_t)(rec | 1);
    records_to_rows_kernel<<<tiles_grid(n), kAosThreads, smem, st>>>(n, rec, recs, rows);
    return launched("records_to_rows_kernel", err);
}

int launch_rows_to_records(int64_t n, int rec, int ncols, const double *rows, double *recs,
                           const double *W, int nsp, cudaStream_t st, std::string &err) {
    if (n <= 0) return HC_OK;
    if (rec < 1 || rec > kAosMaxRec || ncols < 0 || ncols > rec || (W && nsp + 2 > rec)) {
        err = "record width out of range";
        return HC_E_INVALID;
    }
    const size_t smem = sizeof(double) * kAosTile * (size_t)(rec | 1);
    rows_to_records_kernel<<<tiles_grid(n), kAosThreads, smem, st>>>(n, rec, ncols, rows, recs,
                                                                     W, nsp);
    return launched("rows_to_records_kernel", err);
}

// dst = src * factor (the first warm-start sub-steps, dtInit = dt dtFactor)
int launch_scaled_copy(int64_t n, const double *src, double factor, double *dst, cudaStream_t st,
                       std::string &err) {
    if (n <= 0) return HC_OK;
    const int64_t blocks = (n + 255) / 256;
    scaled_copy_kernel<<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), 256, 0, st>>>(
        n, src, factor, dst);
    return launched("scaled_copy_kernel", err);
}

int launch_ideal_gas_p(int64_t n, int nsp, const double *W, const double *T, const double *rho,
                       const double *Y, double *p, cudaStream_t st, std::string &err) {
    if (n <= 0) return HC_OK;
    const int64_t blocks = (n + 255) / 256;
    ideal_gas_p_kernel<<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), 256, 0, st>>>(
        n, nsp, W, T, rho, Y, p);
    return launched("ideal_gas_p_kernel", err);
}

}  // namespace hc
