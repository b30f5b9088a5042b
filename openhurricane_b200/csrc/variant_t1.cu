// Thread-per-cell integrator variants (N = 10 exact, N <= 16 padded).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../../include/hurchem_b200.h"
#include "integrator_t1.cuh"
#include "launch.cuh"
#include "variants.h"

namespace hc {

template <int N>
static int launch_t1(const DevMech &m, int num_sms, const IntegratorParams &P, const CellIO &io,
                     double *ylast, int block, cudaStream_t st, std::string &err) {
    using L = T1Layout<N>;
    auto kern = integrate_t1_kernel<N>;
    const size_t sm = (sizeof(double) * L::kSlots + sizeof(int) * L::kPivSlots) * (size_t)block;
    HC_LCUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int per_sm = 0;
    HC_LCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, block, sm));
    if (per_sm < 1) {
        err = "thread-per-cell kernel does not fit on an SM";
        return HC_E_UNSUPPORTED;
    }
    const int64_t blocks_needed = (io.ncells + block - 1) / block;
    const int64_t grid = std::min<int64_t>(blocks_needed, (int64_t)per_sm * num_sms);
    if (grid <= 0) return HC_OK;
    kern<<<(unsigned)grid, block, sm, st>>>(m, P, io, ylast);
    HC_LCUDA(cudaGetLastError());
    return HC_OK;
}

}  // namespace hc

int variant_integrate_t1(int N, const hc::DevMech &m, int num_sms, const hc::IntegratorParams &P,
                         const hc::CellIO &io, double *ylast, int block, cudaStream_t st,
                         std::string &err) {
    if (N == 10) return hc::launch_t1<10>(m, num_sms, P, io, ylast, block, st, err);
    if (N <= 16) return hc::launch_t1<16>(m, num_sms, P, io, ylast, block, st, err);
    err = "thread-per-cell integrator is built for N <= 16";
    return HC_E_UNSUPPORTED;
}
