// Compact thread-per-cell integrator variants (N = 10 exact, N <= 16 padded;
// 32, 64 or 128 threads per block).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../../include/hurchem_b200.h"
#include "integrator_t2.cuh"
#include "launch.cuh"

namespace hc {

// kernel parameters are limited to 32764 bytes
static_assert(sizeof(T2Mech) + sizeof(IntegratorParams) + sizeof(CellIO) + sizeof(double *) <= 32764,
              "T2Mech exceeds the kernel parameter space");

template <int N, int B>
static int launch_t2(const T2Mech &m, int num_sms, const IntegratorParams &P, const CellIO &io,
                     double *ylast, cudaStream_t st, std::string &err) {
    auto kern = integrate_t2_kernel<N, B>;
    const size_t sm = sizeof(double) * T2Cell<N, B>::kSlots * (size_t)B;
    HC_LCUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int per_sm = 0;
    HC_LCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, B, sm));
    if (per_sm < 1) {
        err = "compact thread-per-cell kernel does not fit on an SM";
        return HC_E_UNSUPPORTED;
    }
    const int64_t blocks_needed = (io.nqueue + B - 1) / B;
    const int64_t grid = std::min<int64_t>(blocks_needed, (int64_t)per_sm * num_sms);
    if (grid <= 0) return HC_OK;
    kern<<<(unsigned)grid, B, sm, st>>>(m, P, io, ylast);
    HC_LCUDA(cudaGetLastError());
    return HC_OK;
}

template <int N>
static int launch_t2_b(const T2Mech &m, int num_sms, const IntegratorParams &P, const CellIO &io,
                       double *ylast, int block, cudaStream_t st, std::string &err) {
    if (block == 32) return launch_t2<N, 32>(m, num_sms, P, io, ylast, st, err);
    if (block == 128) return launch_t2<N, 128>(m, num_sms, P, io, ylast, st, err);
    return launch_t2<N, 64>(m, num_sms, P, io, ylast, st, err);
}

}  // namespace hc

int variant_integrate_t2(int N, const hc::T2Mech &m, int num_sms, const hc::IntegratorParams &P,
                         const hc::CellIO &io, double *ylast, int block, cudaStream_t st,
                         std::string &err) {
    if (N == 10) return hc::launch_t2_b<10>(m, num_sms, P, io, ylast, block, st, err);
    if (N <= 16) return hc::launch_t2_b<16>(m, num_sms, P, io, ylast, block, st, err);
    err = "compact thread-per-cell integrator is built for N <= 16";
    return HC_E_UNSUPPORTED;
}
