// Warp-per-cell (wcell.cuh) and segment-per-cell (scell.cuh) integrators:
// instantiations for N <= 10 and 16 unknowns and their launch.
#include <algorithm>
#include <string>

#include "../../include/hurchem_b200.h"
#include "launch.cuh"
#include "scell.cuh"
#include "wcell.cuh"

namespace hc {

template <int N>
static int launch_w(const WMech &m, int num_sms, const IntegratorParams &P, const CellIO &io,
                    cudaStream_t st, std::string &err) {
    auto kern = integrate_w_kernel<N>;
    const size_t sm = w_tables_bytes(m.nsp, m.nrc, m.nrc32, m.nent, m.ntb, m.njob32) +
                      WSmem<N>::bytes(m.nrc32, m.njob32) * kWWarps;
    HC_LCUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int per_sm = 0;
    HC_LCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * kWWarps, sm));
    if (per_sm < 1) {
        err = "warp-per-cell kernel does not fit on an SM";
        return HC_E_UNSUPPORTED;
    }
    const int64_t blocks_needed = (io.nqueue + kWWarps - 1) / kWWarps;
    const int64_t grid = std::min<int64_t>(blocks_needed, (int64_t)per_sm * num_sms);
    if (grid <= 0) return HC_OK;
    kern<<<(unsigned)grid, 32 * kWWarps, sm, st>>>(m, P, io);
    HC_LCUDA(cudaGetLastError());
    return HC_OK;
}

int launch_integrate_w(const WMech &m, int num_sms, const IntegratorParams &P, const CellIO &io,
                       cudaStream_t st, std::string &err) {
    const int N = m.nsp + 1;
    if (N <= 10) return launch_w<10>(m, num_sms, P, io, st, err);
    if (N <= 16) return launch_w<16>(m, num_sms, P, io, st, err);
    err = "warp-per-cell kernel takes nsp + 1 <= 16";
    return HC_E_UNSUPPORTED;
}

template <int N>
static int launch_s(const WMech &m, int num_sms, const IntegratorParams &P, const CellIO &io,
                    cudaStream_t st, std::string &err) {
    auto kern = integrate_s_kernel<N>;
    constexpr int G = SLayout<N>::G;
    const size_t sm = w_tables_bytes(m.nsp, m.nrc, m.nrc32, m.nent, m.ntb, m.njob32) +
                      sizeof(double) * SLayout<N>::doubles(m.nrc, m.njob) * G * kSWarps;
    HC_LCUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int per_sm = 0;
    HC_LCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * kSWarps, sm));
    if (per_sm < 1) {
        err = "segment-per-cell kernel does not fit on an SM";
        return HC_E_UNSUPPORTED;
    }
    const int64_t blocks_needed = (io.nqueue + G * kSWarps - 1) / (G * kSWarps);
    const int64_t grid = std::min<int64_t>(blocks_needed, (int64_t)per_sm * num_sms);
    if (grid <= 0) return HC_OK;
    kern<<<(unsigned)grid, 32 * kSWarps, sm, st>>>(m, P, io);
    HC_LCUDA(cudaGetLastError());
    return HC_OK;
}

int launch_integrate_s(const WMech &m, int num_sms, const IntegratorParams &P, const CellIO &io,
                       cudaStream_t st, std::string &err) {
    const int N = m.nsp + 1;
    if (N <= 10) return launch_s<10>(m, num_sms, P, io, st, err);
    if (N <= 16) return launch_s<16>(m, num_sms, P, io, st, err);
    err = "segment-per-cell kernel takes nsp + 1 <= 16";
    return HC_E_UNSUPPORTED;
}

}  // namespace hc
