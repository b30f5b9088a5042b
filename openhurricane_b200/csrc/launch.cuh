// Launch helpers shared by the per-size variant translation units.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../../include/hurchem_b200.h"
#include "integrator.cuh"

namespace hc {

#define HC_LCUDA(call)                                                  \
    do {                                                                \
        cudaError_t e_ = (call);                                        \
        if (e_ != cudaSuccess) {                                        \
            err = std::string(#call) + ": " + cudaGetErrorString(e_);   \
            return HC_E_CUDA;                                           \
        }                                                               \
    } while (0)

template <int N, int G>
struct Launch {
    static constexpr int kCellsPerBlock = cells_per_block(G);
    static size_t smem_bytes() { return sizeof(double) * Smem<N, G>::kSize * kCellsPerBlock; }

    static int integrate(const DevMech &m, int num_sms, const IntegratorParams &P,
                         const CellIO &io, cudaStream_t st, std::string &err) {
        // the instantiation without the rarer rate forms and the constant-volume
        // reactor unless the mechanism or the options need them
        auto kern = (m.ext || P.reactor == 1) ? integrate_kernel<N, G, true>
                                              : integrate_kernel<N, G, false>;
        const size_t sm = smem_bytes();
        HC_LCUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        int per_sm = 0;
        HC_LCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, G * kCellsPerBlock, sm));
        if (per_sm < 1) {
            err = "integrator kernel does not fit on an SM";
            return HC_E_UNSUPPORTED;
        }
        const int64_t blocks_needed = (io.nqueue + kCellsPerBlock - 1) / kCellsPerBlock;
        const int64_t grid = std::min<int64_t>(blocks_needed, (int64_t)per_sm * num_sms);
        if (grid <= 0) return HC_OK;
        kern<<<(unsigned)grid, G * kCellsPerBlock, sm, st>>>(m, P, io);
        HC_LCUDA(cudaGetLastError());
        return HC_OK;
    }

    static int rhsjac(const DevMech &m, int64_t n, const double *c, const double *T,
                      const double *p, double *dydt, double *J, cudaStream_t st,
                      std::string &err) {
        auto kern = rhs_jac_kernel<N, G>;
        const size_t sm = smem_bytes();
        HC_LCUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        const int64_t grid = (n + kCellsPerBlock - 1) / kCellsPerBlock;
        if (grid <= 0) return HC_OK;
        kern<<<(unsigned)grid, G * kCellsPerBlock, sm, st>>>(m, n, c, T, p, dydt, J);
        HC_LCUDA(cudaGetLastError());
        return HC_OK;
    }

    static int source(const DevMech &m, int64_t n, const double *T, const double *p,
                      const double *rho, const double *Y, double *Ri, cudaStream_t st,
                      std::string &err) {
        auto kern = source_kernel<N, G>;
        const size_t sm = smem_bytes();
        HC_LCUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        const int64_t grid = (n + kCellsPerBlock - 1) / kCellsPerBlock;
        if (grid <= 0) return HC_OK;
        kern<<<(unsigned)grid, G * kCellsPerBlock, sm, st>>>(m, n, T, p, rho, Y, Ri);
        HC_LCUDA(cudaGetLastError());
        return HC_OK;
    }

    static int srcimp(const DevMech &m, int64_t n, const double *T, const double *p,
                      const double *rho, const double *Y, double *Ri, double *diag,
                      cudaStream_t st, std::string &err) {
        auto kern = source_imp_kernel<N, G>;
        const size_t sm = smem_bytes();
        HC_LCUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        const int64_t grid = (n + kCellsPerBlock - 1) / kCellsPerBlock;
        if (grid <= 0) return HC_OK;
        kern<<<(unsigned)grid, G * kCellsPerBlock, sm, st>>>(m, n, T, p, rho, Y, Ri, diag);
        HC_LCUDA(cudaGetLastError());
        return HC_OK;
    }
};

}  // namespace hc

#define HC_DEFINE_VARIANT(S, N, G)                                                              \
    int variant_integrate_##S(const hc::DevMech &m, int num_sms, const hc::IntegratorParams &P, \
                              const hc::CellIO &io, cudaStream_t st, std::string &err) {         \
        return hc::Launch<N, G>::integrate(m, num_sms, P, io, st, err);                         \
    }                                                                                           \
    int variant_rhsjac_##S(const hc::DevMech &m, int64_t n, const double *c, const double *T,   \
                           const double *p, double *dydt, double *J, cudaStream_t st,           \
                           std::string &err) {                                                  \
        return hc::Launch<N, G>::rhsjac(m, n, c, T, p, dydt, J, st, err);                       \
    }                                                                                           \
    int variant_source_##S(const hc::DevMech &m, int64_t n, const double *T, const double *p,   \
                           const double *rho, const double *Y, double *Ri, cudaStream_t st,     \
                           std::string &err) {                                                  \
        return hc::Launch<N, G>::source(m, n, T, p, rho, Y, Ri, st, err);                       \
    }                                                                                           \
    int variant_srcimp_##S(const hc::DevMech &m, int64_t n, const double *T, const double *p,   \
                           const double *rho, const double *Y, double *Ri, double *diag,        \
                           cudaStream_t st, std::string &err) {                                 \
        return hc::Launch<N, G>::srcimp(m, n, T, p, rho, Y, Ri, diag, st, err);                 \
    }
