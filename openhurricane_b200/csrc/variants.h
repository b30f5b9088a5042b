// Per-size kernel variants of the cell-group integrator, right-hand-side /
// Jacobian and source-term kernels (one translation unit each, see
// variant_*.cu), the thread-per-cell integrator (variant_t1.cu) and the
// property kernel (props.cu). Each entry returns an HC_* status and writes a
// message to err on failure.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "integrator.cuh"

#define HC_DECLARE_VARIANT(S)                                                                   \
    int variant_integrate_##S(const hc::DevMech &m, int num_sms, const hc::IntegratorParams &P, \
                              const hc::CellIO &io, cudaStream_t st, std::string &err);          \
    int variant_rhsjac_##S(const hc::DevMech &m, int64_t n, const double *c, const double *T,   \
                           const double *p, double *dydt, double *J, cudaStream_t st,           \
                           std::string &err);                                                   \
    int variant_source_##S(const hc::DevMech &m, int64_t n, const double *T, const double *p,   \
                           const double *rho, const double *Y, double *Ri, cudaStream_t st,     \
                           std::string &err);                                                   \
    int variant_srcimp_##S(const hc::DevMech &m, int64_t n, const double *T, const double *p,   \
                           const double *rho, const double *Y, double *Ri, double *diag,        \
                           cudaStream_t st, std::string &err);

HC_DECLARE_VARIANT(10)
HC_DECLARE_VARIANT(16)
HC_DECLARE_VARIANT(32)
HC_DECLARE_VARIANT(54)
HC_DECLARE_VARIANT(64)

int variant_integrate_t1(int N, const hc::DevMech &m, int num_sms, const hc::IntegratorParams &P,
                         const hc::CellIO &io, double *ylast, int block, cudaStream_t st,
                         std::string &err);

namespace hc {
struct WMech;
// the warp-per-cell integrator (variant_w.cu, wcell.cuh)
int launch_integrate_w(const WMech &m, int num_sms, const IntegratorParams &P, const CellIO &io,
                       cudaStream_t st, std::string &err);
int launch_integrate_s(const WMech &m, int num_sms, const IntegratorParams &P, const CellIO &io,
                       cudaStream_t st, std::string &err);
int launch_properties(const DevMech &m, int64_t n, const double *T, const double *p,
                      const double *Y, double *ha, double *cp, double *mu, double *kappa,
                      double *D, cudaStream_t st, std::string &err);
}

namespace hc {
struct T2Mech;
}
int variant_integrate_t2(int N, const hc::T2Mech &m, int num_sms, const hc::IntegratorParams &P,
                         const hc::CellIO &io, double *ylast, int block, cudaStream_t st,
                         std::string &err);
namespace hc {
int launch_t_from_ha(const DevMech &m, int64_t n, const double *ha, const double *Y,
                     const double *T0, double TLow, double THigh, double *T, int32_t *flag,
                     cudaStream_t st, std::string &err);
int launch_t_from_ea(const DevMech &m, int64_t n, const double *ea, const double *Y,
                     const double *rho, const double *T0, double TLow, double THigh, double *T,
                     int32_t *flag, cudaStream_t st, std::string &err);
}

namespace hc {
// record-per-cell buffers <-> species-major rows (aos.cu)
constexpr int kAosMaxRec = 66;
int launch_records_to_rows(int64_t n, int rec, const double *recs, double *rows,
                           cudaStream_t st, std::string &err);
int launch_rows_to_records(int64_t n, int rec, int ncols, const double *rows, double *recs,
                           const double *W, int nsp, cudaStream_t st, std::string &err);
int launch_ideal_gas_p(int64_t n, int nsp, const double *W, const double *T, const double *rho,
                       const double *Y, double *p, cudaStream_t st, std::string &err);
int launch_scaled_copy(int64_t n, const double *src, double factor, double *dst, cudaStream_t st,
                       std::string &err);
}
