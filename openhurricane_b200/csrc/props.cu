// Mixture property kernel: per-species enthalpy, mixture cp, Wilke viscosity
// and conductivity, mixture-averaged diffusion coefficients.
//
//   h_i, cp        thermo/src/JANAF.cpp:155-199, thermoList.cpp:165-190
//   mu_i, kappa_i  transport/src/kineticTheory.cpp:37-57, kineticTheory.inl:32-34
//   mu, kappa      transport/src/transportList.cpp:238-284 (muKappa, Wilke)
//   x_i            species/src/speciesList.cpp:208-224 (Yi2Xi)
//   D_i            transport/src/kineticTheory.cpp:118-163 (Di), T^1.5 = T sqrt(T)
//
// One warp per cell, lane i handling species i, i+32, ...; the O(nsp^2) pair
// loops run with per-pair constants precomputed on the host at mechanism
// upload (the reference caches the same constants on first use). The binary
// collision integral exp(-0.145 ln T*_ij) is evaluated as
// T^-0.145 * (1/sqrt(eps_i eps_j))^-0.145, one power per cell instead of one
// per pair. Outputs are species-major [nsp][n].
#include <cuda_runtime.h>

#include <string>

#include "../../include/hurchem_b200.h"
#include "launch.cuh"
#include "variants.h"

namespace hc {

constexpr int kPropWarps = 8;
constexpr int kPropMaxSp = 64;

__global__ void __launch_bounds__(32 * kPropWarps)
properties_kernel(const __grid_constant__ DevMech m, int64_t n, const double *__restrict__ T_,
                  const double *__restrict__ p_, const double *__restrict__ Y, double *ha,
                  double *cpm, double *mu, double *kappa, double *D) {
    __shared__ double sx[kPropWarps][kPropMaxSp];
    __shared__ double smu[kPropWarps][kPropMaxSp];
    const int w = threadIdx.x / 32, lane = threadIdx.x & 31;
    const int nsp = m.nsp;
    const double muPre = 2.6693e-6, omegaPre = 1.147, omegaExp = -0.145;
    for (int64_t cell = (int64_t)blockIdx.x * kPropWarps + w; cell < n;
         cell += (int64_t)gridDim.x * kPropWarps) {
        const double T = T_[cell], p = p_[cell];
        // Yi2Xi
        double wsum = 0.0, cps = 0.0;
        for (int i = lane; i < nsp; i += 32) {
            const double yi = Y[(int64_t)i * n + cell];
            wsum += yi / ldg(&m.W[i]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
        const double Wmean = 1.0 / hmax(wsum, kVeryTiny);
        double xt = 0.0;
        for (int i = lane; i < nsp; i += 32) {
            const double yi = Y[(int64_t)i * n + cell];
            double xi = yi * Wmean / ldg(&m.W[i]);
            xi = hmax(0.0, hmin(1.0, xi));
            sx[w][i] = xi;
            xt += xi;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) xt += __shfl_xor_sync(0xffffffffu, xt, o);
        __syncwarp();
        if (xt != 1.0)
            for (int i = lane; i < nsp; i += 32) sx[w][i] /= xt;
        // species viscosity, conductivity, enthalpy
        double kap[2] = {0.0, 0.0};
        int q = 0;
        for (int i = lane; i < nsp; i += 32, ++q) {
            double cp0, h0;
            species_cp_h(m, i, T, cp0, h0);
            if (ha) ha[(int64_t)i * n + cell] = h0;
            cps += cp0 * Y[(int64_t)i * n + cell];
            const double Wi = ldg(&m.W[i]);
            const double Tstar = T * (1.0 / ldg(&m.eps_k[i]));
            const double om = omegaPre * exp(omegaExp * log(Tstar)) +
                              1.0 / ((Tstar + 0.5) * (Tstar + 0.5));
            const double sg = ldg(&m.sigma[i]);
            const double mui = muPre * sqrt(Wi * T) / ((sg * sg) * om);
            smu[w][i] = mui;
            const double Ri = kRu / Wi;
            kap[q] = mui * Ri * (cp0 / Ri + 1.25);
        }
        __syncwarp();
        // Wilke mixing (transportList::muKappa) and mixture-averaged D_i
        const double Tv1p5 = T * sqrt(T);
        const double Tpow = exp(omegaExp * log(T));
        double mum = 0.0, kappam = 0.0;
        q = 0;
        for (int i = lane; i < nsp; i += 32, ++q) {
            const double mui = smu[w][i];
            double phi = 0.0, sumD = 0.0;
            const double *phiP = &m.pair_phi[(int64_t)i * nsp];
            const double *rD = &m.pair_D[(int64_t)i * nsp];
            const double *rP = &m.pair_Dpow[(int64_t)i * nsp];
            const double *rr = &m.pair_r[(int64_t)i * nsp];
            for (int j = 0; j < nsp; ++j) {
                const double xj = sx[w][j];
                const double tmp = 1.0 + sqrt(mui / smu[w][j] * ldg(&m.pair_w[(int64_t)j * nsp + i]));
                phi += ldg(&phiP[j]) * xj * (tmp * tmp);
                if (j != i) {
                    const double Tstar = T * ldg(&rr[j]);
                    const double Tss = 1.0 / ((Tstar + 0.5) * (Tstar + 0.5));
                    const double OmegaDij = Tpow * ldg(&rP[j]) + Tss;
                    const double Dij = Tv1p5 * ldg(&rD[j]) / (p * OmegaDij);
                    sumD += xj / Dij;
                }
            }
            const double xi = sx[w][i];
            mum += mui * xi / phi;
            kappam += kap[q] * xi / phi;
            if (D) {
                double Dim = 0.0;
                if (xi < 1.0 - kVeryTiny) Dim = (1.0 - xi) / sumD;
                if (isinf(Dim)) Dim = 0.0;
                D[(int64_t)i * n + cell] = Dim;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mum += __shfl_xor_sync(0xffffffffu, mum, o);
            kappam += __shfl_xor_sync(0xffffffffu, kappam, o);
            cps += __shfl_xor_sync(0xffffffffu, cps, o);
        }
        if (lane == 0) {
            if (mu) mu[cell] = mum;
            if (kappa) kappa[cell] = kappam;
            if (cpm) cpm[cell] = cps;
        }
        __syncwarp();
    }
}

int launch_properties(const DevMech &m, int64_t n, const double *T, const double *p,
                      const double *Y, double *ha, double *cp, double *mu, double *kappa,
                      double *D, cudaStream_t st, std::string &err) {
    if (m.nsp > kPropMaxSp) {
        err = "property kernel is built for at most 64 species";
        return HC_E_UNSUPPORTED;
    }
    if (!m.pair_D) {
        err = "mechanism has no transport pair tables";
        return HC_E_INVALID;
    }
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t blocks = std::min<int64_t>((n + kPropWarps - 1) / kPropWarps, (int64_t)sms * 8);
    properties_kernel<<<(unsigned)blocks, 32 * kPropWarps, 0, st>>>(m, n, T, p, Y, ha, cp, mu,
                                                                     kappa, D);
    HC_LCUDA(cudaGetLastError());
    return HC_OK;
}

// Temperature from the mixture's mass enthalpy at constant pressure,
// thermoList::THa_p (thermoList.cpp:501-533): Newton steps
// T <- limit(T - (h(T) - ha) / cp(T)) from T0 until |dT| <= T0 tol, at most
// max_iter + 1 steps; limit clamps to [TLow, THigh] and sets the flag
// (0 below, 1 inside, 2 above; thermoList.cpp:152-163). Thread per cell.
__global__ void t_from_ha_kernel(const __grid_constant__ DevMech m, int64_t n,
                                 const double *__restrict__ ha, const double *__restrict__ Y,
                                 const double *__restrict__ T0, double TLow, double THigh,
                                 double tol, int max_iter, double *__restrict__ Tout,
                                 int32_t *__restrict__ flag) {
    const int nsp = m.nsp;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        double Tnew = T0[c];
        const double Ttol = T0[c] * tol;
        int it = 0, f = 1;
        while (true) {
            const double Test = Tnew;
            double hm = 0.0, cpm = 0.0;
            for (int i = 0; i < nsp; ++i) {
                double cp, h;
                species_cp_h(m, i, Test, cp, h);
                const double yi = Y[(int64_t)i * n + c];
                hm += h * yi;
                cpm += cp * yi;
            }
            const double v = Test - (hm - ha[c]) / cpm;
            if (v < TLow) {
                f = 0;
                Tnew = TLow;
            } else if (v > THigh) {
                f = 2;
                Tnew = THigh;
            } else {
                f = 1;
                Tnew = v;
            }
            if (it++ > max_iter) break;
            if (!(fabs(Tnew - Test) > Ttol)) break;
        }
        Tout[c] = Tnew;
        if (flag) flag[c] = f;
    }
}

// thermoList::TEa_rho (thermoList.inl:343-348 through thermoList.cpp:501-533):
// the same Newton iteration on the mixture's internal energy at fixed
// density, e(T) = sum_i Y_i h_i(T) - p / rho with p = rho Rm T, and
// de/dT = sum_i Y_i cp_i(T) - Rm (thermoList.inl:145-162, 302-306)
__global__ void t_from_ea_kernel(const __grid_constant__ DevMech m, int64_t n,
                                 const double *__restrict__ ea, const double *__restrict__ Y,
                                 const double *__restrict__ rho, const double *__restrict__ T0,
                                 double TLow, double THigh, double tol, int max_iter,
                                 double *__restrict__ Tout, int32_t *__restrict__ flag) {
    const int nsp = m.nsp;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        double w = 0.0;
        for (int i = 0; i < nsp; ++i) w += Y[(int64_t)i * n + c] / ldg(&m.W[i]);
        const double Rm = kRu / (1.0 / hmax(w, kVeryTiny));
        const double r = rho[c];
        double Tnew = T0[c];
        const double Ttol = T0[c] * tol;
        int it = 0, f = 1;
        while (true) {
            const double Test = Tnew;
            double hm = 0.0, cpm = 0.0;
            for (int i = 0; i < nsp; ++i) {
                double cp, h;
                species_cp_h(m, i, Test, cp, h);
                const double yi = Y[(int64_t)i * n + c];
                hm += h * yi;
                cpm += cp * yi;
            }
            const double em = hm - (r * Rm * Test) / r;
            const double cvm = cpm - Rm;
            const double v = Test - (em - ea[c]) / cvm;
            if (v < TLow) {
                f = 0;
                Tnew = TLow;
            } else if (v > THigh) {
                f = 2;
                Tnew = THigh;
            } else {
                f = 1;
                Tnew = v;
            }
            if (it++ > max_iter) break;
            if (!(fabs(Tnew - Test) > Ttol)) break;
        }
        Tout[c] = Tnew;
        if (flag) flag[c] = f;
    }
}

int launch_t_from_ea(const DevMech &m, int64_t n, const double *ea, const double *Y,
                     const double *rho, const double *T0, double TLow, double THigh, double *T,
                     int32_t *flag, cudaStream_t st, std::string &err) {
    if (n <= 0) return HC_OK;
    const int64_t blocks = (n + 127) / 128;
    t_from_ea_kernel<<<(unsigned)(blocks < 148 * 64 ? blocks : 148 * 64), 128, 0, st>>>(
        m, n, ea, Y, rho, T0, TLow, THigh, 1.0e-4, 100, T, flag);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        err = std::string("t_from_ea_kernel: ") + cudaGetErrorString(e);
        return HC_E_CUDA;
    }
    return HC_OK;
}

int launch_t_from_ha(const DevMech &m, int64_t n, const double *ha, const double *Y,
                     const double *T0, double TLow, double THigh, double *T, int32_t *flag,
                     cudaStream_t st, std::string &err) {
    if (n <= 0) return HC_OK;
    const int64_t blocks = (n + 127) / 128;
    t_from_ha_kernel<<<(unsigned)(blocks < 148 * 64 ? blocks : 148 * 64), 128, 0, st>>>(
        m, n, ha, Y, T0, TLow, THigh, 1.0e-4, 100, T, flag);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        err = std::string("t_from_ha_kernel: ") + cudaGetErrorString(e);
        return HC_E_CUDA;
    }
    return HC_OK;
}

}  // namespace hc
