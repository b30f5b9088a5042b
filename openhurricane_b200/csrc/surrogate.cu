// Surrogate path around the network: input features, and the FP64
// conservation + confidence gate that accepts a predicted chemistry
// increment or sends the cell back to the FP64 integrator.
//
// Gate, per cell (thread per cell, FP64):
//   1. de-normalise the prediction: dT_p, dY_p[i];
//   2. project dY_p onto the element-conserving subspace, dY = P dY_p with
//      P = I - A^T (A A^T)^-1 A, A[e][i] = (atoms of element e in species i)
//      / W_i (P is built on the host); this also makes sum_i dY_i = 0, since
//      W_i = sum_e (atoms) * (atomic weight);
//   3. Y' = Y + dY; a component below -y_neg rejects the cell, components in
//      [-y_neg, 0) are set to 0;
//   4. T' from the conserved mixture enthalpy of the constant-pressure
//      reactor, sum_i Y'_i h_i(T') = sum_i Y_i h_i(T), by Newton's method on
//      the NASA-7 polynomials (thermoList::THa_p, thermoList.cpp:470-533),
//      started from T + dT_p;
//   5. accept when |T' - (T + dT_p)| <= tol_T (the network's temperature
//      agrees with the conserved enthalpy), the projection changed the
//      prediction by at most tol_proj * max(|dY_p|_inf, 1e-6), every input
//      feature lies within +-x_max standard deviations of the training data
//      and T' lies in [T_min, T_max];
//   6. accepted cells get T', Y' and rho = p / (R_m T'); rejected cells are
//      left untouched and appended to the rejected-cell list.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/hurchem_b200.h"
#include "mech.cuh"
#include "surrogate.cuh"

namespace hc {
void set_last_error(const std::string &msg);
}

namespace hc {

constexpr int kSurMaxSp = 64;

__global__ void features_kernel(int nsp, int64_t n, const double *__restrict__ T,
                                const double *__restrict__ p, const double *__restrict__ Y,
                                const double *__restrict__ dt, double dt_factor,
                                const double *__restrict__ mean, const double *__restrict__ inv_std,
                                float *__restrict__ X) {
    const int n_in = nsp + 3;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        float *x = X + c * n_in;
        x[0] = (float)((T[c] - mean[0]) * inv_std[0]);
        x[1] = (float)((log(p[c]) - mean[1]) * inv_std[1]);
        for (int i = 0; i < nsp; ++i)
            x[2 + i] = (float)((Y[(int64_t)i * n + c] - mean[2 + i]) * inv_std[2 + i]);
        x[n_in - 1] = (float)((log(dt[c] * dt_factor) - mean[n_in - 1]) * inv_std[n_in - 1]);
    }
}


__global__ void gate_kernel(const __grid_constant__ DevMech m, const __grid_constant__ GateArgs a) {
    const int nsp = m.nsp;
    const int n_in = nsp + 3, n_out = nsp + 1;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < a.n;
         c += (int64_t)gridDim.x * blockDim.x) {
        bool ok = true;
        for (int j = 0; j < n_in; ++j) {
            const float x = a.X[c * n_in + j];
            if (!(fabsf(x) <= (float)a.x_max)) ok = false;
        }
        const double T0 = a.T[c];
        const float *pr = a.pred + c * n_out;
        const double dTp = (double)pr[0] * a.out_std[0] + a.out_mean[0];
        double dyp[kSurMaxSp], y[kSurMaxSp];
        double pmax = 0.0;
        for (int i = 0; i < nsp; ++i) {
            dyp[i] = (double)pr[1 + i] * a.out_std[1 + i] + a.out_mean[1 + i];
            pmax = hmax(pmax, fabs(dyp[i]));
        }
        // enthalpy of the initial state
        double h0 = 0.0;
        for (int i = 0; i < nsp; ++i) {
            double cp, h;
            species_cp_h(m, i, T0, cp, h);
            h0 += a.Y[(int64_t)i * a.n + c] * h;
        }
        double corr = 0.0;
        for (int i = 0; i < nsp; ++i) {
            double d = 0.0;
            for (int k = 0; k < nsp; ++k) d += a.proj[i * nsp + k] * dyp[k];
            corr = hmax(corr, fabs(d - dyp[i]));
            double yi = a.Y[(int64_t)i * a.n + c] + d;
            if (yi < -a.y_neg) ok = false;
            y[i] = (yi < 0.0) ? 0.0 : yi;
        }
        if (corr > a.tol_proj * hmax(pmax, 1e-6)) ok = false;
        // T' from sum Y' h(T') = h0
        double Tn = T0 + dTp;
        if (!(Tn > a.T_min && Tn < a.T_max)) ok = false;
        if (ok) {
            bool conv = false;
            for (int it = 0; it < 30; ++it) {
                double hm = 0.0, cpm = 0.0;
                for (int i = 0; i < nsp; ++i) {
                    double cp, h;
                    species_cp_h(m, i, Tn, cp, h);
                    hm += y[i] * h;
                    cpm += y[i] * cp;
                }
                const double dT = (hm - h0) / cpm;
                Tn -= dT;
                if (!(Tn > a.T_min && Tn < a.T_max)) break;
                if (fabs(dT) <= 1e-10 * Tn) {
                    conv = true;
                    break;
                }
            }
            if (!conv || fabs(Tn - (T0 + dTp)) > a.tol_T) ok = false;
        }
        a.accept[c] = ok ? 1 : 0;
        if (ok) {
            double wsum = 0.0;
            for (int i = 0; i < nsp; ++i) {
                a.Y[(int64_t)i * a.n + c] = y[i];
                wsum += y[i] / ldg(&m.W[i]);
            }
            a.T[c] = Tn;
            a.rho[c] = a.p[c] / (kRu * wsum * Tn);
        } else {
            const unsigned long long slot = atomicAdd(a.n_rejected, 1ULL);
            a.rejected[slot] = (int32_t)c;
        }
    }
}

int launch_features(const DevMech &m, int64_t n, const double *T, const double *p,
                    const double *Y, const double *dt, double dt_factor, const double *mean,
                    const double *inv_std, float *X, cudaStream_t st) {
    if (n <= 0) return HC_OK;
    const int64_t blocks = (n + 255) / 256;
    features_kernel<<<(unsigned)(blocks < 148 * 32 ? blocks : 148 * 32), 256, 0, st>>>(
        m.nsp, n, T, p, Y, dt, dt_factor, mean, inv_std, X);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_last_error(std::string("features_kernel: ") + cudaGetErrorString(e));
        return HC_E_CUDA;
    }
    return HC_OK;
}

int launch_gate(const DevMech &m, const GateArgs &a, cudaStream_t st) {
    if (a.n <= 0) return HC_OK;
    if (m.nsp > kSurMaxSp) {
        set_last_error("surrogate gate supports at most 64 species");
        return HC_E_UNSUPPORTED;
    }
    const int64_t blocks = (a.n + 127) / 128;
    gate_kernel<<<(unsigned)(blocks < 148 * 64 ? blocks : 148 * 64), 128, 0, st>>>(m, a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_last_error(std::string("gate_kernel: ") + cudaGetErrorString(e));
        return HC_E_CUDA;
    }
    return HC_OK;
}

}  // namespace hc
