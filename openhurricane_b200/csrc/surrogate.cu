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
//      [-y_neg, 0) are set to 0, and the element mass those clipped
//      components carried is taken from the major species (Y' > 1e-3) by the
//      minimum-norm correction on them, so elements stay conserved;
//   4. T' from the conserved mixture enthalpy of the constant-pressure
//      reactor, sum_i Y'_i h_i(T') = sum_i Y_i h_i(T), by Newton's method on
//      the NASA-7 polynomials (thermoList::THa_p, thermoList.cpp:470-533),
//      started from T + dT_p;
//   5. accept when |T' - (T + dT_p)| <= tol_T (the network's temperature
//      agrees with the conserved enthalpy), the projection changed the
//      prediction by at most tol_proj * max(|dY_p|_inf, 1e-6), every input
//      feature lies within +-x_max standard deviations of the training data,
//      T' lies in [T_min, T_max] and, when an ensemble's disagreement is
//      given, it is at most tol_spread;
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
constexpr int kSurMaxEl = 8;
constexpr double kSurYFloor = 1e-20;   // mass fractions enter the network as ln(max(Y, floor))

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
        for (int i = 0; i < nsp; ++i) {
            const double yi = Y[(int64_t)i * n + c];
            x[2 + i] = (float)((log(yi > kSurYFloor ? yi : kSurYFloor) - mean[2 + i]) * inv_std[2 + i]);
        }
        x[n_in - 1] = (float)((log(dt[c] * dt_factor) - mean[n_in - 1]) * inv_std[n_in - 1]);
    }
}


__global__ void gate_kernel(const __grid_constant__ DevMech m, const __grid_constant__ GateArgs a) {
    const int nsp = m.nsp;
    const int n_in = nsp + 3, n_out = nsp + 1;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < a.n;
         c += (int64_t)gridDim.x * blockDim.x) {
        bool ok = true;
        if (a.spread && !(a.spread[c] <= (float)a.tol_spread)) ok = false;
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
        // element mass of the clipped components, returned through the major species
        if (ok) {
            const int ne = a.nel;
            double r[kSurMaxEl];
            bool clipped = false;
            for (int e = 0; e < ne; ++e) r[e] = 0.0;
            for (int i = 0; i < nsp; ++i) {
                double d = 0.0;
                for (int k = 0; k < nsp; ++k) d += a.proj[i * nsp + k] * dyp[k];
                const double ex = a.Y[(int64_t)i * a.n + c] + d;   // unclipped
                if (y[i] != ex) {
                    clipped = true;
                    for (int e = 0; e < ne; ++e) r[e] += a.elem[e * nsp + i] * (y[i] - ex);
                }
            }
            if (clipped) {
                // (A_S A_S^T) lam = r over the major species S, then y_S -= A_S^T lam
                double M[kSurMaxEl][kSurMaxEl + 1];
                for (int e = 0; e < ne; ++e) {
                    for (int f = 0; f < ne; ++f) {
                        double sum = 0.0;
                        for (int i = 0; i < nsp; ++i)
                            if (y[i] > 1e-3) sum += a.elem[e * nsp + i] * a.elem[f * nsp + i];
                        M[e][f] = sum;
                    }
                    M[e][ne] = r[e];
                }
                bool solvable = true;
                for (int k = 0; k < ne && solvable; ++k) {
                    int pv = k;
                    for (int i = k + 1; i < ne; ++i)
                        if (fabs(M[i][k]) > fabs(M[pv][k])) pv = i;
                    if (!(fabs(M[pv][k]) > 1e-300)) {
                        // an element without a major carrier: its residual must already be 0
                        if (fabs(M[pv][ne]) > 0.0) solvable = false;
                        for (int j = 0; j <= ne; ++j) M[pv][j] = (j == k) ? 1.0 : 0.0;
                    }
                    if (pv != k)
                        for (int j = 0; j <= ne; ++j) {
                            const double tmp = M[k][j];
                            M[k][j] = M[pv][j];
                            M[pv][j] = tmp;
                        }
                    for (int i = 0; i < ne; ++i) {
                        if (i == k) continue;
                        const double l = M[i][k] / M[k][k];
                        for (int j = k; j <= ne; ++j) M[i][j] -= l * M[k][j];
                    }
                }
                if (!solvable) {
                    ok = false;
                } else {
                    for (int i = 0; i < nsp; ++i) {
                        if (!(y[i] > 1e-3)) continue;
                        double adj = 0.0;
                        for (int e = 0; e < ne; ++e) adj += a.elem[e * nsp + i] * (M[e][ne] / M[e][e]);
                        y[i] -= adj;
                    }
                }
            }
        }
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
