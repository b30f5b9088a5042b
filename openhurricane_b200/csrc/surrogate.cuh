// Surrogate gate / feature kernels shared between the C ABI and their
// translation unit (surrogate.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "mech.cuh"

namespace hc {

struct GateArgs {
    int64_t n;
    double *T;
    const double *p;
    double *rho;
    double *Y;                 // [nsp][n]
    const float *pred;         // [n][nsp+1] normalised (dT, dY_1..dY_nsp)
    const float *X;            // [n][nsp+3] normalised features
    const double *out_mean;    // [nsp+1]
    const double *out_std;     // [nsp+1]
    const double *proj;        // [nsp][nsp]
    const double *elem;        // [nel][nsp] atoms of element e per kg of species i (E / W)
    int nel;
    double tol_T, tol_proj, y_neg, x_max, T_min, T_max;
    const float *spread;       // [n] ensemble disagreement (optional), accept <= tol_spread
    double tol_spread;
    int32_t *accept;           // [n] 1 accepted, 0 rejected
    int32_t *rejected;         // [n] list of rejected cells
    unsigned long long *n_rejected;
};

int launch_features(const DevMech &m, int64_t n, const double *T, const double *p,
                    const double *Y, const double *dt, double dt_factor, const double *mean,
                    const double *inv_std, float *X, cudaStream_t st);
int launch_gate(const DevMech &m, const GateArgs &a, cudaStream_t st);

}  // namespace hc
