// Thread-per-cell implicit-Euler integrator for small mechanisms
// (N = nsp + 1 <= 16 equations), FP64.
//
// Each thread owns one cell and evaluates it as the reference's CPU code
// does, in the same floating-point order: the reaction loop of
// chemistrySource::jacobian (chemistrySource.cpp:967-1021, reactionTypes.cpp
// q/DqDci/DqDT), the Doolittle LU with row swaps (SquareMatrix.hpp:185-237)
// and LUBacksubstituteDPivoting (LUDecompose.hpp:68-100). All lanes of a warp
// walk the same reaction list, so the kinetics run without divergence.
//
// Lockstep. The reference's nested loops (cell -> ODE interval -> step ->
// step attempt -> Newton iteration) are flattened into one state machine per
// thread whose only heavy state is "evaluate J at y_k, factor, solve". Every
// trip round the main loop runs that heavy block for all lanes, then each
// lane advances its own bookkeeping (accept/reject, step control, next cell
// from the device work queue) until it needs the next evaluation. Lanes in
// one warp therefore spend their time in the same instructions although
// their cells are at different steps.
//
// Shared memory holds, per thread and interleaved across the block (slot k of
// thread t at s[k*B + t], conflict-free): the Jacobian / LU (N*N), dydt,
// clamped c, G0, dG0/dT (N each), the LU row scratch (N) and the pivots. The
// two previous step states of ImplicitEuler (yklast_) live in a global
// per-cell buffer, touched once per step.
#pragma once

#include "integrator.cuh"
#include "mech.cuh"
#include "t1_body.cuh"

namespace hc {

template <int N>
struct T1Layout {
    static constexpr int kJ = 0;
    static constexpr int kF = N * N;
    static constexpr int kC = kF + N;
    static constexpr int kG0 = kC + N;
    static constexpr int kDG0 = kG0 + N;
    static constexpr int kS = kDG0 + N;
    static constexpr int kSlots = kS + N;     // doubles per thread
    static constexpr int kPivSlots = N;       // ints per thread (after the doubles)
};


template <int N>
struct T1Cell {
    // temperature sits in the last slot of the state vector; species 0..nsp-1
    // come first and any padding species between them and T stay zero
    static constexpr int TI = N - 1;
    static constexpr bool kAssemblesA = false;
    const DevMech &m;
    double *s;      // block shared memory base
    int *piv;       // block pivot base
    int B, tid;
    int nsp;

    __device__ __forceinline__ double &S(int k) const { return s[k * B + tid]; }
    __device__ __forceinline__ double &Jm(int i, int j) const { return s[(i * N + j) * B + tid]; }
    __device__ __forceinline__ int &Piv(int k) const { return piv[k * B + tid]; }
    __device__ __forceinline__ double F(int i) const { return S(T1Layout<N>::kF + i); }
    __device__ __forceinline__ double W(int i) const { return ldg(&m.W[i]); }

    // chemistrySource::jacobian (chemistrySource.cpp:967-1021); jac = false
    // computes only f (DyDt, :863-883, identical f values).
    __device__ void evaluate(const double (&y)[N], bool jac) {
        using L = T1Layout<N>;
        const double T = y[TI];
        const double logT = log(T);
        const double Tm = hmax(T, kTiny);
#pragma unroll
        for (int i = 0; i < N; ++i) {
            if (i < nsp) S(L::kC + i) = hmax(y[i], 0.0);
            S(L::kF + i) = 0.0;
        }
        if (jac) {
            for (int k = 0; k < N * N; ++k) s[k * B + tid] = 0.0;
        }
        // updateG0 (reactionList.hpp:83-86)
#pragma unroll
        for (int i = 0; i < N; ++i) {
            if (i < nsp) {
                const SpeciesThermo th = species_thermo(m, i, T, logT);
                S(L::kG0 + i) = th.G0;
                S(L::kDG0 + i) = th.DG0DT;
            }
        }
        const double invT = 1.0 / Tm;
        for (int r = 0; r < m.nrc; ++r) {
            const int type = ldg(&m.rate_type[r]);
            const double A = ldg(&m.arr[3 * r]), b = ldg(&m.arr[3 * r + 1]);
            const double Ta = ldg(&m.arr[3 * r + 2]);
            const int nf = ldg(&m.nf[r]), nb = ldg(&m.nb[r]);
            int fi[kMaxSide], bi[kMaxSide];
            double fo[kMaxSide], bo[kMaxSide], fnu[kMaxSide], bnu[kMaxSide];
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k) {
                fi[k] = (k < nf) ? ldg(&m.fidx[kMaxSide * r + k]) : 0;
                bi[k] = (k < nb) ? ldg(&m.bidx[kMaxSide * r + k]) : 0;
                fo[k] = (k < nf) ? ldg(&m.ford[kMaxSide * r + k]) : 0.0;
                bo[k] = (k < nb) ? ldg(&m.bord[kMaxSide * r + k]) : 0.0;
                fnu[k] = (k < nf) ? ldg(&m.fnu[kMaxSide * r + k]) : 0.0;
                bnu[k] = (k < nb) ? ldg(&m.bnu[kMaxSide * r + k]) : 0.0;
            }
            double M = 0.0;
            if (type != kArrhenius) {
                const double *e = &m.eff[(int64_t)r * nsp];
                for (int i = 0; i < nsp; ++i) M += ldg(&e[i]) * S(L::kC + i);
            }
            double kf, k0 = 0.0, kinf = 0.0, Pr = 0.0, F = 1.0, lf = 0.0;
            double b0 = 0.0, Ta0 = 0.0;
            if (type == kArrhenius) {
                kf = arrK_log(A, b, Ta, T, logT);
            } else if (type == kThirdBody) {
                kf = M * arrK_log(A, b, Ta, T, logT);
            } else {
                const double A0 = ldg(&m.arr0[3 * r]);
                b0 = ldg(&m.arr0[3 * r + 1]);
                Ta0 = ldg(&m.arr0[3 * r + 2]);
                k0 = arrK_log(A0, b0, Ta0, T, logT);
                kinf = arrK_log(A, b, Ta, T, logT);
                Pr = k0 / notZeroD(kinf) * M;
                if (type != kLindemann) lf = troe_logfcent(&m.troe[4 * r], type == kTroe4, T);
                F = fall_F(type, lf, Pr);
                kf = kinf * (Pr / (1.0 + Pr)) * F;
            }
            double kr = 0.0, Kc = 0.0, DKcDT = 0.0;
            const bool rev = ldg(&m.reversible[r]) != 0;
            if (rev) {
                const T1Cell *self = this;
                const EquilK eq = equilibrium(
                    m, r, T, [self](int i) { return self->S(L::kG0 + i); },
                    [self](int i) { return self->S(L::kDG0 + i); });
                Kc = eq.Kc;
                DKcDT = eq.DKcDT;
                kr = (fabs(Kc) > kVeryTiny) ? kf / Kc : 0.0;
            }
            double pf[kMaxSide], pb[kMaxSide];
            double qf = kf, qr = kr;
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k) {
                pf[k] = 1.0;
                pb[k] = 1.0;
                if (k < nf) {
                    pf[k] = conc_pow(S(L::kC + fi[k]), fo[k]);
                    qf *= pf[k];
                }
                if (k < nb) {
                    pb[k] = conc_pow(S(L::kC + bi[k]), bo[k]);
                    qr *= pb[k];
                }
            }
            const double q = qf - qr;
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k)
                if (k < nf) S(L::kF + fi[k]) -= fnu[k] * q;
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k)
                if (k < nb) S(L::kF + bi[k]) += bnu[k] * q;
            if (!jac) continue;
            // DqDci (reactionTypes.cpp:354-445)
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k) {
                if (k < nf) {
                    double d = kf;
#pragma unroll
                    for (int j = 0; j < kMaxSide; ++j) {
                        if (j < nf) {
                            const double ord = fo[j];
                            const double cj = S(L::kC + fi[j]);
                            if (j == k) {
                                if (ord == 1.0) continue;
                                if (ord < 1.0) d *= (cj > kTiny) ? ord * pow_n(cj, ord - 1.0) : 0.0;
                                else d *= ord * pow_n(hmax(cj, 0.0), ord - 1.0);
                            } else {
                                d *= pf[j];
                            }
                        }
                    }
#pragma unroll
                    for (int j = 0; j < kMaxSide; ++j)
                        if (j < nf) Jm(fi[j], fi[k]) -= fnu[j] * d;
#pragma unroll
                    for (int j = 0; j < kMaxSide; ++j)
                        if (j < nb) Jm(bi[j], fi[k]) += bnu[j] * d;
                }
            }
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k) {
                if (k < nb) {
                    double d = kr;
#pragma unroll
                    for (int j = 0; j < kMaxSide; ++j) {
                        if (j < nb) {
                            const double ord = bo[j];
                            const double cj = S(L::kC + bi[j]);
                            if (j == k) {
                                if (ord == 1.0) continue;
                                if (ord < 1.0) d *= (cj > kTiny) ? ord * pow_n(cj, ord - 1.0) : 0.0;
                                else d *= ord * pow_n(hmax(cj, 0.0), ord - 1.0);
                            } else {
                                d *= pb[j];
                            }
                        }
                    }
#pragma unroll
                    for (int j = 0; j < kMaxSide; ++j)
                        if (j < nf) Jm(fi[j], bi[k]) += fnu[j] * d;
#pragma unroll
                    for (int j = 0; j < kMaxSide; ++j)
                        if (j < nb) Jm(bi[j], bi[k]) -= bnu[j] * d;
                }
            }
            double dgdT = 0.0;
            if (type == kThirdBody) {
                const double *e = &m.eff[(int64_t)r * nsp];
                const double Mm = hmax(M, kTiny);
                for (int i = 0; i < nsp; ++i) {
                    const double g = ldg(&e[i]) / Mm;
                    if (finite(g)) {
#pragma unroll
                        for (int j = 0; j < kMaxSide; ++j)
                            if (j < nf) Jm(fi[j], i) -= fnu[j] * g * q;
#pragma unroll
                        for (int j = 0; j < kMaxSide; ++j)
                            if (j < nb) Jm(bi[j], i) += bnu[j] * g * q;
                    }
                }
            } else if (type != kArrhenius && M > kTiny) {
                // unimolecularFallOffRR::gamDGamDCi / gamDGamDT (unimolecularFallOffRR.cpp:55-91)
                const double Pr2 = k0 * M / notZeroD(kinf);
                const double F2 = fall_F(type, lf, Pr2);
                const double fabc = troe_dfdci_factor(type, lf, Pr2, F2);
                const double *e = &m.eff[(int64_t)r * nsp];
                for (int i = 0; i < nsp; ++i) {
                    const double dPrdci = ldg(&e[i]) * k0 / notZeroD(kinf);
                    const double dFdci = fabc * (1.0 / (Pr2)*dPrdci);
                    const double g = (dPrdci / (Pr2 * (1 + Pr2)) + dFdci / F2);
                    if (finite(g)) {
#pragma unroll
                        for (int j = 0; j < kMaxSide; ++j)
                            if (j < nf) Jm(fi[j], i) -= fnu[j] * g * q;
#pragma unroll
                        for (int j = 0; j < kMaxSide; ++j)
                            if (j < nb) Jm(bi[j], i) += bnu[j] * g * q;
                    }
                }
                const double dPrdT = Pr2 * ((k0 * invT * (b0 + Ta0 * invT)) / notZeroD(k0) -
                                            (kinf * invT * (b + Ta * invT)) / notZeroD(kinf));
                const double dFdT = troe_dfdt(type, &m.troe[4 * r], T, Pr2, F2, dPrdT);
                dgdT = q * (dPrdT / (Pr2 * (1 + Pr2)) + dFdT / F2);
            }
            // DqDT (reactionTypes.cpp:843-876)
            double dkfdT;
            if (type == kArrhenius || type == kThirdBody) dkfdT = kf * invT * (b + Ta * invT);
            else dkfdT = (Pr / (1.0 + Pr)) * F * (kinf * invT * (b + Ta * invT));
            double dkrdT = rev ? (dkfdT - kr * DKcDT) / hmax(Kc, kVeryTiny) : 0.0;
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k) {
                if (k < nf) dkfdT *= pf[k];
                if (k < nb) dkrdT *= pb[k];
            }
            double dqjdT = dkfdT - dkrdT;
            if (!finite(dqjdT)) dqjdT = 0;
            if (!finite(dgdT)) dgdT = 0;
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k)
                if (k < nf) Jm(fi[k], TI) -= fnu[k] * (dqjdT + dgdT);
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k)
                if (k < nb) Jm(bi[k], TI) += bnu[k] * (dqjdT + dgdT);
        }
        // temperature equation (constant pressure)
        double cCp = 0.0, DTdt = 0.0, dcCpdT = 0.0;
        double cp[N], h[N];
#pragma unroll
        for (int i = 0; i < N; ++i) {
            cp[i] = 0.0;
            h[i] = 0.0;
            if (i < nsp) {
                const SpeciesThermo th = species_thermo(m, i, T, logT);
                cp[i] = th.cp;
                h[i] = th.h;
                cCp += y[i] * th.cp;
                dcCpdT += y[i] * th.dcp;
                DTdt += S(L::kF + i) * th.h;
            }
        }
        DTdt /= cCp;
        S(L::kF + TI) = -DTdt;
        if (!jac) return;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            if (i < nsp) {
                double d = Jm(TI, i);
#pragma unroll
                for (int j = 0; j < N; ++j)
                    if (j < nsp) d -= Jm(j, i) * h[j];
                d += cp[i] * DTdt;
                d /= cCp;
                Jm(TI, i) = d;
            }
        }
        double dd = 0.0;
#pragma unroll
        for (int i = 0; i < N; ++i)
            if (i < nsp) dd -= (cp[i] * S(L::kF + i) + h[i] * Jm(i, TI));
        dd += dcCpdT * DTdt;
        dd /= cCp;
        Jm(TI, TI) = dd;
    }

    // I - dt J in place, then LUDecomposeDPivoting (SquareMatrix.hpp:185-237)
    __device__ void factor(double dt) {
        using L = T1Layout<N>;
#pragma unroll
        for (int i = 0; i < N; ++i) {
#pragma unroll
            for (int j = 0; j < N; ++j) Jm(i, j) = -dt * Jm(i, j);
            Jm(i, i) += 1.0;
        }
        for (int k = 0; k < N; ++k) {
            double maxs = Jm(k, k);
            int ik = k;
            for (int i = k; i < N; ++i) {
                double sumlu = 0.0;
                for (int t = 0; t < k; ++t) sumlu += Jm(i, t) * Jm(t, k);
                const double si = Jm(i, k) - sumlu;
                S(L::kS + i) = si;
                if (i == k) maxs = si;
                if (fabs(si) > fabs(maxs)) {
                    ik = i;
                    maxs = si;
                }
            }
            Piv(k) = ik;
            if (ik != k) {
                for (int t = 0; t < N; ++t) {
                    const double tmp = Jm(k, t);
                    Jm(k, t) = Jm(ik, t);
                    Jm(ik, t) = tmp;
                }
                const double tmp = S(L::kS + k);
                S(L::kS + k) = S(L::kS + ik);
                S(L::kS + ik) = tmp;
            }
            Jm(k, k) = S(L::kS + k);
            for (int j = k + 1; j < N; ++j) {
                double sumlu = 0.0;
                for (int t = 0; t < k; ++t) sumlu += Jm(k, t) * Jm(t, j);
                Jm(k, j) -= sumlu;
            }
            for (int i = k + 1; i < N; ++i) Jm(i, k) = S(L::kS + i) / Jm(k, k);
        }
    }

    // LUBacksubstituteDPivoting (LUDecompose.hpp:68-100); b in registers
    __device__ void solve(double (&b)[N]) {
        using L = T1Layout<N>;
#pragma unroll
        for (int i = 0; i < N; ++i) S(L::kS + i) = b[i];
        for (int k = 0; k < N - 1; ++k) {
            const int t = Piv(k);
            if (t != k) {
                const double tmp = S(L::kS + k);
                S(L::kS + k) = S(L::kS + t);
                S(L::kS + t) = tmp;
            }
        }
        for (int i = 0; i < N; ++i) {
            double sumly = 0.0;
            for (int t = 0; t < i; ++t) sumly += Jm(i, t) * S(L::kS + t);
            S(L::kS + i) -= sumly;
        }
        for (int i = N - 1; i >= 0; --i) {
            double sumux = 0.0;
            for (int t = i + 1; t < N; ++t) sumux += Jm(i, t) * S(L::kS + t);
            S(L::kS + i) = (S(L::kS + i) - sumux) / Jm(i, i);
        }
#pragma unroll
        for (int i = 0; i < N; ++i) b[i] = S(L::kS + i);
    }
};

template <int N>
__global__ void __launch_bounds__(128)
integrate_t1_kernel(const __grid_constant__ DevMech m, const __grid_constant__ IntegratorParams P,
                    const __grid_constant__ CellIO io, double *ylast) {
    using L = T1Layout<N>;
    extern __shared__ double smem_t1[];
    const int B = blockDim.x, tid = threadIdx.x;
    T1Cell<N> cell{m, smem_t1, reinterpret_cast<int *>(smem_t1 + (size_t)L::kSlots * B), B, tid,
                   m.nsp};
    t1_run<N>(cell, P, io, ylast);
}

}  // namespace hc
