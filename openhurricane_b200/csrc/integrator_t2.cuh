// Thread-per-cell implicit-Euler integrator, compact form, for mechanisms of
// N = nsp + 1 <= 16 unknowns (FP64).
//
// The mechanism travels in the kernel's constant parameter bank (T2Mech, a
// __grid_constant__ argument of at most ~24 KB): every lane of a warp walks
// the same reaction at the same time, so each table read is one uniform
// constant-bank load, and branches on a reaction's kind are warp-uniform.
// Per-thread state that is indexed by species (clamped concentrations c,
// molar G0 and dG0/dT, f and the Jacobian / LU) lives in shared memory,
// interleaved across the block at compile-time offsets (slot k of thread t
// at s[k*B + t], conflict-free). The kernel body is loops over reactions and
// species, small enough to stay in the instruction cache.
//
// Arithmetic: the precompiled thread-per-cell kernel's (integrator_t1.cuh,
// restating chemistrySource::jacobian, chemistrySource.cpp:967-1021, and
// reactionTypes.cpp q / Kc / DqDci / DqDT), with three reorderings that stay
// far inside the integrator's tolerance: third-body and fall-off columns are
// added as eff_i * (coef * g_r) with g_r = q/M or the fall-off factor
// (rank one in the efficiencies, zero efficiencies skipped); the LU
// factorisation is right-looking (same pivots and factors as
// LUDecomposeDPivoting, SquareMatrix.hpp:185-237) and multiplies by the
// pivot's reciprocal.
#pragma once

#include "rtc_base.cuh"
#include "t1_body.cuh"

namespace hc {

constexpr int kT2MaxSp = 15;
constexpr int kT2MaxRxn = 64;
constexpr int kT2MaxEff = 512;

struct T2Rxn {
    double A, b, Ta;          // (high-pressure) Arrhenius
    double A0, b0, Ta0;       // low-pressure limit (fall-off)
    double troe[4];
    double fnu[kMaxSide], bnu[kMaxSide], ford[kMaxSide], bord[kMaxSide];
    double sum_stoi;
    int8_t type, rev, nf, nb;
    int8_t fidx[kMaxSide], bidx[kMaxSide];
    int16_t eff_begin, eff_end;   // range in T2Mech::eff_val / eff_idx
};

struct T2Mech {
    int32_t nsp, nrc;
    double W[kT2MaxSp];
    double thermo[kT2MaxSp][17];  // Tlow, Tcommon, Thigh, low a0..a6, high a0..a6
    T2Rxn rxn[kT2MaxRxn];
    double eff_val[kT2MaxEff];
    int8_t eff_idx[kT2MaxEff];
};

template <int N, int B>
struct T2Cell {
    static constexpr int TI = N - 1;
    static constexpr bool kAssemblesA = false;
    static constexpr int kJ = 0, kF = N * N, kC = kF + N, kG = kC + N, kD = kG + N;
    static constexpr int kSlots = kD + N;   // doubles per thread
    const T2Mech &m;
    double *s;     // this thread's first slot
    int nsp;
    int piv[N];

    __device__ T2Cell(const T2Mech &mm, double *smem, int tid) : m(mm), s(smem + tid), nsp(mm.nsp) {}

    __device__ __forceinline__ double &S(int k) const { return s[k * B]; }
    __device__ __forceinline__ double &Jm(int i, int j) const { return s[(i * N + j) * B]; }
    __device__ __forceinline__ double F(int i) const { return s[(kF + i) * B]; }
    __device__ __forceinline__ double W(int i) const { return m.W[i]; }

    // molar thermo of species i (mech.cuh species_thermo, JANAF.cpp:142-219)
    __device__ __forceinline__ void thermo(int i, double T, double logT, bool gibbs, double &o1,
                                           double &o2, double &o3) const {
        const double *th = m.thermo[i];
        const double tl = th[0], tc = th[1], thh = th[2];
        const double *a = (T < tc) ? &th[3] : &th[10];
        const double a0 = a[0], a1 = a[1], a2 = a[2], a3 = a[3], a4 = a[4], a5 = a[5], a6 = a[6];
        const double W = m.W[i];
        const bool out = (T < tl || T > thh);
        const double T0 = out ? hmin(hmax(T, tl), thh) : T;
        const double cp0 = ((((a4 * T0 + a3) * T0 + a2) * T0 + a1) * T0 + a0);
        if (gibbs) {
            const double lT = (T > kTiny) ? logT : log(kTiny);
            const double s0 = ((((a4 / 4.0 * T + a3 / 3.0) * T + a2 / 2.0) * T + a1) * T + a0 * lT + a6);
            const double g0 = (((((-a4 / 20.0 * T - a3 / 12.0) * T - a2 / 6.0) * T - a1 / 2.0) * T +
                                a0 * (1 - lT) - a6) * T + a5);
            const double ds0 = (a0 / hmax(T, kTiny) + a1 + (a2 + (a3 + a4 * T) * T) * T);
            o1 = g0 * W;                        // G0
            o2 = (cp0 - (s0 + T * ds0)) * W;    // dG0/dT
        } else {
            double h0 = ((((a4 / 5.0 * T0 + a3 / 4.0) * T0 + a2 / 3.0) * T0 + a1 / 2.0) * T0 + a0) * T0 + a5;
            if (out) h0 += cp0 * (T - T0);
            o1 = cp0 * W;
            o2 = h0 * W;
            o3 = (a1 + T * (2.0 * a2 + T * (3.0 * a3 + 4.0 * a4 * T))) * W;
        }
    }

    __device__ __forceinline__ void evaluate(const double (&y)[N], bool jac) {
        const double T = y[TI];
        const double logT = log(T);
        const double Tm = hmax(T, kTiny);
        const double invT = 1.0 / Tm;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            if (i < nsp) S(kC + i) = hmax(y[i], 0.0);
            S(kF + i) = 0.0;
        }
        if (jac) {
#pragma unroll
            for (int k = 0; k < N * N; ++k) s[k * B] = 0.0;
        }
        for (int i = 0; i < nsp; ++i) {
            double g, d, unused;
            thermo(i, T, logT, true, g, d, unused);
            S(kG + i) = g;
            S(kD + i) = d;
        }
        const double patm_rt = kPatm / (kRu * T);
        for (int r = 0; r < m.nrc; ++r) {
            const T2Rxn &R = m.rxn[r];
            const int type = R.type, nf = R.nf, nb = R.nb;
            int fi[kMaxSide], bi[kMaxSide];
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k) {
                fi[k] = R.fidx[k];
                bi[k] = R.bidx[k];
            }
            double M = 0.0;
            if (type != kArrhenius)
                for (int e = R.eff_begin; e < R.eff_end; ++e) M += m.eff_val[e] * S(kC + m.eff_idx[e]);
            double kf, k0 = 0.0, kinf = 0.0, Pr = 0.0, F = 1.0, lf = 0.0;
            if (type == kArrhenius) {
                kf = arrK_log(R.A, R.b, R.Ta, T, logT);
            } else if (type == kThirdBody) {
                kf = M * arrK_log(R.A, R.b, R.Ta, T, logT);
            } else {
                k0 = arrK_log(R.A0, R.b0, R.Ta0, T, logT);
                kinf = arrK_log(R.A, R.b, R.Ta, T, logT);
                Pr = k0 / notZeroD(kinf) * M;
                if (type != kLindemann)
                    lf = troe_logfcent_p(R.troe[0], R.troe[1], R.troe[2], R.troe[3], type == kTroe4, T);
                F = fall_F(type, lf, Pr);
                kf = kinf * (Pr / (1.0 + Pr)) * F;
            }
            double kr = 0.0, Kc = 0.0, DKcDT = 0.0;
            if (R.rev) {
                // equilibrium constant (mech.cuh equilibrium(), reactionTypes.cpp:178-241)
                double kp = 0.0, dk = 0.0;
#pragma unroll
                for (int k = 0; k < kMaxSide; ++k)
                    if (k < nf) {
                        const double G = S(kG + fi[k]);
                        kp -= G * R.fnu[k];
                        dk -= (S(kD + fi[k]) - G / Tm) * R.fnu[k];
                    }
#pragma unroll
                for (int k = 0; k < kMaxSide; ++k)
                    if (k < nb) {
                        const double G = S(kG + bi[k]);
                        kp += G * R.bnu[k];
                        dk += (S(kD + bi[k]) - G / Tm) * R.bnu[k];
                    }
                kp /= (Tm * kRu);
                double Kp = exp(-kp);
                if (!finite(Kp)) Kp = kRootVeryLarge;
                dk /= (Tm * kRu);
                double DKp = Kp * dk;
                if (!finite(DKp)) DKp = kVeryLarge;
                const double sst = R.sum_stoi;
                if (fabs(sst) < kVeryTiny) {
                    Kc = Kp;
                    DKcDT = DKp;
                } else {
                    const double fs = pow_n(patm_rt, sst);
                    Kc = hmin(Kp * fs, kVeryLarge);
                    double v = (DKp + Kp * (-sst) / T) * fs;
                    if (!finite(v)) v = kVeryLarge;
                    DKcDT = v;
                }
                kr = (fabs(Kc) > kVeryTiny) ? kf / Kc : 0.0;
            }
            double pf[kMaxSide], pb[kMaxSide];
            double qf = kf, qr = kr;
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k) {
                pf[k] = 1.0;
                pb[k] = 1.0;
                if (k < nf) {
                    pf[k] = pow_n(S(kC + fi[k]), R.ford[k]);
                    qf *= pf[k];
                }
                if (k < nb) {
                    pb[k] = pow_n(S(kC + bi[k]), R.bord[k]);
                    qr *= pb[k];
                }
            }
            const double q = qf - qr;
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k)
                if (k < nf) S(kF + fi[k]) -= R.fnu[k] * q;
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k)
                if (k < nb) S(kF + bi[k]) += R.bnu[k] * q;
            if (!jac) continue;
            // DqDci (reactionTypes.cpp:354-445)
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k) {
                if (k < nf) {
                    double d = kf;
#pragma unroll
                    for (int j = 0; j < kMaxSide; ++j) {
                        if (j < nf) {
                            const double ord = R.ford[j];
                            const double cj = S(kC + fi[j]);
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
                        if (j < nf) Jm(fi[j], fi[k]) -= R.fnu[j] * d;
#pragma unroll
                    for (int j = 0; j < kMaxSide; ++j)
                        if (j < nb) Jm(bi[j], fi[k]) += R.bnu[j] * d;
                }
            }
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k) {
                if (k < nb) {
                    double d = kr;
#pragma unroll
                    for (int j = 0; j < kMaxSide; ++j) {
                        if (j < nb) {
                            const double ord = R.bord[j];
                            const double cj = S(kC + bi[j]);
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
                        if (j < nf) Jm(fi[j], bi[k]) += R.fnu[j] * d;
#pragma unroll
                    for (int j = 0; j < kMaxSide; ++j)
                        if (j < nb) Jm(bi[j], bi[k]) -= R.bnu[j] * d;
                }
            }
            double dgdT = 0.0;
            double g = 0.0;   // d q / d c_i = eff_i * g (third body / fall-off)
            bool rank1 = false;
            if (type == kThirdBody) {
                g = q / hmax(M, kTiny);
                rank1 = true;
            } else if (type != kArrhenius && M > kTiny) {
                // unimolecularFallOffRR::gamDGamDCi / gamDGamDT (unimolecularFallOffRR.cpp:55-91)
                const double Pr2 = k0 * M / notZeroD(kinf);
                const double F2 = fall_F(type, lf, Pr2);
                const double fabc = troe_dfdci_factor(type, lf, Pr2, F2);
                g = q * (k0 / notZeroD(kinf)) * (1.0 / (Pr2 * (1 + Pr2)) + fabc * (1.0 / Pr2) / F2);
                rank1 = finite(g);
                const double dPrdT = Pr2 * ((k0 * invT * (R.b0 + R.Ta0 * invT)) / notZeroD(k0) -
                                            (kinf * invT * (R.b + R.Ta * invT)) / notZeroD(kinf));
                const double dFdT = troe_dfdt_p(type, R.troe[0], R.troe[1], R.troe[2], R.troe[3],
                                                T, Pr2, F2, dPrdT);
                dgdT = q * (dPrdT / (Pr2 * (1 + Pr2)) + dFdT / F2);
            }
            if (rank1) {
                for (int e = R.eff_begin; e < R.eff_end; ++e) {
                    const int i = m.eff_idx[e];
                    const double ge = m.eff_val[e] * g;
#pragma unroll
                    for (int j = 0; j < kMaxSide; ++j)
                        if (j < nf) Jm(fi[j], i) -= R.fnu[j] * ge;
#pragma unroll
                    for (int j = 0; j < kMaxSide; ++j)
                        if (j < nb) Jm(bi[j], i) += R.bnu[j] * ge;
                }
            }
            // DqDT (reactionTypes.cpp:843-876)
            double dkfdT;
            if (type == kArrhenius || type == kThirdBody) dkfdT = kf * invT * (R.b + R.Ta * invT);
            else dkfdT = (Pr / (1.0 + Pr)) * F * (kinf * invT * (R.b + R.Ta * invT));
            double dkrdT = R.rev ? (dkfdT - kr * DKcDT) / hmax(Kc, kVeryTiny) : 0.0;
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k) {
                if (k < nf) dkfdT *= pf[k];
                if (k < nb) dkrdT *= pb[k];
            }
            double dqjdT = dkfdT - dkrdT;
            if (!finite(dqjdT)) dqjdT = 0;
            if (!finite(dgdT)) dgdT = 0;
            const double dq = dqjdT + dgdT;
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k)
                if (k < nf) Jm(fi[k], TI) -= R.fnu[k] * dq;
#pragma unroll
            for (int k = 0; k < kMaxSide; ++k)
                if (k < nb) Jm(bi[k], TI) += R.bnu[k] * dq;
        }
        // temperature equation of the constant-pressure reactor
        double cp[N], h[N];
        double cCp = 0.0, DTdt = 0.0, dcCpdT = 0.0;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            cp[i] = 0.0;
            h[i] = 0.0;
            if (i < nsp) {
                double dcp;
                thermo(i, T, logT, false, cp[i], h[i], dcp);
                cCp += y[i] * cp[i];
                dcCpdT += y[i] * dcp;
                DTdt += S(kF + i) * h[i];
            }
        }
        DTdt /= cCp;
        S(kF + TI) = -DTdt;
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
            if (i < nsp) dd -= (cp[i] * S(kF + i) + h[i] * Jm(i, TI));
        dd += dcCpdT * DTdt;
        dd /= cCp;
        Jm(TI, TI) = dd;
    }

    // I - dt J, then LU with partial pivoting, right-looking, in place
    __device__ __forceinline__ void factor(double dt) {
#pragma unroll
        for (int i = 0; i < N; ++i)
#pragma unroll
            for (int j = 0; j < N; ++j) Jm(i, j) = -dt * Jm(i, j) + (i == j ? 1.0 : 0.0);
#pragma unroll
        for (int k = 0; k < N; ++k) {
            double amax = fabs(Jm(k, k));
            int p = k;
#pragma unroll
            for (int i = k + 1; i < N; ++i) {
                const double v = fabs(Jm(i, k));
                if (v > amax) {
                    amax = v;
                    p = i;
                }
            }
            piv[k] = p;
            if (p != k) {
                double *rp = s + p * (N * B);
#pragma unroll
                for (int j = 0; j < N; ++j) {
                    const double t = Jm(k, j);
                    Jm(k, j) = rp[j * B];
                    rp[j * B] = t;
                }
            }
            const double inv = 1.0 / Jm(k, k);
            double u[N];
#pragma unroll
            for (int j = k + 1; j < N; ++j) u[j] = Jm(k, j);
#pragma unroll
            for (int i = k + 1; i < N; ++i) {
                const double l = Jm(i, k) * inv;
                Jm(i, k) = l;
#pragma unroll
                for (int j = k + 1; j < N; ++j) Jm(i, j) -= l * u[j];
            }
        }
    }

    // LUBacksubstituteDPivoting (LUDecompose.hpp:68-100)
    __device__ __forceinline__ void solve(double (&b)[N]) {
#pragma unroll
        for (int k = 0; k + 1 < N; ++k) {
            const int p = piv[k];
#pragma unroll
            for (int i = k + 1; i < N; ++i) {
                if (p == i) {
                    const double t = b[k];
                    b[k] = b[i];
                    b[i] = t;
                }
            }
        }
#pragma unroll
        for (int i = 1; i < N; ++i) {
            double sum = 0.0;
#pragma unroll
            for (int t = 0; t < i; ++t) sum += Jm(i, t) * b[t];
            b[i] -= sum;
        }
#pragma unroll
        for (int i = N - 1; i >= 0; --i) {
            double sum = 0.0;
#pragma unroll
            for (int t = i + 1; t < N; ++t) sum += Jm(i, t) * b[t];
            b[i] = (b[i] - sum) / Jm(i, i);
        }
    }
};

template <int N, int B>
__global__ void __launch_bounds__(B)
integrate_t2_kernel(const __grid_constant__ T2Mech m, const __grid_constant__ IntegratorParams P,
                    const __grid_constant__ CellIO io, double *ylast) {
    extern __shared__ double smem_t2[];
    T2Cell<N, B> cell(m, smem_t2, threadIdx.x);
    t1_run<N>(cell, P, io, ylast);
}

}  // namespace hc
