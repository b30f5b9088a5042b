// Device-side mechanism tables and the per-species / per-reaction kinetics
// functions shared by the integrator, source-term and property kernels.
//
// Every function restates the reference's CPU formula (file:line cited at
// each) in FP64. Floating-point operations keep the reference's order where
// that is natural on the GPU; remaining differences are the CUDA libm
// (exp/log/pow within a few ulp of glibc), FMA contraction and the fused
// Arrhenius form noted at arrK_log.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace hc {

constexpr double kTiny = 1.0e-15;          // doubleRealTiny (doubleReal.hpp:43)
constexpr double kVeryTiny = 1.0e-300;     // doubleRealVeryTiny
constexpr double kVeryLarge = 1.0e+300;    // doubleRealVeryLarge
constexpr double kRootVeryLarge = 1.0e+150;
constexpr double kPatm = 1.01325e5;        // physicalConstant.hpp:186
// Ru = (kB * NA) * 1e3 [J/kmol/K], evaluated like physicalConstant.hpp:158,183
constexpr double kRu = (1.380649e-23 * 6.02214076e23) * 1e3;
constexpr int kMaxSide = 4;

enum RateType : int32_t { kArrhenius = 0, kThirdBody = 1, kLindemann = 2, kTroe3 = 3, kTroe4 = 4 };

struct DevMech {
    int32_t nsp, nrc;
    const double *W;        // [nsp]
    const double *Trange;   // [nsp*3]
    const double *nasa;     // [nsp*14] low a0..a6, high a0..a6 (mass basis)
    const int32_t *rate_type, *reversible;
    const double *arr, *arr0, *troe;  // [nrc*3], [nrc*3], [nrc*4]
    const double *eff;      // [nrc*nsp]
    const int32_t *nf, *nb; // [nrc]
    const int32_t *fidx, *bidx;       // [nrc*4]
    const double *ford, *bord;        // [nrc*4]
    const double *fnu, *bnu;          // [nrc*4]
    const double *sum_stoi;           // [nrc]
    // participation lists per species (sorted by reaction): coef = -fnu (reactant) / +bnu (product)
    const int32_t *sp_ptr;  // [nsp+1]
    const int32_t *sp_rxn;  // [npart]
    const double *sp_coef;  // [npart]
    // kinetic-theory transport
    const int32_t *geom;
    const double *eps_k, *sigma;
    // pair constants of the mixture-averaged transport, [nsp*nsp] (i*nsp + j)
    const double *pair_D;     // 1.858e-7 sqrt(1/Wi + 1/Wj) / sigma_ij^2 * Patm
    const double *pair_Dpow;  // (1/sqrt(eps_i eps_j))^-0.145
    const double *pair_r;     // 1/sqrt(eps_i eps_j)
    const double *pair_phi;   // (1/sqrt 8) / sqrt(1 + Wi/Wj)
    const double *pair_w;     // sqrt(Wi/Wj)
};

template <typename V>
__device__ __forceinline__ V ldg(const V *p) {
    return __ldg(p);
}

__device__ __forceinline__ double hmax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double hmin(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double notZeroD(double s) { return (s != 0) ? s : kVeryTiny; }
__device__ __forceinline__ bool finite(double x) { return !isnan(x) && !isinf(x); }

// x^y, with the exponents mechanisms use in practice done exactly as a
// correctly rounded pow returns them (y = 1: x; y = 2: one rounded multiply;
// y = 0: 1; y = -1: one rounded division); any other exponent calls pow().
__device__ __forceinline__ double pow_n(double x, double y) {
    if (y == 1.0) return x;
    if (y == 2.0) return x * x;
    if (y == 0.0) return 1.0;
    if (y == -1.0) return 1.0 / x;
    return pow(x, y);
}

__device__ __forceinline__ double conc_pow(double c, double ord) {
    return pow_n(hmax(c, 0.0), ord);
}

// ---------------------------------------------------------------- thermo
// JANAF (thermo/src/JANAF.cpp:142-219, thermo/include/JANAF.inl:33-86).
struct SpeciesThermo {
    double cp;     // molar Cp  (Cp0 = cp0 * W, thermo.inl:44)
    double h;      // molar H   (Ha0)
    double dcp;    // molar dCp/dT (JANAF::Dcp_pDT * W)
    double G0;     // molar Gibbs (JANAF::g0 * W)
    double DG0DT;  // molar dG/dT (thermo.inl:197-203)
};

__device__ __forceinline__ SpeciesThermo species_thermo(const DevMech &m, int i, double T,
                                                        double logT) {
    const double tl = ldg(&m.Trange[3 * i]), tc = ldg(&m.Trange[3 * i + 1]);
    const double th = ldg(&m.Trange[3 * i + 2]);
    const double *a = (T < tc) ? &m.nasa[14 * i] : &m.nasa[14 * i + 7];
    const double a0 = ldg(&a[0]), a1 = ldg(&a[1]), a2 = ldg(&a[2]), a3 = ldg(&a[3]);
    const double a4 = ldg(&a[4]), a5 = ldg(&a[5]), a6 = ldg(&a[6]);
    const double W = ldg(&m.W[i]);
    const bool out = (T < tl || T > th);
    const double T0 = out ? hmin(hmax(T, tl), th) : T;
    const double cp0 = ((((a4 * T0 + a3) * T0 + a2) * T0 + a1) * T0 + a0);
    double h0 = ((((a4 / 5.0 * T0 + a3 / 4.0) * T0 + a2 / 3.0) * T0 + a1 / 2.0) * T0 + a0) * T0 + a5;
    if (out) h0 += cp0 * (T - T0);
    // s0 and g0 use the unclamped T (JANAF.cpp:201-213); log(max(T, tiny))
    const double lT = (T > kTiny) ? logT : log(kTiny);
    const double s0 = ((((a4 / 4.0 * T + a3 / 3.0) * T + a2 / 2.0) * T + a1) * T + a0 * lT + a6);
    const double g0 = (((((-a4 / 20.0 * T - a3 / 12.0) * T - a2 / 6.0) * T - a1 / 2.0) * T +
                        a0 * (1 - lT) - a6) * T + a5);
    const double ds0 = (a0 / hmax(T, kTiny) + a1 + (a2 + (a3 + a4 * T) * T) * T);
    const double dcp = (a1 + T * (2.0 * a2 + T * (3.0 * a3 + 4.0 * a4 * T)));
    SpeciesThermo r;
    r.cp = cp0 * W;
    r.h = h0 * W;
    r.dcp = dcp * W;
    r.G0 = g0 * W;
    r.DG0DT = (cp0 - (s0 + T * ds0)) * W;
    return r;
}

// mass-basis cp0 and ha0 only (property kernels)
__device__ __forceinline__ void species_cp_h(const DevMech &m, int i, double T, double &cp,
                                             double &h) {
    const double tl = ldg(&m.Trange[3 * i]), tc = ldg(&m.Trange[3 * i + 1]);
    const double th = ldg(&m.Trange[3 * i + 2]);
    const double *a = (T < tc) ? &m.nasa[14 * i] : &m.nasa[14 * i + 7];
    const double a0 = ldg(&a[0]), a1 = ldg(&a[1]), a2 = ldg(&a[2]), a3 = ldg(&a[3]);
    const double a4 = ldg(&a[4]), a5 = ldg(&a[5]);
    const bool out = (T < tl || T > th);
    const double T0 = out ? hmin(hmax(T, tl), th) : T;
    cp = ((((a4 * T0 + a3) * T0 + a2) * T0 + a1) * T0 + a0);
    h = ((((a4 / 5.0 * T0 + a3 / 4.0) * T0 + a2 / 3.0) * T0 + a1 / 2.0) * T0 + a0) * T0 + a5;
    if (out) h += cp * (T - T0);
}

// ---------------------------------------------------------------- rate laws
// ArrheniusRR::k (ArrheniusRR.cpp:37-47), A T^b e^{-Ta/T}, evaluated as one
// exponential of b ln T - Ta/T with ln T shared by all reactions of a cell.
__device__ __forceinline__ double arrK_log(double A, double b, double Ta, double T, double logT) {
    double e = 0.0;
    if (fabs(b) > kVeryTiny) e = b * logT;
    if (fabs(Ta) > kVeryTiny) e -= Ta / T;
    return A * exp(e);
}

__device__ __forceinline__ double troe_logfcent(const double *tr, bool four, double T) {
    const double alpha = ldg(&tr[0]), Tsss = ldg(&tr[1]), Ts = ldg(&tr[2]), Tss = ldg(&tr[3]);
    double s = (1.0 - alpha) * exp(-T / Tsss) + alpha * exp(-T / Ts);
    if (four) s += exp(-Tss / T);
    return log10(hmax(s, kTiny));
}

// fallOffFunctions.cpp:81-100 (Troe::F); Lindemann F = 1
__device__ __forceinline__ double fall_F(int type, double logFcent, double Pr) {
    if (type == kLindemann) return 1.0;
    const double c = -0.4 - 0.67 * logFcent;
    const double n = 0.75 - 1.27 * logFcent;
    const double d = 0.14;
    const double logPr = log10(hmax(Pr, kTiny));
    const double x = (logPr + c) / (n - d * (logPr + c));
    return pow(10.0, logFcent / (1.0 + x * x));
}

// The Pr-independent product of Troe::DFDci (fallOffFunctions.cpp:102-129):
// DFDci = [F * A * B * C] * (1/Pr * dPr/dci); returns F*A*B*C.
__device__ __forceinline__ double troe_dfdci_factor(int type, double logFcent, double Pr,
                                                    double F) {
    if (type == kLindemann) return 0.0;
    const double logPr = log10(hmax(Pr, kTiny));
    const double c = -0.4 - 0.67 * logFcent;
    const double n = 0.75 - 1.27 * logFcent;
    const double d = 0.14;
    const double logPrpc = logPr + c;
    const double nm = n - d * logPrpc;
    const double inv = logPrpc / nm;
    const double s1 = 1.0 + inv * inv;
    return F * ((-logFcent) / (s1 * s1)) * (2.0 * logPrpc / (nm * nm)) * (1.0 + d * inv);
}

// Troe::DFDT (fallOffFunctions.cpp:131-157)
__device__ __forceinline__ double troe_dfdt(int type, const double *tr, double T, double Pr,
                                            double F, double DPrDT) {
    if (type == kLindemann) return 0.0;
    const double alpha = ldg(&tr[0]), Tsss = ldg(&tr[1]), Ts = ldg(&tr[2]), Tss = ldg(&tr[3]);
    const double ln10 = log(10.0);
    const double logPr = log10(hmax(Pr, kTiny));
    double Fcent, DFcentDT;
    const double e1 = exp(-T / Tsss), e2 = exp(-T / Ts);
    if (type == kTroe3) {
        Fcent = hmax((1.0 - alpha) * e1 + alpha * e2, kTiny);
        DFcentDT = (1.0 - alpha) * e1 / (-Tsss) + alpha * e2 / (-Ts);
    } else {
        const double e3 = exp(-Tss / T);
        Fcent = hmax((1.0 - alpha) * e1 + alpha * e2 + e3, kTiny);
        DFcentDT = (1.0 - alpha) * e1 / (-Tsss) + alpha * e2 / (-Ts) + e3 * (Tss / (T * T));
    }
    const double logFcent = log10(Fcent);
    const double DlogFcentDT = 1.0 / (Fcent * ln10) * DFcentDT;
    const double c = -0.4 - 0.67 * logFcent;
    const double DcDT = -0.67 * DlogFcentDT;
    const double n = 0.75 - 1.27 * logFcent;
    const double DnDT = -1.27 * DlogFcentDT;
    const double d = 0.14;
    const double dlogPrDT = DPrDT / Pr / ln10;
    const double logPrpc = logPr + c;
    const double nm = n - d * logPrpc;
    const double inv = logPrpc / nm;
    const double dPPDT =
        2.0 * logPrpc / (nm * nm) * ((dlogPrDT + DcDT) - logPrpc / nm * (DnDT - d * (dlogPrDT + DcDT)));
    const double s1 = 1.0 + inv * inv;
    return (F * ln10 * (DlogFcentDT / s1 - logFcent / (s1 * s1) * dPPDT));
}

// Equilibrium constants (reactionTypes.cpp:178-241) from molar G0 / DG0DT
// read through accessors (shared memory layouts differ between kernels).
struct EquilK {
    double Kc, DKcDT;
};

template <typename GAt, typename DAt>
__device__ __forceinline__ EquilK equilibrium(const DevMech &m, int r, double T, GAt G0, DAt DG0) {
    double kp = 0.0, dk = 0.0;
    const double Tm = hmax(T, kTiny);
    const int nf = ldg(&m.nf[r]), nb = ldg(&m.nb[r]);
#pragma unroll
    for (int k = 0; k < kMaxSide; ++k) {
        if (k < nf) {
            const int i = ldg(&m.fidx[kMaxSide * r + k]);
            const double nu = ldg(&m.fnu[kMaxSide * r + k]);
            const double G = G0(i);
            kp -= G * nu;
            dk -= (DG0(i) - G / Tm) * nu;
        }
    }
#pragma unroll
    for (int k = 0; k < kMaxSide; ++k) {
        if (k < nb) {
            const int i = ldg(&m.bidx[kMaxSide * r + k]);
            const double nu = ldg(&m.bnu[kMaxSide * r + k]);
            const double G = G0(i);
            kp += G * nu;
            dk += (DG0(i) - G / Tm) * nu;
        }
    }
    kp /= (Tm * kRu);
    double Kp = exp(-kp);
    if (!finite(Kp)) Kp = kRootVeryLarge;
    dk /= (Tm * kRu);
    double DKp = Kp * dk;
    if (!finite(DKp)) DKp = kVeryLarge;
    const double s = ldg(&m.sum_stoi[r]);
    EquilK e;
    if (fabs(s) < kVeryTiny) {
        e.Kc = Kp;
        e.DKcDT = DKp;
    } else {
        const double f = pow_n(kPatm / (kRu * T), s);
        e.Kc = hmin(Kp * f, kVeryLarge);
        double v = (DKp + Kp * (-s) / T) * f;
        if (!finite(v)) v = kVeryLarge;
        e.DKcDT = v;
    }
    return e;
}

}  // namespace hc
