// Device helpers of the direct-assembly thread-per-cell kernel (kernel 5),
// generated per mechanism by jit_t3.cu and compiled with NVRTC. The common
// path of that kernel is straight-line code with every mechanism constant a
// literal; the helpers here are the rare paths, kept out of line so that
// they cost the common path neither instructions nor instruction-cache room:
//   * species thermo when T lies outside a species' fitted range (cp and h
//     clamped / extrapolated as the reference does);
//   * the equilibrium constant when ln Kc is so large in magnitude that the
//     reference's own overflow clamps apply;
//   * the fall-off function F and its derivatives (Troe, Lindemann).
#pragma once

#include "rtc_base.cuh"

namespace hc {

// JANAF (thermo/src/JANAF.cpp:142-219, thermo/include/JANAF.inl:33-86) for one
// species from its mass-basis coefficients a[0..6] of the range T selects:
// molar cp and h at the clamped temperature (h extrapolated linearly beyond
// the range), dcp/dT, and the two Gibbs terms the rates use: g = G0 / (Ru Tm)
// and dgt = DG0/DT - G0 / Tm (thermo.inl:189-203), both at the unclamped T.
static __device__ __noinline__ void t3_thermo_slow(const double *a, double tl, double th, double W,
                                                   double T, double logT, double invRuT,
                                                   double &cp, double &h, double &dcp, double &g,
                                                   double &dgt) {
    const double a0 = a[0], a1 = a[1], a2 = a[2], a3 = a[3], a4 = a[4], a5 = a[5], a6 = a[6];
    const bool out = (T < tl || T > th);
    const double T0 = out ? hmin(hmax(T, tl), th) : T;
    const double cp0 = ((((a4 * T0 + a3) * T0 + a2) * T0 + a1) * T0 + a0);
    double h0 = ((((a4 / 5.0 * T0 + a3 / 4.0) * T0 + a2 / 3.0) * T0 + a1 / 2.0) * T0 + a0) * T0 + a5;
    if (out) h0 += cp0 * (T - T0);
    const double lT = (T > kTiny) ? logT : log(kTiny);
    const double s0 = ((((a4 / 4.0 * T + a3 / 3.0) * T + a2 / 2.0) * T + a1) * T + a0 * lT + a6);
    const double g0 = (((((-a4 / 20.0 * T - a3 / 12.0) * T - a2 / 6.0) * T - a1 / 2.0) * T +
                        a0 * (1 - lT) - a6) * T + a5);
    const double Tm = hmax(T, kTiny);
    const double ds0 = (a0 / Tm + a1 + (a2 + (a3 + a4 * T) * T) * T);
    cp = cp0 * W;
    h = h0 * W;
    dcp = (a1 + T * (2.0 * a2 + T * (3.0 * a3 + 4.0 * a4 * T))) * W;
    const double G0 = g0 * W;
    const double DG0 = (cp0 - (s0 + T * ds0)) * W;
    g = G0 * invRuT;
    dgt = DG0 - G0 / Tm;
}

// reactionTypes::Kc / ::DKcDT (reactionTypes.cpp:178-241) with their overflow
// clamps, from kp = sum nu G0 / (Tm Ru) and dk = sum nu (DG0/DT - G0/Tm) / (Tm Ru)
static __device__ __noinline__ void t3_kc_slow(double kp, double dk, double s, double T, double &Kc,
                                               double &DKcDT) {
    double Kp = exp(-kp);
    if (isnan(Kp) || isinf(Kp)) Kp = kRootVeryLarge;
    double DKp = Kp * dk;
    if (isnan(DKp) || isinf(DKp)) DKp = kVeryLarge;
    if (fabs(s) < kVeryTiny) {
        Kc = Kp;
        DKcDT = DKp;
    } else {
        const double fs = pow(kPatm / (kRu * T), s);
        Kc = hmin(Kp * fs, kVeryLarge);
        double v = (DKp + Kp * (-s) / T) * fs;
        if (isnan(v) || isinf(v)) v = kVeryLarge;
        DKcDT = v;
    }
}

// log10 of the Troe centering factor (fallOffFunctions.cpp:81-100)
static __device__ __noinline__ double t3_troe_logfcent(double alpha, double Tsss, double Ts,
                                                       double Tss, int four, double T) {
    return troe_logfcent_p(alpha, Tsss, Ts, Tss, four != 0, T);
}

// Troe::F (fallOffFunctions.cpp:81-100); Lindemann F = 1
static __device__ __noinline__ double t3_fall_F(int type, double logFcent, double Pr) {
    return fall_F(type, logFcent, Pr);
}

// the fall-off reaction's derivative pieces (unimolecularFallOffRR::gamDGamDCi,
// ::gamDGamDT, unimolecularFallOffRR.cpp:55-91, with Troe::DFDci / ::DFDT,
// fallOffFunctions.cpp:102-157) for q = kinf Pr/(1+Pr) F ...:
//   gq   = q (k0/kinf) (1/(Pr(1+Pr)) + F'/(Pr F)), so that the column of
//          species i gets eff_i * gq (rank one in the efficiencies);
//   dgdT = q (dPr/dT / (Pr(1+Pr)) + dF/dT / F).
// Both are zero when M <= tiny, as in the reference.
static __device__ __noinline__ void t3_falloff_jac(int type, double alpha, double Tsss,
                                                   double Ts, double Tss, double k0,
                                                   double kinf, double b0, double Ta0, double b,
                                                   double Ta, double M, double lf, double q,
                                                   double T, double invT, double &gq,
                                                   double &dgdT) {
    gq = 0.0;
    dgdT = 0.0;
    if (!(M > kTiny)) return;
    const double Pr2 = k0 * M / notZeroD(kinf);
    const double F2 = fall_F(type, lf, Pr2);
    const double fabc = troe_dfdci_factor(type, lf, Pr2, F2);
    double g = q * (k0 / notZeroD(kinf)) * (1.0 / (Pr2 * (1 + Pr2)) + fabc * (1.0 / Pr2) / F2);
    gq = finite(g) ? g : 0.0;
    const double dPrdT = Pr2 * ((k0 * invT * (b0 + Ta0 * invT)) / notZeroD(k0) -
                                (kinf * invT * (b + Ta * invT)) / notZeroD(kinf));
    const double dFdT = troe_dfdt_p(type, alpha, Tsss, Ts, Tss, T, Pr2, F2, dPrdT);
    const double d = q * (dPrdT / (Pr2 * (1 + Pr2)) + dFdT / F2);
    dgdT = finite(d) ? d : 0.0;
}

}  // namespace hc

namespace hc {

// Troe centering factor from its three exponentials e1 = exp(-T/T***),
// e2 = exp(-T/T*), e3 = exp(-T**/T) (e3 unused by the three-parameter form):
// lf = log10 Fcent, dlf = d lf / dT (fallOffFunctions.cpp:81-157)
struct T3Cent {
    double lf, dlf;
};

__device__ __forceinline__ T3Cent t3_troe_cent(bool four, double alpha, double iTsss, double iTs,
                                               double Tss, double e1, double e2, double e3,
                                               double invT) {
    double Fc = (1.0 - alpha) * e1 + alpha * e2;
    double dFc = (1.0 - alpha) * e1 * (-iTsss) + alpha * e2 * (-iTs);
    if (four) {
        Fc += e3;
        dFc += e3 * (Tss * invT * invT);
    }
    Fc = hmax(Fc, kTiny);
    T3Cent r;
    r.lf = log10(Fc);
    r.dlf = fdiv(dFc, Fc * 2.302585092994045684);
    return r;
}

// Troe::F at log10 Pr (fallOffFunctions.cpp:81-100)
__device__ __forceinline__ double t3_troe_F(double lf, double logPr) {
    const double c = -0.4 - 0.67 * lf;
    const double n = 0.75 - 1.27 * lf;
    const double x = fdiv(logPr + c, n - 0.14 * (logPr + c));
    return exp10(lf / (1.0 + x * x));
}

// the fall-off reaction's Jacobian pieces (as t3_falloff_jac) from the
// quantities the rate evaluation already holds: F and log10 Pr at Pr, the
// centering factor and its T derivative (Troe::DFDci, ::DFDT,
// fallOffFunctions.cpp:102-157; unimolecularFallOffRR::gamDGamDCi,
// ::gamDGamDT, unimolecularFallOffRR.cpp:55-91); troe = false: Lindemann
__device__ __forceinline__ void t3_falloff_jac_fast(bool troe, T3Cent cent, double F, double logPr,
                                                    double k0, double kinf, double b0, double Ta0,
                                                    double b, double Ta, double M, double q,
                                                    double invT, double &gq, double &dgdT) {
    gq = 0.0;
    dgdT = 0.0;
    if (!(M > kTiny)) return;
    const double ikinf = frcp(notZeroD(kinf));
    const double Pr2 = k0 * M * ikinf;
    const double dPrdT = Pr2 * (fdiv(k0 * invT * (b0 + Ta0 * invT), notZeroD(k0)) -
                                (kinf * invT * (b + Ta * invT)) * ikinf);
    double fabc = 0.0, dFdT = 0.0;
    if (troe) {
        const double ln10 = 2.302585092994045684;
        const double lf = cent.lf, dlf = cent.dlf;
        const double c = -0.4 - 0.67 * lf, n = 0.75 - 1.27 * lf, d = 0.14;
        const double logPrpc = logPr + c;
        const double nm = n - d * logPrpc;
        const double inm = frcp(nm);
        const double inv = logPrpc * inm;
        const double s1 = 1.0 + inv * inv;
        const double is1 = frcp(s1);
        fabc = F * ((-lf) * is1 * is1) * (2.0 * logPrpc * inm * inm) * (1.0 + d * inv);
        const double DcDT = -0.67 * dlf, DnDT = -1.27 * dlf;
        const double dlogPrDT = dPrdT * frcp(Pr2 * ln10);
        const double dPPDT = 2.0 * logPrpc * inm * inm *
                             ((dlogPrDT + DcDT) - logPrpc * inm * (DnDT - d * (dlogPrDT + DcDT)));
        dFdT = F * ln10 * (dlf * is1 - lf * is1 * is1 * dPPDT);
    }
    const double iP = frcp(Pr2 * (1 + Pr2)), iF = frcp(F);
    const double g = q * (k0 * ikinf) * (iP + fabc * frcp(Pr2) * iF);
    gq = finite(g) ? g : 0.0;
    const double dd = q * (dPrdT * iP + dFdT * iF);
    dgdT = finite(dd) ? dd : 0.0;
}

}  // namespace hc

namespace hc {

// x^nu for the small stoichiometric coefficients of 1/Kc products
__device__ __forceinline__ double pow_small(double x, double nu) {
    if (nu == 1.0) return x;
    if (nu == 2.0) return x * x;
    if (nu == 3.0) return x * x * x;
    return pow_out(x, nu);
}

// tables of the compact thread-per-cell kernel (t4_cell.cuh)
struct T4Range {
    double h[5], h5;      // h  = T (h0 + T (h1 + ...)) + h5          (molar, W a_k/(k+1))
    double s0, s[4], s6;  // s  = s0 ln T + T (s1 + T (s2 + ...)) + s6  (W a0, W a_k/k)
    double cp[5];         // cp = cp0 + T (cp1 + ...)                 (W a_k)
    double dcp[4];        // dcp/dT = W (a1 + 2 a2 T + 3 a3 T^2 + 4 a4 T^3)
};

struct T4Species {
    double tl, tc, th, W;
    T4Range lo, hi;
    double raw[2][7];     // mass-basis coefficients for the out-of-range forms
};

struct T4Rxn {
    int type, rev, nf, nb;
    int fi[kMaxSide], bi[kMaxSide];
    double fnu[kMaxSide], bnu[kMaxSide], ford[kMaxSide], bord[kMaxSide];
    double A, b, Ta, A0, b0, Ta0;
    double alpha, iTsss, iTs, Tss;   // Troe (1/T***, 1/T*)
    double Tsss, Ts;                 // Troe as given (out-of-line forms)
    double s;                        // sum of stoichiometric coefficients (products - reactants)
    int eff_begin, eff_end;
};

struct T4Eff {
    int sp;
    double e;
};

}  // namespace hc
