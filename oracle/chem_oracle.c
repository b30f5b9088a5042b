/*
 * chem_oracle.c -- CPU restatement of OpenHurricane's chemistry source-term
 * path, used as the ORACLE of this repository.
 *
 * TEST INFRASTRUCTURE ONLY. Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load this code, as the checker; the product
 * path (libhurchem_b200.so) never calls it.
 *
 * It restates, function by function and in the same floating-point order,
 * the reference's CPU algorithm for one cell:
 *   thermo        thermo/src/JANAF.cpp:142-219, thermo/include/JANAF.inl:33-86,
 *                 thermo/include/thermo.inl:44-203 (molar = mass x W)
 *   rate laws     reactionRateTypes/src/ArrheniusRR.cpp:37-47 (+ hpp:96-99),
 *                 ArrheniusThirdBodyRR.cpp:37-57, unimolecularFallOffRR.cpp:37-91,
 *                 fallOffFunctions.cpp:81-157 (Troe), :54-79 (SRI), fallOffFunctions.hpp
 *                 (Lindemann); reversibleReactionWithRevPars.hpp:68-122 (Chemkin REV);
 *                 logInterpolationRR.cpp:78-226 (PLOG), LandauTellerRR.cpp:37-99 (LT),
 *                 chemicallyActicatedBimolecularRR.cpp:36-96 (HIGH), JanevRR.cpp:37-88 (JAN),
 *                 powerSeriesRateRR.cpp:37-74 (FIT1)
 *   reactions     reactionTypes/src/reactionTypes.cpp:178-352 (Kp, DKpDT, Kc, DKcDT, q),
 *                 :354-445 (DqDci), :843-876 (DqDT); reversibleReactions.hpp:62-127;
 *                 irreversibleReactions.hpp; reactionList.hpp:83-86 (updateG0)
 *   reactor RHS   chemistrySource/src/chemistrySource.cpp:863-907 (DyDt),
 *                 :967-1021 (jacobian), :1152-1164 (checkNewY),
 *                 :1225-1246 (ciToYi), :1494-1556 (cell loop)
 *   integrator    Hurricane/mathematicalTools/ODEs/src/ImplicitEuler.cpp:40-52
 *                 (maxIncrement), :101-142 (solve), :161-251 (NewtonIteration),
 *                 :253-292 (adaptiveSolve), :294-342 (solve over [t0, tn]);
 *                 ODEsSolver.cpp:37-46 (maxError)
 *   linear solve  Hurricane/dataStructure/containers/Matrices/include/SquareMatrix.hpp:185-237
 *                 (LUDecomposeDPivoting), LinearEquations/include/LUDecompose.hpp:68-100
 *                 (LUBacksubstituteDPivoting)
 *   properties    transport/src/kineticTheory.cpp:37-116, kineticTheory.inl:32-34,
 *                 transport/src/transportList.cpp:31-56, :238-284 (muKappa)
 *
 * Built with the reference's own flags (-O3 -mavx2, no FMA contraction) so
 * that, with glibc's exp/log/pow, it reproduces the reference bit for bit on
 * the constant-pressure path; tests/test_oracle_pin.py checks that against
 * the reference compiled from source.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/hurchem_b200.h"

#define TINY 1.0e-15
#define VERY_TINY 1.0e-300
#define VERY_LARGE 1.0e+300
#define ROOT_VERY_LARGE 1.0e+150

static const double KB = 1.380649e-23;
static const double NA_ = 6.02214076e23;
#define RU ((KB * NA_) * 1e3)
#define PATM 1.01325e5

/* std::max / std::min semantics: max(a,b) = (a < b) ? b : a */
static inline double hmax(double a, double b) { return (a < b) ? b : a; }
static inline double hmin(double a, double b) { return (b < a) ? b : a; }

typedef struct {
    const hc_mech_desc *m;
    double *G0, *DG0DT;     /* [nsp] */
    double p;               /* the cell's pressure (pressure-dependent rate tables) */
} mech_ctx;

/* ---------------- thermo (mass basis coefficients) ---------------- */

static inline const double *coeffs(const hc_mech_desc *m, int i, double T) {
    return (T < m->Trange[3 * i + 1]) ? &m->nasa[14 * i] : &m->nasa[14 * i + 7];
}

static inline double limitT(const hc_mech_desc *m, int i, double T) {
    const double tl = m->Trange[3 * i], th = m->Trange[3 * i + 2];
    if (T < tl || T > th) return hmin(hmax(T, tl), th);
    return T;
}

static double cp0(const hc_mech_desc *m, int i, double T) {
    const double *a = coeffs(m, i, T);
    const double T0 = limitT(m, i, T);
    return ((((a[4] * T0 + a[3]) * T0 + a[2]) * T0 + a[1]) * T0 + a[0]);
}

static double ha0(const hc_mech_desc *m, int i, double T) {
    const double *a = coeffs(m, i, T);
    const double tl = m->Trange[3 * i], th = m->Trange[3 * i + 2];
    if (T < tl || T > th) {
        const double T0 = (T < tl) ? tl : th;
        double h0 = ((((a[4] / 5.0 * T0 + a[3] / 4.0) * T0 + a[2] / 3.0) * T0 + a[1] / 2.0) * T0 +
                     a[0]) * T0 + a[5];
        const double c = ((((a[4] * T0 + a[3]) * T0 + a[2]) * T0 + a[1]) * T0 + a[0]);
        h0 += c * (T - T0);
        return h0;
    }
    return (((((a[4] / 5.0 * T + a[3] / 4.0) * T + a[2] / 3.0) * T + a[1] / 2.0) * T + a[0]) * T +
            a[5]);
}

static double s0(const hc_mech_desc *m, int i, double T) {
    const double *a = coeffs(m, i, T);
    return ((((a[4] / 4.0 * T + a[3] / 3.0) * T + a[2] / 2.0) * T + a[1]) * T +
            a[0] * log(hmax(T, TINY)) + a[6]);
}

static double g0(const hc_mech_desc *m, int i, double T) {
    const double *a = coeffs(m, i, T);
    return (((((-a[4] / 20.0 * T - a[3] / 12.0) * T - a[2] / 6.0) * T - a[1] / 2.0) * T +
             a[0] * (1 - log(hmax(T, TINY))) - a[6]) * T + a[5]);
}

static double Ds0DT(const hc_mech_desc *m, int i, double T) {
    const double *a = coeffs(m, i, T);
    return (a[0] / hmax(T, TINY) + a[1] + (a[2] + (a[3] + a[4] * T) * T) * T);
}

static double Dcp_pDT(const hc_mech_desc *m, int i, double T) {
    const double *a = coeffs(m, i, T);
    return (a[1] + T * (2.0 * a[2] + T * (3.0 * a[3] + 4.0 * a[4] * T)));
}

/* molar quantities (thermo.inl: X0 = x0 * Wi) */
static inline double Cp_p(const hc_mech_desc *m, int i, double T) { return cp0(m, i, T) * m->W[i]; }
static inline double Ha_p(const hc_mech_desc *m, int i, double T) { return ha0(m, i, T) * m->W[i]; }
static inline double DCp_pDT(const hc_mech_desc *m, int i, double T) {
    return Dcp_pDT(m, i, T) * m->W[i];
}
static inline double G0m(const hc_mech_desc *m, int i, double T) { return g0(m, i, T) * m->W[i]; }
static inline double DG0DTm(const hc_mech_desc *m, int i, double T) {
    const double dg = cp0(m, i, T) - (s0(m, i, T) + T * Ds0DT(m, i, T));
    return dg * m->W[i];
}

static void updateG0(mech_ctx *x, double T) {
    for (int i = 0; i < x->m->nsp; ++i) {
        x->G0[i] = G0m(x->m, i, T);
        x->DG0DT[i] = DG0DTm(x->m, i, T);
    }
}

/* ---------------- rate laws ---------------- */

static double arrK(const double *a, double T) {
    double k = a[0];
    if (fabs(a[1]) > VERY_TINY) k *= pow(T, a[1]);
    if (fabs(a[2]) > VERY_TINY) k *= exp(-a[2] / T);
    return k;
}

static double arrDkDT(const double *a, double kj, double T) {
    const double invT = 1.0 / hmax(T, TINY);
    return kj * invT * (a[1] + a[2] * invT);
}

static inline double notZeroD(double s) { return (s != 0) ? s : VERY_TINY; }

static double thirdM(const hc_mech_desc *m, int r, const double *c) {
    double mm = 0.0;
    const double *e = &m->eff[(int64_t)r * m->nsp];
    for (int i = 0; i < m->nsp; ++i) mm += e[i] * c[i];
    return mm;
}

static void troeLogFcent(const double *tr, int four, double T, double *logFcent) {
    const double alpha = tr[0], Tsss = tr[1], Ts = tr[2], Tss = tr[3];
    if (!four)
        *logFcent = log10(hmax((1.0 - alpha) * exp(-T / Tsss) + alpha * exp(-T / Ts), TINY));
    else
        *logFcent = log10(hmax((1.0 - alpha) * exp(-T / Tsss) + alpha * exp(-T / Ts) +
                                   exp(-Tss / T), TINY));
}

/* SRI (fallOffFunctions.cpp:54-79): a, b, c, d, e */
static double sriF(const double *s, double T, double Pr) {
    const double logPr = log10(hmax(Pr, TINY));
    const double X = 1.0 / (1.0 + logPr * logPr);
    return s[3] * pow(s[0] * exp(-s[1] / T) + exp(-T / s[2]), X) * pow(T, s[4]);
}

static double sriDFDci(const double *s, double T, double Pr, double F, double DPrDci) {
    const double lp = log10(hmax(Pr, TINY));
    const double X = 1.0 / (1.0 + lp * lp);
    const double dXdc = -X * X * 2.0 * log10(Pr) / Pr / log(10.0) * DPrDci;
    return (F * dXdc * log(s[0] * exp(-s[1] / T) + exp(-T / s[2])));
}

static double sriDFDT(const double *s, double T, double Pr, double F, double DPrDT) {
    const double lp = log10(hmax(Pr, TINY));
    const double X = 1.0 / (1.0 + lp * lp);
    const double dXdPr = -X * X * 2.0 * log10(Pr) / Pr / log(10.0);
    return (F * (s[4] / T + dXdPr * DPrDT * log(s[0] * exp(-s[1] / T) + exp(-T / s[2])) +
                 X * (s[0] * s[1] * exp(-s[1] / T) / (T * T) - exp(-T / s[2]) / s[2]) /
                     (s[0] * exp(-s[1] / T) + exp(-T / s[2]))));
}

static double fallF(const hc_mech_desc *m, int r, double T, double Pr) {
    const int t = m->rate_type[r];
    if (t == HC_RATE_LINDEMANN) return 1.0;
    if (t == HC_RATE_SRI) return sriF(&m->sri[5 * r], T, Pr);
    double logFcent;
    troeLogFcent(&m->troe[4 * r], t == HC_RATE_TROE4, T, &logFcent);
    const double c = -0.4 - 0.67 * logFcent;
    const double n = 0.75 - 1.27 * logFcent;
    const double d = 0.14;
    const double logPr = log10(hmax(Pr, TINY));
    const double x = (logPr + c) / (n - d * (logPr + c));
    return pow(10.0, logFcent / (1.0 + x * x));
}

static double fallDFDci(const hc_mech_desc *m, int r, double T, double Pr, double F,
                        double DPrDci) {
    const int t = m->rate_type[r];
    if (t == HC_RATE_LINDEMANN) return 0.0;
    if (t == HC_RATE_SRI) return sriDFDci(&m->sri[5 * r], T, Pr, F, DPrDci);
    const double logPr = log10(hmax(Pr, TINY));
    double logFcent;
    troeLogFcent(&m->troe[4 * r], t == HC_RATE_TROE4, T, &logFcent);
    const double c = -0.4 - 0.67 * logFcent;
    const double n = 0.75 - 1.27 * logFcent;
    const double d = 0.14;
    const double logPrpc = logPr + c;
    const double dlogPrpc = d * (logPrpc);
    const double nmdlogPrpc = n - dlogPrpc;
    const double invnmdlogPrpc = logPrpc / nmdlogPrpc;
    const double s1 = 1.0 + invnmdlogPrpc * invnmdlogPrpc;
    return (F * ((-logFcent) / (s1 * s1)) * (2.0 * logPrpc / (nmdlogPrpc * nmdlogPrpc)) *
            (1.0 + d * invnmdlogPrpc) * (1.0 / (Pr)*DPrDci));
}

static double fallDFDT(const hc_mech_desc *m, int r, double T, double Pr, double F,
                       double DPrDT) {
    const int t = m->rate_type[r];
    if (t == HC_RATE_LINDEMANN) return 0.0;
    if (t == HC_RATE_SRI) return sriDFDT(&m->sri[5 * r], T, Pr, F, DPrDT);
    const double *tr = &m->troe[4 * r];
    const double alpha = tr[0], Tsss = tr[1], Ts = tr[2], Tss = tr[3];
    const double ln10 = log(10.0);
    const double logPr = log10(hmax(Pr, TINY));
    double Fcent, DFcentDT;
    if (t == HC_RATE_TROE3) {
        Fcent = hmax((1.0 - alpha) * exp(-T / Tsss) + alpha * exp(-T / Ts), TINY);
        DFcentDT = (1.0 - alpha) * exp(-T / Tsss) / (-Tsss) + alpha * exp(-T / Ts) / (-Ts);
    } else {
        Fcent = hmax((1.0 - alpha) * exp(-T / Tsss) + alpha * exp(-T / Ts) + exp(-Tss / T), TINY);
        DFcentDT = (1.0 - alpha) * exp(-T / Tsss) / (-Tsss) + alpha * exp(-T / Ts) / (-Ts) +
                   exp(-Tss / T) * (Tss / (T * T));
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
    const double dlogPrpc = d * (logPrpc);
    const double nmdlogPrpc = n - dlogPrpc;
    const double invnmdlogPrpc = logPrpc / nmdlogPrpc;
    const double dPPDT = 2.0 * logPrpc / (nmdlogPrpc * nmdlogPrpc) *
                         ((dlogPrDT + DcDT) - logPrpc / nmdlogPrpc * (DnDT - d * (dlogPrDT + DcDT)));
    const double s1 = 1.0 + invnmdlogPrpc * invnmdlogPrpc;
    return (F * ln10 * (DlogFcentDT / s1 - logFcent / (s1 * s1) * dPPDT));
}

/* PLOG (logInterpolationRR.cpp:78-147 k, :149-226 DkDT): the entries of
   reaction r sorted by pressure, equal pressures adding their rates. Restated
   loop for loop: inside the table the loop over intervals does not stop at
   the first one that brackets p, so the last interval (the two highest
   pressures) is the one evaluated. At the top the reference adds duplicated
   highest pressures, and its derivative indexes one past its list there;
   tables with a duplicated highest pressure are rejected by the reader and
   by hc_mech_create, so that branch only ever sees its first entry. */
static double plogK(const hc_mech_desc *m, int r, double p, double T) {
    const int b = m->plog_ptr[r], n = m->plog_ptr[r + 1] - b;
    const double *pp = &m->plog_p[b], *pa = &m->plog_arr[3 * b];
    double k = 0.0;
    if (p <= pp[0]) {
        k = arrK(&pa[0], T);
        for (int i = 0; i < n - 1; i++) {
            if (pp[i + 1] > pp[i]) break;
            k += arrK(&pa[3 * (i + 1)], T);
        }
    } else if (p >= pp[n - 1]) {
        k = arrK(&pa[3 * (n - 1)], T);
        for (int i = n - 1; i > 1; i--) {
            if (pp[i - 1] < pp[i]) break;
            k += arrK(&pa[3 * (i - 1)], T);
        }
    } else {
        for (int i = 0; i < n - 1; i++) {
            if (p < pp[i + 1]) {
                double k0 = arrK(&pa[3 * i], T);
                for (int j = i - 1; j >= 0; j--) {
                    if (pp[j + 1] > pp[j]) break;
                    k0 += arrK(&pa[3 * j], T);
                }
                double k1 = arrK(&pa[3 * (i + 1)], T);
                for (int j = i + 1; j < n - 1; j++) {
                    if (pp[j + 1] > pp[j]) break;
                    k1 += arrK(&pa[3 * (j + 1)], T);
                }
                const double lnk0 = log(k0);
                const double lnk1 = log(k1);
                const double lnp0 = log(pp[i]);
                const double lnp1 = log(pp[i + 1]);
                const double lnp = log(p);
                const double lnk = lnk0 + (lnk1 - lnk0) * (lnp - lnp0) / (lnp1 - lnp0);
                k = exp(lnk);
            }
        }
    }
    return k;
}

static double plogDkDT(const hc_mech_desc *m, int r, double kj, double p, double T) {
    const int b = m->plog_ptr[r], n = m->plog_ptr[r + 1] - b;
    const double *pp = &m->plog_p[b], *pa = &m->plog_arr[3 * b];
    double dkdT = 0.0;
    if (p <= pp[0]) {
        const double k0 = arrK(&pa[0], T);
        dkdT = arrDkDT(&pa[0], k0, T);
        for (int i = 0; i < n - 1; i++) {
            if (pp[i + 1] > pp[i]) break;
            const double ki = arrK(&pa[3 * (i + 1)], T);
            dkdT += arrDkDT(&pa[3 * (i + 1)], ki, T);
        }
    } else if (p >= pp[n - 1]) {
        const double kl = arrK(&pa[3 * (n - 1)], T);
        dkdT = arrDkDT(&pa[3 * (n - 1)], kl, T);
        for (int i = n - 1; i > 1; i--) {
            if (pp[i - 1] < pp[i]) break;
            const double ki = arrK(&pa[3 * (i - 1)], T);
            dkdT += arrDkDT(&pa[3 * (i - 1)], ki, T);
        }
    } else {
        for (int i = 0; i < n - 1; i++) {
            if (p < pp[i + 1]) {
                double k0 = arrK(&pa[3 * i], T);
                double dk0dT = arrDkDT(&pa[3 * i], k0, T);
                for (int j = i - 1; j >= 0; j--) {
                    if (pp[j + 1] > pp[j]) break;
                    const double kj0 = arrK(&pa[3 * j], T);
                    k0 += kj0;
                    dk0dT += arrDkDT(&pa[3 * j], kj0, T);
                }
                double k1 = arrK(&pa[3 * (i + 1)], T);
                double dk1dT = arrDkDT(&pa[3 * (i + 1)], k1, T);
                for (int j = i + 1; j < n - 1; j++) {
                    if (pp[j + 1] > pp[j]) break;
                    const double kj1 = arrK(&pa[3 * (j + 1)], T);
                    k1 += kj1;
                    dk1dT += arrDkDT(&pa[3 * (j + 1)], kj1, T);
                }
                const double lnp0 = log(pp[i]);
                const double lnp1 = log(pp[i + 1]);
                const double lnp = log(p);
                const double dlnkdT =
                    1.0 / k0 * dk0dT + (1.0 / k1 * dk1dT - 1.0 / k0 * dk0dT) * (lnp - lnp0) / (lnp1 - lnp0);
                dkdT = kj * dlnkdT;
            }
        }
    }
    return dkdT;
}

/* Landau-Teller (LandauTellerRR.cpp:37-99) */
static double ltK(const double *a, const double *bc, double T) {
    double lta = a[0];
    if (fabs(a[1]) > VERY_TINY) lta *= pow(T, a[1]);
    double expAgr = 0.0;
    if (fabs(a[2]) > VERY_TINY) expAgr -= a[2] / T;
    if (fabs(bc[0]) > VERY_TINY) expAgr += bc[0] / pow(T, 1.0 / 3.0);
    if (fabs(bc[1]) > VERY_TINY) expAgr += bc[1] / pow(T, 2.0 / 3.0);
    if (fabs(expAgr) > VERY_TINY) lta *= exp(expAgr);
    return lta;
}

static double ltDkDT(const double *a, const double *bc, double T) {
    double lta = a[0];
    if (fabs(a[1]) > VERY_TINY) lta *= pow(T, a[1]);
    double expArg = 0, deriv = 0;
    if (fabs(a[2]) > VERY_TINY) {
        const double TaT = a[2] / T;
        expArg -= TaT;
        deriv += TaT;
    }
    if (fabs(bc[0]) > VERY_TINY) {
        const double BT = bc[0] / cbrt(T);
        expArg += BT;
        deriv -= BT / 3;
    }
    if (fabs(bc[1]) > VERY_TINY) {
        const double CT = bc[1] / pow(T, 2.0 / 3.0);
        expArg += CT;
        deriv -= 2 * CT / 3;
    }
    if (fabs(expArg) > VERY_TINY) lta *= exp(expArg);
    return lta * (a[1] + deriv) / T;
}

/* Janev (JanevRR.cpp:37-88) and power series (powerSeriesRateRR.cpp:37-74) */
static double janevK(const hc_mech_desc *m, int r, double T) {
    const double *a = &m->arr[3 * r], *b = &m->xcoef[9 * r];
    double lta = a[0];
    if (fabs(a[1]) > VERY_TINY) lta *= pow(T, a[1]);
    double expArg = 0.0;
    if (fabs(a[2]) > VERY_TINY) expArg -= a[2] / T;
    const double lnT = log(T);
    for (int n = 0; n < 9; n++) expArg += b[n] * pow(lnT, n);
    lta *= exp(expArg);
    return lta;
}

static double janevDkDT(const hc_mech_desc *m, int r, double T) {
    const double *a = &m->arr[3 * r], *b = &m->xcoef[9 * r];
    double lta = a[0];
    if (fabs(a[1]) > VERY_TINY) lta *= pow(T, a[1]);
    double expArg = 0;
    if (fabs(a[2]) > VERY_TINY) expArg -= a[2] / T;
    const double lnT = log(T);
    for (int n = 0; n < 9; n++) expArg += b[n] * pow(lnT, n);
    double deriv = b[1];
    for (int n = 2; n < 9; n++) deriv += n * b[n] * pow(lnT, n - 1);
    lta *= exp(expArg);
    return lta * (a[1] + a[2] / T + deriv) / T;
}

static double pseriesK(const hc_mech_desc *m, int r, double T) {
    const double *a = &m->arr[3 * r], *b = &m->xcoef[9 * r];
    double lta = a[0];
    if (fabs(a[1]) > VERY_TINY) lta *= pow(T, a[1]);
    double expArg = 0.0;
    for (int n = 0; n < 4; n++) expArg += b[n] / pow(T, n + 1);
    lta *= exp(expArg);
    return lta;
}

static double pseriesDkDT(const hc_mech_desc *m, int r, double T) {
    const double *a = &m->arr[3 * r], *b = &m->xcoef[9 * r];
    double lta = a[0];
    if (fabs(a[1]) > VERY_TINY) lta *= pow(T, a[1]);
    double expArg = 0, deriv = 0;
    for (int n = 0; n < 4; n++) {
        const double cT = b[n] / pow(T, n + 1);
        expArg += cT;
        deriv -= (n + 1) * cT;
    }
    lta *= exp(expArg);
    return lta * (a[1] + deriv) / T;
}

/* collision efficiency (Chemkin COLLEFF; collisionRR.hpp:94-107, 146-169,
   collisionRR.cpp:36-46): k = min(1, Arrhenius) Zb(T), Zb = N_A d^2
   sqrt(8 pi RAB T); dk/dT = (k > 1 ? Arrhenius DkDT at k : 0) dZb/dT with
   dZb/dT = N_A d^2 sqrt(2 pi RAB / T), as the reference states them.
   xcoef = (N_A d^2, 8 pi RAB, 2 pi RAB), RAB = Ru / W_AB, made by the reader */
static double collisionK(const hc_mech_desc *m, int r, double T) {
    const double *x = &m->xcoef[9 * r];
    const double g = arrK(&m->arr[3 * r], T);
    const double gam = (g < 1.0) ? g : 1.0; /* std::min(1, g) */
    return gam * (x[0] * sqrt(x[1] * T));
}

static double collisionDkDT(const hc_mech_desc *m, int r, double kj, double T) {
    const double *x = &m->xcoef[9 * r];
    return (kj > 1.0 ? arrDkDT(&m->arr[3 * r], kj, T) : 0.0) * (x[0] * sqrt(x[2] / T));
}

/* chemically activated bimolecular (Chemkin HIGH,
   chemicallyActicatedBimolecularRR.cpp:36-96): k = k0 F / (1 + Pr) */
static int activated(const hc_mech_desc *m, int r) { return m->activated && m->activated[r]; }

static double rateK(const hc_mech_desc *m, int r, double p, double T, const double *c) {
    const int t = m->rate_type[r];
    const double *a = &m->arr[3 * r];
    if (t == HC_RATE_ARRHENIUS) return arrK(a, T);
    if (t == HC_RATE_PLOG) return plogK(m, r, p, T);
    if (t == HC_RATE_LANDAU_TELLER) return ltK(&m->arr[3 * r], &m->lt[2 * r], T);
    if (t == HC_RATE_JANEV) return janevK(m, r, T);
    if (t == HC_RATE_POWER_SERIES) return pseriesK(m, r, T);
    if (t == HC_RATE_COLLISION) return collisionK(m, r, T);
    if (t == HC_RATE_THIRD_BODY) {
        const double M = thirdM(m, r, c);
        return (M * arrK(a, T));
    }
    const double k0 = arrK(&m->arr0[3 * r], T);
    const double kinf = arrK(a, T);
    const double Pr = k0 / notZeroD(kinf) * thirdM(m, r, c);
    if (activated(m, r)) return k0 * (1.0 / (1.0 + Pr)) * fallF(m, r, T, Pr);
    return kinf * (Pr / (1.0 + Pr)) * fallF(m, r, T, Pr);
}

static double rateDkDT(const hc_mech_desc *m, int r, double kj, double p, double T,
                       const double *c) {
    const int t = m->rate_type[r];
    const double *a = &m->arr[3 * r];
    if (t == HC_RATE_ARRHENIUS || t == HC_RATE_THIRD_BODY) return arrDkDT(a, kj, T);
    if (t == HC_RATE_PLOG) return plogDkDT(m, r, kj, p, T);
    if (t == HC_RATE_LANDAU_TELLER) return ltDkDT(&m->arr[3 * r], &m->lt[2 * r], T);
    if (t == HC_RATE_JANEV) return janevDkDT(m, r, T);
    if (t == HC_RATE_POWER_SERIES) return pseriesDkDT(m, r, T);
    if (t == HC_RATE_COLLISION) return collisionDkDT(m, r, kj, T);
    const double k0 = arrK(&m->arr0[3 * r], T);
    const double kinf = arrK(a, T);
    const double Pr = k0 / notZeroD(kinf) * thirdM(m, r, c);
    if (activated(m, r))
        return (1.0 / (1.0 + Pr)) * fallF(m, r, T, Pr) * arrDkDT(&m->arr0[3 * r], k0, T);
    return (Pr / (1.0 + Pr)) * fallF(m, r, T, Pr) * arrDkDT(a, kinf, T);
}

static void gamDGamDCi(const hc_mech_desc *m, int r, double T, const double *c, double *g) {
    const int t = m->rate_type[r];
    const int nsp = m->nsp;
    const double *e = &m->eff[(int64_t)r * nsp];
    if (t == HC_RATE_THIRD_BODY) {
        const double MM = thirdM(m, r, c);
        for (int i = 0; i < nsp; ++i) g[i] = e[i] / hmax(MM, TINY);
        return;
    }
    const double M = thirdM(m, r, c);
    if (M > TINY) {
        const double k0 = arrK(&m->arr0[3 * r], T);
        const double kinf = arrK(&m->arr[3 * r], T);
        const double Pr = k0 * M / notZeroD(kinf);
        const double F = fallF(m, r, T, Pr);
        for (int i = 0; i < nsp; ++i) {
            const double dPrdci = e[i] * k0 / notZeroD(kinf);
            const double dFdci = fallDFDci(m, r, T, Pr, F, dPrdci);
            if (activated(m, r)) g[i] = (-dPrdci / (1 + Pr) + dFdci / F);
            else g[i] = (dPrdci / (Pr * (1 + Pr)) + dFdci / F);
        }
    } else {
        for (int i = 0; i < nsp; ++i) g[i] = 0.0;
    }
}

static double gamDGamDT(const hc_mech_desc *m, int r, double T, const double *c) {
    const int t = m->rate_type[r];
    if (t == HC_RATE_ARRHENIUS || t == HC_RATE_THIRD_BODY || t >= HC_RATE_PLOG) return 0.0;
    const double M = thirdM(m, r, c);
    if (M > TINY) {
        const double *a0 = &m->arr0[3 * r], *a = &m->arr[3 * r];
        const double k0 = arrK(a0, T);
        const double kinf = arrK(a, T);
        const double Pr = k0 * M / notZeroD(kinf);
        const double F = fallF(m, r, T, Pr);
        const double dPrdT =
            Pr * (arrDkDT(a0, k0, T) / notZeroD(k0) - arrDkDT(a, kinf, T) / notZeroD(kinf));
        const double dFdT = fallDFDT(m, r, T, Pr, F, dPrdT);
        if (activated(m, r)) return (-dPrdT / (1 + Pr) + dFdT / F);
        return (dPrdT / (Pr * (1 + Pr)) + dFdT / F);
    }
    return 0.0;
}

/* ---------------- equilibrium constants ---------------- */

static double Kp(const mech_ctx *x, int r, double T) {
    const hc_mech_desc *m = x->m;
    double kp = 0.0;
    for (int k = 0; k < m->nf[r]; ++k) kp -= x->G0[m->fidx[HC_MAX_SIDE * r + k]] * m->fnu[HC_MAX_SIDE * r + k];
    for (int k = 0; k < m->nb[r]; ++k) kp += x->G0[m->bidx[HC_MAX_SIDE * r + k]] * m->bnu[HC_MAX_SIDE * r + k];
    kp /= (hmax(T, TINY) * RU);
    const double e = exp(-kp);
    if (isnan(e) || isinf(e)) return ROOT_VERY_LARGE;
    return e;
}

static double DKpDT(const mech_ctx *x, int r, double T) {
    const hc_mech_desc *m = x->m;
    const double kp = Kp(x, r, T);
    double d = 0.0;
    for (int k = 0; k < m->nf[r]; ++k) {
        const int i = m->fidx[HC_MAX_SIDE * r + k];
        d -= (x->DG0DT[i] - x->G0[i] / hmax(T, TINY)) * m->fnu[HC_MAX_SIDE * r + k];
    }
    for (int k = 0; k < m->nb[r]; ++k) {
        const int i = m->bidx[HC_MAX_SIDE * r + k];
        d += (x->DG0DT[i] - x->G0[i] / hmax(T, TINY)) * m->bnu[HC_MAX_SIDE * r + k];
    }
    d /= (hmax(T, TINY) * RU);
    const double v = kp * d;
    if (isnan(v) || isinf(v)) return VERY_LARGE;
    return v;
}

static double sumStoi(const hc_mech_desc *m, int r) {
    double s = 0.0;
    for (int k = 0; k < m->nf[r]; ++k) s -= m->fnu[HC_MAX_SIDE * r + k];
    for (int k = 0; k < m->nb[r]; ++k) s += m->bnu[HC_MAX_SIDE * r + k];
    return s;
}

static double Kc(const mech_ctx *x, int r, double T) {
    const double s = sumStoi(x->m, r);
    if (fabs(s) < VERY_TINY) return Kp(x, r, T);
    return hmin(Kp(x, r, T) * pow(PATM / (RU * T), s), VERY_LARGE);
}

static double DKcDT(const mech_ctx *x, int r, double T) {
    const double s = sumStoi(x->m, r);
    if (fabs(s) < VERY_TINY) return DKpDT(x, r, T);
    const double f = pow(PATM / (RU * T), s);
    const double kp = Kp(x, r, T);
    const double v = (DKpDT(x, r, T) + kp * (-s) / T) * f;
    if (isnan(v) || isinf(v)) return VERY_LARGE;
    return v;
}

/* explicit reverse rate (reversibleReactionWithRevPars::kr): the reverse
   Arrhenius law, the third-body one (M times it), or for a Landau-Teller
   reaction the reverse Landau-Teller law of Chemkin RLT (B, C in xcoef,
   chemkinFileRead.cpp:441-478, 1507-1512) */
static double kRevExplicit(const hc_mech_desc *m, int r, double T, const double *c) {
    const double *a = &m->arr_rev[3 * r];
    if (m->rate_type[r] == HC_RATE_LANDAU_TELLER) return ltK(a, &m->xcoef[9 * r], T);
    if (m->rate_type[r] == HC_RATE_THIRD_BODY) {
        const double M = thirdM(m, r, c);
        return (M * arrK(a, T));
    }
    return arrK(a, T);
}

static double kRev(const mech_ctx *x, int r, double kfwd, double T, const double *c) {
    if (x->m->reversible[r] == HC_REVERSIBLE_REV) return kRevExplicit(x->m, r, T, c);
    if (!x->m->reversible[r]) return 0.0;
    const double kc = Kc(x, r, T);
    if (fabs(kc) > VERY_TINY) return kfwd / kc;
    return 0.0;
}

static double DkrDT(const mech_ctx *x, int r, double kr, double T, double dkfdT) {
    if (x->m->reversible[r] == HC_REVERSIBLE_REV) {
        if (x->m->rate_type[r] == HC_RATE_LANDAU_TELLER)
            return ltDkDT(&x->m->arr_rev[3 * r], &x->m->xcoef[9 * r], T);
        return arrDkDT(&x->m->arr_rev[3 * r], kr, T);
    }
    if (!x->m->reversible[r]) return 0.0;
    const double kc = hmax(Kc(x, r, T), VERY_TINY);
    return (dkfdT - kr * DKcDT(x, r, T)) / kc;
}

/* q: rate of progress; accumulates into dcdt (reactionTypes.cpp:263-280, 331-352) */
static double qRate(const mech_ctx *x, int r, double T, const double *c, double *dcdt, double *kfo,
                    double *kro) {
    const hc_mech_desc *m = x->m;
    double qf = rateK(m, r, x->p, T, c);
    if (kfo) *kfo = qf;
    double qr = kRev(x, r, qf, T, c);
    if (kro) *kro = qr;
    for (int k = 0; k < m->nf[r]; ++k)
        qf *= pow(hmax(c[m->fidx[HC_MAX_SIDE * r + k]], 0.0), m->ford[HC_MAX_SIDE * r + k]);
    for (int k = 0; k < m->nb[r]; ++k)
        qr *= pow(hmax(c[m->bidx[HC_MAX_SIDE * r + k]], 0.0), m->bord[HC_MAX_SIDE * r + k]);
    const double q = qf - qr;
    if (dcdt) {
        for (int k = 0; k < m->nf[r]; ++k) dcdt[m->fidx[HC_MAX_SIDE * r + k]] -= m->fnu[HC_MAX_SIDE * r + k] * q;
        for (int k = 0; k < m->nb[r]; ++k) dcdt[m->bidx[HC_MAX_SIDE * r + k]] += m->bnu[HC_MAX_SIDE * r + k] * q;
    }
    return q;
}

static void DqDci(const mech_ctx *x, int r, double kf, double kr, double qfr, double T,
                  const double *c, double *J, int n, double *scratch) {
    const hc_mech_desc *m = x->m;
    const int nf = m->nf[r], nb = m->nb[r];
    const int *fi = &m->fidx[HC_MAX_SIDE * r], *bi = &m->bidx[HC_MAX_SIDE * r];
    const double *fnu = &m->fnu[HC_MAX_SIDE * r], *bnu = &m->bnu[HC_MAX_SIDE * r];
    const double *fo = &m->ford[HC_MAX_SIDE * r], *bo = &m->bord[HC_MAX_SIDE * r];
    for (int i = 0; i < nf; ++i) {
        const int si = fi[i];
        double d = kf;
        for (int j = 0; j < nf; ++j) {
            const int sj = fi[j];
            const double ord = fo[j];
            if (i == j) {
                if (ord == 1.0) continue;
                else if (ord < 1.0) {
                    if (c[sj] > TINY) d *= ord * pow(c[sj], ord - 1.0);
                    else d *= 0.0;
                } else d *= ord * pow(hmax(c[sj], 0.0), ord - 1.0);
            } else d *= pow(hmax(c[sj], 0.0), ord);
        }
        for (int j = 0; j < nf; ++j) J[fi[j] * n + si] -= fnu[j] * d;
        for (int j = 0; j < nb; ++j) J[bi[j] * n + si] += bnu[j] * d;
    }
    for (int i = 0; i < nb; ++i) {
        const int si = bi[i];
        double d = kr;
        for (int j = 0; j < nb; ++j) {
            const int sj = bi[j];
            const double ord = bo[j];
            if (i == j) {
                if (ord == 1.0) continue;
                else if (ord < 1.0) {
                    if (c[sj] > TINY) d *= ord * pow(c[sj], ord - 1.0);
                    else d *= 0.0;
                } else d *= ord * pow(hmax(c[sj], 0.0), ord - 1.0);
            } else d *= pow(hmax(c[sj], 0.0), ord);
        }
        for (int j = 0; j < nf; ++j) J[fi[j] * n + si] += fnu[j] * d;
        for (int j = 0; j < nb; ++j) J[bi[j] * n + si] -= bnu[j] * d;
    }
    const int t = m->rate_type[r];
    if (t != HC_RATE_ARRHENIUS && t < HC_RATE_PLOG) {   /* hasThirdBodyTerms() */
        double *g = scratch;
        gamDGamDCi(m, r, T, c, g);
        for (int i = 0; i < m->nsp; ++i) {
            for (int j = 0; j < nf; ++j)
                if (!isnan(g[i]) && !isinf(g[i])) J[fi[j] * n + i] -= fnu[j] * g[i] * qfr;
            for (int j = 0; j < nb; ++j)
                if (!isnan(g[i]) && !isinf(g[i])) J[bi[j] * n + i] += bnu[j] * g[i] * qfr;
        }
    }
}

static void DqDT(const mech_ctx *x, int r, double kf, double kr, double qfr, double T,
                 const double *c, double *J, int n) {
    const hc_mech_desc *m = x->m;
    const int nf = m->nf[r], nb = m->nb[r], nsp = m->nsp;
    const int *fi = &m->fidx[HC_MAX_SIDE * r], *bi = &m->bidx[HC_MAX_SIDE * r];
    const double *fnu = &m->fnu[HC_MAX_SIDE * r], *bnu = &m->bnu[HC_MAX_SIDE * r];
    double dkfdT = rateDkDT(m, r, kf, x->p, T, c);
    double dkrdT = DkrDT(x, r, kr, T, dkfdT);
    for (int i = 0; i < nf; ++i) dkfdT *= pow(hmax(c[fi[i]], 0.0), m->ford[HC_MAX_SIDE * r + i]);
    for (int i = 0; i < nb; ++i) dkrdT *= pow(hmax(c[bi[i]], 0.0), m->bord[HC_MAX_SIDE * r + i]);
    double dqjdT = dkfdT - dkrdT;
    double dgdT = qfr * gamDGamDT(m, r, T, c);
    if (isnan(dqjdT) || isinf(dqjdT)) dqjdT = 0;
    if (isnan(dgdT) || isinf(dgdT)) dgdT = 0;
    for (int i = 0; i < nf; ++i) J[fi[i] * n + nsp] -= fnu[i] * (dqjdT + dgdT);
    for (int i = 0; i < nb; ++i) J[bi[i] * n + nsp] += bnu[i] * (dqjdT + dgdT);
}

/* ---------------- reactor (constant pressure) ---------------- */

typedef struct {
    mech_ctx x;
    int nsp, n;
    double p;
    double *ci, *g, *J, *s;     /* work */
    hc_counters cnt;
    int cv;                     /* constant volume (else constant pressure) */
    double rho0;                /* the cell's density (constant volume) */
    double *yt;                 /* [nsp] mass fractions of the current state */
} reactor;

/* speciesList::MWbyYi / Rm (speciesList.cpp:106-116, speciesList.inl:58-61) */
static double mwByYi(const hc_mech_desc *m, const double *yi) {
    if (m->nsp == 1) return m->W[0];
    double w = 0.0;
    for (int i = 0; i < m->nsp; ++i) w += yi[i] / m->W[i];
    return 1.0 / hmax(w, VERY_TINY);
}

/* constant volume: p = rho Rm T (perfectGas::pm, perfectGas.cpp:49-53) with
   Y = c W / rho0 (chemistrySource.cpp:885-906 uses c as given, :975-981 the
   clamped c), molar internal energy e_i W_i = (h_i - R_i T) W_i
   (thermo.inl:168-171) and cv_i = cp_i - R_i (thermo.inl:80-94) */
static double cvPressure(reactor *R, const double *c, double T) {
    const hc_mech_desc *m = R->x.m;
    for (int i = 0; i < R->nsp; ++i) R->yt[i] = c[i] * m->W[i] / R->rho0;
    const double Rm = RU / mwByYi(m, R->yt);
    return R->rho0 * Rm * T;
}

static inline double ea_m(const hc_mech_desc *m, int i, double T) {
    return ha0(m, i, T) - (RU / m->W[i]) * T;
}

static inline double Cv_p(const hc_mech_desc *m, int i, double T) {
    return (cp0(m, i, T) - RU / m->W[i]) * m->W[i];
}

static void DyDt(reactor *R, const double *y, double *dydt) {
    const hc_mech_desc *m = R->x.m;
    const int nsp = R->nsp;
    const double T = y[nsp];
    R->cnt.n_rhs++;
    if (R->cv) {
        /* chemistrySource::DyDt, constant volume (chemistrySource.cpp:885-906) */
        for (int i = 0; i < R->n; ++i) dydt[i] = 0.0;
        R->p = R->x.p = cvPressure(R, y, T);
        for (int i = 0; i < nsp; ++i) R->ci[i] = y[i];
        updateG0(&R->x, T);
        for (int r = 0; r < m->nrc; ++r) qRate(&R->x, r, T, R->ci, dydt, NULL, NULL);
        double cvmix = 0.0, DTdt = 0.0;
        for (int i = 0; i < nsp; ++i) {
            cvmix += R->yt[i] * (cp0(m, i, T) - RU / m->W[i]);   /* cv_p */
            DTdt += dydt[i] * ea_m(m, i, T) * m->W[i];
        }
        DTdt /= (cvmix * R->rho0);
        dydt[nsp] = -DTdt;
        return;
    }
    for (int i = 0; i < R->n; ++i) dydt[i] = 0.0;
    for (int i = 0; i < nsp; ++i) R->ci[i] = hmax(y[i], 0.0);
    updateG0(&R->x, T);
    for (int i = 0; i < R->n; ++i) dydt[i] = 0.0;
    for (int r = 0; r < m->nrc; ++r) qRate(&R->x, r, T, R->ci, dydt, NULL, NULL);
    double cCp = 0.0, DTdt = 0.0;
    for (int i = 0; i < nsp; ++i) {
        cCp += y[i] * Cp_p(m, i, T);
        DTdt += dydt[i] * Ha_p(m, i, T);
    }
    DTdt /= cCp;
    dydt[nsp] = -DTdt;
}

static void jacobian(reactor *R, const double *y, double *dfdt, double *J) {
    const hc_mech_desc *m = R->x.m;
    const int nsp = R->nsp, n = R->n;
    const double T = y[nsp];
    R->cnt.n_jac++;
    updateG0(&R->x, T);
    for (int i = 0; i < nsp; ++i) R->ci[i] = hmax(y[i], 0.0);
    if (R->cv) R->p = R->x.p = cvPressure(R, R->ci, T);
    for (int i = 0; i < n * n; ++i) J[i] = 0.0;
    for (int i = 0; i < n; ++i) dfdt[i] = 0.0;
    for (int r = 0; r < m->nrc; ++r) {
        double kf, kr;
        const double qfr = qRate(&R->x, r, T, R->ci, dfdt, &kf, &kr);
        DqDci(&R->x, r, kf, kr, qfr, T, R->ci, J, n, R->g);
        DqDT(&R->x, r, kf, kr, qfr, T, R->ci, J, n);
    }
    if (R->cv) {
        /* chemistrySource::jacobian, constant volume (chemistrySource.cpp:1022-1055) */
        double cCv = 0.0, DTdt = 0.0, dcCvdT = 0.0;
        for (int i = 0; i < nsp; ++i) {
            cCv += y[i] * Cv_p(m, i, T);
            dcCvdT += y[i] * DCp_pDT(m, i, T);
            DTdt += dfdt[i] * ea_m(m, i, T) * m->W[i];
        }
        DTdt /= cCv;
        dfdt[nsp] = -DTdt;
        for (int i = 0; i < nsp; ++i) {
            double d = J[nsp * n + i];
            for (int j = 0; j < nsp; ++j) d -= J[j * n + i] * ea_m(m, j, T) * m->W[j];
            d += Cv_p(m, i, T) * DTdt;
            d /= cCv;
            J[nsp * n + i] = d;
        }
        double dd = 0.0;
        for (int i = 0; i < nsp; ++i)
            dd -= (Cv_p(m, i, T) * dfdt[i] + ea_m(m, i, T) * m->W[i] * J[i * n + nsp]);
        dd += dcCvdT * DTdt;
        dd /= cCv;
        J[nsp * n + nsp] = dd;
        return;
    }
    double cCp = 0.0, DTdt = 0.0, dcCpdT = 0.0;
    for (int i = 0; i < nsp; ++i) {
        cCp += y[i] * Cp_p(m, i, T);
        dcCpdT += y[i] * DCp_pDT(m, i, T);
        DTdt += dfdt[i] * Ha_p(m, i, T);
    }
    DTdt /= cCp;
    dfdt[nsp] = -DTdt;
    for (int i = 0; i < nsp; ++i) {
        double d = J[nsp * n + i];
        for (int j = 0; j < nsp; ++j) d -= J[j * n + i] * Ha_p(m, j, T);
        d += Cp_p(m, i, T) * DTdt;
        d /= cCp;
        J[nsp * n + i] = d;
    }
    double dd = 0.0;
    for (int i = 0; i < nsp; ++i) dd -= (Cp_p(m, i, T) * dfdt[i] + Ha_p(m, i, T) * J[i * n + nsp]);
    dd += dcCpdT * DTdt;
    dd /= cCp;
    J[nsp * n + nsp] = dd;
}

/* ---------------- dense LU with partial pivoting ---------------- */

static void luDecompose(double *A, int n, int *M, double *s) {
    for (int k = 0; k < n; ++k) {
        double maxs = A[k * n + k];
        int ik = k;
        for (int i = k; i < n; ++i) {
            double sumlu = 0.0;
            for (int t = 0; t < k; ++t) sumlu += A[i * n + t] * A[t * n + k];
            s[i] = A[i * n + k] - sumlu;
            if (i == k) maxs = s[i];
            if (fabs(s[i]) > fabs(maxs)) {
                ik = i;
                maxs = s[i];
            }
        }
        M[k] = ik;
        if (ik != k) {
            for (int t = 0; t < n; ++t) {
                const double tmp = A[k * n + t];
                A[k * n + t] = A[ik * n + t];
                A[ik * n + t] = tmp;
            }
            const double tmp = s[k];
            s[k] = s[ik];
            s[ik] = tmp;
        }
        A[k * n + k] = s[k];
        for (int j = k + 1; j < n; ++j) {
            double sumlu = 0.0;
            for (int t = 0; t < k; ++t) sumlu += A[k * n + t] * A[t * n + j];
            A[k * n + j] -= sumlu;
        }
        for (int i = k + 1; i < n; ++i)
            if (k < n - 1) A[i * n + k] = s[i] / A[k * n + k];
    }
}

static void luSolve(const double *A, int n, const int *M, double *b) {
    for (int k = 0; k < n - 1; ++k) {
        const int t = M[k];
        if (t != k) {
            const double tmp = b[k];
            b[k] = b[t];
            b[t] = tmp;
        }
    }
    for (int i = 0; i < n; ++i) {
        double sumly = 0.0;
        for (int t = 0; t < i; ++t) sumly += A[i * n + t] * b[t];
        b[i] -= sumly;
    }
    for (int i = n - 1; i >= 0; --i) {
        double sumux = 0.0;
        for (int t = i + 1; t < n; ++t) sumux += A[i * n + t] * b[t];
        b[i] = (b[i] - sumux) / A[i * n + i];
    }
}

/* ---------------- implicit Euler ---------------- */

typedef struct {
    reactor *R;
    const hc_opts *o;
    int n;
    int countStep;
    double lastTimeStep[2];
    double *yklast0, *yklast1, *yk, *yTemp, *dydt, *err, *dfdy, *s;
    int *piv;
    int status;
} ieuler;

static double maxError(const ieuler *E, const double *y0, const double *y, const double *e) {
    double m = 0.0;
    for (int i = 0; i < E->n; ++i) {
        const double tol = E->o->atol + E->o->rtol * hmax(fabs(y0[i]), fabs(y[i]));
        m = hmax(m, fabs(e[i]) / tol);
    }
    return m;
}

static double maxIncrement(const ieuler *E, const double *y0, const double *y, const double *e) {
    double m = 0.0;
    for (int i = 0; i < E->n; ++i) {
        if (isnan(y[i])) return 1.5;
        const double tol = E->o->atol_increment + E->o->rtol_increment * hmax(fabs(y0[i]), fabs(y[i]));
        m = hmax(m, fabs(e[i]) / tol);
    }
    return m;
}

static void formNewton(ieuler *E, double dt) {
    const int n = E->n;
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) E->dfdy[i * n + j] = -dt * E->dfdy[i * n + j];
        E->dfdy[i * n + i] += 1.0;
    }
    luDecompose(E->dfdy, n, E->piv, E->s);
    E->R->cnt.n_lu++;
}

static double newton(ieuler *E, const double *y0, double dt, double *ykp1, int *conv) {
    const int n = E->n;
    int count = 0;
    double maxErr = 0.0, lastErr = 0.0;
    const int autoJ = E->o->auto_update_jacobian;
    const int stepJ = E->o->step_to_update_jac;
    do {
        if (autoJ) {
            if (count == 0 || count % stepJ == 0) {
                jacobian(E->R, ykp1, E->dydt, E->dfdy);
                formNewton(E, dt);
            } else {
                DyDt(E->R, ykp1, E->dydt);
            }
        } else {
            jacobian(E->R, ykp1, E->dydt, E->dfdy);
            formNewton(E, dt);
        }
        for (int i = 0; i < n; ++i) E->err[i] = (-ykp1[i] + y0[i]) + dt * E->dydt[i];
        luSolve(E->dfdy, n, E->piv, E->err);
        E->R->cnt.n_newton++;
        for (int i = 0; i < n; ++i) {
            if (isnan(E->err[i]) || isinf(E->err[i])) {
                *conv = 0;
                return 1000.0;
            }
            ykp1[i] += E->err[i];
        }
        maxErr = maxError(E, ykp1, ykp1, E->err);
        if (count > 0) {
            const double diver = maxErr / hmax(lastErr, TINY);
            if (autoJ) {
                const int lim = (30 * stepJ > 50) ? 30 * stepJ : 50;
                if (diver > 2 && count > lim) {
                    *conv = 0;
                    return 1000.0;
                }
            } else if (diver > 2 && count > 5) {
                *conv = 0;
                return 1000.0;
            }
        }
        lastErr = maxErr;
        count++;
        if (isnan(maxErr)) {
            *conv = 0;
            return 1000.0;
        }
        if (count > 1000) {
            *conv = 0;
            return maxErr;
        }
    } while (maxErr > 1.0);
    *conv = 1;
    return maxErr;
}

static double stepSolve(ieuler *E, const double *y0, double dt, double *y) {
    const int n = E->n;
    E->R->cnt.n_attempts++;
    memcpy(E->yk, y0, sizeof(double) * n);
    int conv = 1;
    const double errN = newton(E, y0, dt, E->yk, &conv);
    memcpy(y, E->yk, sizeof(double) * n);
    if (!conv) return errN;
    if (E->countStep == 0) {
        DyDt(E->R, E->yk, E->dydt);
        for (int i = 0; i < n; ++i) E->err[i] = E->yk[i] - y0[i] - dt * E->dydt[i];
        return maxIncrement(E, y0, E->yk, E->err);
    }
    const double dtn = E->lastTimeStep[0], dtn1 = E->lastTimeStep[1];
    const double f1 = 2.0 / (dtn * (dtn + dtn1));
    const double f2 = 2.0 / (dtn1 * (dtn + dtn1));
    const double LTEF = (dtn * dtn) * 0.5;
    for (int i = 0; i < n; ++i) {
        E->err[i] = f1 * (E->yk[i] - y0[i]) - f2 * (y0[i] - E->yklast1[i]);
        E->err[i] *= LTEF;
    }
    return maxIncrement(E, y0, E->yk, E->err);
}

static int checkNewY(const ieuler *E, double *dt, const double *yOld, const double *yNew) {
    const int last = E->n - 1;
    if ((yNew[last] - yOld[last]) > E->o->T_alpha * yOld[last]) {
        *dt *= E->o->T_beta;
        return 0;
    }
    return 1;
}

/* returns 0 ok, nonzero = step-size underflow (the reference aborts) */
static int adaptiveSolve(ieuler *E, double *t, double *dt0, double *y) {
    const hc_opts *o = E->o;
    const int n = E->n;
    double dt = *dt0;
    double error = 0.0;
    memcpy(E->yTemp, y, sizeof(double) * n);
    E->lastTimeStep[1] = E->lastTimeStep[0];
    int count = 0;
    do {
        E->lastTimeStep[0] = dt;
        error = stepSolve(E, y, dt, E->yTemp);
        if (!checkNewY(E, &dt, y, E->yTemp) && count < 100) {
            error = 2;
            count++;
            if (dt <= VERY_TINY) return 1;
            continue;
        }
        if (error > 1.0) {
            const double scale = hmax(o->safescale * pow(error, -o->alphainc), o->minscale);
            dt *= scale;
            if (dt <= VERY_TINY) return 1;
        }
    } while (error > 1.0);
    *t += dt;
    memcpy(y, E->yTemp, sizeof(double) * n);
    E->R->cnt.n_steps++;
    if (error > pow(o->maxscale / o->safescale, -1.0 / o->alphainc))
        *dt0 = hmin(hmax(o->safescale * pow(error, -o->alphainc), o->minscale), o->maxscale) * dt;
    else
        *dt0 = hmax(o->safescale * o->maxscale * dt, dt);
    return 0;
}

/* ImplicitEuler::solve(t0, tn, dt0, y); returns 0, or 1 on underflow; sets *reached */
static int solveInterval(ieuler *E, double t0, double *tn, double *dt0, double *y) {
    double t = t0;
    double dt = 0.2 * (*dt0);
    double dtReached = t0;
    int last = 0;
    for (int nstep = 0; nstep < E->o->maxstep; ++nstep) {
        E->countStep = nstep;
        if (nstep == 0) {
            memcpy(E->yklast0, y, sizeof(double) * E->n);
        } else {
            memcpy(E->yklast1, E->yklast0, sizeof(double) * E->n);
            memcpy(E->yklast0, y, sizeof(double) * E->n);
        }
        const double dtTry0 = dt;
        if ((t + dt - *tn) * (t + dt - t0) > 0) {
            dt = *tn - t;
            last = 1;
        } else if (t + dt == *tn) {
            last = 1;
        }
        if (adaptiveSolve(E, &t, &dt, y)) return 1;
        dtReached = t;
        if ((t - *tn) * (*tn - t0) >= 0) {
            if (nstep > 0 && last) *dt0 = hmin(dtTry0, *tn);
            return 0;
        }
    }
    E->status |= HC_CELL_MAXSTEP;
    *tn = dtReached;
    return 0;
}

/* ---------------- public oracle entry points ---------------- */

typedef struct {
    hc_mech_desc m;
} oracle_mech;

static void *xcalloc(size_t n, size_t s) {
    void *p = calloc(n ? n : 1, s);
    return p;
}

/* thermo values for KAT comparisons: out[7*nsp] = cp0, ha0, s0, g0, G0, DG0DT, Dcp_pDT */
void oracle_thermo(const hc_mech_desc *m, double T, double *out) {
    for (int i = 0; i < m->nsp; ++i) {
        out[7 * i + 0] = cp0(m, i, T);
        out[7 * i + 1] = ha0(m, i, T);
        out[7 * i + 2] = s0(m, i, T);
        out[7 * i + 3] = g0(m, i, T);
        out[7 * i + 4] = G0m(m, i, T);
        out[7 * i + 5] = DG0DTm(m, i, T);
        out[7 * i + 6] = Dcp_pDT(m, i, T);
    }
}

/* rate constants at (p, T, c): out[3*nrc] = kf, Kc, kr */
void oracle_rates(const hc_mech_desc *m, double p, double T, const double *c, double *out) {
    mech_ctx x = {m, (double *)xcalloc(m->nsp, 8), (double *)xcalloc(m->nsp, 8), p};
    double *cc = (double *)xcalloc(m->nsp, 8);
    for (int i = 0; i < m->nsp; ++i) cc[i] = hmax(c[i], 0.0);
    updateG0(&x, T);
    for (int r = 0; r < m->nrc; ++r) {
        const double kf = rateK(m, r, p, T, cc);
        out[3 * r] = kf;
        out[3 * r + 1] = Kc(&x, r, T);
        out[3 * r + 2] = kRev(&x, r, kf, T, cc);
    }
    free(x.G0); free(x.DG0DT); free(cc);
}

static void reactorInit(reactor *R, const hc_mech_desc *m) {
    memset(R, 0, sizeof(*R));
    R->x.m = m;
    R->x.G0 = (double *)xcalloc(m->nsp, 8);
    R->x.DG0DT = (double *)xcalloc(m->nsp, 8);
    R->nsp = m->nsp;
    R->n = m->nsp + 1;
    R->ci = (double *)xcalloc(m->nsp, 8);
    R->g = (double *)xcalloc(m->nsp, 8);
    R->yt = (double *)xcalloc(m->nsp, 8);
}

static void reactorFree(reactor *R) {
    free(R->x.G0); free(R->x.DG0DT); free(R->ci); free(R->g); free(R->yt);
}

/* DyDt and Jacobian at states: y = [c, T] per state, at pressures p[ns]
   (NULL: one atmosphere; only pressure-dependent rate tables read it) */
void oracle_rhs_jac(const hc_mech_desc *m, int64_t ns, const double *c /*[nsp*ns]*/,
                    const double *T, const double *p, double *dydt /*[ns*n]*/,
                    double *J /*[ns*n*n]*/) {
    reactor R;
    reactorInit(&R, m);
    const int n = R.n;
    double *y = (double *)xcalloc(n, 8), *f = (double *)xcalloc(n, 8);
    for (int64_t k = 0; k < ns; ++k) {
        for (int i = 0; i < m->nsp; ++i) y[i] = c[(int64_t)i * ns + k];
        y[m->nsp] = T[k];
        R.p = R.x.p = p ? p[k] : PATM;
        if (dydt) DyDt(&R, y, &dydt[k * n]);
        if (J) jacobian(&R, y, f, &J[k * n * n]);
    }
    free(y); free(f);
    reactorFree(&R);
}

/*
 * Integrate cells (chemistrySource::solve(dt, dtFactor) body per cell).
 * Arrays are SoA [nsp][ncells]. On return: T, rho, Y updated, c = final
 * concentrations, subdt = new warm-start step, status per cell, and the
 * counters summed into cnt.
 */
int oracle_integrate(const hc_mech_desc *m, const hc_opts *o, int64_t ncells, double *T,
                     const double *p, double *rho, double *Y, const double *dt, double dtFactor,
                     double *subdt, double *cout, int32_t *status, hc_counters *cnt) {
    reactor R;
    reactorInit(&R, m);
    const int nsp = m->nsp, n = R.n;
    ieuler E;
    memset(&E, 0, sizeof(E));
    E.R = &R;
    E.o = o;
    E.n = n;
    E.yklast0 = (double *)xcalloc(n, 8);
    E.yklast1 = (double *)xcalloc(n, 8);
    E.yk = (double *)xcalloc(n, 8);
    E.yTemp = (double *)xcalloc(n, 8);
    E.dydt = (double *)xcalloc(n, 8);
    E.err = (double *)xcalloc(n, 8);
    E.s = (double *)xcalloc(n, 8);
    E.dfdy = (double *)xcalloc((size_t)n * n, 8);
    E.piv = (int *)xcalloc(n, sizeof(int));
    double *y = (double *)xcalloc(n, 8);
    double *yi = (double *)xcalloc(nsp, 8);
    int bad = 0;
    for (int64_t cell = 0; cell < ncells; ++cell) {
        E.status = 0;
        const double Ti = T[cell];
        const double tstep = dt[cell] * dtFactor;
        for (int i = 0; i < nsp; ++i) y[i] = rho[cell] * Y[(int64_t)i * ncells + cell] / m->W[i];
        if (Ti < o->T_threshold) {
            subdt[cell] = tstep;
            for (int i = 0; i < nsp; ++i) cout[(int64_t)i * ncells + cell] = y[i];
            if (status) status[cell] = HC_CELL_SKIPPED;
            continue;
        }
        R.p = p[cell];
        R.x.p = p[cell];
        R.cv = o->reactor == 1;
        R.rho0 = rho[cell];
        double leftTime = tstep;
        double sub = hmin(leftTime, hmin(subdt[cell], o->dt_max));
        double Tcur = Ti;
        while (leftTime > 0.0) {
            double d = leftTime;
            y[nsp] = Tcur;
            if (solveInterval(&E, 0.0, &d, &sub, y)) {
                E.status |= HC_CELL_UNDERFLOW;
                Tcur = y[nsp];
                break;
            }
            Tcur = y[nsp];
            leftTime -= d;
        }
        subdt[cell] = sub;
        /* ciToYi(ci, yi): clamp, rho from c, normalise (chemistrySource.cpp:1225-1246) */
        double rr = 0.0;
        for (int i = 0; i < nsp; ++i) yi[i] = hmax(0.0, y[i]);
        for (int i = 0; i < nsp; ++i) rr += yi[i] * m->W[i];
        double ys = 0.0;
        for (int i = 0; i < nsp; ++i) {
            yi[i] = yi[i] * m->W[i] / hmax(rr, TINY);
            ys += yi[i];
        }
        if (ys != 1.0)
            for (int i = 0; i < nsp; ++i) yi[i] /= ys;
        /* constant pressure: rho = p / (Rm T), Rm = Ru / Wmean, Wmean =
           1/max(sum yi/Wi, veryTiny) (perfectGas.cpp:36-40, speciesList.inl:58-61,
           speciesList.cpp:106-116); constant volume: rho is kept and the reference
           updates p instead (chemistrySource.cpp:1317-1323) */
        double wsum = 0.0;
        for (int i = 0; i < nsp; ++i) wsum += yi[i] / m->W[i];
        const double Rm = RU / (1.0 / hmax(wsum, VERY_TINY));
        T[cell] = Tcur;
        if (!R.cv) rho[cell] = p[cell] / (Rm * Tcur);
        for (int i = 0; i < nsp; ++i) {
            Y[(int64_t)i * ncells + cell] = yi[i];
            cout[(int64_t)i * ncells + cell] = y[i];
        }
        if (status) status[cell] = E.status;
        if (E.status & ~HC_CELL_MAXSTEP) bad++;
    }
    if (cnt) *cnt = R.cnt;
    free(E.yklast0); free(E.yklast1); free(E.yk); free(E.yTemp); free(E.dydt); free(E.err);
    free(E.s); free(E.dfdy); free(E.piv); free(y); free(yi);
    reactorFree(&R);
    return bad;
}
