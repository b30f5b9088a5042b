// Cell-group implicit-Euler integrator (N = nsp + 1 up to 64 equations),
// FP64 throughout, for mechanisms too large for one thread per cell.
//
// One cell group (G lanes, see group.cuh) integrates one cell at a time and
// pulls the next cell index from a device work queue (one atomicAdd per
// cell), so cells whose sub-step counts differ by 100x do not leave SMs idle:
// the grid is persistent (a multiple of the SM count) and the queue is
// ordered most-expensive-first when a cost estimate from the previous flow
// step is available.
//
// Per cell, the control flow is the reference's, unchanged:
//   chemistrySource::solve(dt, dtFactor) cell loop  chemistrySource.cpp:1511-1555
//   ImplicitEuler::solve(t0, tn, dt0, y)            ODEs/src/ImplicitEuler.cpp:294-342
//   ImplicitEuler::adaptiveSolve                    :253-292
//   ImplicitEuler::solve(t0, y0, dydt0, dt, y)      :101-142
//   ImplicitEuler::NewtonIteration                  :161-251
// and the arithmetic is distributed over the lanes:
//   * species thermo: lane i evaluates species i (one log(T) per lane);
//   * reactions: lanes take G reactions at a time and write a small record
//     per reaction (q, dq/dc of each reactant/product, dq/dT, third-body
//     data) to shared memory; lane i then builds row i of the Jacobian from
//     the reactions species i takes part in, in reaction order (the order in
//     which reactionTypes::DqDci / DqDT accumulate, reactionTypes.cpp:354-445,843-876);
//   * the temperature row/column (chemistrySource.cpp:991-1021) from group
//     reductions and column reads;
//   * the Newton matrix I - dt J is factored with partial pivoting, lane i
//     keeping row i in registers; the pivot row is broadcast through shared
//     memory and the factor is written there in pivot order (P A = L U, the
//     layout LUDecomposeDPivoting produces, SquareMatrix.hpp:185-237);
//   * the triangular solves run on the first warp, row-oriented forward
//     (same summation order as LUBacksubstituteDPivoting) and column-
//     oriented backward.
// Every loop is bounded: the reference's own caps (maxstep, 1000 Newton
// iterations, step-size underflow) plus a per-cell cap on total Newton
// iterations, after which the cell stops with HC_CELL_ITER_LIMIT.
#pragma once

#include "group.cuh"
#include "mech.cuh"

namespace hc {

constexpr int kRec = 16;   // doubles per reaction record

// cells integrated by one block of 128 threads (a cell group of G lanes each)
__host__ __device__ constexpr int cells_per_block(int G) { return 128 / G; }

template <int N, int G>
struct Smem {
    static constexpr int LD = (N % 2 == 0) ? N + 1 : N;   // odd row stride: conflict-free columns
    static constexpr int kJ = 0;                            // J / LU rows, N x LD
    static constexpr int kRecOff = kJ + N * LD;             // G x kRec
    static constexpr int kC = kRecOff + G * kRec;           // clamped c
    static constexpr int kG0 = kC + N;
    static constexpr int kDG0 = kG0 + N;
    static constexpr int kCp = kDG0 + N;
    static constexpr int kH = kCp + N;
    static constexpr int kDCp = kH + N;
    static constexpr int kB = kDCp + N;                     // permuted rhs
    static constexpr int kX = kB + N;                       // solution
    static constexpr int kMisc = kX + N;                    // T, scalars
    static constexpr int kRed = kMisc + 8;                  // 4 doubles
    static constexpr int kRedI = kRed + 4;                  // 4 ints (2 doubles' room)
    static constexpr int kSize = kRedI + 4;                 // doubles
};

// X: the mechanism may use the rate forms only some mechanisms need (SRI
// fall-off, explicit reverse parameters, PLOG tables). The integrator is
// instantiated with and without them and launched without them when the
// mechanism has none, so that their branches cost the common forms nothing.
template <int N, int G, bool X = true>
struct CellCtx {
    const DevMech &m;
    const IntegratorParams &P;
    Group<G> g;
    double *s;        // this cell's shared memory
    int nsp;
    double p;
    double rho0;      // the cell's density (constant-volume reactor)
    int n_jac, n_rhs, n_lu, n_newton, n_steps, n_attempts;
    int status;

    __device__ CellCtx(const DevMech &mm, const IntegratorParams &pp, Group<G> gg, double *sm)
        : m(mm), P(pp), g(gg), s(sm), nsp(mm.nsp), p(0), rho0(0), n_jac(0), n_rhs(0), n_lu(0),
          n_newton(0), n_steps(0), n_attempts(0), status(0) {}

    // ---------------------------------------------------------------------
    // f(y) and, if jac, the analytic Jacobian rows into shared memory.
    // y is this lane's element (lane < N). Returns this lane's f element.
    // chemistrySource::DyDt (chemistrySource.cpp:863-883) / ::jacobian (:967-1021);
    // constant volume (X and P.reactor == 1): :885-906 / :975-981, 1022-1055
    __device__ __forceinline__ double evaluate(double y, bool jac) {
        using L = Smem<N, G>;
        const int lane = g.lane;
        const bool cv = X && P.reactor == 1;
        if (jac) ++n_jac; else ++n_rhs;
        // the constant-volume right-hand side takes c as given, the Jacobian and the
        // constant-pressure forms the clamped c
        if (lane < nsp) s[L::kC + lane] = (cv && !jac) ? y : hmax(y, 0.0);
        if (lane == nsp) s[L::kMisc] = y;
        g.sync();
        const double T = s[L::kMisc];
        const double logT = log(T);
        if (cv) {
            // p = rho0 Rm T with Y = c W / rho0 (perfectGas::pm, speciesList::MWbyYi)
            double t = 0.0;
            if (lane < nsp) {
                const double Wl = ldg(&m.W[lane]);
                t = (s[L::kC + lane] * Wl / rho0) / Wl;
            }
            const double wsum = g.sum(t);
            p = rho0 * (kRu / (1.0 / hmax(wsum, kVeryTiny))) * T;
        }
        if (lane < nsp) {
            const SpeciesThermo th = species_thermo(m, lane, T, logT);
            s[L::kG0 + lane] = th.G0;
            s[L::kDG0 + lane] = th.DG0DT;
            // constant volume: molar Cv = Cp - Ru and E = H - Ru T take the place of
            // Cp and H in the temperature equation (thermo.inl:80-94, 168-171)
            s[L::kCp + lane] = cv ? th.cp - kRu : th.cp;
            s[L::kH + lane] = cv ? th.h - kRu * T : th.h;
            s[L::kDCp + lane] = th.dcp;
        }
        double *Jrow = &s[L::kJ + lane * L::LD];
        if (jac && lane < N) {
            // species rows, the temperature row and any padding rows start at zero
            for (int j = 0; j < N; ++j) Jrow[j] = 0.0;
        }
        g.sync();
        const double *c = &s[L::kC];
        double f = 0.0;
        int ptr = 0, pend = 0;
        if (lane < nsp) {
            ptr = ldg(&m.sp_ptr[lane]);
            pend = ldg(&m.sp_ptr[lane + 1]);
        }
        for (int base = 0; base < m.nrc; base += G) {
            const int r = base + lane;
            if (r < m.nrc) reaction_record(r, T, logT, c, jac, &s[L::kRecOff + lane * kRec]);
            g.sync();
            if (lane < nsp) {
                while (ptr < pend) {
                    const int rr = ldg(&m.sp_rxn[ptr]);
                    if (rr >= base + G) break;
                    apply_record(rr, ldg(&m.sp_coef[ptr]), &s[L::kRecOff + (rr - base) * kRec], jac,
                                 Jrow, f);
                    ++ptr;
                }
            }
            g.sync();
        }
        // temperature equation: constant pressure (cp, h) or constant volume (cv, e)
        const bool sp = lane < nsp;
        const double cpi = sp ? s[L::kCp + lane] : 0.0;
        const double hi = sp ? s[L::kH + lane] : 0.0;
        const double cCp = g.sum(sp ? y * cpi : 0.0);
        const double dcCpdT = jac ? g.sum(sp ? y * s[L::kDCp + lane] : 0.0) : 0.0;
        double DTdt = g.sum(sp ? f * hi : 0.0);
        DTdt /= cCp;
        if (lane == nsp) f = -DTdt;
        if (jac) {
            // d(dT/dt)/dc_i: column i of the species block (chemistrySource.cpp:1003-1011)
            if (sp) {
                double d = 0.0;
                for (int j = 0; j < nsp; ++j) d -= s[L::kJ + j * L::LD + lane] * s[L::kH + j];
                d += cpi * DTdt;
                d /= cCp;
                s[L::kJ + nsp * L::LD + lane] = d;
            }
            const double part = sp ? (cpi * f + hi * Jrow[nsp]) : 0.0;
            double dd = -g.sum(part);
            dd += dcCpdT * DTdt;
            dd /= cCp;
            if (lane == nsp) s[L::kJ + nsp * L::LD + nsp] = dd;
            g.sync();
        }
        return f;
    }

    // one reaction: q and the derivative pieces (reactionTypes.cpp:263-352, 354-445, 843-876)
    __device__ __forceinline__ void reaction_record(int r, double T, double logT, const double *c,
                                                 bool jac, double *rec) {
        using L = Smem<N, G>;
        const int type = ldg(&m.rate_type[r]);
        const double A = ldg(&m.arr[3 * r]), b = ldg(&m.arr[3 * r + 1]), Ta = ldg(&m.arr[3 * r + 2]);
        const int nf = ldg(&m.nf[r]), nb = ldg(&m.nb[r]);
        int fi[kMaxSide], bi[kMaxSide];
        double fo[kMaxSide], bo[kMaxSide];
#pragma unroll
        for (int k = 0; k < kMaxSide; ++k) {
            fi[k] = (k < nf) ? ldg(&m.fidx[kMaxSide * r + k]) : 0;
            bi[k] = (k < nb) ? ldg(&m.bidx[kMaxSide * r + k]) : 0;
            fo[k] = (k < nf) ? ldg(&m.ford[kMaxSide * r + k]) : 0.0;
            bo[k] = (k < nb) ? ldg(&m.bord[kMaxSide * r + k]) : 0.0;
        }
        double M = 0.0;
        // PLOG, Landau-Teller, Janev and power series (codes 6 and up) carry no third body
        if (type != kArrhenius && !(X && type >= kPLOG)) {
            const double *e = &m.eff[(int64_t)r * nsp];
            for (int i = 0; i < nsp; ++i) M += ldg(&e[i]) * c[i];
        }
        double kf, k0 = 0.0, kinf = 0.0, Pr = 0.0, F = 1.0, lf = 0.0;
        double b0 = 0.0, Ta0 = 0.0;
        if (type == kArrhenius) {
            kf = arrK_log(A, b, Ta, T, logT);
        } else if (type == kThirdBody) {
            kf = M * arrK_log(A, b, Ta, T, logT);
        } else if (X && type == kPLOG) {
            kf = plog_k_global(m.plog_ptr, m.plog_p, m.plog_arr, r, p, T, logT);
        } else if (X && type == kLandauTeller) {
            kf = lt_k_global(&m.arr[3 * r], &m.lt[2 * r], T, logT);
        } else if (X && type >= kJanev) {
            kf = xrate_k_global(type, &m.arr[3 * r], &m.xcoef[9 * r], T, logT);
        } else {
            const double A0 = ldg(&m.arr0[3 * r]);
            b0 = ldg(&m.arr0[3 * r + 1]);
            Ta0 = ldg(&m.arr0[3 * r + 2]);
            k0 = arrK_log(A0, b0, Ta0, T, logT);
            kinf = arrK_log(A, b, Ta, T, logT);
            Pr = k0 / notZeroD(kinf) * M;
            if (X && type == kSRI) {
                F = sri_F_global(&m.sri[5 * r], T, Pr);
            } else {
                if (type != kLindemann) lf = troe_logfcent(&m.troe[4 * r], type == kTroe4, T);
                F = fall_F(type, lf, Pr);
            }
            // chemicallyActicatedBimolecularRR::k (chemicallyActicatedBimolecularRR.cpp:36-44)
            if (X && ldg(&m.activated[r])) kf = k0 * (1.0 / (1.0 + Pr)) * F;
            else kf = kinf * (Pr / (1.0 + Pr)) * F;
        }
        double kr = 0.0, Kc = 0.0, DKcDT = 0.0;
        const int rev_kind = ldg(&m.reversible[r]);
        const bool rev = rev_kind != 0;
        if (X && rev_kind == kRevExplicit) {
            // reversibleReactionWithRevPars::kr (reversibleReactionWithRevPars.hpp:68-76):
            // the reverse rate law of the same kind, M times it for third-body;
            // a Landau-Teller reaction's reverse B, C (Chemkin RLT) sit in xcoef
            if (type == kLandauTeller) kr = lt_k_global(&m.arr_rev[3 * r], &m.xcoef[9 * r], T, logT);
            else kr = arr_global(&m.arr_rev[3 * r], T, logT);
            if (type == kThirdBody) kr = M * kr;
        } else if (rev) {
            const double *sg = s;
            const EquilK eq = equilibrium(
                m, r, T, [sg](int i) { return sg[L::kG0 + i]; },
                [sg](int i) { return sg[L::kDG0 + i]; });
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
                pf[k] = conc_pow(c[fi[k]], fo[k]);
                qf *= pf[k];
            }
            if (k < nb) {
                pb[k] = conc_pow(c[bi[k]], bo[k]);
                qr *= pb[k];
            }
        }
        const double q = qf - qr;
        rec[0] = q;
        if (!jac) return;
        // d q / d c_k of each reactant (DqDci forward part) and product (reverse part)
#pragma unroll
        for (int k = 0; k < kMaxSide; ++k) {
            if (k < nf) {
                double d = kf;
#pragma unroll
                for (int j = 0; j < kMaxSide; ++j) {
                    if (j < nf) {
                        const double ord = fo[j];
                        const double cj = c[fi[j]];
                        if (j == k) {
                            if (ord == 1.0) continue;
                            if (ord < 1.0) d *= (cj > kTiny) ? ord * pow_n(cj, ord - 1.0) : 0.0;
                            else d *= ord * pow_n(hmax(cj, 0.0), ord - 1.0);
                        } else {
                            d *= pf[j];
                        }
                    }
                }
                rec[2 + k] = d;
            }
            if (k < nb) {
                double d = kr;
#pragma unroll
                for (int j = 0; j < kMaxSide; ++j) {
                    if (j < nb) {
                        const double ord = bo[j];
                        const double cj = c[bi[j]];
                        if (j == k) {
                            if (ord == 1.0) continue;
                            if (ord < 1.0) d *= (cj > kTiny) ? ord * pow_n(cj, ord - 1.0) : 0.0;
                            else d *= ord * pow_n(hmax(cj, 0.0), ord - 1.0);
                        } else {
                            d *= pb[j];
                        }
                    }
                }
                rec[6 + k] = d;
            }
        }
        // d q / d T (DqDT)
        const double invT = 1.0 / hmax(T, kTiny);
        double dkfdT;
        if (type == kArrhenius || type == kThirdBody) {
            dkfdT = kf * invT * (b + Ta * invT);
        } else if (X && type == kPLOG) {
            dkfdT = plog_dkdt_global(m.plog_ptr, m.plog_p, m.plog_arr, r, kf, p, T, logT);
        } else if (X && type == kLandauTeller) {
            dkfdT = lt_dkdt_global(&m.arr[3 * r], &m.lt[2 * r], kf, T);
        } else if (X && type >= kJanev) {
            dkfdT = xrate_dkdt_global(type, &m.arr[3 * r], &m.xcoef[9 * r], kf, T, logT);
        } else if (X && ldg(&m.activated[r])) {
            dkfdT = (1.0 / (1.0 + Pr)) * F * (k0 * invT * (b0 + Ta0 * invT));
        } else {
            dkfdT = (Pr / (1.0 + Pr)) * F * (kinf * invT * (b + Ta * invT));
        }
        double dkrdT = 0.0;
        if (X && rev_kind == kRevExplicit && type == kLandauTeller)
            dkrdT = lt_dkdt_global(&m.arr_rev[3 * r], &m.xcoef[9 * r], kr, T);
        else if (X && rev_kind == kRevExplicit)
            dkrdT = kr * invT * (ldg(&m.arr_rev[3 * r + 1]) + ldg(&m.arr_rev[3 * r + 2]) * invT);
        else if (rev) dkrdT = (dkfdT - kr * DKcDT) / hmax(Kc, kVeryTiny);
#pragma unroll
        for (int k = 0; k < kMaxSide; ++k) {
            if (k < nf) dkfdT *= pf[k];
            if (k < nb) dkrdT *= pb[k];
        }
        double dqjdT = dkfdT - dkrdT;
        double dgdT = 0.0;
        double kind = 0.0;
        // third-body and fall-off columns are rank one in the efficiencies:
        // d q / d c_i = eff_i * g_r, with g_r = q / M (third body) or
        // q (k0/kinf) (1/(Pr(1+Pr)) + F'/(Pr F)) (fall-off,
        // unimolecularFallOffRR::gamDGamDCi, unimolecularFallOffRR.cpp:55-91);
        // the record carries g_r so that each row adds eff_i * (coef g_r)
        if (type == kThirdBody) {
            kind = 1.0;
            rec[11] = q / hmax(M, kTiny);
        } else if (type != kArrhenius && !(X && type >= kPLOG)) {
            if (M > kTiny) {
                // unimolecularFallOffRR::gamDGamDT (unimolecularFallOffRR.cpp:55-91)
                const double Pr2 = k0 * M / notZeroD(kinf);
                const double F2 =
                    (X && type == kSRI) ? sri_F_global(&m.sri[5 * r], T, Pr2) : fall_F(type, lf, Pr2);
                const double dPrdT = Pr2 * ((k0 * invT * (b0 + Ta0 * invT)) / notZeroD(k0) -
                                            (kinf * invT * (b + Ta * invT)) / notZeroD(kinf));
                const double dFdT = (X && type == kSRI)
                                        ? sri_dfdt_global(&m.sri[5 * r], T, Pr2, F2, dPrdT)
                                        : troe_dfdt(type, &m.troe[4 * r], T, Pr2, F2, dPrdT);
                const double fabc = (X && type == kSRI)
                                        ? sri_dfdci_factor_global(&m.sri[5 * r], T, Pr2, F2)
                                        : troe_dfdci_factor(type, lf, Pr2, F2);
                double g;
                if (X && ldg(&m.activated[r])) {
                    // chemicallyActicatedBimolecularRR::gamDGamDT / gamDGamDCi
                    // (chemicallyActicatedBimolecularRR.cpp:56-96)
                    dgdT = q * (-dPrdT / (1 + Pr2) + dFdT / F2);
                    g = q * (k0 / notZeroD(kinf)) * (-1.0 / (1 + Pr2) + fabc * (1.0 / Pr2) / F2);
                } else {
                    dgdT = q * (dPrdT / (Pr2 * (1 + Pr2)) + dFdT / F2);
                    g = q * (k0 / notZeroD(kinf)) *
                        (1.0 / (Pr2 * (1 + Pr2)) + fabc * (1.0 / Pr2) / F2);
                }
                kind = finite(g) ? 2.0 : 3.0;
                rec[11] = g;
            } else {
                kind = 3.0;
            }
        }
        if (!finite(dqjdT)) dqjdT = 0;
        if (!finite(dgdT)) dgdT = 0;
        rec[1] = dqjdT + dgdT;
        rec[10] = kind;
    }

    // species row `lane` gets reaction r's contributions (coef = -nu' or +nu'')
    __device__ __forceinline__ void apply_record(int r, double coef, const double *rec, bool jac,
                                                 double *Jrow, double &f) {
        const double q = rec[0];
        f += coef * q;
        if (!jac) return;
        const int nf = ldg(&m.nf[r]), nb = ldg(&m.nb[r]);
        for (int k = 0; k < nf; ++k) Jrow[ldg(&m.fidx[kMaxSide * r + k])] += coef * rec[2 + k];
        for (int k = 0; k < nb; ++k) Jrow[ldg(&m.bidx[kMaxSide * r + k])] += (-coef) * rec[6 + k];
        const double kind = rec[10];
        if (kind == 1.0 || kind == 2.0) {
            const double *e = &m.eff[(int64_t)r * nsp];
            const double s = coef * rec[11];
            for (int i = 0; i < nsp; ++i) Jrow[i] += ldg(&e[i]) * s;
        }
        Jrow[nsp] += coef * rec[1];
    }

    // ---------------------------------------------------------------------
    // Newton matrix I - dt J, LU with partial pivoting; rows left in smem in
    // pivot order. Returns this lane's pivot step (or -1 for padding lanes).
    // The elimination steps are instantiated one by one (lu_step<K>) so that
    // the lane's row stays in registers with static indices.
    template <int K>
    __device__ __forceinline__ void lu_step(double (&a)[N], bool &act, int &mystep) {
        using L = Smem<N, G>;
        const int p = g.argmax(act ? fabs(a[K]) : -1.0);
        if (g.lane == p) {
            mystep = K;
            act = false;
#pragma unroll
            for (int j = 0; j < N; ++j) s[L::kJ + K * L::LD + j] = a[j];
        }
        g.sync();
        if (act) {
            const double *pr = &s[L::kJ + K * L::LD];
            const double l = a[K] / pr[K];
            a[K] = l;
#pragma unroll
            for (int j = K + 1; j < N; ++j) a[j] -= l * pr[j];
        }
        if constexpr (K + 1 < N) lu_step<K + 1>(a, act, mystep);
    }

    __device__ __forceinline__ int factor(double dt) {
        using L = Smem<N, G>;
        const int lane = g.lane;
        double a[N];
        if (lane < N) {
#pragma unroll
            for (int j = 0; j < N; ++j) a[j] = -dt * s[L::kJ + lane * L::LD + j];
#pragma unroll
            for (int j = 0; j < N; ++j)
                if (j == lane) a[j] += 1.0;
        } else {
#pragma unroll
            for (int j = 0; j < N; ++j) a[j] = 0.0;
        }
        ++n_lu;
        g.sync();   // every row read before the factor overwrites the buffer
        bool act = lane < N;
        int mystep = -1;
        lu_step<0>(a, act, mystep);
        return mystep;
    }

    // solve (LU) x = b; b is this lane's element; returns x element
    __device__ __forceinline__ double solve(int mystep, double b) {
        using L = Smem<N, G>;
        const int lane = g.lane;
        if (mystep >= 0) s[L::kB + mystep] = b;
        g.sync();
        if (g.warp == 0) {
            constexpr int GW = Group<G>::GW;
            constexpr int R = (N + GW - 1) / GW;
            const int wl = g.wlane;
            double z[R], acc[R];
#pragma unroll
            for (int q = 0; q < R; ++q) {
                const int i = wl + GW * q;
                z[q] = (i < N) ? s[L::kB + i] : 0.0;
                acc[q] = 0.0;
            }
            // forward: z_i = b_i - sum_{t<i} L(i,t) z_t (ascending t)
#pragma unroll
            for (int t = 0; t < N; ++t) {
                const int q_t = t / GW, l_t = t % GW;
                const double mine = z[q_t] - acc[q_t];
                const double zt = __shfl_sync(g.mask, mine, g.base + l_t);
                if (wl == l_t) z[q_t] = zt;
#pragma unroll
                for (int q = 0; q < R; ++q) {
                    const int i = wl + GW * q;
                    if (i > t && i < N) acc[q] += s[L::kJ + i * L::LD + t] * zt;
                }
            }
            // backward: x_t = (z_t - sum_{j>t} U(t,j) x_j) / U(t,t)
#pragma unroll
            for (int q = 0; q < R; ++q) acc[q] = 0.0;
#pragma unroll
            for (int t = N - 1; t >= 0; --t) {
                const int q_t = t / GW, l_t = t % GW;
                const double mine = (z[q_t] - acc[q_t]) / s[L::kJ + t * L::LD + t];
                const double xt = __shfl_sync(g.mask, mine, g.base + l_t);
                if (wl == 0) s[L::kX + t] = xt;
#pragma unroll
                for (int q = 0; q < R; ++q) {
                    const int i = wl + GW * q;
                    if (i < t) acc[q] += s[L::kJ + i * L::LD + t] * xt;
                }
            }
        }
        g.sync();
        return (lane < N) ? s[L::kX + lane] : 0.0;
    }
};

enum CellRc : int { kRcOk = 0, kRcUnderflow = 1, kRcIterLimit = 2 };

template <int N, int G, bool X = true>
struct CellIntegrator : CellCtx<N, G, X> {
    using Base = CellCtx<N, G, X>;
    using Base::g;
    using Base::P;
    using Base::nsp;
    int countStep;
    double lts0, lts1;          // lastTimeStep_[0], [1]
    double yk0, yk1;            // yklast_[0], [1] (this lane's element)

    __device__ CellIntegrator(const DevMech &mm, const IntegratorParams &pp, Group<G> gg,
                              double *sm)
        : Base(mm, pp, gg, sm), countStep(0), lts0(0), lts1(0), yk0(0), yk1(0) {}

    // ODEsSolver::maxError (ODEsSolver.cpp:37-46); NaN terms do not raise the max
    __device__ double max_error(double y0, double y, double e) {
        double v = 0.0;
        if (g.lane < N) {
            const double tol = P.atol + P.rtol * hmax(fabs(y0), fabs(y));
            v = fabs(e) / tol;
            if (isnan(v)) v = 0.0;
        }
        return g.max(v);
    }

    // ImplicitEuler::maxIncrement (ImplicitEuler.cpp:40-52)
    __device__ double max_increment(double y0, double y, double e) {
        const bool nan_y = (g.lane < N) && isnan(y);
        if (g.any(nan_y)) return 1.5;
        double v = 0.0;
        if (g.lane < N) {
            const double tol = P.atol_inc + P.rtol_inc * hmax(fabs(y0), fabs(y));
            v = fabs(e) / tol;
            if (isnan(v)) v = 0.0;
        }
        return g.max(v);
    }

    // ImplicitEuler::NewtonIteration (ImplicitEuler.cpp:161-251)
    __device__ double newton(double y0, double dt, double &yk, bool &conv, int &rc) {
        int count = 0;
        double maxErr = 0.0, lastErr = 0.0;
        int mystep = -1;
        const bool autoJ = P.auto_update_jacobian != 0;
        const int stepJ = P.step_to_update_jac;
        do {
            double f;
            if (!autoJ || count == 0 || count % stepJ == 0) {
                f = this->evaluate(yk, true);
                mystep = this->factor(dt);
            } else {
                f = this->evaluate(yk, false);
            }
            const double rhs = (g.lane < N) ? ((-yk + y0) + dt * f) : 0.0;
            const double x = this->solve(mystep, rhs);
            ++this->n_newton;
            const bool bad = (g.lane < N) && !finite(x);
            const int firstBad = g.min_int(bad ? g.lane : 1 << 30);
            if (firstBad < (1 << 30)) {
                if (g.lane < firstBad) yk += x;
                conv = false;
                return 1000.0;
            }
            if (g.lane < N) yk += x;
            maxErr = max_error(yk, yk, x);
            if (count > 0) {
                const double diver = maxErr / hmax(lastErr, kTiny);
                if (autoJ) {
                    const int lim = (30 * stepJ > 50) ? 30 * stepJ : 50;
                    if (diver > 2 && count > lim) {
                        conv = false;
                        return 1000.0;
                    }
                } else if (diver > 2 && count > 5) {
                    conv = false;
                    return 1000.0;
                }
            }
            lastErr = maxErr;
            count++;
            if (isnan(maxErr)) {
                conv = false;
                return 1000.0;
            }
            if (count > 1000) {
                conv = false;
                return maxErr;
            }
            if (P.max_newton_total > 0 && this->n_newton >= P.max_newton_total) {
                rc = kRcIterLimit;
                conv = false;
                return 1000.0;
            }
        } while (maxErr > 1.0);
        conv = true;
        return maxErr;
    }

    // ImplicitEuler::solve(t0, y0, dydt0, dt, y) (ImplicitEuler.cpp:101-142)
    __device__ double step(double y0, double dt, double &y, int &rc) {
        ++this->n_attempts;
        double yk = y0;
        bool conv = true;
        const double errN = newton(y0, dt, yk, conv, rc);
        y = yk;
        if (!conv) return errN;
        double e = 0.0;
        if (countStep == 0) {
            const double f = this->evaluate(yk, false);
            e = yk - y0 - dt * f;
        } else {
            const double dtn = lts0, dtn1 = lts1;
            const double f1 = 2.0 / (dtn * (dtn + dtn1));
            const double f2 = 2.0 / (dtn1 * (dtn + dtn1));
            const double LTEF = (dtn * dtn) * 0.5;
            e = f1 * (yk - y0) - f2 * (y0 - yk1);
            e *= LTEF;
        }
        return max_increment(y0, yk, e);
    }

    __device__ double bcast_T(double v) {
        using L = Smem<N, G>;
        if (g.lane == nsp) this->s[L::kMisc + 1] = v;
        g.sync();
        const double r = this->s[L::kMisc + 1];
        g.sync();
        return r;
    }

    // ImplicitEuler::adaptiveSolve (ImplicitEuler.cpp:253-292) with checkNewY
    // (chemistrySource.cpp:1152-1164)
    __device__ int adaptive(double &t, double &dt0, double &y) {
        double dt = dt0;
        double error = 0.0;
        double yTemp = y;
        lts1 = lts0;
        int count = 0;
        const double Told = bcast_T(y);
        do {
            lts0 = dt;
            int rc = kRcOk;
            error = step(y, dt, yTemp, rc);
            if (rc != kRcOk) return rc;
            const double Tnew = bcast_T(yTemp);
            bool ok = true;
            if ((Tnew - Told) > P.T_alpha * Told) {
                dt *= P.T_beta;
                ok = false;
            }
            if (!ok && count < 100) {
                error = 2;
                count++;
                if (dt <= kVeryTiny) return kRcUnderflow;
                continue;
            }
            if (error > 1.0) {
                const double scale = hmax(P.safescale * pow(error, -P.alphainc), P.minscale);
                dt *= scale;
                if (dt <= kVeryTiny) return kRcUnderflow;
            }
        } while (error > 1.0);
        t += dt;
        y = yTemp;
        ++this->n_steps;
        if (error > P.err_accept_limit)
            dt0 = hmin(hmax(P.safescale * pow(error, -P.alphainc), P.minscale), P.maxscale) * dt;
        else
            dt0 = hmax(P.safescale * P.maxscale * dt, dt);
        return kRcOk;
    }

    // ImplicitEuler::solve(t0, tn, dt0, y) (ImplicitEuler.cpp:294-342), t0 = 0
    __device__ int interval(double &tn, double &dt0, double &y) {
        double t = 0.0;
        double dt = 0.2 * dt0;
        double dtReached = 0.0;
        bool last = false;
        for (int n = 0; n < P.maxstep; ++n) {
            countStep = n;
            if (n == 0) {
                yk0 = y;
            } else {
                yk1 = yk0;
                yk0 = y;
            }
            const double dtTry0 = dt;
            if ((t + dt - tn) * (t + dt - 0.0) > 0) {
                dt = tn - t;
                last = true;
            } else if (t + dt == tn) {
                last = true;
            }
            const int rc = adaptive(t, dt, y);
            if (rc != kRcOk) return rc;
            dtReached = t;
            if ((t - tn) * (tn - 0.0) >= 0) {
                if (n > 0 && last) dt0 = hmin(dtTry0, tn);
                return kRcOk;
            }
        }
        this->status |= 2;  // HC_CELL_MAXSTEP
        tn = dtReached;
        return kRcOk;
    }
};

template <int G>
__device__ __forceinline__ Group<G> make_group(double *s, int gid, int red_off, int redi_off) {
    Group<G> g;
    g.lane = threadIdx.x % G;
    g.wlane = (G < 32) ? g.lane : (threadIdx.x & 31);
    g.warp = g.lane >> 5;
    g.base = (G < 32) ? ((threadIdx.x & 31) & ~(G - 1)) : 0;
    g.mask = (G < 32) ? (((1u << G) - 1u) << g.base) : 0xffffffffu;
    g.barid = 1 + gid;
    g.red = s + red_off;
    g.redi = reinterpret_cast<int *>(s + redi_off);
    return g;
}

// evaluation-only kernels use no integrator option
__device__ const IntegratorParams kNoParams{};

template <int N, int G, bool X = true>
#ifndef HC_GROUP_MIN_BLOCKS
#define HC_GROUP_MIN_BLOCKS 4   // blocks of 128 threads per SM the 32-lane groups are built for (measured best)
#endif
#ifndef HC_GROUP64_MIN_BLOCKS
#define HC_GROUP64_MIN_BLOCKS 2   // the same for the 64-lane groups
#endif
__global__ void __launch_bounds__(128, (G == 64) ? HC_GROUP64_MIN_BLOCKS : HC_GROUP_MIN_BLOCKS)
integrate_kernel(const __grid_constant__ DevMech m, const __grid_constant__ IntegratorParams P,
                 const __grid_constant__ CellIO io) {
    using L = Smem<N, G>;
    extern __shared__ double smem_all[];
    const int gid = threadIdx.x / G;
    double *s = smem_all + (size_t)gid * L::kSize;
    const Group<G> g = make_group<G>(s, gid, L::kRed, L::kRedI);
    const int nsp = m.nsp;
    const int lane = g.lane;
    while (true) {
        long long *slot = reinterpret_cast<long long *>(s + L::kMisc + 2);
        if (lane == 0) *slot = (long long)atomicAdd(io.queue_head, 1ULL);
        g.sync();
        const long long k = *slot;
        g.sync();
        if (k >= io.nqueue) break;
        const int64_t cell = io.order ? (int64_t)io.order[k] : (int64_t)k;
        CellIntegrator<N, G, X> ci(m, P, g, s);
        const double Ti = io.T[cell];
        const double tstep = io.dt[cell] * io.dt_factor;
        const double rho0 = io.rho[cell];
        const double W = (lane < nsp) ? ldg(&m.W[lane]) : 1.0;
        double y = 0.0;
        if (lane < nsp) y = rho0 * io.Y[(int64_t)lane * io.ncells + cell] / W;
        const double c0 = y;
        if (Ti < P.T_threshold) {
            if (lane == 0) {
                io.subdt[cell] = tstep;
                if (io.status) io.status[cell] = 1;  // HC_CELL_SKIPPED
                if (io.cost) io.cost[cell] = 0;
            }
            if (io.Ri && lane < nsp) io.Ri[(int64_t)lane * io.ncells + cell] = 0.0;
            continue;
        }
        ci.p = io.p[cell];
        ci.rho0 = io.rho[cell];
        double leftTime = tstep;
        double sub = hmin(leftTime, hmin(io.subdt[cell], P.dt_max));
        if (lane == nsp) y = Ti;
        int rc = kRcOk;
        while (leftTime > 0.0) {
            double d = leftTime;
            rc = ci.interval(d, sub, y);
            if (rc != kRcOk) break;
            leftTime -= d;
        }
        if (rc == kRcUnderflow) ci.status |= 4;
        if (rc == kRcIterLimit) ci.status |= 8;
        // ciToYi (chemistrySource.cpp:1225-1246) and rho = p / (Rm T)
        const double Tn = ci.bcast_T(y);
        double yi = (lane < nsp) ? hmax(0.0, y) : 0.0;
        const double rr = g.sum(yi * ((lane < nsp) ? W : 0.0));
        yi = (lane < nsp) ? yi * W / hmax(rr, kTiny) : 0.0;
        const double ys = g.sum(yi);
        if (ys != 1.0) yi /= ys;
        const double wsum = g.sum((lane < nsp) ? yi / W : 0.0);
        const double Rm = kRu / (1.0 / hmax(wsum, kVeryTiny));
        if (lane < nsp) {
            io.Y[(int64_t)lane * io.ncells + cell] = yi;
            if (io.Ri) io.Ri[(int64_t)lane * io.ncells + cell] = (y - c0) / tstep * W;
        }
        if (lane == 0) {
            io.T[cell] = Tn;
            // constant volume keeps the density (the reference updates p instead,
            // chemistrySource.cpp:1317-1323)
            if (!(X && P.reactor == 1)) io.rho[cell] = ci.p / (Rm * Tn);
            io.subdt[cell] = sub;
            if (io.status) io.status[cell] = ci.status;
            if (io.cost) io.cost[cell] = ci.n_newton;
            if (io.counters) {
                atomicAdd(&io.counters[0], (unsigned long long)ci.n_jac);
                atomicAdd(&io.counters[1], (unsigned long long)ci.n_rhs);
                atomicAdd(&io.counters[2], (unsigned long long)ci.n_lu);
                atomicAdd(&io.counters[3], (unsigned long long)ci.n_newton);
                atomicAdd(&io.counters[4], (unsigned long long)ci.n_steps);
                atomicAdd(&io.counters[5], (unsigned long long)ci.n_attempts);
            }
        }
    }
}

// f(y) and the analytic Jacobian at given states (chemistrySource::DyDt,
// ::jacobian); one cell group per state.
template <int N, int G>
__global__ void __launch_bounds__(128)
rhs_jac_kernel(const __grid_constant__ DevMech m, int64_t n, const double *c, const double *T,
               const double *p, double *dydt, double *J) {
    using L = Smem<N, G>;
    extern __shared__ double smem_all[];
    constexpr int CPB = cells_per_block(G);
    const int gid = threadIdx.x / G;
    double *s = smem_all + (size_t)gid * L::kSize;
    const int64_t k = (int64_t)blockIdx.x * CPB + gid;
    if (k >= n) return;
    const Group<G> g = make_group<G>(s, gid, L::kRed, L::kRedI);
    CellCtx<N, G> ctx(m, kNoParams, g, s);
    ctx.p = p[k];
    const int nsp = m.nsp, lane = g.lane, n1 = nsp + 1;
    double y = 0.0;
    if (lane < nsp) y = c[(int64_t)lane * n + k];
    if (lane == nsp) y = T[k];
    const double f = ctx.evaluate(y, J != nullptr);
    if (dydt && lane < n1) dydt[k * n1 + lane] = f;
    if (J && lane < n1) {
        for (int j = 0; j < n1; ++j)
            J[k * n1 * n1 + (int64_t)lane * n1 + j] = s[L::kJ + lane * L::LD + j];
    }
}

// explicit source terms omega_i W_i (chemistrySource::calculateSourceTerms,
// chemistrySource.cpp:1370-1406)
template <int N, int G>
__global__ void __launch_bounds__(128)
source_kernel(const __grid_constant__ DevMech m, int64_t n, const double *T, const double *p,
              const double *rho, const double *Y, double *Ri) {
    using L = Smem<N, G>;
    extern __shared__ double smem_all[];
    constexpr int CPB = cells_per_block(G);
    const int gid = threadIdx.x / G;
    double *s = smem_all + (size_t)gid * L::kSize;
    const int64_t k = (int64_t)blockIdx.x * CPB + gid;
    if (k >= n) return;
    const Group<G> g = make_group<G>(s, gid, L::kRed, L::kRedI);
    CellCtx<N, G> ctx(m, kNoParams, g, s);
    ctx.p = p[k];
    const int nsp = m.nsp, lane = g.lane;
    double y = 0.0;
    if (lane < nsp) y = rho[k] * Y[(int64_t)lane * n + k] / ldg(&m.W[lane]);
    if (lane == nsp) y = T[k];
    const double f = ctx.evaluate(y, false);
    if (lane < nsp) Ri[(int64_t)lane * n + k] = f * ldg(&m.W[lane]);
}

// point-implicit source terms (chemistrySource::calculateSourceTermsImp with
// withoutLastSpec = true, chemistrySource.cpp:1412-1450, via omegaCoupled,
// :422-480): Ri_i = omega_i W_i for every species and, for j < nsp - 1,
//   diag_j = J_jj - (W_j / W_L) J_jL + J_jT W_j (e_L - e_j) / (rho c_v)
// with L the last species (c_L follows from the others at fixed density,
// reactionTypes.cpp:761-832), e_i = h_i - R_i T (thermo.inl:168-171) and
// c_v = c_p - R_mix (thermoList.inl:145-149)
template <int N, int G>
__global__ void __launch_bounds__(128)
source_imp_kernel(const __grid_constant__ DevMech m, int64_t n, const double *T, const double *p,
                  const double *rho, const double *Y, double *Ri, double *diag) {
    using L = Smem<N, G>;
    extern __shared__ double smem_all[];
    constexpr int CPB = cells_per_block(G);
    const int gid = threadIdx.x / G;
    double *s = smem_all + (size_t)gid * L::kSize;
    const int64_t k = (int64_t)blockIdx.x * CPB + gid;
    if (k >= n) return;
    const Group<G> g = make_group<G>(s, gid, L::kRed, L::kRedI);
    CellCtx<N, G> ctx(m, kNoParams, g, s);
    ctx.p = p[k];
    const int nsp = m.nsp, lane = g.lane, Ls = nsp - 1;
    const double W = (lane < nsp) ? ldg(&m.W[lane]) : 1.0;
    const double Yi = (lane < nsp) ? Y[(int64_t)lane * n + k] : 0.0;
    const double Tk = T[k], rk = rho[k];
    double y = 0.0;
    if (lane < nsp) y = rk * Yi / W;
    if (lane == nsp) y = Tk;
    const double f = ctx.evaluate(y, true);
    if (lane < nsp) Ri[(int64_t)lane * n + k] = f * W;
    double cpi = 0.0, hi = 0.0;
    if (lane < nsp) species_cp_h(m, lane, Tk, cpi, hi);
    const double cp_mix = g.sum(Yi * cpi);
    const double ymw = g.sum((lane < nsp) ? Yi / W : 0.0);
    const double cv = cp_mix - kRu * ymw;
    const double ei = hi - (kRu / W) * Tk;
    if (lane == Ls) s[L::kMisc + 5] = ei;
    g.sync();
    const double eL = s[L::kMisc + 5];
    if (lane < Ls) {
        const double *row = &s[L::kJ + lane * L::LD];
        const double WL = ldg(&m.W[Ls]);
        diag[(int64_t)lane * n + k] =
            row[lane] - (W / WL) * row[Ls] + row[nsp] * W * (eL - ei) / (rk * cv);
    }
}

}  // namespace hc
