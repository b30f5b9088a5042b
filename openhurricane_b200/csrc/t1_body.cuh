// The per-thread implicit-Euler state machine of the thread-per-cell
// integrators, shared by the precompiled kernel (mechanism read from tables,
// integrator_t1.cuh) and the kernels generated for one mechanism and
// compiled at run time (jit.cu). `Cell` supplies the chemistry of one cell:
//   int nsp;                                    species count
//   double W(int i);                            molecular weight
//   void evaluate(const double (&y)[N], bool jac)   f (and J) at y
//   double F(int i);                            f_i of the last evaluation
//   void factor(double dt);                     LU of I - dt J, pivoted
//   static constexpr bool kAssemblesA;          true: evaluate(y, jac, dt) writes
//                                               I - dt J itself and factor()
//                                               only factors it
//   void solve(double (&b)[N]);                 b <- (I - dt J)^-1 b
//
// The reference's nested loops (cell -> ODE interval -> step -> step
// attempt -> Newton iteration; chemistrySource.cpp:1511-1555,
// ImplicitEuler.cpp:101-342, ODEsSolver.cpp:148-225) are flattened into one
// state machine per thread whose only heavy state is "evaluate, factor,
// solve". Every trip round the main loop runs that heavy block for all lanes
// of a warp, then each lane advances its own bookkeeping (accept/reject,
// step control, next cell from the device work queue). The two previous
// step states of ImplicitEuler (yklast_) live in a global per-cell buffer.
#pragma once

#include "rtc_base.cuh"

namespace hc {

enum T1State : int {
    kT1Fetch = 0,
    kT1Interval,
    kT1Step,
    kT1Attempt,
    kT1Newton,      // heavy: J(yk), LU, solve, Newton update
    kT1Err0,        // heavy: f(yk) for the first-step error estimate
    kT1AttemptEnd,
    kT1Done
};

// Lockstep: every thread of the block passes one block barrier per trip of
// the main loop (threads without a cell keep looping until the whole block is
// done), so that the block's warps run the heavy block together and share
// its instruction fetches.
template <int N, bool Lockstep = false, class Cell>
__device__ __forceinline__ void t1_run(Cell &cell, const IntegratorParams &P, const CellIO &io,
                                       double *__restrict__ ylast) {
    constexpr int TI = N - 1;
    const int nsp = cell.nsp;
    double y[N], yk[N];
#pragma unroll
    for (int i = 0; i < N; ++i) y[i] = yk[i] = 0.0;
    int state = kT1Fetch;
    int64_t cellid = -1;
    double leftTime = 0, sub = 0, tstep = 0, p = 0;
    double t = 0, tn = 0, dt = 0, dtReached = 0, dtTry0 = 0, adt = 0, lts0 = 0, lts1 = 0;
    double lastErr = 0, Told = 0, error = 0;
    int nstep = 0, tcount = 0, ncount = 0, cstatus = 0;
    bool last = false;
    int n_jac = 0, n_rhs = 0, n_lu = 0, n_newton = 0, n_steps = 0, n_att = 0;
    double *yk0 = nullptr, *yk1 = nullptr;   // yklast_[0], yklast_[1] in global scratch

    while (true) {
        // ---------------- bookkeeping until the next heavy evaluation
        int guard = 0;
        while (state != kT1Newton && state != kT1Err0 && state != kT1Done && guard < 64) {
            ++guard;
            if (state == kT1Fetch) {
                if (cellid >= 0) {
                    // finish the previous cell: ciToYi and rho (chemistrySource.cpp:1225-1246)
                    double rr = 0.0, yi[N];
#pragma unroll
                    for (int i = 0; i < N; ++i) {
                        yi[i] = 0.0;
                        if (i < nsp) {
                            yi[i] = hmax(0.0, y[i]);
                            rr += yi[i] * cell.W(i);
                        }
                    }
                    const double irr = frcp(hmax(rr, kTiny));
                    double ys = 0.0;
#pragma unroll
                    for (int i = 0; i < N; ++i)
                        if (i < nsp) {
                            yi[i] = yi[i] * cell.W(i) * irr;
                            ys += yi[i];
                        }
                    const double iys = frcp(ys);
                    if (ys != 1.0) {
#pragma unroll
                        for (int i = 0; i < N; ++i)
                            if (i < nsp) yi[i] *= iys;
                    }
                    double wsum = 0.0;
#pragma unroll
                    for (int i = 0; i < N; ++i)
                        if (i < nsp) wsum += yi[i] * (1.0 / cell.W(i));
                    const double Rm = kRu * hmax(wsum, kVeryTiny);
                    const double Tn = y[TI];
                    const double rho0 = io.rho[cellid];
                    const double itstep = frcp(tstep);
#pragma unroll
                    for (int i = 0; i < N; ++i) {
                        if (i < nsp) {
                            const double Wi = cell.W(i);
                            const int64_t at = (int64_t)i * io.ncells + cellid;
                            if (io.Ri) {
                                const double c0 = rho0 * io.Y[at] * (1.0 / Wi);
                                io.Ri[at] = (y[i] - c0) * itstep * Wi;
                            }
                            io.Y[at] = yi[i];
                        }
                    }
                    io.T[cellid] = Tn;
                    io.rho[cellid] = fdiv(p, Rm * Tn);
                    io.subdt[cellid] = sub;
                    if (io.status) io.status[cellid] = cstatus;
                    if (io.cost) io.cost[cellid] = n_newton;
                    if (io.counters) {
                        atomicAdd(&io.counters[0], (unsigned long long)n_jac);
                        atomicAdd(&io.counters[1], (unsigned long long)n_rhs);
                        atomicAdd(&io.counters[2], (unsigned long long)n_lu);
                        atomicAdd(&io.counters[3], (unsigned long long)n_newton);
                        atomicAdd(&io.counters[4], (unsigned long long)n_steps);
                        atomicAdd(&io.counters[5], (unsigned long long)n_att);
                    }
                    cellid = -1;
                }
                const unsigned long long k = atomicAdd(io.queue_head, 1ULL);
                if ((long long)k >= io.nqueue) {
                    state = kT1Done;
                    break;
                }
                cellid = io.order ? (int64_t)io.order[k] : (int64_t)k;
                yk0 = ylast + (size_t)cellid * 2 * N;
                yk1 = yk0 + N;
                n_jac = n_rhs = n_lu = n_newton = n_steps = n_att = 0;
                cstatus = 0;
                const double Ti = io.T[cellid];
                tstep = io.dt[cellid] * io.dt_factor;
                const double rho0 = io.rho[cellid];
                if (Ti < P.T_threshold) {
                    io.subdt[cellid] = tstep;
                    if (io.status) io.status[cellid] = 1;   // HC_CELL_SKIPPED
                    if (io.cost) io.cost[cellid] = 0;
                    if (io.Ri)
                        for (int i = 0; i < nsp; ++i) io.Ri[(int64_t)i * io.ncells + cellid] = 0.0;
                    cellid = -1;
                    continue;
                }
#pragma unroll
                for (int i = 0; i < N; ++i) {
                    y[i] = 0.0;
                    if (i < nsp) y[i] = rho0 * io.Y[(int64_t)i * io.ncells + cellid] * (1.0 / cell.W(i));
                }
                y[TI] = Ti;
                p = io.p[cellid];
                leftTime = tstep;
                sub = hmin(leftTime, hmin(io.subdt[cellid], P.dt_max));
                state = kT1Interval;
            } else if (state == kT1Interval) {
                // ImplicitEuler::solve(t0 = 0, tn = leftTime, dt0 = sub, y)
                tn = leftTime;
                t = 0.0;
                dt = 0.2 * sub;
                dtReached = 0.0;
                last = false;
                nstep = 0;
                state = kT1Step;
            } else if (state == kT1Step) {
                if (nstep >= P.maxstep) {
                    cstatus |= 2;       // HC_CELL_MAXSTEP
                    tn = dtReached;
                    leftTime -= tn;
                    state = (leftTime > 0.0) ? kT1Interval : kT1Fetch;
                    continue;
                }
                if (nstep == 0) {
#pragma unroll
                    for (int i = 0; i < N; ++i) yk0[i] = y[i];
                } else {
#pragma unroll
                    for (int i = 0; i < N; ++i) {
                        yk1[i] = yk0[i];
                        yk0[i] = y[i];
                    }
                }
                dtTry0 = dt;
                if ((t + dt - tn) * (t + dt - 0.0) > 0) {
                    dt = tn - t;
                    last = true;
                } else if (t + dt == tn) {
                    last = true;
                }
                // ImplicitEuler::adaptiveSolve start
                adt = dt;
                lts1 = lts0;
                tcount = 0;
                Told = y[TI];
                state = kT1Attempt;
            } else if (state == kT1Attempt) {
                lts0 = adt;
                ++n_att;
#pragma unroll
                for (int i = 0; i < N; ++i) yk[i] = y[i];
                ncount = 0;
                lastErr = 0.0;
                state = kT1Newton;
            } else if (state == kT1AttemptEnd) {
                // adaptiveSolve after solve(): checkNewY, then the error test
                const double Tnew = yk[TI];
                bool ok = true;
                if ((Tnew - Told) > P.T_alpha * Told) {
                    adt *= P.T_beta;
                    ok = false;
                }
                if (!ok && tcount < 100) {
                    error = 2;
                    tcount++;
                    if (adt <= kVeryTiny) {
                        cstatus |= 4;
                        state = kT1Fetch;
                        continue;
                    }
                    state = kT1Attempt;
                    continue;
                }
                if (error > 1.0) {
                    const double scale = hmax(P.safescale * fpow_pos(error, -P.alphainc), P.minscale);
                    adt *= scale;
                    if (adt <= kVeryTiny) {
                        cstatus |= 4;
                        state = kT1Fetch;
                        continue;
                    }
                    state = kT1Attempt;
                    continue;
                }
                // accepted
                t += adt;
#pragma unroll
                for (int i = 0; i < N; ++i) y[i] = yk[i];
                ++n_steps;
                if (error > P.err_accept_limit)
                    dt = hmin(hmax(P.safescale * fpow_pos(error, -P.alphainc), P.minscale), P.maxscale) * adt;
                else
                    dt = hmax(P.safescale * P.maxscale * adt, adt);
                dtReached = t;
                if ((t - tn) * (tn - 0.0) >= 0) {
                    if (nstep > 0 && last) sub = hmin(dtTry0, tn);
                    leftTime -= tn;
                    state = (leftTime > 0.0) ? kT1Interval : kT1Fetch;
                } else {
                    ++nstep;
                    state = kT1Step;
                }
            }
        }
        if constexpr (Lockstep) {
            if (!__syncthreads_or(state != kT1Done)) break;   // the whole block is done
            if (state != kT1Newton && state != kT1Err0) continue;
        } else {
            if (state == kT1Done) break;      // no cell left for this thread
            if (guard >= 64 && state != kT1Newton && state != kT1Err0) continue;
        }
        // ---------------- heavy block: J at yk, LU, solve
        const bool newton = (state == kT1Newton);
        if constexpr (Cell::kAssemblesA) {
            // the cell writes the Newton matrix I - dt J while it evaluates J
            cell.evaluate(yk, newton, lts0);
        } else {
            cell.evaluate(yk, newton);
        }
        if (newton) {
            ++n_jac;
            cell.factor(lts0);
            ++n_lu;
            double b[N];
#pragma unroll
            for (int i = 0; i < N; ++i) b[i] = (-yk[i] + y[i]) + lts0 * cell.F(i);
            cell.solve(b);
            ++n_newton;
            // ImplicitEuler::NewtonIteration update and tests
            int firstBad = N;
#pragma unroll
            for (int i = N - 1; i >= 0; --i)
                if (!finite(b[i])) firstBad = i;
            if (firstBad < N) {
#pragma unroll
                for (int i = 0; i < N; ++i)
                    if (i < firstBad) yk[i] += b[i];
                error = 1000.0;
                state = kT1AttemptEnd;
            } else {
                double maxErr = 0.0;
#pragma unroll
                for (int i = 0; i < N; ++i) {
                    yk[i] += b[i];
                    const double tol = P.atol + P.rtol * hmax(fabs(yk[i]), fabs(yk[i]));
                    maxErr = hmax(maxErr, fabs(b[i]) * frcp(tol));
                }
                bool fail = false;
                if (ncount > 0) {
                    const double diver = maxErr * frcp(hmax(lastErr, kTiny));
                    if (diver > 2 && ncount > 5) fail = true;
                }
                if (fail) {
                    error = 1000.0;
                    state = kT1AttemptEnd;
                } else {
                    lastErr = maxErr;
                    ncount++;
                    if (isnan(maxErr)) {
                        error = 1000.0;
                        state = kT1AttemptEnd;
                    } else if (ncount > 1000) {
                        error = maxErr;
                        state = kT1AttemptEnd;
                    } else if (P.max_newton_total > 0 && n_newton >= P.max_newton_total) {
                        cstatus |= 8;
                        state = kT1Fetch;
                    } else if (maxErr > 1.0) {
                        state = kT1Newton;
                    } else if (nstep == 0) {
                        state = kT1Err0;     // first step: error from f(y_k)
                    } else {
                        // 3-point error estimate (ImplicitEuler.cpp:121-140)
                        const double dtn = lts0, dtn1 = lts1;
                        const double f1 = 2.0 * frcp(dtn * (dtn + dtn1));
                        const double f2 = 2.0 * frcp(dtn1 * (dtn + dtn1));
                        const double LTEF = (dtn * dtn) * 0.5;
                        double me = 0.0;
                        bool nan_y = false;
#pragma unroll
                        for (int i = 0; i < N; ++i) {
                            double e = f1 * (yk[i] - y[i]) - f2 * (y[i] - yk1[i]);
                            e *= LTEF;
                            if (isnan(yk[i])) nan_y = true;
                            const double tol =
                                P.atol_inc + P.rtol_inc * hmax(fabs(y[i]), fabs(yk[i]));
                            me = hmax(me, fabs(e) * frcp(tol));
                        }
                        error = nan_y ? 1.5 : me;
                        state = kT1AttemptEnd;
                    }
                }
            }
        } else {
            // kT1Err0: error = maxIncrement(y0, yk, yk - y0 - dt f(yk))
            ++n_rhs;
            double me = 0.0;
            bool nan_y = false;
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const double e = yk[i] - y[i] - lts0 * cell.F(i);
                if (isnan(yk[i])) nan_y = true;
                const double tol = P.atol_inc + P.rtol_inc * hmax(fabs(y[i]), fabs(yk[i]));
                me = hmax(me, fabs(e) * frcp(tol));
            }
            error = nan_y ? 1.5 : me;
            state = kT1AttemptEnd;
        }
    }
}

}  // namespace hc
