// Oracle driver around the reference's own CPU chemistry path.
//
// TEST INFRASTRUCTURE ONLY: this program links the OpenHurricane sources
// (compiled unmodified by oracle/Makefile.ref) and runs their chemistry
// source term on seeded inputs so that the parity tests and the CPU-baseline
// leg of bench.py have the reference's own numbers. It is never part of the
// product path.
//
// Set-up mirrors the reference's 0-D application
// (applications/chemSolvers/chemSolvers.cpp:42-66): the built-in XML/mesh
// strings of chemSolvers.hpp are merged with the case file given by "-i",
// then the flow model and its mixture (mechanism, thermo, transport) are
// created through the reference's factories (flowModel::creator).
//
// The chemistry object is the reference's ODESolver<chemistrySource>
// (chemistryODESolvers/include/ODESolver.inl:42-66) with the "solver"
// sub-controller of the case file. OracleChem only adds a public per-cell
// entry that reproduces the body of chemistrySource::solve(dt, dtFactor)
// (chemistrySource.cpp:1494-1556) for one cell, because the reference loops
// over mesh cells and our inputs are a flat list of seeded cells.
//
// Modes (environment variable HC_MODE):
//   integrate : cells file -> integrated T, Y, c, rho, subDt per cell, and the
//               wall time of the integration loop only (stderr).
//   kat       : states file -> DyDt and analytic Jacobian per state
//               (chemistrySource.cpp:863 and :967), plus per-species thermo
//               and per-reaction kf/Kc values at the state's T.
//   props     : cells file -> per-species ha_i, mixture cp, mu, kappa and
//               mixture-averaged D_i (thermoList / transportList).
//   tha       : cells file (dt column = target mass enthalpy ha, subDt0
//               column = starting temperature T0) -> T from
//               thermoList::THa_p(ha, p, T0, iFlag, yi) (thermoList.cpp:501-533)
//               and iFlag per cell.
//   srcimp    : cells file -> the point-implicit source terms the flow solver
//               asks for (chemistrySource::calculateSourceTermsImp with its
//               default withoutLastSpec = true, chemistrySource.cpp:1412-1450):
//               Ri = omega_i W_i for every species and the diagonal source
//               Jacobian of the first nsp - 1 species, from omegaCoupled
//               (chemistrySource.cpp:422-480) at the cell's state.
//
// Binary formats (little endian, all int64 header words then float64):
//   cells  : nsp, n, T[n], p[n], rho[n], dt[n], subDt0[n], Y[nsp*n] (species-major)
//   result : nsp, n, T[n], p[n], rho[n], subDt[n], status[n], Y[nsp*n], c[nsp*n]
//   states : nsp, n, p[n], T[n], c[nsp*n]
//   katout : nsp, nrc, n, per state: dydt[nsp+1], J[(nsp+1)^2] row-major,
//            per species (cp0, ha0, s0, g0, G0, DG0DT, Dcp_pDT), per reaction (kf, Kc, kr)
//   props  : nsp, n, per cell: ha[nsp], cp, mu, kappa, D[nsp]
//   srcimp : nsp, n, per cell: Ri[nsp], diag[nsp-1]
//   tha    : n, per cell: T, iFlag

#include "commonInclude.hpp"
#include "dataStructure.hpp"
#include "flowModel.hpp"
#include "makeChemistryODESolvers.hpp"
#include "chemSolvers.hpp"

#include <chrono>
#include <csignal>
#include <execinfo.h>
#include <unistd.h>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <stdexcept>
#include <vector>

using namespace OpenHurricane;

namespace {

std::vector<double> readDoubles(std::ifstream &f, size_t n) {
    std::vector<double> v(n);
    f.read(reinterpret_cast<char *>(v.data()), sizeof(double) * n);
    if (!f) throw std::runtime_error("short read");
    return v;
}

void writeDoubles(std::ofstream &f, const std::vector<double> &v) {
    f.write(reinterpret_cast<const char *>(v.data()), sizeof(double) * v.size());
}

const char *envOr(const char *k, const char *d) {
    const char *v = std::getenv(k);
    return v ? v : d;
}

} // namespace

class OracleChem : public ODESolver<chemistrySource> {
public:
    OracleChem(flowModel &flows, const controller &cont) : ODESolver<chemistrySource>(flows, cont) {}

    double W(integer i) const { return species_.W(i); }

    // One cell of chemistrySource::solve(dt, dtFactor) (chemistrySource.cpp:1511-1555),
    // dtFactor = 1, returning the final concentrations as well as the
    // renormalised mass fractions that solve(t, dT, p, T, rho, yi) returns
    // (chemistrySource.cpp:1300-1325).
    int cell(double T, double p, double rho, double dt, double subDt0, realArray &yi,
             realArray &ci, double &Tout, double &pout, double &rhoout, double &subDtOut) {
        const integer nsp = nsp_;
        if (T < TemperatureThreshold_) {
            for (integer i = 0; i < nsp; ++i) ci[i] = rho * yi[i] / species_.W(i);
            Tout = T; pout = p; rhoout = rho; subDtOut = dt;
            return 1;
        }
        for (integer i = 0; i < nsp; ++i) ci[i] = rho * yi[i] / species_.W(i);
        this->p0_ = this->p_ = p;
        this->rho0_ = this->rho_ = rho;
        T_ = T;
        real leftTime = dt;
        real subDt = min(leftTime, min(subDt0, dtMax_));
        while (leftTime > 0.0) {
            real d = leftTime;
            this->solve(ci, d, subDt);
            leftTime -= d;
        }
        subDtOut = subDt;
        ciToYi(ci, yi);
        if (reactionFlowType_ == ReactionFlowType::ConstantPressure) {
            rho_ = therm().rho(p_, T_, yi);
        } else {
            p_ = therm().p(rho_, T_, yi);
        }
        Tout = T_; pout = p_; rhoout = rho_;
        return 0;
    }

    void setState(double p, double rho) {
        p0_ = p_ = p;
        rho0_ = rho_ = rho;
    }
};

static int runIntegrate(OracleChem &chem) {
    std::ifstream fin(envOr("HC_IN", "cells.bin"), std::ios::binary);
    int64_t hdr[2];
    fin.read(reinterpret_cast<char *>(hdr), sizeof(hdr));
    const int64_t nsp = hdr[0], n = hdr[1];
    if (nsp != chem.nsp()) {
        std::fprintf(stderr, "species mismatch %ld vs %d\n", (long)nsp, (int)chem.nsp());
        return 2;
    }
    auto T = readDoubles(fin, n), p = readDoubles(fin, n), rho = readDoubles(fin, n);
    auto dt = readDoubles(fin, n), sub0 = readDoubles(fin, n), Y = readDoubles(fin, nsp * n);
    const int64_t b = std::atoll(envOr("HC_BEGIN", "0"));
    int64_t e = std::atoll(envOr("HC_END", "-1"));
    if (e < 0 || e > n) e = n;
    const int64_t m = e - b;
    std::vector<double> To(m), po(m), ro(m), so(m), st(m), Yo(nsp * m), co(nsp * m);
    realArray yi(nsp), ci(nsp);
    auto t0 = std::chrono::steady_clock::now();
    for (int64_t k = 0; k < m; ++k) {
        const int64_t c = b + k;
        for (int64_t i = 0; i < nsp; ++i) yi[i] = Y[i * n + c];
        double Tt, pp, rr, ss;
        int s = chem.cell(T[c], p[c], rho[c], dt[c], sub0[c], yi, ci, Tt, pp, rr, ss);
        To[k] = Tt; po[k] = pp; ro[k] = rr; so[k] = ss; st[k] = s;
        for (int64_t i = 0; i < nsp; ++i) {
            Yo[i * m + k] = yi[i];
            co[i * m + k] = ci[i];
        }
    }
    auto t1 = std::chrono::steady_clock::now();
    std::fprintf(stderr, "HC_INTEGRATE_SECONDS %.9f cells %ld\n",
                 std::chrono::duration<double>(t1 - t0).count(), (long)m);
    std::ofstream fout(envOr("HC_OUT", "result.bin"), std::ios::binary);
    int64_t oh[2] = {nsp, m};
    fout.write(reinterpret_cast<const char *>(oh), sizeof(oh));
    writeDoubles(fout, To); writeDoubles(fout, po); writeDoubles(fout, ro);
    writeDoubles(fout, so); writeDoubles(fout, st); writeDoubles(fout, Yo); writeDoubles(fout, co);
    return 0;
}

static int runKat(OracleChem &chem, flowModel &flows) {
    std::ifstream fin(envOr("HC_IN", "states.bin"), std::ios::binary);
    int64_t hdr[2];
    fin.read(reinterpret_cast<char *>(hdr), sizeof(hdr));
    const int64_t nsp = hdr[0], n = hdr[1];
    auto p = readDoubles(fin, n), T = readDoubles(fin, n), c = readDoubles(fin, nsp * n);
    auto &mix = flows.mixtures();
    const auto &thl = mix.thermalTable();
    auto &reacs = mix.reactions();
    const int64_t nrc = reacs.size();
    const int64_t neq = nsp + 1;
    std::ofstream fout(envOr("HC_OUT", "kat.bin"), std::ios::binary);
    int64_t oh[3] = {nsp, nrc, n};
    fout.write(reinterpret_cast<const char *>(oh), sizeof(oh));
    realArray y(neq), dydt(neq), dfdt(neq), cc(nsp);
    realSquareMatrix J(neq);
    for (int64_t k = 0; k < n; ++k) {
        for (int64_t i = 0; i < nsp; ++i) y[i] = c[i * n + k];
        y[nsp] = T[k];
        chem.setState(p[k], 1.0);
        chem.DyDt(0, y, dydt);
        chem.jacobian(0, y, dfdt, J);
        std::vector<double> out;
        for (int64_t i = 0; i < neq; ++i) out.push_back(dydt[i]);
        for (int64_t i = 0; i < neq; ++i)
            for (int64_t j = 0; j < neq; ++j) out.push_back(J(i, j));
        for (int64_t i = 0; i < nsp; ++i) {
            const auto &th = thl[i];
            out.push_back(th.cp0(T[k]));
            out.push_back(th.ha0(T[k]));
            out.push_back(th.s0(T[k]));
            out.push_back(th.g0(T[k]));
            out.push_back(th.G0(T[k]));
            out.push_back(th.DG0DT(T[k]));
            out.push_back(th.Dcp_pDT(p[k], T[k]));
        }
        for (int64_t i = 0; i < nsp; ++i) cc[i] = std::max(c[i * n + k], 0.0);
        reacs.updateG0(T[k]);
        for (int64_t r = 0; r < nrc; ++r) {
            const real kf = reacs[r].kf(p[k], T[k], cc);
            out.push_back(kf);
            out.push_back(reacs[r].Kc(T[k]));
            out.push_back(reacs[r].kr(kf, p[k], T[k], cc));
        }
        writeDoubles(fout, out);
    }
    return 0;
}

static int runProps(flowModel &flows) {
    std::ifstream fin(envOr("HC_IN", "cells.bin"), std::ios::binary);
    int64_t hdr[2];
    fin.read(reinterpret_cast<char *>(hdr), sizeof(hdr));
    const int64_t nsp = hdr[0], n = hdr[1];
    auto T = readDoubles(fin, n), p = readDoubles(fin, n), rho = readDoubles(fin, n);
    auto dt = readDoubles(fin, n), sub0 = readDoubles(fin, n), Y = readDoubles(fin, nsp * n);
    auto &mix = flows.mixtures();
    const auto &thl = mix.thermalTable();
    const auto &trl = mix.transTable();
    std::ofstream fout(envOr("HC_OUT", "props.bin"), std::ios::binary);
    int64_t oh[2] = {nsp, n};
    fout.write(reinterpret_cast<const char *>(oh), sizeof(oh));
    realArray yi(nsp), cpi(nsp), Di(nsp);
    auto t0 = std::chrono::steady_clock::now();
    std::vector<double> out;
    out.reserve((2 * nsp + 3) * n);
    for (int64_t k = 0; k < n; ++k) {
        for (int64_t i = 0; i < nsp; ++i) yi[i] = Y[i * n + k];
        for (int64_t i = 0; i < nsp; ++i) out.push_back(thl[i].ha_p(p[k], T[k]));
        for (int64_t i = 0; i < nsp; ++i) cpi[i] = thl[i].cp_p(p[k], T[k]);
        out.push_back(thl.cp_p(p[k], T[k], yi));
        real mum, kappam;
        trl.muKappa(p[k], T[k], cpi, yi, mum, kappam);
        out.push_back(mum);
        out.push_back(kappam);
        Di = trl.Df(p[k], T[k], yi);
        for (int64_t i = 0; i < nsp; ++i) out.push_back(Di[i]);
    }
    auto t1 = std::chrono::steady_clock::now();
    std::fprintf(stderr, "HC_PROPS_SECONDS %.9f cells %ld\n",
                 std::chrono::duration<double>(t1 - t0).count(), (long)n);
    writeDoubles(fout, out);
    return 0;
}

static int runTHa(flowModel &flows) {
    std::ifstream fin(envOr("HC_IN", "cells.bin"), std::ios::binary);
    int64_t hdr[2];
    fin.read(reinterpret_cast<char *>(hdr), sizeof(hdr));
    const int64_t nsp = hdr[0], n = hdr[1];
    auto T = readDoubles(fin, n), p = readDoubles(fin, n), rho = readDoubles(fin, n);
    auto ha = readDoubles(fin, n), T0 = readDoubles(fin, n), Y = readDoubles(fin, nsp * n);
    const auto &thl = flows.mixtures().thermalTable();
    std::ofstream fout(envOr("HC_OUT", "tha.bin"), std::ios::binary);
    int64_t oh[1] = {n};
    fout.write(reinterpret_cast<const char *>(oh), sizeof(oh));
    realArray yi(nsp);
    std::vector<double> out;
    for (int64_t k = 0; k < n; ++k) {
        for (int64_t i = 0; i < nsp; ++i) yi[i] = Y[i * n + k];
        integer flag = 1;
        out.push_back(thl.THa_p(ha[k], p[k], T0[k], flag, yi));
        out.push_back((double)flag);
    }
    writeDoubles(fout, out);
    return 0;
}

static int runSrcImp(OracleChem &chem) {
    std::ifstream fin(envOr("HC_IN", "cells.bin"), std::ios::binary);
    int64_t hdr[2];
    fin.read(reinterpret_cast<char *>(hdr), sizeof(hdr));
    const int64_t nsp = hdr[0], n = hdr[1];
    auto T = readDoubles(fin, n), p = readDoubles(fin, n), rho = readDoubles(fin, n);
    auto dt = readDoubles(fin, n), sub0 = readDoubles(fin, n), Y = readDoubles(fin, nsp * n);
    std::ofstream fout(envOr("HC_OUT", "srcimp.bin"), std::ios::binary);
    int64_t oh[2] = {nsp, n};
    fout.write(reinterpret_cast<const char *>(oh), sizeof(oh));
    realArray yi(nsp), ci(nsp), w(nsp), diag(nsp);
    std::vector<double> out;
    out.reserve((2 * nsp - 1) * n);
    for (int64_t k = 0; k < n; ++k) {
        for (int64_t i = 0; i < nsp; ++i) {
            yi[i] = Y[i * n + k];
            ci[i] = rho[k] * yi[i] / chem.W(i);
        }
        chem.omegaCoupled(rho[k], p[k], T[k], ci, yi, w, diag);
        for (int64_t i = 0; i < nsp; ++i) out.push_back(w[i] * chem.W(i));
        for (int64_t i = 0; i + 1 < nsp; ++i) out.push_back(diag[i]);
    }
    writeDoubles(fout, out);
    return 0;
}

// thermoList::TEa_rho for each cell: the cells format carries rho, the
// mixture's internal energy in the dt column and T0 in the sub-step column
static int runTEa(flowModel &flows) {
    std::ifstream fin(envOr("HC_IN", "cells.bin"), std::ios::binary);
    int64_t hdr[2];
    fin.read(reinterpret_cast<char *>(hdr), sizeof(hdr));
    const int64_t nsp = hdr[0], n = hdr[1];
    auto T = readDoubles(fin, n), p = readDoubles(fin, n), rho = readDoubles(fin, n);
    auto ea = readDoubles(fin, n), T0 = readDoubles(fin, n), Y = readDoubles(fin, nsp * n);
    const auto &thl = flows.mixtures().thermalTable();
    std::ofstream fout(envOr("HC_OUT", "tea.bin"), std::ios::binary);
    int64_t oh[1] = {n};
    fout.write(reinterpret_cast<const char *>(oh), sizeof(oh));
    realArray yi(nsp);
    std::vector<double> out;
    for (int64_t k = 0; k < n; ++k) {
        for (int64_t i = 0; i < nsp; ++i) yi[i] = Y[i * n + k];
        integer flag = 1;
        out.push_back(thl.TEa_rho(ea[k], rho[k], T0[k], flag, yi));
        out.push_back((double)flag);
    }
    writeDoubles(fout, out);
    return 0;
}

static void onSegv(int) {
    void *bt[64];
    int n = backtrace(bt, 64);
    backtrace_symbols_fd(bt, n, 2);
    _exit(139);
}

int main(int argc, char *argv[]) {
    std::signal(SIGSEGV, onSegv);
    initializing(&argc, &argv);
    argParse myArg(argc, argv, "chemSolvers");
    iteration iter("CFDIter", myArg, contStr);
    myArg.clear();
    std::fprintf(stderr, "HC_STAGE mesh\n");
    runtimeMesh gm(object(iter.name(), iter, object::WRITE_RELAY_OUTPUT), iter.cont(), meshStr);
    std::fprintf(stderr, "HC_STAGE config\n");
    iter.readAndAddCont(iter.configName());
    std::fprintf(stderr, "HC_STAGE flow\n");

    auto flows = flowModel::creator(gm, iter.cont().subController("flow"));
    const auto &reacCont =
        iter.cont().subController("flow").subController("mixture").subController("reactions");
    std::fprintf(stderr, "HC_STAGE chem\n");
    OracleChem chem(*flows, reacCont.subController("chemistrySource"));
    std::fprintf(stderr, "HC_STAGE ready\n");
    if (iter.cont().found("chemSolvers")) {
        auto w = iter.cont().subController("chemSolvers").findWord("type");
        trim(w);
        if (w == "constVolume") chem.setConstantVolume();
        else chem.setConstantPressure();
    }

    const std::string mode = envOr("HC_MODE", "integrate");
    int rc = 0;
    if (mode == "integrate") rc = runIntegrate(chem);
    else if (mode == "kat") rc = runKat(chem, *flows);
    else if (mode == "props") rc = runProps(*flows);
    else if (mode == "srcimp") rc = runSrcImp(chem);
    else if (mode == "tha") rc = runTHa(*flows);
    else if (mode == "tea") rc = runTEa(*flows);
    else rc = 3;
    std::fflush(stdout);
    std::fflush(stderr);
    // The reference's finish() tears down MPI/logging; exit directly so that
    // nothing it prints at shutdown mixes with our results.
    std::_Exit(rc);
}
