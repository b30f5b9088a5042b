/*
 * hurchem_b200.hpp -- C++ host interface over the C ABI of libhurchem_b200.so.
 *
 * Header-only; needs no CUDA headers. Mirrors the all-cell interface of the
 * reference's chemistrySource (speciesTransport/chemistrySource/include/
 * chemistrySource.hpp:576-662) over caller-owned host fields in the flow
 * solver's structure-of-arrays layout:
 *
 *   double solve(const double *dt, double dtFactor)      chemistrySource.cpp:1494-1556
 *   void   solveUpdate(const double *dt, double dtFactor) chemistrySource.cpp:1558-1609
 *   void   calculateSourceTerms()                        chemistrySource.cpp:1370-1406
 *   const double *Ri(int i)                              chemistrySource.hpp:641
 *   double solve(t, dT, p, T, rho, yi)  (one cell)        chemistrySource.cpp:1300-1325
 *
 * Errors: a negative status from the library throws hurchem::Error with the
 * library's message (the reference aborts through LFatal instead).
 */
#ifndef HURCHEM_B200_HPP
#define HURCHEM_B200_HPP

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "hurchem_b200.h"

namespace hurchem {

class Error : public std::runtime_error {
public:
    explicit Error(const std::string &what) : std::runtime_error(what) {}
};

inline int check(int rc, const char *what) {
    if (rc < 0) throw Error(std::string(what) + ": " + hc_last_error());
    return rc;
}

inline hc_opts defaultOptions() {
    hc_opts o;
    hc_default_opts(&o);
    return o;
}

/* A mechanism uploaded to the current device. */
class Mechanism {
public:
    explicit Mechanism(const hc_mech_desc &desc) { check(hc_mech_create(&desc, &h_), "hc_mech_create"); }
    ~Mechanism() {
        if (h_) hc_mech_destroy(h_);
    }
    Mechanism(const Mechanism &) = delete;
    Mechanism &operator=(const Mechanism &) = delete;

    int nsp() const { return hc_mech_nsp(h_); }
    int nrc() const { return hc_mech_nrc(h_); }
    hc_mech_t handle() const { return h_; }
    void setTuning(int kernel, int block) { check(hc_set_tuning(h_, kernel, block), "hc_set_tuning"); }

    /*
     * The reference's CUDA-path buffers, one record of nsp + 2 doubles per cell
     * in host memory. integrateRecords: records [T, Y..., rho] over dt (already
     * times dtFactor) from the warm-start sub-steps subdt (updated), as
     * calcChemODEsArray (CUDAChemistrySourceODEs.cu:823-858) leaves them:
     * T and c_i with the record's rho when returnCi, else T, Y and the new rho.
     * Returns the number of cells that hit the step-size floor or the Newton cap.
     * p may be null (ideal-gas pressure from the record).
     */
    int integrateRecords(int64_t ncells, double *TYiRho, const double *dt, double *subdt,
                         bool returnCi, const hc_opts &opts = defaultOptions(),
                         const double *p = nullptr) {
        return check(hc_integrate_aos_host(h_, &opts, ncells, TYiRho, p, dt, subdt,
                                           returnCi ? 1 : 0, nullptr, nullptr),
                     "hc_integrate_aos_host");
    }
    /*
     * Source terms from records [Y..., rho, T] into RRi[cell * nsp + i], enqueued
     * on `stream` (a cudaStream_t) without waiting: the caller does its own work
     * and synchronises the stream before reading RRi (calculateSourceTermsAsync,
     * CUDAChemistrySource.cpp:189-198). Pinned host buffers make the copies
     * asynchronous.
     */
    void sourceTermsRecordsAsync(int64_t ncells, const double *YiRhoT, double *RRi,
                                 void *stream, const double *p = nullptr) {
        check(hc_source_terms_aos_async(h_, ncells, YiRhoT, p, RRi, stream),
              "hc_source_terms_aos_async");
    }

private:
    hc_mech_t h_ = nullptr;
};

/*
 * Chemistry source over host fields of ncells cells: T[n], p[n], rho[n] and
 * Y[nsp][n] (species-major), all owned by the caller (the flow model).
 */
class ChemistrySource {
public:
    ChemistrySource(Mechanism &mech, int64_t ncells, double *T, const double *p, double *rho,
                    double *Y, const hc_opts &opts = defaultOptions())
        : mech_(mech), n_(ncells), T_(T), p_(p), rho_(rho), Y_(Y), opts_(opts),
          Ri_((size_t)mech.nsp() * (size_t)ncells, 0.0), status_((size_t)ncells, 0) {}

    /* Integrate every cell over dt*dtFactor, fill Ri and leave the fields
     * unchanged; returns the smallest warm-start sub-step. */
    double solve(const double *dt, double dtFactor) {
        const size_t n = (size_t)n_, ns = (size_t)mech_.nsp();
        std::vector<double> T(T_, T_ + n), rho(rho_, rho_ + n), Y(Y_, Y_ + n * ns);
        initDt(dt, dtFactor);
        lastBad_ = check(hc_integrate_host(mech_.handle(), &opts_, n_, T.data(), p_, rho.data(),
                                           Y.data(), dt, dtFactor, dtInit_.data(), Ri_.data(),
                                           status_.data(), &counters_, nullptr),
                         "hc_integrate_host");
        return n ? *std::min_element(dtInit_.begin(), dtInit_.end()) : 0.0;
    }

    /* Integrate every cell and write Y, T and rho back into the fields. */
    void solveUpdate(const double *dt, double dtFactor) {
        initDt(dt, dtFactor);
        lastBad_ = check(hc_integrate_host(mech_.handle(), &opts_, n_, T_, p_, rho_, Y_, dt,
                                           dtFactor, dtInit_.data(), nullptr, status_.data(),
                                           &counters_, nullptr),
                         "hc_integrate_host");
    }

    /* Ri = omega_i W_i at the current state. */
    void calculateSourceTerms() {
        check(hc_source_terms_host(mech_.handle(), n_, T_, p_, rho_, Y_, Ri_.data(), nullptr),
              "hc_source_terms_host");
    }

    /* One cell over t with first sub-step dT (the per-cell solve of finiteRate);
     * yi is updated, T and rho are returned through the references. */
    double solve(double t, double dT, double p, double &T, double &rho, double *yi) {
        double dt = t, sub = dT;
        check(hc_integrate_host(mech_.handle(), &opts_, 1, &T, &p, &rho, yi, &dt, 1.0, &sub,
                                nullptr, nullptr, nullptr, nullptr),
              "hc_integrate_host");
        return sub;
    }

    const double *Ri(int i) const { return Ri_.data() + (size_t)i * (size_t)n_; }
    const std::vector<int32_t> &status() const { return status_; }
    const hc_counters &counters() const { return counters_; }
    int lastBadCells() const { return lastBad_; }
    hc_opts &options() { return opts_; }

private:
    void initDt(const double *dt, double dtFactor) {
        if (dtInit_.size() != (size_t)n_) {
            dtInit_.resize((size_t)n_);
            for (int64_t i = 0; i < n_; ++i) dtInit_[(size_t)i] = dt[i] * dtFactor;
        }
    }

    Mechanism &mech_;
    int64_t n_;
    double *T_;
    const double *p_;
    double *rho_;
    double *Y_;
    hc_opts opts_;
    std::vector<double> Ri_;
    std::vector<int32_t> status_;
    std::vector<double> dtInit_;
    hc_counters counters_{};
    int lastBad_ = 0;
};

}  // namespace hurchem

#endif /* HURCHEM_B200_HPP */
