/*
 * hurchem_b200.h -- C ABI of the B200 chemistry source-term library
 * (libhurchem_b200.so, built from openhurricane_b200/csrc/).
 *
 * The library integrates OpenHurricane's chemistry source term on an NVIDIA
 * B200 (sm_100a): per-cell stiff integration of finite-rate kinetics over
 * one flow time step with the reference's implicit-Euler scheme in FP64, the
 * source terms omega_i * W_i, and the NASA-7 / kinetic-theory mixture
 * properties. Every entry point takes plain pointers and sizes; no CUDA or
 * torch type appears in a signature (streams are passed as void*).
 *
 * Layout: per-cell fields are structure-of-arrays. A species field is
 * [nsp][ncells] (species-major, cell index fastest), the layout the
 * reference's flow solver keeps its PtrList<cellRealArray> yi_ in.
 *
 * Errors: every function returns an int status: 0 = success, > 0 = number
 * of cells that ended with a non-OK per-cell status (see HC_CELL_*), < 0 =
 * fatal (HC_E_*). hc_last_error() returns a message for the last failure on
 * the calling thread. The library never aborts the host process.
 *
 * Ownership: handles (hc_mech_t, hc_workspace_t) own device memory; host
 * arrays are caller-owned. Calls taking a stream are stream-ordered and
 * asynchronous unless their name ends in _host, which copies to and from
 * host memory and synchronises the stream before returning.
 */
#ifndef HURCHEM_B200_H
#define HURCHEM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HC_ABI_VERSION 2

/* fatal status codes */
#define HC_OK 0
#define HC_E_INVALID (-1)     /* bad argument (null pointer, size, option) */
#define HC_E_CUDA (-2)        /* CUDA runtime error */
#define HC_E_UNSUPPORTED (-3) /* mechanism / option outside the kernel's range */
#define HC_E_NOMEM (-4)

/* per-cell status words written by the integrators */
#define HC_CELL_OK 0
#define HC_CELL_SKIPPED 1       /* T below the temperature threshold: not integrated */
#define HC_CELL_MAXSTEP 2       /* an ODE solve hit maxstep (the reference then restarts it) */
#define HC_CELL_UNDERFLOW 4     /* step size fell below 1e-300 (the reference aborts here) */
#define HC_CELL_ITER_LIMIT 8    /* safety cap on total Newton iterations reached */

/* rate-law codes of hc_mech_desc.rate_type */
#define HC_RATE_ARRHENIUS 0
#define HC_RATE_THIRD_BODY 1
#define HC_RATE_LINDEMANN 2
#define HC_RATE_TROE3 3
#define HC_RATE_TROE4 4
#define HC_RATE_SRI 5       /* fall-off with the SRI function (fallOffFunctions::SRI) */
#define HC_RATE_PLOG 6      /* pressure-dependent Arrhenius table with logarithmic
                               interpolation, Chemkin PLOG (logInterpolationRR) */
#define HC_RATE_LANDAU_TELLER 7   /* A T^b exp(-Ta/T + B/T^(1/3) + C/T^(2/3)), Chemkin LT
                                     (LandauTellerRR) */
#define HC_RATE_JANEV 8     /* A T^b exp(-Ta/T + sum_{n<9} b_n (ln T)^n), Chemkin JAN (JanevRR) */
#define HC_RATE_POWER_SERIES 9  /* A T^b exp(sum_{n<4} b_n / T^(n+1)), Chemkin FIT1 (powerSeriesRR) */
#define HC_RATE_COLLISION 10    /* min(1, A T^b exp(-Ta/T)) x0 sqrt(x1 T), Chemkin COLLEFF
                                   (collisionRR); xcoef = N_A d^2, 8 pi Ru / W_AB, 2 pi Ru / W_AB
                                   with d the mean Lennard-Jones diameter of the two reactants
                                   as read (angstrom) and W_AB their reduced molar mass */

/* hc_mech_desc.reversible */
#define HC_IRREVERSIBLE 0
#define HC_REVERSIBLE 1         /* kr = kf / Kc (reversibleReactions) */
#define HC_REVERSIBLE_REV 2     /* kr from explicit reverse Arrhenius parameters, Chemkin REV
                                   (reversibleReactionWithRevPars); Arrhenius, third-body and
                                   Landau-Teller rate laws (the last with the reverse B, C of
                                   Chemkin RLT in xcoef), as in the reference */

#define HC_MAX_SIDE 4

/*
 * Flattened mechanism (SI units: kg, m, s, kmol, K, J). Produced on the host
 * from Chemkin / NASA-7 / transport files (openhurricane_b200/mechanism.py
 * applies the reference's unit conversions). Mirrors the data the reference's
 * mixture flattens for its GPU path (reactions/cuda/include/cuChemInterface.hpp:39-342),
 * but structure-of-arrays per reaction.
 */
typedef struct hc_mech_desc {
    int32_t nsp;             /* species */
    int32_t nrc;             /* reactions */
    const double *W;         /* [nsp] molecular weights kg/kmol */
    const double *Trange;    /* [nsp*3] Tlow, Tcommon, Thigh */
    const double *nasa;      /* [nsp*14] mass-basis NASA-7: low a0..a6, high a0..a6 */
    const int32_t *rate_type;  /* [nrc] HC_RATE_* */
    const int32_t *reversible; /* [nrc] HC_IRREVERSIBLE, HC_REVERSIBLE or HC_REVERSIBLE_REV */
    const double *arr;       /* [nrc*3] A, beta, Ta (high-pressure limit for fall-off) */
    const double *arr0;      /* [nrc*3] low-pressure limit (fall-off only) */
    const double *troe;      /* [nrc*4] alpha, T***, T*, T** */
    const double *eff;       /* [nrc*nsp] third-body efficiencies */
    const int32_t *nf;       /* [nrc] reactants */
    const int32_t *nb;       /* [nrc] products */
    const int32_t *fidx;     /* [nrc*HC_MAX_SIDE] */
    const int32_t *bidx;
    const double *fnu;       /* [nrc*HC_MAX_SIDE] stoichiometric coefficients */
    const double *bnu;
    const double *ford;      /* [nrc*HC_MAX_SIDE] reaction orders */
    const double *bord;
    /* kinetic-theory transport data (transport/include/kineticTheory.hpp) */
    const int32_t *geom;     /* [nsp] */
    const double *eps_k;     /* [nsp] well depth / kB, K */
    const double *sigma;     /* [nsp] collision diameter, Angstrom */
    /* since ABI 2; NULL when no reaction uses them */
    const double *sri;       /* [nrc*5] SRI a, b, c, d, e (HC_RATE_SRI reactions) */
    const double *arr_rev;   /* [nrc*3] reverse A, beta, Ta (HC_REVERSIBLE_REV reactions; for a
                                third-body reaction the reverse rate is M times this) */
    /* PLOG tables: entries plog_ptr[r] .. plog_ptr[r+1]-1 of reaction r, sorted by
       pressure (equal pressures keep their file order and their rates add), the
       two highest pressures distinct; NULL when no reaction is HC_RATE_PLOG */
    const int32_t *plog_ptr; /* [nrc+1] */
    const double *plog_p;    /* [plog_ptr[nrc]] pressures, Pa */
    const double *plog_arr;  /* [plog_ptr[nrc]*3] A, beta, Ta of each entry */
    /* chemically activated bimolecular reactions (Chemkin HIGH,
       chemicallyActicatedBimolecularRR): 1 where the fall-off reaction r
       (HC_RATE_LINDEMANN / TROE3 / TROE4 / SRI) is one, with arr0 = k0 (its main
       line) and arr = kinf (HIGH); k = k0 F / (1 + Pr). NULL: none */
    const int32_t *activated; /* [nrc] */
    const double *lt;        /* [nrc*2] Landau-Teller B, C (HC_RATE_LANDAU_TELLER); NULL: none */
    const double *xcoef;     /* [nrc*9] Janev b_0..b_8, power-series b_0..b_3 or collision
                                x0..x2 (then zeros);
                                for a Landau-Teller reaction with HC_REVERSIBLE_REV, the
                                reverse rate's B, C (Chemkin RLT): kr is then the
                                Landau-Teller law on arr_rev and these. NULL: none */
} hc_mech_desc;

/*
 * Integrator options. Names and defaults follow the reference's controller
 * keys: solver/{maxstep, atol, rtol, safescale, minscale, maxScale, alphainc}
 * (Hurricane/mathematicalTools/ODEs/src/ODEsSolver.cpp:80-92),
 * ImplicitEuler/{autoUpdateJacobian, stepToUpdateJac, ATolIncrement,
 * RTolIncrement} (ODEs/src/ImplicitEuler.cpp:68-84),
 * solveOptions/{TemperatureThreshold, TemperatureAlpha, TemperatureBeta} and
 * chemicalMaxStep (chemistrySource/src/chemistrySource.cpp:42-84).
 */
typedef struct hc_opts {
    int32_t maxstep;             /* 10000 */
    int32_t auto_update_jacobian;/* 0 */
    int32_t step_to_update_jac;  /* 10 */
    int32_t reactor;             /* chemSolvers type: 0 constant pressure, 1 constant volume
                                    (cell-group kernels: the density is held and not written,
                                    the pressure follows the state inside the step and is not
                                    written back, as in the reference's solveUpdate) */
    double atol;                 /* 1e-15 (reference default "tiny") */
    double rtol;                 /* 1e-4 */
    double safescale;            /* 0.8 */
    double minscale;             /* 0.25 */
    double maxscale;             /* 2.0 */
    double alphainc;             /* 0.25 */
    double atol_increment;       /* 1e-7 */
    double rtol_increment;       /* 1e-3 */
    double T_threshold;          /* 200 K */
    double T_alpha;              /* 0.2 */
    double T_beta;               /* 0.25 */
    double dt_max;               /* chemicalMaxStep, 1e15 ("large") */
    int64_t max_newton_total;    /* safety cap per cell per call, 0 = none */
} hc_opts;

/* per-call work counters (summed over cells) */
typedef struct hc_counters {
    int64_t n_jac;       /* Jacobian evaluations (each also yields f) */
    int64_t n_rhs;       /* right-hand-side-only evaluations */
    int64_t n_lu;        /* LU factorisations */
    int64_t n_newton;    /* Newton iterations */
    int64_t n_steps;     /* accepted steps */
    int64_t n_attempts;  /* step attempts */
} hc_counters;

typedef struct hc_mech_s *hc_mech_t;

int hc_abi_version(void);
const char *hc_last_error(void);
void hc_default_opts(hc_opts *opts);

/*
 * Kernel selection for hc_integrate*: kernel 0 = automatic (the warp per
 * cell, kernel 6, wherever it takes the mechanism and the reactor, else the
 * cell group: their lanes share each Newton iteration of one cell, which
 * bounds the step's duration when per-cell costs are uneven), 1 = table-driven thread per
 * cell, 2 = cell group (32 lanes up to 32 unknowns, 64 above),
 * 3 = thread per cell generated for this mechanism (every index and
 * coefficient a literal; compiled with NVRTC for sm_100a on first use, which
 * must precede any stream capture), 4 = compact thread per cell (mechanism
 * in the kernel's constant parameter bank: nsp <= 15, <= 64 reactions),
 * 5 = thread per cell generated for this mechanism with the Newton matrix
 * I - dt J assembled column by column from register-held rates and written
 * once per entry, no divisions on the common path and a small instruction
 * footprint (NVRTC on first use, like 3), 6 = warp per cell (one cell per
 * warp, lane i holding element i and row i of the Newton matrix; nsp + 1 <= 16),
 * 7 = segment per cell (32 / (nsp + 1) cells per warp, one per segment of
 * nsp + 1 lanes, each segment with its own step-control state; nsp + 1 <= 16);
 * block = threads per block of the thread-per-cell kernels (32, 64 or 128;
 * kernels 6 and 7 run 256-thread blocks whatever it says). Set by the
 * autotuner (openhurricane_b200/autotune.py).
 * The thread-per-cell kernels (1, 3, 4, 5) take nsp <= 15, the constant-pressure
 * reactor and the common rate forms (Arrhenius, third body, Lindemann / Troe
 * fall-off); a call that asks for one of them outside that range fails with
 * HC_E_UNSUPPORTED; kernels 6 and 7 take the same rate forms and reactor,
 * and autoUpdateJacobian. The cell group takes everything hc_mech_create accepts.
 * No reference counterpart.
 */
int hc_set_tuning(hc_mech_t mech, int kernel, int block);

/* The generated kernel's CUDA source for a mechanism (len = its length; up to
 * cap-1 bytes and a terminating 0 are written to buf when buf != NULL).
 * Host-only: needs no GPU. */
int hc_jit_source(const hc_mech_desc *desc, int block, char *buf, int64_t cap, int64_t *len);
/* Compile that source with NVRTC for sm_100a without loading it (host only);
 * cubin_bytes receives the size of the compiled image. */
int hc_jit_compile(const hc_mech_desc *desc, int block, int64_t *cubin_bytes);
/* The same for a chosen generated kernel: 3 (thread per cell, Jacobian
 * scattered into shared memory) or 5 (thread per cell, Newton matrix
 * assembled column by column from register-held rates). */
int hc_jit_source_kernel(const hc_mech_desc *desc, int kernel, int block, char *buf, int64_t cap,
                         int64_t *len);
int hc_jit_compile_kernel(const hc_mech_desc *desc, int kernel, int block, int64_t *cubin_bytes);

/* Upload a mechanism; selects the compiled kernel variant for nsp. */
int hc_mech_create(const hc_mech_desc *desc, hc_mech_t *out);
int hc_mech_destroy(hc_mech_t mech);
int hc_mech_nsp(hc_mech_t mech);
int hc_mech_nrc(hc_mech_t mech);

/*
 * Integrate ncells cells over dt[cell] * dt_factor with device pointers.
 * Replaces chemistrySource::solve(const realArray &dt, real dtFactor) and
 * chemistrySource::solveUpdate (chemistrySource/src/chemistrySource.cpp:1494-1609)
 * for the ODESolver<chemistrySource> + ImplicitEuler configuration.
 *   T[ncells]        in: temperature; out: T after the step
 *   p[ncells]        pressure (constant during the step)
 *   rho[ncells]      in: density; out: rho(p, T, Y) after the step
 *   Y[nsp*ncells]    in: mass fractions; out: renormalised mass fractions
 *   dt[ncells]       flow time step per cell
 *   subdt[ncells]    in/out warm-start sub-step (the reference's dtInit);
 *                    pass dt on the first flow step
 *   Ri[nsp*ncells]   optional out (may be NULL): (c_new - c_old)/(dt*dt_factor)*W_i
 *   status[ncells]   optional out: HC_CELL_* bits
 *   counters         optional out (host struct; forces a stream sync)
 * The device work queue and the counters live in the mechanism (one set per
 * hc_mech_t): calls of hc_integrate* on the same mechanism that overlap in
 * time on different streams race on them, so callers that integrate on
 * several streams at once create one hc_mech_t per stream.
 */
int hc_integrate(hc_mech_t mech, const hc_opts *opts, int64_t ncells, double *T, const double *p,
                 double *rho, double *Y, const double *dt, double dt_factor, double *subdt,
                 double *Ri, int32_t *status, hc_counters *counters, void *stream);

/*
 * hc_integrate with a work-queue order and a per-cell cost output: cells are
 * taken from the device queue in the order order[0..ncells) (NULL: natural
 * order), and cost[cell] receives the cell's Newton-iteration count (NULL:
 * not written). Feeding a descending sort of the previous flow step's cost
 * back as the next step's order starts the stiffest cells first
 * (stiffness re-binning). No reference counterpart: the reference integrates
 * cells in mesh order (chemistrySource.cpp:1511).
 */
int hc_integrate_ordered(hc_mech_t mech, const hc_opts *opts, int64_t ncells, double *T,
                         const double *p, double *rho, double *Y, const double *dt,
                         double dt_factor, double *subdt, double *Ri, int32_t *status,
                         const int32_t *order, int64_t *cost, hc_counters *counters,
                         void *stream);

/*
 * Integrate only the cells sel[0..nsel) of fields of length ncells (device
 * pointers; species fields keep the stride ncells); other cells are not
 * touched. Used for the surrogate's rejected cells. No reference
 * counterpart.
 */
int hc_integrate_subset(hc_mech_t mech, const hc_opts *opts, int64_t ncells, int64_t nsel,
                        const int32_t *sel, double *T, const double *p, double *rho, double *Y,
                        const double *dt, double dt_factor, double *subdt, double *Ri,
                        int32_t *status, int64_t *cost, hc_counters *counters, void *stream);

/*
 * Allocation-free integration. No counterpart in the reference.
 *
 * Same contract as hc_integrate (device pointers, stream-ordered) for
 * mechanisms of nsp <= 15 species and <= 64 reactions, integrated with the
 * compact thread-per-cell kernel, for callers that must not allocate device
 * memory during the call: a solver that runs under a fixed device-memory
 * budget or its own memory pool, code that calls the chemistry where the
 * CUDA allocator must not be entered (a host callback, a section holding its
 * own allocator's lock), or a loop that cannot afford the stream
 * synchronisation a growing allocation brings. hc_integrate grows a per-cell
 * scratch buffer with cudaMalloc when a call brings more cells than before;
 * this call allocates nothing: its scratch is a fixed file-scope device array
 * for at most HC_NOALLOC_MAX_CELLS cells (16 MiB, part of the library's
 * device image, placed in device memory when the CUDA runtime loads that
 * image), and larger calls are rejected with HC_E_INVALID. Every call made
 * outside a stream capture looks up that array's address on the current
 * device (cudaGetSymbolAddress; after a cudaDeviceReset the next call finds
 * the array's new place); a call under capture uses the address of the last
 * lookup on that device, so make one call on each device before capturing
 * (the first may also load the library's device image under lazy module
 * loading). The kernel is always the compact thread-per-cell kernel
 * (hc_set_tuning kernel 4): the kernel chosen with hc_set_tuning is not
 * consulted, only its block size applies. The work queue in the array is zeroed with
 * cudaMemsetAsync at every call. All calls share the array: calls that
 * overlap in time (other streams, other host threads) race on it, so callers
 * serialise them. Returns HC_OK or a negative HC_E_* code; per-cell statuses
 * go to status (no count is returned, which would need a host copy).
 */
#define HC_NOALLOC_MAX_CELLS 65536
int hc_integrate_noalloc(hc_mech_t mech, const hc_opts *opts, int64_t ncells, double *T,
                         const double *p, double *rho, double *Y, const double *dt,
                         double dt_factor, double *subdt, double *Ri, int32_t *status,
                         void *stream);

/* Same as hc_integrate with host buffers: H2D, integrate, D2H, synchronise. */
int hc_integrate_host(hc_mech_t mech, const hc_opts *opts, int64_t ncells, double *T,
                      const double *p, double *rho, double *Y, const double *dt, double dt_factor,
                      double *subdt, double *Ri, int32_t *status, hc_counters *counters,
                      void *stream);

/*
 * Right-hand side and analytic Jacobian of the constant-pressure reactor at
 * given states (chemistrySource::DyDt / ::jacobian, chemistrySource.cpp:863,967).
 *   c[nsp*n], T[n], p[n] -> dydt[(nsp+1)*n] (optional), J[(nsp+1)^2 * n] row-major
 *   per state (optional).
 */
int hc_rhs_jacobian(hc_mech_t mech, int64_t n, const double *c, const double *T, const double *p,
                    double *dydt, double *J, void *stream);

/*
 * Explicit source terms omega_i * W_i [kg/m^3/s] (chemistrySource::calculateSourceTerms,
 * chemistrySource.cpp:1370-1406): T, p, rho, Y -> Ri[nsp*n].
 */
int hc_source_terms(hc_mech_t mech, int64_t n, const double *T, const double *p, const double *rho,
                    const double *Y, double *Ri, void *stream);

/*
 * Temperature from the mixture's mass enthalpy at constant pressure
 * (thermoList::THa_p, thermoList.cpp:501-533, with the reference's step
 * tolerance 1e-4 T0 and 100-iteration cap): ha[n] J/kg, Y[nsp*n], starting
 * temperatures T0[n] -> T[n]; flag[n] (optional) = 0 clamped at TLow,
 * 1 inside, 2 clamped at THigh (the reference's defaults: 50 K, 5000 K).
 */
int hc_temperature_from_enthalpy(hc_mech_t mech, int64_t n, const double *ha, const double *Y,
                                 const double *T0, double TLow, double THigh, double *T,
                                 int32_t *flag, void *stream);

/*
 * Temperature from the mixture's mass internal energy at constant density
 * (thermoList::TEa_rho, thermoList.inl:343-348, the same Newton iteration,
 * tolerance, cap and clamp as hc_temperature_from_enthalpy):
 * ea[n] J/kg with e = sum_i Y_i h_i - p/rho, p = rho Rm T; Y[nsp*n], rho[n],
 * starting temperatures T0[n] -> T[n]; flag[n] (optional) as above.
 */
int hc_temperature_from_energy(hc_mech_t mech, int64_t n, const double *ea, const double *Y,
                               const double *rho, const double *T0, double TLow, double THigh,
                               double *T, int32_t *flag, void *stream);

/*
 * Point-implicit source terms for the flow solver's species equations
 * (chemistrySource::calculateSourceTermsImp with its default
 * withoutLastSpec = true, chemistrySource.cpp:1412-1450, via omegaCoupled,
 * :422-480): Ri[nsp*n] = omega_i W_i [kg/m^3/s] and diag[(nsp-1)*n], the
 * diagonal of the source Jacobian of the first nsp - 1 species with the last
 * species' concentration eliminated at fixed density and the temperature
 * coupling at constant internal energy (the reference's diagSource()).
 */
int hc_source_terms_imp(hc_mech_t mech, int64_t n, const double *T, const double *p,
                        const double *rho, const double *Y, double *Ri, double *diag,
                        void *stream);

/*
 * Mixture properties (thermoList / transportList, kinetic theory + Wilke):
 * T, p, Y -> ha[nsp*n] (J/kg per species), cp[n] (J/kg/K), mu[n] (Pa s),
 * kappa[n] (W/m/K), D[nsp*n] (m^2/s mixture-averaged). Any output may be NULL.
 */
int hc_properties(hc_mech_t mech, int64_t n, const double *T, const double *p, const double *Y,
                  double *ha, double *cp, double *mu, double *kappa, double *D, void *stream);

/*
 * Host-buffer forms of hc_source_terms and hc_properties: copy in, compute,
 * copy out, synchronise the stream. They serve the reference's host-side
 * callers, which pass host arrays: chemistrySource::calculateSourceTerms
 * (chemistrySource.cpp:1370-1406), CUDAThermo::calchaicp
 * (thermo/include/thermoListCUDA.hpp:40-58) and
 * CUDATransport::calcTransportProperties (transport/src/transportListCUDA.cu:236).
 */
int hc_source_terms_host(hc_mech_t mech, int64_t n, const double *T, const double *p,
                         const double *rho, const double *Y, double *Ri, void *stream);
int hc_properties_host(hc_mech_t mech, int64_t n, const double *T, const double *p,
                       const double *Y, double *ha, double *cp, double *mu, double *kappa,
                       double *D, void *stream);

/* ------------------------------------------------------------------------
 * Record-per-cell forms: the buffers of the reference's CUDA path, one
 * record of nsp + 2 doubles per cell. The records are transposed on the
 * device into the species-major fields of the entry points above, computed,
 * and transposed back. p[n] is optional: NULL takes p from the ideal-gas law,
 * p = rho Ru T sum_i Y_i / W_i, with the record's rho, T and Y. The records
 * live in the mechanism's workspace while a call is in flight, so calls on
 * one mechanism are issued on one stream (or synchronised between streams).
 * Mechanisms of up to 64 species.
 *
 * hc_integrate_aos / hc_integrate_aos_host: records [T, Y_0..Y_{nsp-1}, rho]
 * (calcChemODEsArray, chemistrySource/src/CUDAChemistrySourceODEs.cu:823-858,
 * called from CUDAChemistrySource.cpp:377-399) integrated over dt[n]
 * (already multiplied by dtFactor, as the reference's caller does) with the
 * warm-start sub-steps subdt[n] (in/out), by this library's implicit-Euler
 * integrator (the same kernels as hc_integrate). On return each record
 * holds T and either, return_ci != 0, the concentrations
 * c_i = Y_i rho_new / W_i [kmol/m^3] with the record's own rho left in place
 * (the reference's returnCi form, from which its caller forms Ri), or the
 * mass fractions and the new density. status[n] is optional. The _aos form
 * takes device pointers and is stream-ordered; the _aos_host form takes host
 * pointers, synchronises, and returns the number of cells with
 * HC_CELL_UNDERFLOW or HC_CELL_ITER_LIMIT like hc_integrate_host.
 */
int hc_integrate_aos(hc_mech_t mech, const hc_opts *opts, int64_t ncells, double *TYiRho,
                     const double *p, const double *dt, double *subdt, int return_ci,
                     int32_t *status, void *stream);
int hc_integrate_aos_host(hc_mech_t mech, const hc_opts *opts, int64_t ncells, double *TYiRho,
                          const double *p, const double *dt, double *subdt, int return_ci,
                          int32_t *status, void *stream);

/*
 * Explicit source terms from records [Y_0..Y_{nsp-1}, rho, T] (getYiRhoT,
 * CUDAChemistrySource.cpp:73-81) into RRi[cell * nsp + i] [kg/m^3/s]
 * (calcOnlyChemSourceTermsAsync via CUDAChemistrySource::calculateSourceTermsAsync,
 * CUDAChemistrySource.cpp:189-198; read back by laminarSpeciesSolverCUDA.cpp:326-330).
 * hc_source_terms_aos takes device pointers. hc_source_terms_aos_async takes
 * host pointers and only enqueues the copies and kernels on the stream: it
 * returns before the results arrive, the caller does its own host work
 * meanwhile (the reference computes the viscous fluxes) and synchronises the
 * stream before reading RRi. With pageable host memory the CUDA runtime
 * performs the copies synchronously, so pinned buffers (cudaHostAlloc, as
 * the reference allocates them) are what makes the overlap happen.
 */
int hc_source_terms_aos(hc_mech_t mech, int64_t n, const double *YiRhoT, const double *p,
                        double *RRi, void *stream);
int hc_source_terms_aos_async(hc_mech_t mech, int64_t n, const double *YiRhoT, const double *p,
                              double *RRi, void *stream);

/*
 * Mixture properties from records [Y_0..Y_{nsp-1}, T, p] (nsp + 2 doubles per
 * cell), the input of CUDAThermo::calchaicp (thermo/include/thermoListCUDA.hpp:40-58,
 * thermo/src/thermoListCUDA.cu:84-123) and CUDATransport::calcTransportProperties
 * (transport/src/transportListCUDA.cu:236-276), into their outputs:
 * haicp[cell * (nsp + 1) + i] = h_i [J/kg] and, at i = nsp, the mixture cp
 * [J/kg/K]; DMuKappa[cell * (nsp + 2) + i] = D_i [m^2/s], then mu [Pa s] and
 * kappa [W/m/K]. Either output may be NULL. hc_properties_aos takes device
 * pointers (stream-ordered); hc_properties_aos_host host pointers
 * (synchronous, as the reference's non-Async calls).
 */
/* ------------------------------------------------------------------------
 * Device state: a flow's cells resident on the device between calls, for
 * callers that keep the fields there (hc_upload once, then integrate /
 * source terms / properties every step, hc_download when the host needs
 * them). The state owns device fields T[n], p[n], rho[n], Y[nsp*n]
 * (species-major), the warm-start sub-steps subdt[n], Ri[nsp*n] and the
 * per-cell statuses; hc_state_fields returns their device addresses. Calls
 * are stream-ordered; downloads synchronise the stream. A state belongs to
 * the mechanism it was made with, which must outlive it; record layouts go
 * through the mechanism's workspace, so calls on one mechanism are issued
 * on one stream.
 */
typedef struct hc_state_s *hc_state_t;

/* record layouts (nsp + 2 doubles per cell) of the reference's CUDA path */
#define HC_RECORDS_T_Y_RHO 0   /* [T, Y..., rho]: calcChemODEsArray */
#define HC_RECORDS_Y_RHO_T 1   /* [Y..., rho, T]: calculateSourceTermsAsync (getYiRhoT) */
#define HC_RECORDS_Y_T_P 2     /* [Y..., T, p]: calchaicp / calcTransportProperties */

int hc_state_create(hc_mech_t mech, int64_t ncells, hc_state_t *out);
int hc_state_destroy(hc_state_t state);
int hc_state_fields(hc_state_t state, double **T, double **p, double **rho, double **Y,
                    double **subdt, double **Ri, int32_t **status);
/* host species-major fields in; any may be NULL (kept). Passing subdt sets the
   warm-start sub-steps; otherwise the first integration starts from dt dtFactor. */
int hc_upload(hc_state_t state, const double *T, const double *p, const double *rho,
              const double *Y, const double *subdt, void *stream);
/* host records in (HC_RECORDS_*); for layouts 0 and 1, p[n] (host) or NULL for
   the ideal-gas pressure of the record's rho, T and Y */
int hc_upload_records(hc_state_t state, int layout, const double *recs, const double *p,
                      void *stream);
/* host species-major fields out (any may be NULL); synchronises */
int hc_download(hc_state_t state, double *T, double *rho, double *Y, double *Ri, double *subdt,
                int32_t *status, void *stream);
/* host records out, layout HC_RECORDS_T_Y_RHO or HC_RECORDS_Y_RHO_T; synchronises */
int hc_download_records(hc_state_t state, int layout, double *recs, void *stream);
/* one flow step of every cell over dt[n] (device) * dt_factor, as hc_integrate:
   T, Y (and rho at constant pressure) updated, Ri, subdt and statuses written */
int hc_state_integrate(hc_state_t state, const hc_opts *opts, const double *dt, double dt_factor,
                       void *stream);
/* Ri = omega_i W_i at the state's fields */
int hc_state_source_terms(hc_state_t state, void *stream);
/* mixture properties at the state's fields into device outputs (any may be NULL) */
int hc_state_properties(hc_state_t state, double *ha, double *cp, double *mu, double *kappa,
                        double *D, void *stream);

int hc_properties_aos(hc_mech_t mech, int64_t n, const double *YiTP, double *haicp,
                      double *DMuKappa, void *stream);
int hc_properties_aos_host(hc_mech_t mech, int64_t n, const double *YiTP, double *haicp,
                           double *DMuKappa, void *stream);

/*
 * Measurement utility, no reference counterpart: runs an FP64 FMA-throughput
 * probe on the current device (independent FMA chains on every SM) and
 * returns the achieved TFLOP/s, the denominator of the integrator's roofline.
 */
int hc_probe_fp64_peak(int iters, double *tflops, void *stream);

/* ------------------------------------------------------------------------
 * Surrogate network (no reference counterpart): a multilayer perceptron
 * n_in -> n_hidden x width (GELU) -> n_out with BF16 tensor-core (tcgen05)
 * forward and backward kernels accumulating in FP32, FP32 master parameters
 * and Adam. Inputs and targets are device fp32 row-major [B][n_in] /
 * [B][n_out], already normalised by the caller. Errors are reported through
 * hc_last_error().
 */
typedef struct hc_mlp_s *hc_mlp_t;

int hc_mlp_create(int n_in, int n_out, int n_hidden, int width, int max_batch, uint64_t seed,
                  hc_mlp_t *out);
int hc_mlp_destroy(hc_mlp_t mlp);
int64_t hc_mlp_num_params(hc_mlp_t mlp);
/* host parameter layout, layer by layer: W [out][in] row-major, then b [out] */
int hc_mlp_get_params(hc_mlp_t mlp, float *host);
int hc_mlp_set_params(hc_mlp_t mlp, const float *host);
/* gradients of the mean-squared error (parameter layout), no update; synchronises */
int hc_mlp_grad(hc_mlp_t mlp, const float *X, const float *Y, int B, float *grad_host,
                float *loss_host, void *stream);
/* one Adam step; loss_host != NULL or check != 0 make the call synchronous */
int hc_mlp_train_step(hc_mlp_t mlp, const float *X, const float *Y, int B, float lr,
                      float *loss_host, int check, void *stream);
/* Y = net(X) for any B (processed in chunks of max_batch rows) */
int hc_mlp_forward(hc_mlp_t mlp, const float *X, int64_t B, float *Y, void *stream);
/* reads and clears the tensor-core pipelines' timeout flag; synchronises */
int hc_mlp_check(hc_mlp_t mlp, void *stream);
/* test entry: C[M][N] = act(A[M][K] B[N][K]^T + bias), bf16 in, fp32 out,
 * M % 128 == 0, N % 32 == 0, K % 64 == 0; act 0 identity, 1 GELU */
int hc_gemm_bf16_tn(const void *A, const void *B, int M, int N, int K, const float *bias,
                    int act, float *C, void *stream);

/*
 * Surrogate path around the network (no reference counterpart).
 *
 * hc_surrogate_features: X[n][nsp+3] (float) = normalised (T, ln p,
 * ln max(Y_1, 1e-20) .. ln max(Y_nsp, 1e-20), ln(dt*dt_factor)):
 * (value - mean[j]) * inv_std[j].
 *
 * hc_surrogate_gate: pred[n][nsp+1] is the network's normalised increment
 * (dT, dY_1..dY_nsp) over the flow step (de-normalised with out_mean /
 * out_std). Per cell, in FP64: dY is projected onto the element-conserving
 * subspace with proj[nsp][nsp]; Y' = Y + dY (components below -y_neg reject,
 * those in [-y_neg, 0) become 0 and the element mass they carried is taken
 * from the major species, Y' > 1e-3, with elem[nel][nsp] = atoms / W);
 * T' solves sum Y'_i h_i(T') = sum Y_i h_i(T)
 * (constant-pressure enthalpy); the cell is accepted when |T' - (T + dT)| <=
 * tol_T, the projection moved dY by at most tol_proj * max(|dY|_inf, 1e-6),
 * every |X| <= x_max, T_min < T' < T_max and, when spread != NULL (an
 * ensemble's per-cell disagreement), spread <= tol_spread. Accepted cells get T', Y' and
 * rho = p/(R_m T'); rejected cells are untouched, listed in rejected[0..
 * *n_rejected) (any order) for hc_integrate_subset. Synchronises the stream.
 */
typedef struct hc_gate_opts {
    double tol_T;     /* K */
    double tol_proj;  /* relative */
    double y_neg;     /* largest negative mass fraction clipped to zero */
    double x_max;     /* input features' range, in training standard deviations */
    double T_min, T_max;
    double tol_spread; /* largest ensemble disagreement accepted */
} hc_gate_opts;

int hc_surrogate_features(hc_mech_t mech, int64_t n, const double *T, const double *p,
                          const double *Y, const double *dt, double dt_factor, const double *mean,
                          const double *inv_std, float *X, void *stream);
int hc_surrogate_gate(hc_mech_t mech, int64_t n, double *T, const double *p, double *rho,
                      double *Y, const float *pred, const float *X, const double *out_mean,
                      const double *out_std, const double *proj, const double *elem, int nel,
                      const float *spread, const hc_gate_opts *gate, int32_t *accept,
                      int32_t *rejected, int64_t *n_rejected, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* HURCHEM_B200_H */
