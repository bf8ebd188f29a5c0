/*
 * espec_gpu.h -- C-ABI of the B200 wave-packet propagator (libespecgpu.so).
 *
 * Two layers:
 *   1. Fortran-callable drop-ins for eSPec's propagators (lower-case name
 *      with trailing underscore, every argument by reference, one hidden
 *      size_t length per CHARACTER*(*) argument appended in order).  They
 *      take the same arguments as the reference routines and leave the same
 *      outputs in the caller's arrays.
 *   2. Plan-based batched entry points used by the drop-ins and by batched
 *      scans (thousands of independent packets in one launch).
 *
 * All functions return ESPEC_OK (0) or a negative error code; the message of
 * the last error of the calling thread is espec_last_error().  Nothing here
 * aborts the process.  A library built without a usable GPU fails every call
 * with ESPEC_ECUDA -- there is no CPU fallback.
 */
#ifndef ESPEC_GPU_H
#define ESPEC_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* return codes */
#define ESPEC_OK 0
#define ESPEC_EINVAL (-1)   /* invalid argument / unsupported case          */
#define ESPEC_ECUDA (-2)    /* CUDA runtime or launch error                 */
#define ESPEC_ENOMEM (-3)   /* device allocation failed                     */

/* arithmetic forms */
#define ESPEC_FP64 0        /* plain FP64 form (parity form)                */
#define ESPEC_MIXED 1       /* FP32 data, FP64 phases and C(t) accumulation */

/* absorber kinds (absorb.f: .VOPTIC_* complex potentials, .SMOOTHW mask) */
#define ESPEC_ABS_NONE 0
#define ESPEC_ABS_VOPTIC 1
#define ESPEC_ABS_SMOOTHW 2

/* propagation methods */
#define ESPEC_SPO 0         /* split operator, FFT kinetic term (.PFSPO)     */
#define ESPEC_SOD 1         /* second-order differences, FFT kinetic (.PFSOD) */
#define ESPEC_SIL 2         /* short-iterative Lanczos, FD Hamiltonian (.PSIL) */
#define ESPEC_PSOD 3        /* second-order differences, FD Hamiltonian (.PSOD) */

/* reproduce reference defects on request (FP64 form only) */
#define ESPEC_Q_SPO_INPLACE 1   /* spofft.f:150-153 kinetic multiply            */
#define ESPEC_Q_SOD_SMOOTHW 2   /* sodfft.f:108 never applies the .SMOOTHW mask */
#define ESPEC_Q_SIL_INPLACE 4   /* sil.f:145-148 sin term uses the cos-scaled U   */
#define ESPEC_Q_FFTNT_SP 8      /* cfft.f:35 TWOPI from a single-precision literal */
#define ESPEC_Q_DIGT_ND 16      /* dkeft.f:80-137 2D/3D kinetic table as written   */
#define ESPEC_Q_PSOD_COPY 32    /* psod.f:136-141 restart copy sets V1(I+1) = V0(I) */
#define ESPEC_Q_GVPOT_3D 64     /* gvpot.f:96 3D grid takes RX from the z index    */

/* analytic potential forms (potfuncs.f; espec_pot_kind maps the deck's name) */
#define ESPEC_POT_OHS 1          /* 1D/2D/3D harmonic                             */
#define ESPEC_POT_DOHS 2         /* 1D                                            */
#define ESPEC_POT_MORSEM 3       /* 1D                                            */
#define ESPEC_POT_ANTI_MORSEM 4  /* 1D                                            */
#define ESPEC_POT_MOD_MORSE 5    /* 1D                                            */
#define ESPEC_POT_MORSE 6        /* 1D/2D                                         */
#define ESPEC_POT_ANTI_MORSE 7   /* 1D                                            */
#define ESPEC_POT_DMORSE 8       /* 1D                                            */
#define ESPEC_POT_STEP 9         /* 1D/3D                                         */
#define ESPEC_POT_BARRIER 10     /* 1D/2D/3D                                      */
#define ESPEC_POT_CONST 11       /* .CONST / .FREE                                */
#define ESPEC_POT_LSM 12         /* 2D                                            */
#define ESPEC_POT_LS 13
#define ESPEC_POT_LBH_CC 14
#define ESPEC_POT_LBH 15
#define ESPEC_POT_LEPS_CC 16
#define ESPEC_POT_LEPS 17        /* 2D/3D                                         */
#define ESPEC_POT_WELLXY 18
#define ESPEC_POT_WELLX 19
#define ESPEC_POT_WELLY 20
#define ESPEC_POT_WELL 21
#define ESPEC_POT_BARRIERXY 22
#define ESPEC_POT_BARRIERX 23
#define ESPEC_POT_BARRIERY 24

/* memory space of user pointers */
#define ESPEC_MEM_HOST 0
#define ESPEC_MEM_DEVICE 1
/* host memory (page-locked) with the copies left in flight on the stream:
 * espec_spo_load and espec_spo_results return at once, the caller
 * synchronises the stream before it reads or reuses the buffers */
#define ESPEC_MEM_HOST_ASYNC 2

/* launch shape of a batched split-operator run (espec_spo_set_launch) */
#define ESPEC_LAUNCH_CLASSES 0     /* one kernel per packet size, concurrent streams */
#define ESPEC_LAUNCH_PERSISTENT 1  /* one persistent kernel over every packet size   */

#define ESPEC_SHFS 2.4188843243e-2  /* fs per atomic unit of time (pspofft.f:76) */

/* ----------------------------------------------------------------------
 * Fortran-callable drop-ins.  Same arguments, same outputs and the
 * same printed partial auto-correlation table as the reference routines;
 * the defects of the reference's arithmetic are reproduced.  A case the GPU
 * path does not run (PSPOFFT/PSODFFT: unsupported grid sizes; PLNZ: order
 * above 16) or a device error sets INFO = 2 (message on
 * standard error).  Work arrays, XI, XF, VAR, ABSTOL and IWORK are accepted
 * and not touched.
 * ---------------------------------------------------------------------- */
/* replaces SUBROUTINE PSPOFFT (pspofft.f:1-3; called from espec.f:1474), 1D
 * (espec_spo_* plan) and 2D/3D (espec_spond_* plan, the reference's N-D
 * kinetic table) */
void pspofft_(const int* absorb, const char* dim, const char* prtcrl,
              const char* tpabsor, int* info, const int* lc, const int* mp,
              const int* mpi, const int* mpr, const int* mxdct, const int* n,
              const double* dt, const double* ti, const double* tf,
              const double* tol, const int* np, const double* shm,
              const double* sh, const double* sm, double* u1, double* v1,
              const double* xi, const double* xf, double* tc,
              const double* vpot, const double* vabc, double* lnzvc,
              double* wrk1, double* wrk2, const double* var, size_t dim_len,
              size_t prtcrl_len, size_t tpabsor_len);
/* replaces SUBROUTINE PSODFFT (psodfft.f:1-3; called from espec.f:1373), 1D
 * and 2D/3D */
void psodfft_(const int* absorb, const char* dim, const char* prtcrl,
              const char* tpabsor, int* info, const int* lc, const int* mp,
              const int* mpi, const int* mpr, const int* mxdct, const int* n,
              const double* dt, const double* ti, const double* tf,
              const double* tol, const int* np, const double* shm,
              const double* sh, const double* sm, double* u1, double* u2,
              double* v1, double* v2, const double* xi, const double* xf,
              double* tc, const double* vpot, const double* vabc,
              double* wrkr, double* wrki, const double* var, double* lnzvc,
              size_t dim_len, size_t prtcrl_len, size_t tpabsor_len);
/* replaces SUBROUTINE PLNZ (plnz.f:1-4; called from espec.f:1499), 1D/2D/3D;
 * also leaves the last Lanczos basis in LNZVC(1:N, 1:MP) as LNZ does */
void plnz_(const int* absorb, const int* change, const char* dim,
           const char* prtcrl, const char* tpabsor, int* info, const int* lc,
           const int* lmtreort, int* mp, const int* mpi, const int* mpr,
           const int* mxdct, const int* n, const double* abstol,
           const double* dt, const double* ti, const double* tf,
           const double* tol, const int* np, int* iwork, const double* shm,
           const double* vpot, const double* vabc, double* u, double* v,
           const double* xi, const double* xf, double* wu, double* wv,
           double* wp, double* work, const double* var, double* lnzvc,
           size_t dim_len, size_t prtcrl_len, size_t tpabsor_len);
/* replaces SUBROUTINE PSOD (psod.f:1-3; called from espec.f:1362), 1D/2D/3D
 * (espec_grid_* plan, method ESPEC_PSOD, the reference's restart-copy
 * defect): psi(TF) in U2/V2, psi(TF-dt) in U1/V1; an absorber other than
 * .VOPTIC/.SMOOTHW/.SMRS, where the reference STOPs, sets INFO = 2 */
void psod_(const int* absorb, const char* dim, const char* prtcrl,
           const char* tpabsor, int* info, const int* lc, const int* mp,
           const int* mpi, const int* mpr, const int* mxdct, const int* n,
           const double* dt, const double* ti, const double* tf,
           const double* tol, const int* np, const double* shm, double* u1,
           double* u2, double* v1, double* v2, const double* xi,
           const double* xf, const double* vpot, const double* vabc,
           double* work, const double* var, double* lnzvc, size_t dim_len,
           size_t prtcrl_len, size_t tpabsor_len);
/* replaces SUBROUTINE PPSOD (ppsod.f:1-5; called from espec.f:1398): PSOD with
 * the laser pulse EFC (.GAUS, .GGAUS, .SIN2, .NONE; E0, TP, OMG, T0 / TD, SNI,
 * KL as ef.f) and dipole DM, 1D/2D/3D; prints the table of ppsod.f (E with and
 * without the field, C(t), the populations of LNZVC(., KP+1..KP+NPR), the
 * norm); C(t) in LNZVC(., MPR/MPI); psi(TF) in U2/V2, psi(TF - dt) in U1/V1;
 * VPOT left holding VP - DM EF of the last step.  The movie, potential and
 * pulse files of PRTVEFF, PRTEIGVC2, PRTPULS are not written. */
void ppsod_(const int* absorb, const int* prtveff, const int* prteigvc2, const int* prtpuls,
            const char* dim, const char* efc, const char* prtcrl, const char* tpabsor,
            int* info, const int* lc, const int* mp, const int* mpi, const int* mpr,
            const int* mxdct, const int* n, const int* nshot, const int* npr, const int* kp,
            const int* nispg, const double* e0, const double* t0, const double* td,
            const double* tp, const double* omg, const double* sni, const int* kl,
            const double* dt, const double* ti, const double* tf, const double* tol,
            const int* np, const int* nd, const double* sh, const double* shm, double* u1,
            double* u2, double* v1, double* v2, const double* xi, const double* xp,
            const double* xf, const double* dm, double* vpot, const double* vabc, double* work,
            const double* var, double* lnzvc, const int* prtregion, const int* nreg,
            const double* range, const int* prtonlyreim, size_t dim_len, size_t efc_len,
            size_t prtcrl_len, size_t tpabsor_len);
/* replaces SUBROUTINE PPLNZ (pplnz.f:1-5; called from espec.f:1513 for
 * '.PPSIL' / '.PPLNZ'): PLNZ with the laser pulse EFC and dipole DM, 1D/2D/3D;
 * prints pplnz.f's table (E with and without the field, C(t), |C|^2 and the
 * populations of LNZVC(., KP+1..KP+NPR-1), the norm); C(t) in LNZVC(., MPR/MPI),
 * the last step's Lanczos basis in LNZVC(., 1..MP); psi(TF) in U/V; VPOT
 * left holding VP - DM EF of the last step; MP lowered as LNZ lowers it.  The
 * files of PRTVEFF, PRTEIGVC2, PRTPULS and '.LASTWP' are not written. */
void pplnz_(const int* absorb, const int* change, const int* prtveff, const int* prteigvc2,
            const int* prtpuls, const char* dim, const char* efc, const char* prtcrl,
            const char* tpabsor, int* info, const int* lc, const int* lmtreort, int* mp,
            const int* mpi, const int* mpr, const int* mxdct, const int* n, const int* nshot,
            const int* kl, const int* npr, const int* kp, const double* abstol, const double* dt,
            const double* ti, const double* tf, const double* tol, const double* e0,
            const double* t0, const double* td, const double* tp, const double* omg,
            const double* sni, const int* np, const int* nd, int* iwork, const double* sh,
            const double* shm, double* vpot, const double* vabc, double* u, double* v,
            const double* xi, const double* xf, const double* xp, const double* dm, double* wu,
            double* wv, double* wp, double* work, const double* var, double* lnzvc,
            size_t dim_len, size_t efc_len, size_t prtcrl_len, size_t tpabsor_len);
/* replace SUBROUTINE HWHM (hwhm.f:1-80; TAL is scaled in place) and
 * SUBROUTINE SPECTRUMTD (spectrumtd.f:1-116; prints the spectrum table,
 * sets DE < 0 to 0), called at espec.f:1618-1624: the arithmetic runs on the
 * GPU (espec_spectrum_dev), FFTNT's single-precision 2 pi included */
void hwhm_(const int* m, const double* dt, const double* tf, double* tal,
           const double* de, double* u, double* v);
void spectrumtd_(const char* tpwind, const int* m, const double* dt,
                 const double* tf, const double* wp, double* de, double* u,
                 double* v, size_t tpwind_len);
/* Runs an eSPec input deck (time-dependent part of espec.f for one packet
 * with a .FILE potential and its .GETR eigenvector; .PFSPO, .PFSOD, .PSIL,
 * .PSOD, and .PPSOD / .PPSIL with *PULSE_AND_DIPOLE; absorbers, total
 * correlation, HWHM and spectrum) through the GPU
 * drop-ins, printing to stdout what espec.x prints from "Propagating
 * eigenvector..." on.  Files named in the deck are relative to the deck's
 * directory.  An option outside that part is refused (ESPEC_EINVAL, reason
 * on stderr).  No counterpart entry point in the reference: it replaces the
 * executable's driver for these decks. */
int espec_run_deck(const char* deck_path);
/* The same deck over njobs .FILE inputs (each its own initial state and
 * potential, the deck's grid size), replacing one executable run per file:
 * 1D .PFSPO or .PFSOD, all packets in one batched plan and one batched
 * spectrum launch; writes the correlation block to <out_prefix><k>.crl and
 * the spectrum block to <out_prefix><k>.spc (k = 1..njobs, the text espec.x
 * prints for that file).  No counterpart entry point in the reference. */
int espec_run_scan(const char* deck_path, int njobs, const char* const* data_files,
                   const char* out_prefix);
/* one row of the partial auto-correlation table in FORMAT 1021 of
 * pspofft.f:148 (newline included); returns its length */
int espec_format_crl_row(double t, double e, double cr, double ci, double ct,
                         double fnt, char* buf, int len);

const char* espec_last_error(void);
const char* espec_version(void);
/* 1 when a CUDA device of compute capability 10.x is usable, else 0 */
int espec_device_ok(void);

/* ----------------------------------------------------------------------
 * Batched 1D split-operator plans.
 *
 * Replaces the time loop of PSPOFFT (pspofft.f:110-145) with PSPOFFTAUX
 * (spofft.f:3-203) for many independent 1D packets at once.  Packet k has
 * npts[k] points, grid step sh[k] (bohr) and mass sm[k] (electron masses);
 * all packets share dt_fs.  Sizes 256, 384, 512, 768, 1024, 1536, 2048 and
 * 4096 run the register FFT plans (FP64 or mixed); any other even size from 4
 * to 7252 runs, in FP64, one CTA per packet with a shared-memory mixed-radix
 * FFT (any N, as the reference's fft3d.f).
 * Arrays passed to espec_spo_load are concatenated over packets in order.
 * C(t) = <psi(0)|psi(t)> is produced for every step: nsteps+1 complex
 * samples per packet, packet-major.
 * ---------------------------------------------------------------------- */
typedef struct espec_spo_plan espec_spo_plan;

int espec_spo_create(espec_spo_plan** plan, int npk, const int* npts,
                     const double* sh, const double* sm, double dt_fs,
                     int precision, int absorb, int quirks);
/* Same plan for another method: ESPEC_SOD replaces the time loop of PSODFFT
 * (psodfft.f:77-206, sodfft.f:64-126), FP64 only, register plans for sizes
 * 256..2048 and any other even size up to 3626 in shared memory; its first
 * step is the reference's two-half-step start-up and C(t) again has nsteps+1
 * samples.  espec_spo_create(...) = espec_prop_create(..., ESPEC_SPO, ...). */
int espec_prop_create(espec_spo_plan** plan, int npk, const int* npts,
                      const double* sh, const double* sm, double dt_fs, int method,
                      int precision, int absorb, int quirks);
/* SOD plans: psi(TF - dt), the older of the two states the leapfrog keeps */
int espec_prop_previous(espec_spo_plan* plan, double* psi_re, double* psi_im,
                        int where, void* stream);
/* vabc: absorber table (complex-potential values for ESPEC_ABS_VOPTIC, mask
 * for ESPEC_ABS_SMOOTHW), ignored for ESPEC_ABS_NONE; psi_im may be NULL. */
int espec_spo_load(espec_spo_plan* plan, const double* vpot, const double* vabc,
                   const double* psi_re, const double* psi_im, int where,
                   void* stream);
int espec_spo_run(espec_spo_plan* plan, int nsteps, void* stream);
int espec_spo_results(espec_spo_plan* plan, double* c_re, double* c_im,
                      double* psi_re, double* psi_im, int where, void* stream);
/* nsteps more steps from the plan's current state (psi0 right after
 * espec_spo_load, else the state the last run or continuation left; a SOD
 * plan needs one espec_spo_run first).  C(t) stays <psi0|psi(t)>; sample s
 * (1..nsteps) is the s-th step of this call, sample 0 is not written.  The
 * printed rows of PSPOFFT/PSODFFT split a run this way (pspofft.f:125-144). */
int espec_prop_continue(espec_spo_plan* plan, int nsteps, void* stream);
/* energy EFFT4 (eigenergfft.f:58-100: sum V|psi|^2 + B sum TC |F psi|^2, B=1/N,
 * hartree) and norm sum |psi|^2 (pspofft.f:96-98) of each packet's current
 * state, FP64 on the GPU; e and norm are host arrays of npk entries. */
int espec_prop_energies(espec_spo_plan* plan, double* e, double* norm, void* stream);
/* Kernel variant for the packets of size npts (0..espec_spo_variant_count()-1):
 * radix plan, location of the per-point tables and register budget.  Call
 * before espec_spo_load.  Defaults come from autotuning on B200. */
int espec_spo_set_variant(espec_spo_plan* plan, int npts, int variant);
int espec_spo_variant_count(void);
/* ESPEC_VARIANT_TC (256-point packets, mixed form only): the FFT as dense
 * 16-point DFT GEMMs on the tensor cores (tcgen05.mma, BF16 x 3 split
 * operands, FP32 accumulation in tensor memory), 8 packets per CTA; the
 * phases, twiddles and C(t) as the other mixed variants.  No counterpart in
 * the reference (its FFT is fft3d.f).  espec_spo_tc_status: 1 when one of its
 * bounded mbarrier waits gave up since the last call (synchronous; clears). */
#define ESPEC_VARIANT_TC 5
int espec_spo_tc_status(int* timed_out);
/* Launch shape of espec_spo_run / espec_prop_continue.  ESPEC_LAUNCH_CLASSES
 * (the default): one kernel per size class on concurrent streams, each with
 * the variant espec_spo_set_variant chose (setting a variant selects this
 * shape).  ESPEC_LAUNCH_PERSISTENT (available when every packet size is
 * 256..2048 and the plan is an FP64 or mixed split operator without the
 * in-place defect): one kernel whose CTAs claim items -- groups of packets of
 * one size filling a CTA -- from a device counter, longest items first.  Call
 * before espec_spo_load; no counterpart in the reference (its scans run one
 * process per packet). */
int espec_spo_set_launch(espec_spo_plan* plan, int mode);
/* Relative cost of one persistent item of packets of size npts (the claim
 * order is by decreasing cost; default: points of an item x log2 npts). */
int espec_spo_set_item_cost(espec_spo_plan* plan, int npts, double cost);
/* Number of packets whose C(t) became NaN or infinite during the last run or
 * continued segment of a split-operator plan (checked on the device at every
 * C(t) sample, counted once per packet; synchronises with the stream).  The
 * drop-ins keep the reference's INFO (a NaN fails none of its drift tests);
 * a batched caller reads this count after each segment. */
int espec_prop_nonfinite(espec_spo_plan* plan, int* count, void* stream);
/* device pointer of the C(t) buffer (double2, packet-major) */
const void* espec_spo_device_c(const espec_spo_plan* plan);
int espec_spo_npoints(const espec_spo_plan* plan);
void espec_spo_destroy(espec_spo_plan* plan);

/* ----------------------------------------------------------------------
 * Batched 1D split-operator propagation that allocates nothing.
 *
 * No counterpart in the reference: eSPec has no GPU and no allocator to
 * avoid.  For callers that cannot call cudaMalloc -- an application that owns
 * the whole device memory pool, a code under a fixed memory budget, or code
 * running while another component captures or replays GPU work.  Inputs and
 * outputs are device pointers owned by the caller; the intermediate tables
 * live in one fixed __device__ array inside the library (about 3.2 MB, held on
 * every GPU that loads the library until the process exits).
 *
 * npts/sh/sm: host arrays of npk entries (at most 128 packets, at most 32768
 * grid points in total; sizes as espec_spo_create).  vpot: npts-sum doubles.
 * psi0: interleaved complex (re, im) doubles.  c_out: interleaved complex,
 * npk*(nsteps+1) samples, packet-major.  psi_out: interleaved complex or NULL.
 * No absorber; C(t) every step, same arithmetic as variant 0 of the plans.
 * Calls share the array: calls whose GPU work overlaps race; serialise them.
 * The first call on each device resolves the array's address; make it
 * before any stream capture.  A call is not itself capturable into a graph:
 * it copies its packet descriptors from host memory that is gone by the time
 * a graph would replay.  The array's address is cached for the life of the
 * process (one primary context per device; do not call again on a device
 * after cudaDeviceReset).  Sizes beyond the limits return ESPEC_EINVAL.
 * ---------------------------------------------------------------------- */
int espec_spo_run_static(int npk, const int* npts, const double* sh,
                         const double* sm, double dt_fs, int precision,
                         const double* vpot, const double* psi0, int nsteps,
                         double* c_out, double* psi_out, void* stream);

/* ----------------------------------------------------------------------
 * Grid plans: one wave packet on a 1D, 2D or 3D grid (x fastest, the
 * reference's column-major U(N) layout).
 *
 * ESPEC_SIL replaces the time loop of PLNZ (plnz.f:71-151) with PLNZAUX
 * (sil.f:70-181), LNZ (lnz.f:76-119), REORT (reort.f:65-80) and AU
 * (au1d.f, au2di.f, au3d.f): per step two m-step Lanczos chains (real and
 * imaginary part) with full classical Gram-Schmidt reorthogonalisation, the
 * Krylov exponential of the tridiagonal matrix, FP64.  np: points per axis;
 * shm: 1/(24 m_a h_a^2) per axis (espec.f:819); mp: Lanczos order 1..16
 * (already clamped as lnz.f:64-72 does); absorb: ESPEC_ABS_NONE or
 * ESPEC_ABS_SMOOTHW (mask applied after each step, sil.f:171-175); quirks:
 * ESPEC_Q_SIL_INPLACE.  One cooperative launch per run; C(t) = <psi0|psi(t)>
 * every step (nsteps+1 samples).
 *
 * ESPEC_PSOD replaces the time loop of PSOD (psod.f:64-205) with PSODAUX
 * (sod.f:64-123) and the same AU: psi(t+dt) = psi(t-dt) - 2 i dt H psi(t),
 * started by an Euler step to t + dt/2 and a midpoint step to t + dt; mp is
 * ignored; absorb: ESPEC_ABS_NONE, ESPEC_ABS_VOPTIC (vabc = the complex
 * absorbing potential) or ESPEC_ABS_SMOOTHW (vabc = the mask); quirks:
 * ESPEC_Q_PSOD_COPY.  One cooperative launch per run, one grid barrier per
 * step.
 * ---------------------------------------------------------------------- */
typedef struct espec_grid_plan espec_grid_plan;

int espec_grid_create(espec_grid_plan** plan, int method, int ndim, const int* np,
                      const double* shm, double dt_fs, int mp, int precision,
                      int absorb, int quirks);
/* psi_im may be NULL; vabc: the absorber table (ignored without one) */
int espec_grid_load(espec_grid_plan* plan, const double* vpot, const double* vabc,
                    const double* psi_re, const double* psi_im, int where,
                    void* stream);
int espec_grid_run(espec_grid_plan* plan, int nsteps, void* stream);
/* nsteps more steps from the current state; sample 0 is not written */
int espec_grid_continue(espec_grid_plan* plan, int nsteps, void* stream);
/* synchronises; fails with ESPEC_ECUDA if a grid barrier of the kernel
 * gave up waiting */
int espec_grid_results(espec_grid_plan* plan, double* c_re, double* c_im,
                       double* psi_re, double* psi_im, int where, void* stream);
/* EIGENERG (eigenerg.f:56-66): <u|H_FD u> + <v|H_FD v>, and |u|^2 + |v|^2,
 * of the current state */
int espec_grid_energies(espec_grid_plan* plan, double* e, double* norm, void* stream);
/* Lanczos vectors of the last step's chain (0: real part, 1: imaginary part)
 * into dst(1:N, 1:MP) with leading dimension ld >= N (column-major) */
int espec_grid_basis(espec_grid_plan* plan, int chain, double* dst, int ld, int where,
                     void* stream);
/* <u|H u> + <v|H v> and the norm with the potential V - DM EF (a PSOD plan
 * with a pulse; EF = 0 gives espec_grid_energies) */
int espec_grid_energies_at(espec_grid_plan* plan, double ef, double* e, double* norm,
                           void* stream);
/* Laser pulse (chpot.f): dm = the dipole function on the grid, ef = a field
 * table counted from the start of a run and continued through
 * espec_grid_continue.  ESPEC_PSOD plans (PPSOD, ppsod.f): PSODAUX call j
 * uses the potential V - dm * ef[j] (0, 1: the start-up; step s >= 2: call s;
 * espec_ppsod_field).  ESPEC_SIL plans (PPLNZ, pplnz.f): the step landing at
 * step j uses V - dm * ef[j] (espec_pplnz_field).  Copies both tables. */
int espec_grid_set_pulse(espec_grid_plan* plan, const double* dm, const double* ef, long ncalls,
                         int where);
/* <w_j|u> and <w_j|v> of the current state u + i v for nvec <= 8 real
 * device vectors w (column j at w + j N): out[2j], out[2j+1] on the host
 * (the populations of ppsod.f:268-300; synchronises) */
int espec_grid_project(espec_grid_plan* plan, const double* w, int nvec, double* out,
                       void* stream);
/* ESPEC_PSOD plans: psi(TF - dt) of the last run (synchronises) */
int espec_grid_previous(espec_grid_plan* plan, double* psi_re, double* psi_im, int where,
                        void* stream);
long espec_grid_npoints(const espec_grid_plan* plan);
void espec_grid_destroy(espec_grid_plan* plan);
/* Bounded waits of the grid kernels (no counterpart in the reference, which
 * has no device waits).  Every grid-barrier wait of the SIL and PSOD kernels
 * gives up after `polls` polls of the arrival count (0: the default, 2^24,
 * seconds); the kernel then sets its error flag and returns, and
 * espec_grid_results reports ESPEC_ECUDA ("timed out"), the drop-ins INFO = 2.
 * espec_selftest_short_arrivals(k): the next k grid launches start their
 * arrival count one short, so their first barrier never completes and every
 * wait runs out -- the time-out path exercised without any fault; the device
 * stays usable. */
int espec_set_wait_limit(long polls);
int espec_selftest_short_arrivals(int launches);
/* CTAs of the plan's cooperative launches: 1 .. the co-resident maximum chosen
 * at creation (one per SM, or every co-resident CTA for large PSOD grids);
 * 0 restores that maximum.  Fewer CTAs make each grid barrier's reduction
 * cheaper on small grids (a tuning knob; results do not depend on it beyond
 * the order of the partial sums). */
int espec_grid_set_ctas(espec_grid_plan* plan, int nctas);

/* ----------------------------------------------------------------------
 * Analytic potentials on the GPU: the forms of POT1D / POT2D / POT3D
 * (potfuncs.f:3-497) on the grid loop of GVPOT (gvpot.f:1-111), with its
 * shift by the grid minimum when shiftp is set (1D and 3D: when the minimum
 * is above 1e-6; 2D: when its magnitude is).  cst: the 14 constants (MXCST)
 * GVPOT receives, i.e. after MAKECST, in atomic units.
 *
 * espec_pot_kind: ESPEC_POT_* of the name POTCH for a grid of ndim axes (the
 * first of the reference's prefix tests that matches), 0 if none.
 * espec_gvpot_1d: npk packets (a parameter scan; packet k: npts[k] points at
 * xi[k] + i sh[k], constants cst[k*14 .. k*14+13]) in one launch; vpot:
 * device, concatenated; xmin: host [npk] or NULL, the grid point of each
 * minimum (GVPOT's XMIN) when shiftp.  Synchronous.
 * espec_gvpot_nd: one 2D or 3D grid (x fastest); sm: NULL or the three
 * masses SM(1..3) of the .LBH_CC / .LEPS_CC mass-scaled coordinates (unused
 * by the other forms); quirks: ESPEC_Q_GVPOT_3D.
 * ---------------------------------------------------------------------- */
int espec_pot_kind(const char* potch, size_t len, int ndim);
int espec_gvpot_1d(int npk, const int* npts, const double* xi, const double* sh, int kind,
                   const double* cst, int shiftp, double* vpot, double* xmin, void* stream);
int espec_gvpot_nd(int ndim, const int* np, const double* xi, const double* sh,
                   const double* sm, int kind, const double* cst, int shiftp, int quirks,
                   double* vpot, void* stream);

/* ----------------------------------------------------------------------
 * Split-operator propagation on one 2D or 3D grid (PSPOFFT/PSPOFFTAUX,
 * pspofft.f:72-145, spofft.f:64-200, with the N-D kinetic table of DIGT,
 * dkeft.f:80-137).  Axis sizes 32, 64, 128, 256 or 512, x fastest; sh, sm per
 * axis; precision ESPEC_FP64 or ESPEC_MIXED (FP32 state and transforms, FP64
 * tables and C(t)); absorb as the 1D plans; quirks ESPEC_Q_SPO_INPLACE (FP64)
 * and ESPEC_Q_DIGT_ND (the reference's 2D/3D table, only TC(1..NP1) filled;
 * without it the table is the outer sum of the axis tables).  C(t) every step,
 * nsteps+1 samples; psi(TF) returned by espec_spond_results.
 * ---------------------------------------------------------------------- */
typedef struct espec_spond_plan espec_spond_plan;
int espec_spond_create(espec_spond_plan** plan, int ndim, const int* np, const double* sh,
                       const double* sm, double dt_fs, int precision, int absorb, int quirks);
/* the same for a method: ESPEC_SPO, or ESPEC_SOD (PSODFFT, psodfft.f:77-206,
 * sodfft.f:64-126: FP64, two half-step start-up, then leapfrog; quirks
 * ESPEC_Q_SOD_SMOOTHW, ESPEC_Q_DIGT_ND) */
int espec_spond_create_method(espec_spond_plan** plan, int method, int ndim, const int* np,
                              const double* sh, const double* sm, double dt_fs, int precision,
                              int absorb, int quirks);
/* SOD plans: psi(TF - dt) of the last run */
int espec_spond_previous(espec_spond_plan* plan, double* psi_re, double* psi_im, int where,
                         void* stream);
int espec_spond_load(espec_spond_plan* plan, const double* vpot, const double* vabc,
                     const double* psi_re, const double* psi_im, int where, void* stream);
int espec_spond_run(espec_spond_plan* plan, int nsteps, void* stream);
int espec_spond_results(espec_spond_plan* plan, double* c_re, double* c_im, double* psi_re,
                        double* psi_im, int where, void* stream);
/* nsteps more steps from psi of the last run; sample 0 is not written */
int espec_spond_continue(espec_spond_plan* plan, int nsteps, void* stream);
/* EFFT4 (eigenergfft.f:58-100) and sum |psi|^2 of the current state (psi0
 * before any run), FP64 on the GPU */
int espec_spond_energies(espec_spond_plan* plan, double* e, double* norm, void* stream);
void espec_spond_destroy(espec_spond_plan* plan);

/* ----------------------------------------------------------------------
 * Initial-state eigensolver, batched over potentials (2D grids, FP64).
 *
 * LANCZSG (lanczsc.f:56-120): for each of nstates lowest states, restarted
 * Lanczos of length m (full reorthogonalisation, lnz.f/reort.f) from a start
 * vector, restarting from the K-th Ritz vector until |H v - theta v| <= tol
 * (the true residual; one H*v per restart on top of the m Lanczos steps).
 * All pointers are device pointers: vpot [nprob][n], start [nprob][nstates]
 * [n], vec [nprob][nstates][n] (the normalised eigenvectors), eval/resid
 * [nprob][nstates], matvecs [nprob][nstates] (H*v applications per state),
 * work_L [nprob][m][n] and work_v [nprob][n] scratch.  m <= 40, nstates <= 16.
 * A 1D problem is an np[0] x 1 grid with shm[1] = 0.
 * ---------------------------------------------------------------------- */
int espec_eig_solve_dev(int nprob, const int* np, const double* shm,
                        const double* vpot, const double* start, int nstates, int m,
                        double tol, int maxrest, double* vec, double* eval,
                        double* resid, int* matvecs, double* work_L, double* work_v,
                        void* stream);
/* the reference's cold start (rans.f:38-39 LCG from NSEED = 1, the first n
 * draws discarded, then n draws per state; lanczsc.f:56-62) into d_out
 * [nstates][n] */
int espec_eig_lcg_start(double* d_out, int n, int nstates, void* stream);
/* 2D coupled-Morse potentials on an np[0] x np[1] grid over [xi,xf]x[yi,yf]
 * from params [nprob][5] = (De1, a1, De2, a2, lambda) (device pointers) */
int espec_eig_morse2d(int nprob, const double* params, const int* np, double xi,
                      double xf, double yi, double yf, double re1, double re2,
                      double* vpot, void* stream);

/* ----------------------------------------------------------------------
 * Learned warm start for the eigensolver (no counterpart in the reference,
 * which always starts from its LCG vectors).  Kernels of a small multilayer
 * perceptron trained on the eigensolver's own eigenvectors; all pointers are
 * device pointers, matrices row-major.
 * ---------------------------------------------------------------------- */
/* C[M,N] = alpha op(A) op(B) + beta C, op(X) = X^T when t* != 0 */
int espec_gemm_f64(int M, int N, int K, double alpha, const double* A, int lda, int ta,
                   const double* B, int ldb, int tb, double beta, double* C, int ldc,
                   void* stream);
int espec_gemm_f32(int M, int N, int K, float alpha, const float* A, int lda, int ta,
                   const float* B, int ldb, int tb, float beta, float* C, int ldc,
                   void* stream);
/* db[c] = sum_r dy[r,c] */
int espec_mlp_colsum(const float* dy, int rows, int cols, float* db, void* stream);
/* mean squared error: row_loss[r] = sum_c (y-t)^2/(rows cols), dy = its gradient */
int espec_mlp_mse(const float* y, const float* t, int rows, int cols, float* dy,
                  float* row_loss, void* stream);
/* separable basis transform, one vector of nx*ny points (x fastest) per CTA;
 * phi [nb][nx], chi [nb][ny] (float, device); coefficient index a*nb + b:
 * dir 0: c[v][a*nb+b] = scale sum_{x,y} phi[a][x] chi[b][y] psi[v][x+nx*y]
 * dir 1: psi[v][x+nx*y] = scale sum_{a,b} phi[a][x] chi[b][y] c[v][a*nb+b]
 * (FP32 arithmetic; psi double, c float) */
int espec_sep_basis(int dir, int nvec, int nx, int ny, int nb, const float* phi, const float* chi,
                    double* psi, float* c, float scale, void* stream);
/* element-wise f64 -> f32 (to_f32 != 0) or f32 -> f64, times scale */
int espec_convert(const void* src, void* dst, long count, int to_f32, double scale,
                  void* stream);
/* C[M,N] (float) = alpha op(A) op(B) + beta C with A, B bfloat16 (raw 16-bit
 * values), FP32 accumulation on the tensor cores (tcgen05.mma, accumulator in
 * tensor memory); op(X) = X^T when t* != 0, row-major as espec_gemm_f32 */
int espec_gemm_bf16(int M, int N, int K, float alpha, const void* A, int lda, int ta,
                    const void* B, int ldb, int tb, float beta, float* C, int ldc, void* stream);
/* synchronous: 1 when a tensor-core GEMM gave up waiting for its MMAs since
 * the last call (its output is then not written), else 0; clears the flag */
int espec_gemm_bf16_status(int* timed_out);
/* Self-test of the tensor-core GEMM's bounded mbarrier wait: one thread waits
 * on an mbarrier nothing arrives on (no copy or MMA attached) with a limit of
 * `polls` polls; *gave_up = 1 when the wait gave up as it must (the GEMM
 * status flag is set too: read it with espec_gemm_bf16_status).  Synchronous. */
int espec_selftest_mbar_wait(long polls, int* gave_up);
/* z[r,c] += b[c]; h = bf16(GELU(z)) (act != 0) or bf16(z); h may be NULL */
int espec_mlp_bias_gelu(float* z, const float* b, int rows, int cols, int act, void* h_bf16,
                        void* stream);
/* dh *= GELU'(z) (z = the layer's pre-activation); dz_bf16 = bf16(dh) */
int espec_mlp_gelu_back(float* dh, const float* z, long count, void* dz_bf16, void* stream);
/* y = bf16(x) */
int espec_to_bf16(const float* x, void* y, long count, void* stream);
/* one Adam step (Kingma & Ba) on FP32 master weights with hyper = device
 * {lr, 1 - b1^t, 1 - b2^t} (replayable from a captured CUDA graph with new
 * values written into hyper), then w_bf16 = bf16(w) (w_bf16 may be NULL) */
int espec_mlp_adam_bf16(float* w, const float* g, float* m1, float* m2, long count,
                        const float* hyper, float b1, float b2, float eps, void* w_bf16,
                        void* stream);

/* ----------------------------------------------------------------------
 * Laser pulses (ef.f): E(t) in atomic units for the shapes of *PULSE_AND_DIPOLE;
 * par = {E0, TP, OMG, T0 (.GAUS, .GGAUS) or TD (.SIN2), SNI, KL (.GGAUS)}.
 * ---------------------------------------------------------------------- */
#define ESPEC_PULSE_NONE 0
#define ESPEC_PULSE_GAUS 1
#define ESPEC_PULSE_GGAUS 2
#define ESPEC_PULSE_SIN2 3
double espec_pulse_field(int shape, const double* par, double t);
/* the field of every PSODAUX call of a PPSOD run from TI to TF (ppsod.f:252-260,
 * 378-386): ef[0] at (TI+DT)/2, ef[1] at TI+DT, then one per step of DT for
 * NF = NINT((TF + DT/2 - TI - DT)/DT) steps; returns NF + 2 (the run has
 * NF + 1 steps) or a negative error code */
long espec_ppsod_field(int shape, const double* par, double ti, double tf, double dt, double* ef,
                       long cap);
/* the field of every step of a PPLNZ run (pplnz.f:139-141, DO T = TI+DT,
 * TF+DT/2, DT with CHPOT(T) before each step): ef[0] = EF(TI), ef[s] = EF at
 * the time step s lands at; returns the number of steps + 1 */
long espec_pplnz_field(int shape, const double* par, double ti, double tf, double dt, double* ef,
                       long cap);

/* ----------------------------------------------------------------------
 * Spectrum stage on the device, batched over packets (FP64).
 *
 * For each of npk packets: the 2^mf-point time signal -- assembled from the
 * first 2^(mf-1) C(t) samples as espec.f:1545-1576 does (assemble = 1; in =
 * double2 C(t) with stride ld per packet, e.g. espec_spo_device_c with
 * ld = nsteps+1) or read as given (assemble = 0, stride ld) -- then HWHM
 * (hwhm.f:59-77; skipped when tal < 0; de = DE - E1I of espec.f:1618), the
 * window of SPECTRUMTD (window 1 = .SG with parameter wp, 0 = none), the half
 * swap and the backward DFT / N of FFTNT (spectrumtd.f:58-81, cfft.f).
 * spec: device double2 [npk][2^mf] in FFTNT's natural order.  work: device
 * scratch of espec_spectrum_work_bytes(npk, mf).  quirks: ESPEC_Q_FFTNT_SP.
 * ---------------------------------------------------------------------- */
int espec_spectrum_dev(int npk, int mf, const void* in, long ld, int assemble,
                       double dtf, double tf, double tal, double de, int window,
                       double wp, int quirks, void* spec, void* work, void* stream);
size_t espec_spectrum_work_bytes(int npk, int mf);

#ifdef __cplusplus
}
#endif
#endif
