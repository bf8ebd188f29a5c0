/*
 * espec_oracle.h -- CPU FP64 restatement of eSPec's propagation path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * product in espec_b200/: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it.  The product
 * never links or calls it.
 *
 * Every routine follows a Fortran routine of the eSPec sources (cited per
 * function in espec_oracle.cpp as file:line under the reference's src/).
 * Reference defects are reproduced only when the matching ORC_Q_* bit is set
 * in `quirks`; with quirks == 0 the oracle is the corrected method.
 *
 * Parity pin: the restatement is checked against outputs of the shipped
 * eSPec executable (tests/golden/, generated by tests/golden/make_golden.py)
 * at the executable's print precision, and against the reference's own
 * golden test8 spectrum.
 */
#ifndef ESPEC_ORACLE_H
#define ESPEC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* reference defects, reproduced on request */
#define ORC_Q_SPO_INPLACE  1  /* spofft.f:150-153 kinetic multiply reuses updated U */
#define ORC_Q_SIL_INPLACE  2  /* sil.f:145-148 sin term uses the cos-scaled U      */
#define ORC_Q_DIGT_ND      4  /* dkeft.f:80-137 2D/3D kinetic table filled wrongly   */
#define ORC_Q_SOD_SMOOTHW  8  /* sodfft.f:108 mask test never true: no .SMOOTHW   */
#define ORC_Q_FFTNT_SP    16  /* cfft.f TWOPI literal is single precision            */
#define ORC_Q_PSOD_COPY   32  /* psod.f:136-141 restart copy: V1(I+1) = V0(I)        */

enum { ORC_ABS_NONE = 0, ORC_ABS_VOPTIC = 1, ORC_ABS_SMOOTHW = 2 };
enum { ORC_PRT_NONE = 0, ORC_PRT_PARTIAL = 1, ORC_PRT_YES = 2 };

/* physical constants used by the reference (cited in espec_oracle.cpp) */
#define ORC_SHFS 2.4188843243e-2      /* fs per atomic time unit   */
#define ORC_A0A  0.5291772083         /* Angstrom per bohr         */
#define ORC_AMU  1836.152667539       /* electron masses per amu   */
#define ORC_FATE 27.2113834           /* eV per hartree            */

typedef struct {
  int ndim;          /* 1, 2 or 3                                   */
  int np[3];         /* grid points per axis, x fastest             */
  double dt, ti, tf; /* fs                                          */
  double tol;        /* drift tolerance in percent                  */
  double sh[3];      /* grid step per axis, bohr                    */
  double sm[3];      /* mass per axis, electron masses              */
  double shm[3];     /* 1/(24 m h^2) per axis (finite differences)  */
  int lc;            /* C(t) stride in steps                        */
  int absorb;        /* ORC_ABS_*                                   */
  int prtcrl;        /* ORC_PRT_*                                   */
  int quirks;        /* ORC_Q_* bits                                */
  int mp;            /* Lanczos order (SIL)                          */
  int lmtreort;      /* LMTREORT limit (SIL)                         */
  int change;        /* *CHANGE flag (SIL clamps MP to LMTREORT)     */
} orc_prop_t;

/* Fortran real-valued DO loop trip count: max(0, INT((b - a + c) / c)) */
int orc_do_count(double a, double b, double c);

/* multivariate FFT along one variable, Singleton calling convention */
void orc_fft(double* re, double* im, int ntot, int n, int nspan, int isn);

/* kinetic table in FFT order; returns B = 1/N in *b                     */
void orc_digt(int ndim, const int* np, const double* sh, const double* sm,
              double* tc, double* b, int quirks);

/* 4th-order finite-difference H*u with zero Dirichlet boundary          */
void orc_au(int ndim, const int* np, const double* shm, const double* vpot,
            const double* u, double* out);

double orc_fcorrel(int n, const double* a, const double* b);
double orc_ecnorm(int n, const double* a);
double orc_eigenerg(int ndim, const int* np, const double* shm,
                    const double* vpot, const double* u);
double orc_efft4(int ndim, const int* np, double b, const double* u,
                 const double* v, const double* tc, const double* vpot);

/* one propagation step (in place)                                       */
void orc_spo_step(int ndim, const int* np, double b, double cst1,
                  double cst2, const double* tc, const double* vpot,
                  const double* vabc, int absorb, int quirks, double* u,
                  double* v);

/* absorber table on the grid (1D: all types; 2D: SMOOTHW)              */
int orc_absorbingbc(int ndim, const int* np, int type, const double* al,
                    const double* ar, const double* sh, const double* xi,
                    const double* xf, const double* voi, double* vabc);
enum { ORC_ABC_SMOOTHW = 1, ORC_ABC_VOPTIC_LINEAR = 2,
       ORC_ABC_VOPTIC_POLIN = 3, ORC_ABC_SMRS = 4 };

/*
 * Propagators.  u, v (and u2, v2 for SOD) are overwritten with psi(TF).
 * c_re/c_im receive the stored C(t) samples (LNZVC columns), capacity c_cap.
 * rows (6 doubles per printed row: t, E, Cr, Ci, |C| or |C|^2, norm) are
 * filled when prtcrl != NONE, capacity row_cap.  Return value: number of C(t)
 * samples stored, or -1 on a fatal condition (the reference's STOP).
 */
int orc_pspofft(const orc_prop_t* p, const double* vpot, const double* vabc,
                double* u, double* v, double* c_re, double* c_im, int c_cap,
                double* rows, int row_cap, int* nrows, int* info);
int orc_psodfft(const orc_prop_t* p, const double* vpot, const double* vabc,
                double* u1, double* v1, double* u2, double* v2,
                double* c_re, double* c_im, int c_cap, double* rows,
                int row_cap, int* nrows, int* info);
int orc_plnz(const orc_prop_t* p, const double* vpot, const double* vabc,
             double* u, double* v, double* c_re, double* c_im, int c_cap,
             double* rows, int row_cap, int* nrows, int* info);
/* PSOD (psod.f): second-order differences with the finite-difference H;
 * on return (u2, v2) = psi(TF), (u1, v1) = psi(TF - dt) */
int orc_psod(const orc_prop_t* p, const double* vpot, const double* vabc,
             double* u1, double* v1, double* u2, double* v2, double* c_re,
             double* c_im, int c_cap, double* rows, int row_cap, int* nrows,
             int* info);

/* EF (ef.f:20-60): shape 0 none, 1 .GAUS, 2 .GGAUS, 3 .SIN2;
 * par = {E0, TP, OMG, T0 or TD, SNI, KL} */
double orc_ef(int shape, const double* par, double t);
/* PPSOD's propagation (ppsod.f:64-400 without its printed table, files and
 * populations): PSOD's steps with the potential VP - DM EF(t) of chpot.f at
 * (TI+DT)/2, TI+DT and then each step's end time; C(t) every LC steps, the
 * start-up samples included (the reference stores those only while it
 * prints) */
int orc_ppsod(const orc_prop_t* p, const double* vp, const double* vabc, const double* dm,
              int shape, const double* par, double* u1, double* v1, double* u2, double* v2,
              double* c_re, double* c_im, int c_cap);

/* PPSOD with its table and LNZVC rules (ppsod.f:64-400; no files): rows of
 * 7 + npr columns (T, ET, E0, Cr, Ci, |C|^2, |P_k|^2 for the npr real vectors
 * w[k*n..], FNT); C(0) and the start-up sample are stored only when printed,
 * as the reference does (with PRTCRL = NONE the first C slot is a placeholder) */
int orc_ppsod_table(const orc_prop_t* p, const double* vp, const double* vabc, const double* dm,
                    int shape, const double* par, int npr, const double* w, double* u1,
                    double* v1, double* u2, double* v2, double* c_re, double* c_im, int c_cap,
                    double* rows, int row_cap, int* nrows, int* info);
/* PPLNZ's propagation (pplnz.f:139-141, no printing): PLNZ's steps with the
 * potential VP - DM EF(T) at the time each step lands at */
int orc_pplnz(const orc_prop_t* p, const double* vp, const double* vabc, const double* dm,
              int shape, const double* par, double* u, double* v, double* c_re, double* c_im,
              int c_cap);
/* PPLNZ with its table (pplnz.f:76-320): rows of 6 + npr values, LNZVC's
 * C(t) rows and INFO; w holds the npr - 1 printed projection vectors */
int orc_pplnz_table(const orc_prop_t* p, const double* vp, const double* vabc, const double* dm,
                    int shape, const double* par, int npr, const double* w, double* u, double* v,
                    double* c_re, double* c_im, int c_cap, double* rows, int row_cap, int* nrows,
                    int* info);

/* symmetric tridiagonal eigensolver: d[n] diag, e[n-1] offdiag, z[n*n]
 * column-major eigenvectors, eigenvalues ascending in w.  0 on success. */
int orc_tridiag_eig(int n, const double* d, const double* e, double* w,
                    double* z);

/* Spectrum stage (espec.f:1545-1576, hwhm.f, spectrumtd.f, cfft.f)      */
void orc_total_correlation(int mf, const double* c_re, const double* c_im,
                           double* u, double* v);
void orc_hwhm(int mf, double dtf, double tf, double tal, double de,
              double* u, double* v);
void orc_fftnt(double* x, double* y, int n, int m, int itype, int quirks);
/* window + swap + FFTNT; writes energies (eV, without DE) into en[n]     */
int orc_spectrumtd(int window_sg, int mf, double dtf, double tf, double wp,
                   double de, double* u, double* v, double* en, int quirks);

/*
 * Batched 1D split-operator propagation (CPU baseline, host threads over
 * packets).  Packet k owns points [off[k], off[k+1]) of u, v, vpot.  Uses
 * the reference step of spofft.f (per-step trig included).  C(t) of every
 * step goes to c_re/c_im[k*(nsteps+1) + s].  Returns 0.
 */
int orc_spo_batch(int npk, const int* off, const double* sh, const double* sm,
                  const double* vpot, double* u, double* v, double dt_fs,
                  int nsteps, int quirks, double* c_re, double* c_im,
                  int nthreads);

/* Initial-state eigensolver (lanczsc.f LANCZSG with the true residual):
 * start [nstates][n], evecs [nstates][n]; returns 1 if a state did not
 * converge within maxrest restarts.  orc_ran / orc_lcg_start: rans.f LCG. */
double orc_ran(int* nseed);
void orc_lcg_start(int n, int nstates, double* out);
int orc_eig_lanczsg(int ndim, const int* np, const double* shm, const double* vpot,
                    int nstates, int m, double tol, int maxrest, const double* start,
                    double* evals, double* evecs, double* resid, int* matvecs);

/* potfuncs.f POT1D / POT2D / POT3D and gvpot.f GVPOT (CST(1..14) as cst[0..13]) */
double orc_pot1d(const char* potch, const double* cst, double rx);
double orc_pot2d(const char* potch, const double* sm, const double* cst, double rx, double ry);
double orc_pot3d(const char* potch, const double* cst, double rx, double ry, double rz);
void orc_gvpot(int shiftp, const char* potch, int ndim, const int* np, const double* xi,
               const double* sm, const double* sh, const double* cst, int quirk3d,
               double* vpot, double* xmin);

#ifdef __cplusplus
}
#endif
#endif
