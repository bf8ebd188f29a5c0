// sil.cuh -- grid propagators with the finite-difference Hamiltonian:
// second-order differences (.PSOD, psod.f/sod.f), and short-iterative-Lanczos
// propagation (eSPec's .PSIL/.PLNZ:
// plnz.f:71-151, sil.f:70-181, lnz.f:76-119, reort.f:65-80, au1d.f/au2di.f/
// au3d.f) on one 1D, 2D or 3D grid, FP64, as ONE cooperative persistent
// kernel.
//
// Per time step the real part u and the imaginary part v are propagated by
// two independent m-step Lanczos chains (run side by side, sharing every
// grid barrier):
//   vi = work/bt0 ; w = H vi - bt0 v_prev ; al = <vi,w> ;
//   work = w - al vi - sum_q <w - al vi, L_q> L_q   (classical Gram-Schmidt
//   against all stored vectors) ; bt = |work|
// with H the 4th-order finite-difference Hamiltonian.  The two dot-product
// rounds of an iteration are merged into one (<w - al vi, L_q> = <w,L_q> -
// al <vi,L_q>), and the residual's norm joins the next iteration's dot
// products: the residual is formed pointwise, H is applied to it
// unnormalised (H is linear) after a handshake with the neighbouring CTAs
// only, and the one reduction yields bt = |res| together with the next
// iteration's products, rescaled by 1/bt.  An iteration costs one grid
// barrier.  Each barrier is also the reduction: after it every CTA sums the
// per-CTA partials itself in one fixed order, so all CTAs hold the same
// (deterministic) totals.
//
// The Krylov exponential e^{-i cst T} of the m x m tridiagonal T is formed by
// every CTA (same inputs, same result) by Taylor series with scaling and
// squaring in FP64 -- the same matrix function the reference forms through
// the eigenvectors of T (DSTEVX) -- and the new state is the combination of
// the Lanczos vectors (the last one formed from the residual in that pass).
#pragma once
#include <cuda_runtime.h>

namespace espec {

constexpr int kSilMaxM = 16;      // Lanczos order limit
constexpr int kSilThreads = 256;  // threads per CTA
constexpr int kSilNQ = 96;        // partial sums per CTA and barrier (>= 2 (3 + 3 (m-1)))

struct SilArgs {
  int ndim, nx, ny, nz;
  long n;
  double shm[3];  // 1/(24 m_a h_a^2) per axis
  double sht30;   // 30 * (shm[0] + shm[1] + shm[2])
  double inv_nx, inv_ny;  // 1/nx, 1/ny: grid indices by multiplication
  int nstrips;  // PSOD on a 2D grid: column strips of kSilThreads (0: point ranges)
  const double* vpot;
  const double* mask;  // .SMOOTHW mask or null
  double* u;           // state (in / out)
  double* v;
  const double* u0;  // psi(0) for C(t)
  const double* v0;
  double* L;     // [2][m][n] Lanczos vectors of the u and v chains
  double* work;  // [2][n]
  double* wbuf;  // [2][n]
  double* part;  // [2][gridDim.x][kSilNQ]: partial sums, by barrier parity
  unsigned* bar;  // [0..1]: one 64-bit count of the grid barrier arrivals of the launch
  unsigned* nflag;  // [gridDim.x]: neighbour handshake epoch of each CTA (zeroed per launch)
  int* err;       // set when a barrier wait gave up
  long spin_limit;  // polls before a barrier wait gives up
  double2* c_out;  // C(t) of every step: slot s for step s (slot 0 only if write_c0)
  int m, nsteps, quirk, write_c0;
  double cst;  // dt in atomic units (SIL); 2 dt in atomic units (PSOD)
  // second-order differences with the same H (.PSOD, psod.f / sod.f): the
  // state one step before (u, v), the absorber (.VOPTIC potential or
  // .SMOOTHW mask) and its kind, the start-up switch and the restart-copy
  // defect of psod.f:136-141
  double* up;
  double* vp;
  const double* vabc;
  int kabs;  // 0 none, 1 .VOPTIC, 2 .SMOOTHW
  int start, copy_quirk;
  // a laser pulse (chpot.f): PSOD -- the potential of PSODAUX call j is
  // V - dm ef[j], calls counted from the start of the run (0, 1: the
  // start-up; step s >= 2: call s, .PPSOD); SIL -- the step landing at step
  // j uses V - dm ef[j] (.PPSIL); slot0 = the steps done before this launch
  const double* dm;
  const double* ef;
  long slot0;
};

}  // namespace espec
