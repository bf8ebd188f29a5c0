// diag1d.cuh -- per-packet energy and norm of a plan's current state (FP64).
#pragma once
#include "spo1d.cuh"

namespace espec {

struct DiagArgs {
  const double2* psi;   // x order, concatenated
  const double* vpot;   // hartree, x order
  const double* tc;     // kinetic table (DIGT) in FFT order per packet
  const int* kfreq;     // FFT index held at each final position of DefaultPlan<N>
  const SpoPacket* pk;  // off: first point; c_off: output slot
  double2* out;         // (E, norm) per packet
};

cudaError_t diag_launch(int n, const DiagArgs& a, int nblocks, cudaStream_t st);

}  // namespace espec
