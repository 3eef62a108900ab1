// Declarations shared between the translation units of the nsrno_b200 library.
#pragma once

#include "nsr_common.cuh"

// FFT plans and digit-reversed symbol tables of one grid.
struct PrecTables {
  FftPlan px, pz;      // along x (rows) and z (columns)
  const float* s2x;    // sin^2(pi kx / nx) at digit-reversed x positions
  const float* s2z;    // sin^2(pi kz / nz) at digit-reversed z positions
};

inline size_t nsr_align(size_t b) { return (b + 255) & ~(size_t)255; }

int nsr_check_grid(const NsrGrid* g, bool need_fft);
int nsr_prec_setup(const NsrGrid* g, PrecTables* t, void* table_mem, cudaStream_t st);
size_t nsr_prec_table_bytes(const NsrGrid* g);
int nsr_cols_tc(const NsrGrid* g);
size_t nsr_cols_smem(const NsrGrid* g);
int nsr_rows_per_cta(const NsrGrid* g);

int nsr_check_learned(const NsrLearned* L, int n_systems, cudaStream_t st);
