/*
 * Build shim: lets nvcc compile a few of rocHPL's own source files
 * (src/matgen/HPL_pdrandmat_device.cpp, src/matgen/HPL_xjumpm.cpp,
 *  src/pgesv/HPL_pipid.cpp, src/pauxil/HPL_dlaswp00N_device.cpp) unmodified
 * from the read-only reference tree, for a single process (P = Q = 1) on CUDA.
 *
 * It stands in for rocHPL's umbrella header include/hpl.hpp: the HIP, rocBLAS
 * and MPI headers are replaced by the CUDA runtime plus the handful of types,
 * macros and stubs those four files touch. The matgen constants and the
 * block-cyclic index macros still come from the reference's own headers
 * (include/hpl_pmatgen.hpp, include/hpl_pauxil.hpp), pulled in below with the
 * MPI/rocBLAS-dependent headers fenced off by their include guards.
 *
 * Test infrastructure only: the product never includes this file.
 */
#ifndef HPLB_REF_SHIM_HPL_HPP
#define HPLB_REF_SHIM_HPL_HPP

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>

/* Fence off the headers that need MPI, HIP or rocBLAS. */
#define HPL_PMISC_HPP
#define HPL_BLAS_HPP
#define HPL_AUXIL_HPP
#define HPL_GRID_H
#define HPL_GRID_HPP
#define HPL_PGESV_HPP
#define HPL_PTEST_HPP
#define HPL_PANEL_HPP
#define HPL_PFACT_HPP
#define HPL_COMM_HPP
#define HPL_PTIMER_HPP

typedef int MPI_Comm;
typedef int HPL_T_MACH;
typedef int HPL_T_NORM;

/* The single-process grid: only the fields HPL_grid_info reads. */
typedef struct HPL_S_grid {
  int nprow, npcol, myrow, mycol;
} HPL_T_grid;

static inline int HPL_grid_info(const HPL_T_grid* g, int* nprow, int* npcol,
                                int* myrow, int* mycol) {
  *nprow = g->nprow; *npcol = g->npcol; *myrow = g->myrow; *mycol = g->mycol;
  return 0;
}

/* The panel fields HPL_pipid reads (include/hpl_panel.hpp:31-73 has the full struct). */
typedef struct HPL_S_panel {
  int* ipiv;
  int  jb;
  int  ia;
} HPL_T_panel;

typedef struct HPL_S_test HPL_T_test;
typedef struct HPL_S_palg HPL_T_palg;
typedef struct HPL_S_pmat HPL_T_pmat;

/* HIP/rocBLAS spellings used by the device files, mapped onto CUDA. */
#define hipGetLastError cudaGetLastError
#define hipDeviceSynchronize cudaDeviceSynchronize
#define hipStream_t cudaStream_t
#define CHECK_HIP_ERROR(e)                                                    \
  do {                                                                        \
    cudaError_t e__ = (e);                                                    \
    if(e__ != cudaSuccess) {                                                  \
      fprintf(stderr, "ref shim: CUDA error %s\n", cudaGetErrorString(e__));  \
    }                                                                         \
  } while(0)
#define CHECK_ROCBLAS_ERROR(e) (e)
typedef void* rocblas_handle;
extern rocblas_handle handle;
static inline int rocblas_get_stream(rocblas_handle, cudaStream_t* s) {
  *s = 0;
  return 0;
}

#include "hpl_misc.hpp"
#include "hpl_pauxil.hpp"
#include "hpl_pmatgen.hpp"

void HPL_pipid(HPL_T_panel* PANEL, int* K, int* IPID);
void HPL_dlaswp00N(const int M, const int N, double* A, const int LDA, const int* IPIV);

#endif
