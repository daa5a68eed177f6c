/*
 * C entry points into rocHPL's own matgen / pivot / row-swap sources, built by
 * oracle/build_ref.sh into oracle/_ref/libhplref.so.
 *
 * Test infrastructure only: pins the oracle and the CUDA kernels against the
 * reference's own code for
 *   - the LCG matrix   (src/matgen/HPL_pdrandmat_device.cpp:84-201),
 *   - ipiv -> (src,dst) pairs (src/pgesv/HPL_pipid.cpp:19-164) and the permU
 *     unrolling of src/panel/HPL_pdpanel_swapids.cpp:22-44,
 *   - the single-process row swap kernel (src/pauxil/HPL_dlaswp00N_device.cpp).
 */
#include "hpl.hpp"

rocblas_handle handle = nullptr;

extern "C" {

/* Fill the M x N column-major device matrix dA (leading dimension lda) exactly
 * as HPL_pdrandmat does on a 1 x 1 grid. Returns a cudaError_t value. */
int ref_pdrandmat(int M, int N, int NB, double* dA, int lda, int iseed) {
  HPL_T_grid g{1, 1, 0, 0};
  HPL_pdrandmat(&g, M, N, NB, dA, lda, iseed);
  return (int)cudaDeviceSynchronize();
}

/* The local part of process (myrow, mycol) of an nprow x npcol grid, as
 * HPL_pdrandmat generates it (NB x NB block-cyclic, starting in process (0,0)):
 * LocP(M) rows and LocQ(N) columns into dA (leading dimension lda). */
int ref_pdrandmat_grid(int M, int N, int NB, double* dA, int lda, int iseed, int nprow,
                       int npcol, int myrow, int mycol) {
  HPL_T_grid g{nprow, npcol, myrow, mycol};
  HPL_pdrandmat(&g, M, N, NB, dA, lda, iseed);
  return (int)cudaDeviceSynchronize();
}

/* HPL_xjumpm: constants to jump JUMPM steps from IRANN. */
void ref_xjumpm(int jumpm, uint64_t mult, uint64_t iadd, uint64_t irann,
                uint64_t* iranm, uint64_t* iam, uint64_t* icm) {
  HPL_xjumpm(jumpm, mult, iadd, irann, *iranm, *iam, *icm);
}

/* HPL_pipid for a panel whose first global row is ia, with jb pivots ipiv[]
 * (global row indices).  IPID must hold 4*jb ints; *K receives its length. */
void ref_pipid(int ia, int jb, int* ipiv, int* K, int* IPID) {
  HPL_T_panel p;
  p.ipiv = ipiv;
  p.jb   = jb;
  p.ia   = ia;
  HPL_pipid(&p, K, IPID);
}

/* Unroll ipiv into the 2*jb permU map used by the single-process row swap,
 * following src/panel/HPL_pdpanel_swapids.cpp:22-44 on top of HPL_pipid. */
void ref_swapids(int ia, int jb, int* ipiv, int* permU) {
  int* ipid = (int*)malloc(sizeof(int) * 4 * (jb > 0 ? jb : 1));
  int  K    = 0;
  for(int i = 0; i < jb; i++) permU[i + jb] = -1;
  ref_pipid(ia, jb, ipiv, &K, ipid);
  for(int i = 0; i < K; i += 2) {
    int src = ipid[i] - ia;
    int dst = ipid[i + 1] - ia;
    if(dst < jb)
      permU[dst] = src;
    else
      permU[src + jb] = dst;
  }
  free(ipid);
}

/* HPL_dlaswp00N on the device: M pivot rows, N columns, permU (2*M ints) on
 * the device. Returns a cudaError_t value after synchronising. */
int ref_dlaswp00N(int M, int N, double* dA, int lda, const int* dpermU) {
  HPL_dlaswp00N(M, N, dA, lda, dpermU);
  return (int)cudaDeviceSynchronize();
}

}  // extern "C"
