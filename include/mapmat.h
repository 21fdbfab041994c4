/*
 * Drop-in pointing-matrix API of midapack, B200 implementation.
 * Same names, signatures and struct layout as the reference
 * (algebra/include/mapmat/mapmat.h:25-114, built with W_MPI); the numerical
 * work runs on the GPU of the calling thread's current CUDA device.
 *
 * Device residency: MatInit compresses the indices on the GPU (the result is
 * written back to `indices` in place and to `lindices`, as the reference
 * does) and keeps a device copy of the pointing keyed by the Mat address.
 * MatVecProd / TrMatVecProd then move only their input and output vectors.
 * Changing the contents of `values` after MatInit requires MatSetValues (or
 * MatInit) again, which refreshes the device copy.
 */
#ifndef MDP_DROPIN_MAPMAT_H
#define MDP_DROPIN_MAPMAT_H

#include "mdp_mpi_compat.h"

#ifdef __cplusplus
extern "C" {
#endif

/* communication flags (mapmat.h:26-37); a single GPU needs no reduction, so all behave as NONE */
#define NONE        0
#define RING        1
#define BUTTERFLY   2
#define NONBLOCKING 3
#define NOEMPTY     4
#define ALLTOALLV   5
#define ALLREDUCE   6
#define BUTTERFLY_BLOCKING_1 7
#define BUTTERFLY_BLOCKING_2 8
#define NOEMPTYSTEPRING      9
#define SEQ 0
#define OMP 1
#define GPU 2

/* mapmat.h:46-69 (W_MPI layout) */
typedef struct {
    int      flag;
    int      m;
    int      nnz;
    int      trash_pix;
    int     *indices;
    double  *values;
    int     *id_last_pix;
    int     *ll;
    int      lcount;
    int     *lindices;
    MPI_Comm comm;
    int     *com_indices, com_count;
    int      steps;
    int     *nS, *nR;
    int    **R, **S;
} Mat;

/* mapmat.h:71-76 -> replaces mapmat.c:54-73 */
int  MatInit(Mat *A, int m, int nnz, int *indices, double *values, int flag, MPI_Comm comm);
/* mapmat.h:78 -> mapmat.c:83-87 */
void MatSetIndices(Mat *A, int m, int nnz, int *indices);
/* mapmat.h:80 -> mapmat.c:97-102 (also invalidates the device copy of values) */
void MatSetValues(Mat *A, int m, int nnz, double *values);
/* mapmat.h:82 -> mapmat.c:323-400 (frees lindices and the device copy) */
void MatFree(Mat *A);
/* mapmat.h:84 -> mapmat.c:496-521; any sflag gives the counting-sort result */
int  MatLocalShape(Mat *A, int sflag);
/* mapmat.h:88 -> mapmat.c:530-695; single GPU: records comm/flag, no scheme */
int  MatComShape(Mat *A, int flag, MPI_Comm comm);
/* mapmat.h:92 -> mapmat.c:704-729; y[m] = A x */
int  MatVecProd(Mat *A, double *x, double *y, int pflag);
/* mapmat.h:94 -> mapmat.c:819-859; x[lcount - nnz*trash_pix] = A^T y */
int  TrMatVecProd(Mat *A, double *y, double *x, int pflag);
/* mapmat.h:113 -> mapmat.c:1008-1141; single GPU: the reduction is the identity */
int  greedyreduce(Mat *A, double *x);

#ifdef __cplusplus
}
#endif
#endif
