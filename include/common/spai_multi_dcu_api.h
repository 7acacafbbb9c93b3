/*
 * Drop-in replacement of the reference's algorithm API
 * (include/common/spai_multi_dcu_api.h:1-24 in SingkiWong/DCU), C++ linkage,
 * same signatures.  Implemented in dcu_b200/csrc/host_api.cpp on top of the C
 * ABI in dcu_spai.h; one B200 does the work of every "DCU unit".
 *
 * Contract differences from the reference, all deliberate:
 *   - Run*SPAI_MultiDCU_MPI upload CSC_A (host) themselves and return M in
 *     devCSC_M_global as a DEVICE CSC matrix (pattern of A, FP64 values,
 *     arrays cudaMalloc'ed and owned by the caller, free with cudaFree); the
 *     reference needed replicateMatrixA before and aggregateResults after.
 *   - They return the device time of the build in ms, or -1.0f on failure
 *     (the reference exits the process on any HIP error); the message is in
 *     lastErrorMultiDCU(ctx).
 *   - Columns outside [globalColStart, globalColEnd) of M are zero.
 */
#ifndef SPAI_MULTI_DCU_API_H
#define SPAI_MULTI_DCU_API_H

#include "common/dataType.h"

struct MultiDCU_Context;

/* src/spai_multi_dcu.cpp:1296-1350.  Returns NULL (instead of exiting) when
 * no CUDA device is present. */
MultiDCU_Context* initMultiDCU(int requestedDCUs = -1);

/* src/spai_multi_dcu.cpp:2335-2380 */
void cleanupMultiDCU(MultiDCU_Context *ctx);

/* static partition (balanced_columns), src/spai_multi_dcu.cpp:1867-1870 */
float RunStaticSPAI_MultiDCU_MPI(MultiDCU_Context *ctx, const CSC_Matrix *CSC_A,
                                 CSC_Matrix *devCSC_M_global,
                                 int globalColStart, int globalColEnd);

/* dynamic partition (balanced_nnz), src/spai_multi_dcu.cpp:1872-1875 */
float RunDynamicSPAI_MultiDCU_MPI(MultiDCU_Context *ctx, const CSC_Matrix *CSC_A,
                                  CSC_Matrix *devCSC_M_global,
                                  int globalColStart, int globalColEnd);

/* src/spai_multi_dcu.cpp:1878-1951 (non-static, not in the reference header):
 * CSC->CSR of A and M, b = 1, x0 = 1, BiCGSTAB with ||r||_2 < 1e-7 absolute,
 * MAX_ITER 10000.  Returns the reference's iteration counter (0 on invalid
 * arguments or a CUDA failure). */
int runBiCGSTABOnRank0(CSC_Matrix *devCSC_A_full, CSC_Matrix *devCSC_M_global);

/* runBiCGSTABOnRank0 that also reports the solve: device time in ms, whether
 * it converged (0/1), the tolerance and the iteration cap it ran with (each
 * output optional, NULL to skip).  Not in the reference: the command-line
 * driver prints these on its [SOLVER_REPORT] line, which is where the
 * experiment database takes the solver time from. */
int runBiCGSTABOnRank0Info(CSC_Matrix *devCSC_A_full, CSC_Matrix *devCSC_M_global,
                           double *solverMs, int *converged, double *tol, int *maxIters);

/* src/spai_multi_dcu.cpp:1486-1551: copies host A to the device.  Optional
 * here (Run* uploads A itself); kept for callers that follow the reference's
 * call order.  The device copy is reachable through deviceMatrixA(ctx). */
void replicateMatrixA(MultiDCU_Context *ctx, CSC_Matrix *CSC_A);

/* The device copy of A made by the last Run* / replicateMatrixA call (the
 * reference's ctx->devCSC_A[0]), for runBiCGSTABOnRank0. */
CSC_Matrix* deviceMatrixA(MultiDCU_Context *ctx);

/* Number of DCU units the context stands for (always 1: one GPU). */
int numDCUUnits(MultiDCU_Context *ctx);

/* Message of the last failure on this context ("" if none). */
const char* lastErrorMultiDCU(MultiDCU_Context *ctx);

/* The reference's report line (src/spai_multi_dcu.cpp:2572-2574), byte for byte. */
void printAlgoReport(const char *mode, int dcuUnits, const char *partition,
                     float preconditionerMs, int iterationCount);

#endif
