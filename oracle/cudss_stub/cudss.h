/* Link-only stand-in for the cuDSS API, used to build the reference rdcu (its bdf.cu
 * calls cuDSS) in an image that has no cuDSS.  Only the names the reference uses are
 * declared, with signatures inferred from its call sites (reference bdf.cu:26-29,
 * 154-159, 341-368, 450-452, 487-489).  Every function returns
 * CUDSS_STATUS_NOT_SUPPORTED without touching the GPU, so the reference's BDF path
 * reports "CUDSS analysis failed" and stops, while its DP45 path is unaffected.
 * Test infrastructure only: used by oracle/build_ref.sh, never by librdcu. */
#ifndef RDCU_CUDSS_STUB_H
#define RDCU_CUDSS_STUB_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct cudss_stub_handle *cudssHandle_t;
typedef struct cudss_stub_matrix *cudssMatrix_t;
typedef struct cudss_stub_config *cudssConfig_t;
typedef struct cudss_stub_data *cudssData_t;
typedef enum { CUDSS_STATUS_SUCCESS = 0, CUDSS_STATUS_NOT_SUPPORTED = 7 } cudssStatus_t;
typedef enum {
  CUDSS_PHASE_ANALYSIS = 1, CUDSS_PHASE_FACTORIZATION = 2, CUDSS_PHASE_REFACTORIZATION = 4,
  CUDSS_PHASE_SOLVE = 8
} cudssPhase_t;
typedef enum { CUDSS_DATA_INFO = 0 } cudssDataParam_t;
typedef enum { CUDSS_R_32I = 10, CUDSS_R_64F = 1 } cudssStubType_t;
typedef enum { CUDSS_MTYPE_GENERAL = 0 } cudssMatrixType_t;
typedef enum { CUDSS_MVIEW_FULL = 0 } cudssMatrixViewType_t;
typedef enum { CUDSS_BASE_ZERO = 0 } cudssIndexBase_t;
typedef enum { CUDSS_LAYOUT_COL_MAJOR = 0 } cudssLayout_t;

cudssStatus_t cudssCreate(cudssHandle_t *h);
cudssStatus_t cudssDestroy(cudssHandle_t h);
cudssStatus_t cudssConfigCreate(cudssConfig_t *c);
cudssStatus_t cudssConfigDestroy(cudssConfig_t c);
cudssStatus_t cudssDataCreate(cudssHandle_t h, cudssData_t *d);
cudssStatus_t cudssDataDestroy(cudssHandle_t h, cudssData_t d);
cudssStatus_t cudssDataGet(cudssHandle_t h, cudssData_t d, cudssDataParam_t p, void *v, size_t sz,
                           size_t *written);
cudssStatus_t cudssMatrixCreateCsr(cudssMatrix_t *m, int64_t nrows, int64_t ncols, int64_t nnz,
                                   void *rowStart, void *rowEnd, void *colIndices, void *values,
                                   cudssStubType_t rowType, cudssStubType_t colType,
                                   cudssStubType_t valueType, cudssMatrixType_t mtype, cudssMatrixViewType_t mview,
                                   cudssIndexBase_t base);
cudssStatus_t cudssMatrixCreateDn(cudssMatrix_t *m, int64_t nrows, int64_t ncols, int64_t ld,
                                  void *values, cudssStubType_t valueType, cudssLayout_t layout);
cudssStatus_t cudssMatrixDestroy(cudssMatrix_t m);
cudssStatus_t cudssExecute(cudssHandle_t h, cudssPhase_t phase, cudssConfig_t c, cudssData_t d,
                           cudssMatrix_t A, cudssMatrix_t x, cudssMatrix_t b);
#ifdef __cplusplus
}
#endif
#endif
