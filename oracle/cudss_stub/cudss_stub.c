/* Link-only cuDSS stand-in (see cudss.h): every call reports "not supported". */
#include "cudss.h"
#define NS CUDSS_STATUS_NOT_SUPPORTED
cudssStatus_t cudssCreate(cudssHandle_t *h) { if (h) *h = 0; return NS; }
cudssStatus_t cudssDestroy(cudssHandle_t h) { (void)h; return NS; }
cudssStatus_t cudssConfigCreate(cudssConfig_t *c) { if (c) *c = 0; return NS; }
cudssStatus_t cudssConfigDestroy(cudssConfig_t c) { (void)c; return NS; }
cudssStatus_t cudssDataCreate(cudssHandle_t h, cudssData_t *d) { (void)h; if (d) *d = 0; return NS; }
cudssStatus_t cudssDataDestroy(cudssHandle_t h, cudssData_t d) { (void)h; (void)d; return NS; }
cudssStatus_t cudssDataGet(cudssHandle_t h, cudssData_t d, cudssDataParam_t p, void *v, size_t sz,
                           size_t *written) {
  (void)h; (void)d; (void)p;
  if (v && sz >= sizeof(int)) *(int *)v = -1;
  if (written) *written = sizeof(int);
  return NS;
}
cudssStatus_t cudssMatrixCreateCsr(cudssMatrix_t *m, int64_t nrows, int64_t ncols, int64_t nnz,
                                   void *rowStart, void *rowEnd, void *colIndices, void *values,
                                   cudssStubType_t rowType, cudssStubType_t colType,
                                   cudssStubType_t valueType, cudssMatrixType_t mtype, cudssMatrixViewType_t mview,
                                   cudssIndexBase_t base) {
  (void)nrows; (void)ncols; (void)nnz; (void)rowStart; (void)rowEnd; (void)colIndices;
  (void)values; (void)rowType; (void)colType; (void)valueType; (void)mtype; (void)mview; (void)base;
  if (m) *m = 0;
  return NS;
}
cudssStatus_t cudssMatrixCreateDn(cudssMatrix_t *m, int64_t nrows, int64_t ncols, int64_t ld,
                                  void *values, cudssStubType_t valueType, cudssLayout_t layout) {
  (void)nrows; (void)ncols; (void)ld; (void)values; (void)valueType; (void)layout;
  if (m) *m = 0;
  return NS;
}
cudssStatus_t cudssMatrixDestroy(cudssMatrix_t m) { (void)m; return NS; }
cudssStatus_t cudssExecute(cudssHandle_t h, cudssPhase_t phase, cudssConfig_t c, cudssData_t d,
                           cudssMatrix_t A, cudssMatrix_t x, cudssMatrix_t b) {
  (void)h; (void)phase; (void)c; (void)d; (void)A; (void)x; (void)b;
  return NS;
}
