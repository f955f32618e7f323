/* Test-oracle plumbing: the reference LYNX sources call the Fortran BLAS/LAPACK
 * names (dgemm_, dsyev_, ...).  The only LAPACK in this image is the OpenBLAS
 * that ships with SciPy, whose symbols carry a "scipy_" prefix.  These
 * forwarders give the reference sources the names they expect. */
#define FWD(ret, name, params, args) \
    extern ret scipy_##name params;  \
    ret name params { return scipy_##name args; }

typedef int I;
typedef double D;
typedef char C;

FWD(void, dgemm_, (const C* ta, const C* tb, const I* m, const I* n, const I* k, const D* al, const D* a, const I* lda, const D* b, const I* ldb, const D* be, D* c, const I* ldc), (ta, tb, m, n, k, al, a, lda, b, ldb, be, c, ldc))
FWD(void, zgemm_, (const C* ta, const C* tb, const I* m, const I* n, const I* k, const void* al, const void* a, const I* lda, const void* b, const I* ldb, const void* be, void* c, const I* ldc), (ta, tb, m, n, k, al, a, lda, b, ldb, be, c, ldc))
FWD(void, dsymm_, (const C* s, const C* u, const I* m, const I* n, const D* al, const D* a, const I* lda, const D* b, const I* ldb, const D* be, D* c, const I* ldc), (s, u, m, n, al, a, lda, b, ldb, be, c, ldc))
FWD(void, dtrsm_, (const C* s, const C* u, const C* t, const C* d, const I* m, const I* n, const D* al, const D* a, const I* lda, D* b, const I* ldb), (s, u, t, d, m, n, al, a, lda, b, ldb))
FWD(void, ztrsm_, (const C* s, const C* u, const C* t, const C* d, const I* m, const I* n, const void* al, const void* a, const I* lda, void* b, const I* ldb), (s, u, t, d, m, n, al, a, lda, b, ldb))
FWD(void, dpotrf_, (const C* u, const I* n, D* a, const I* lda, I* info), (u, n, a, lda, info))
FWD(void, zpotrf_, (const C* u, const I* n, void* a, const I* lda, I* info), (u, n, a, lda, info))
FWD(void, dsyev_, (const C* j, const C* u, const I* n, D* a, const I* lda, D* w, D* work, const I* lwork, I* info), (j, u, n, a, lda, w, work, lwork, info))
FWD(void, zheev_, (const C* j, const C* u, const I* n, void* a, const I* lda, D* w, void* work, const I* lwork, D* rwork, I* info), (j, u, n, a, lda, w, work, lwork, rwork, info))
FWD(void, dsterf_, (const I* n, D* d, D* e, I* info), (n, d, e, info))
FWD(void, dsyevd_, (const C* j, const C* u, const I* n, D* a, const I* lda, D* w, D* work, const I* lwork, I* iwork, const I* liwork, I* info), (j, u, n, a, lda, w, work, lwork, iwork, liwork, info))
FWD(void, dgesv_, (const I* n, const I* nrhs, D* a, const I* lda, I* ipiv, D* b, const I* ldb, I* info), (n, nrhs, a, lda, ipiv, b, ldb, info))
