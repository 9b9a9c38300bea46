/* Fortran BLAS/LAPACK entry points for the reference build, forwarded to
 * the OpenBLAS that scipy bundles (LP64, symbols with the prefix given by
 * AFQMC_ORACLE_BLAS_PREFIX, library from AFQMC_ORACLE_BLAS), resolved on
 * first use.  The reference compiles against these names with
 * -DUSE_BLAS_LAPACK (common/lapackblasHao/blas_lapack_wrap.h); every argument
 * is a pointer, so each forwarder passes its arguments through unchanged.
 * Oracle reference build only (test infrastructure). */
#include <complex.h>
#include <dlfcn.h>
#include <stdio.h>
#include <stdlib.h>

static void *or_sym(const char *name)
{
    static void *lib = NULL;
    if (!lib) {
        const char *path = getenv("AFQMC_ORACLE_BLAS");
        if (!path) { fprintf(stderr, "reference build: AFQMC_ORACLE_BLAS is not set\n"); exit(1); }
        lib = dlopen(path, RTLD_NOW | RTLD_LOCAL);
        if (!lib) { fprintf(stderr, "reference build: cannot load %s\n", path); exit(1); }
    }
    const char *pre = getenv("AFQMC_ORACLE_BLAS_PREFIX");
    char full[128];
    snprintf(full, sizeof full, "%s%s", pre ? pre : "", name);
    void *f = dlsym(lib, full);
    if (!f) { fprintf(stderr, "reference build: no symbol %s\n", full); exit(1); }
    return f;
}

void cgemm_(void *a0, void *a1, void *a2, void *a3, void *a4, void *a5, void *a6, void *a7, void *a8, void *a9, void *a10, void *a11, void *a12)
{
    static void (*f)(void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *))or_sym("cgemm_");
    f(a0, a1, a2, a3, a4, a5, a6, a7, a8, a9, a10, a11, a12);
}

void dgemm_(void *a0, void *a1, void *a2, void *a3, void *a4, void *a5, void *a6, void *a7, void *a8, void *a9, void *a10, void *a11, void *a12)
{
    static void (*f)(void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *))or_sym("dgemm_");
    f(a0, a1, a2, a3, a4, a5, a6, a7, a8, a9, a10, a11, a12);
}

void sgemm_(void *a0, void *a1, void *a2, void *a3, void *a4, void *a5, void *a6, void *a7, void *a8, void *a9, void *a10, void *a11, void *a12)
{
    static void (*f)(void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *))or_sym("sgemm_");
    f(a0, a1, a2, a3, a4, a5, a6, a7, a8, a9, a10, a11, a12);
}

void zgemm_(void *a0, void *a1, void *a2, void *a3, void *a4, void *a5, void *a6, void *a7, void *a8, void *a9, void *a10, void *a11, void *a12)
{
    static void (*f)(void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *))or_sym("zgemm_");
    f(a0, a1, a2, a3, a4, a5, a6, a7, a8, a9, a10, a11, a12);
}

void zgemv_(void *a0, void *a1, void *a2, void *a3, void *a4, void *a5, void *a6, void *a7, void *a8, void *a9, void *a10)
{
    static void (*f)(void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *))or_sym("zgemv_");
    f(a0, a1, a2, a3, a4, a5, a6, a7, a8, a9, a10);
}

void dgemv_(void *a0, void *a1, void *a2, void *a3, void *a4, void *a5, void *a6, void *a7, void *a8, void *a9, void *a10)
{
    static void (*f)(void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *))or_sym("dgemv_");
    f(a0, a1, a2, a3, a4, a5, a6, a7, a8, a9, a10);
}

void zgetrf_(void *a0, void *a1, void *a2, void *a3, void *a4, void *a5)
{
    static void (*f)(void *, void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *, void *, void *))or_sym("zgetrf_");
    f(a0, a1, a2, a3, a4, a5);
}

void dgetrf_(void *a0, void *a1, void *a2, void *a3, void *a4, void *a5)
{
    static void (*f)(void *, void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *, void *, void *))or_sym("dgetrf_");
    f(a0, a1, a2, a3, a4, a5);
}

void zgetrs_(void *a0, void *a1, void *a2, void *a3, void *a4, void *a5, void *a6, void *a7, void *a8)
{
    static void (*f)(void *, void *, void *, void *, void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *, void *, void *, void *, void *, void *))or_sym("zgetrs_");
    f(a0, a1, a2, a3, a4, a5, a6, a7, a8);
}

void dgetrs_(void *a0, void *a1, void *a2, void *a3, void *a4, void *a5, void *a6, void *a7, void *a8)
{
    static void (*f)(void *, void *, void *, void *, void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *, void *, void *, void *, void *, void *))or_sym("dgetrs_");
    f(a0, a1, a2, a3, a4, a5, a6, a7, a8);
}

void zgetri_(void *a0, void *a1, void *a2, void *a3, void *a4, void *a5, void *a6)
{
    static void (*f)(void *, void *, void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *, void *, void *, void *))or_sym("zgetri_");
    f(a0, a1, a2, a3, a4, a5, a6);
}

void zgeqrf_(void *a0, void *a1, void *a2, void *a3, void *a4, void *a5, void *a6, void *a7)
{
    static void (*f)(void *, void *, void *, void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *, void *, void *, void *, void *))or_sym("zgeqrf_");
    f(a0, a1, a2, a3, a4, a5, a6, a7);
}

void zungqr_(void *a0, void *a1, void *a2, void *a3, void *a4, void *a5, void *a6, void *a7, void *a8)
{
    static void (*f)(void *, void *, void *, void *, void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *, void *, void *, void *, void *, void *))or_sym("zungqr_");
    f(a0, a1, a2, a3, a4, a5, a6, a7, a8);
}

void zheevd_(void *a0, void *a1, void *a2, void *a3, void *a4, void *a5, void *a6, void *a7, void *a8, void *a9, void *a10, void *a11, void *a12)
{
    static void (*f)(void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *))or_sym("zheevd_");
    f(a0, a1, a2, a3, a4, a5, a6, a7, a8, a9, a10, a11, a12);
}

void dsyevd_(void *a0, void *a1, void *a2, void *a3, void *a4, void *a5, void *a6, void *a7, void *a8, void *a9, void *a10)
{
    static void (*f)(void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *))or_sym("dsyevd_");
    f(a0, a1, a2, a3, a4, a5, a6, a7, a8, a9, a10);
}

void zgesvd_(void *a0, void *a1, void *a2, void *a3, void *a4, void *a5, void *a6, void *a7, void *a8, void *a9, void *a10, void *a11, void *a12, void *a13, void *a14)
{
    static void (*f)(void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *))or_sym("zgesvd_");
    f(a0, a1, a2, a3, a4, a5, a6, a7, a8, a9, a10, a11, a12, a13, a14);
}

void zgesdd_(void *a0, void *a1, void *a2, void *a3, void *a4, void *a5, void *a6, void *a7, void *a8, void *a9, void *a10, void *a11, void *a12, void *a13, void *a14)
{
    static void (*f)(void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *, void *))or_sym("zgesdd_");
    f(a0, a1, a2, a3, a4, a5, a6, a7, a8, a9, a10, a11, a12, a13, a14);
}

void dsteqr_(void *a0, void *a1, void *a2, void *a3, void *a4, void *a5, void *a6, void *a7)
{
    static void (*f)(void *, void *, void *, void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *, void *, void *, void *, void *))or_sym("dsteqr_");
    f(a0, a1, a2, a3, a4, a5, a6, a7);
}

void zlarnv_(void *a0, void *a1, void *a2, void *a3)
{
    static void (*f)(void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *))or_sym("zlarnv_");
    f(a0, a1, a2, a3);
}

void dlarnv_(void *a0, void *a1, void *a2, void *a3)
{
    static void (*f)(void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *))or_sym("dlarnv_");
    f(a0, a1, a2, a3);
}

void clarnv_(void *a0, void *a1, void *a2, void *a3)
{
    static void (*f)(void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *))or_sym("clarnv_");
    f(a0, a1, a2, a3);
}

void slarnv_(void *a0, void *a1, void *a2, void *a3)
{
    static void (*f)(void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *))or_sym("slarnv_");
    f(a0, a1, a2, a3);
}

void zaxpy_(void *a0, void *a1, void *a2, void *a3, void *a4, void *a5)
{
    static void (*f)(void *, void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *, void *, void *))or_sym("zaxpy_");
    f(a0, a1, a2, a3, a4, a5);
}

void zcopy_(void *a0, void *a1, void *a2, void *a3, void *a4)
{
    static void (*f)(void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *, void *))or_sym("zcopy_");
    f(a0, a1, a2, a3, a4);
}

void zscal_(void *a0, void *a1, void *a2, void *a3)
{
    static void (*f)(void *, void *, void *, void *) = NULL;
    if (!f) f = (void (*)(void *, void *, void *, void *))or_sym("zscal_");
    f(a0, a1, a2, a3);
}

double dznrm2_(void *a0, void *a1, void *a2)
{
    static double (*f)(void *, void *, void *) = NULL;
    if (!f) f = (double (*)(void *, void *, void *))or_sym("dznrm2_");
    return f(a0, a1, a2);
}

double _Complex zdotc_(void *a0, void *a1, void *a2, void *a3, void *a4)
{
    static double _Complex (*f)(void *, void *, void *, void *, void *) = NULL;
    if (!f) f = (double _Complex (*)(void *, void *, void *, void *, void *))or_sym("zdotc_");
    return f(a0, a1, a2, a3, a4);
}
