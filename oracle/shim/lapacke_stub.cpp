// LAPACKE stubs for the oracle build of the reference library.  The sparse
// path never calls them; reaching one means the harness strayed into the
// dense array::Matrix code, so abort loudly.  Test infrastructure only.
#include <cstdio>
#include <cstdlib>
#include "mkl.h"

extern "C" {
lapack_int LAPACKE_dpotrf(int, char, lapack_int, double*, lapack_int)
{
    std::fprintf(stderr, "oracle shim: LAPACKE_dpotrf is not available\n");
    std::abort();
}
lapack_int LAPACKE_dpotri(int, char, lapack_int, double*, lapack_int)
{
    std::fprintf(stderr, "oracle shim: LAPACKE_dpotri is not available\n");
    std::abort();
}
lapack_int LAPACKE_dgetrf(int, lapack_int, lapack_int, double*, lapack_int, lapack_int*)
{
    std::fprintf(stderr, "oracle shim: LAPACKE_dgetrf is not available\n");
    std::abort();
}
}
