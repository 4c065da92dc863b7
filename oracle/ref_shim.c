/*
 * ref_shim.c -- zero-filling allocator for the reference oracle build.
 * Test infrastructure (linked only into oracle/_ref/libfslref.so).
 *
 * The reference's Array3D (src/helpers.c:58-80) allocates its rows with
 * malloc and never initialises them; src/turbulence.c:17-100 and
 * src/fluxes.c:191,360,531 then read elements that were never written.  The
 * oracle build compiles src/helpers.c with -Dmalloc=fsl_ref_zero_alloc so that
 * every such element reads 0.0 (the calloc convention), which makes the
 * reference deterministic.
 */
#include <stdlib.h>

void *fsl_ref_zero_alloc(size_t n)
{
    return calloc(1, n ? n : 1);
}
