/*
 * ref_patch.h -- forced include (gcc -include) used ONLY when compiling the
 * reference's serial solver sources, in place, into the test oracle
 * oracle/_ref/libfslref.so.  Test infrastructure, never linked by the product.
 *
 * It applies the first half of the two-line oracle patch without touching the
 * reference tree: the reference's src/type.h:1-6 is guarded by TYPE_H and
 * defines `typedef float real;`.  Defining the guard first with `real` as
 * double makes every reference translation unit compute in FP64.
 *
 * The second half (src/helpers.c:73, `malloc` -> zero-filled allocation) is
 * applied by compiling helpers.c with -Dmalloc=fsl_ref_zero_alloc; see
 * ref_shim.c.  With both halves the reference is deterministic: every read of
 * a never-written array element (src/turbulence.c:17-100 zero bands, the
 * ghost layers of mu_SGS and of the A_ij temporaries) reads 0.0.
 */
#ifndef TYPE_H
#define TYPE_H
typedef double real;
#endif
