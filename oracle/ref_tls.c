/*
 * ref_tls.c — compiles the reference's Snac/libSnac/src/Tetrahedra.c, where it
 * lies (its path comes from the Makefile as REF_TETRAHEDRA_C), with its
 * function-local statics made thread-local.
 *
 * TEST INFRASTRUCTURE ONLY: the multi-threaded checker _ref/libsnacref_mt.so.
 * Tetrahedra.c keeps every intermediate of Tetrahedra_Volume,
 * Tetrahedra_SurfaceArea and Tetrahedra_SurfaceNormal in function-local
 * statics (the file's header notes it is not thread-safe); with one copy per
 * thread the arithmetic, and so every result, is the serial build's.  The
 * system headers come first so that the keyword is redefined only for the
 * reference file itself.
 */
#include <assert.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define static static __thread
#include REF_TETRAHEDRA_C
#undef static
