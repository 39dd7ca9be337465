/*
 * ref_pad.c -- test infrastructure: heap padding for the reference build.
 *
 * The reference's HMIS first pass sizes its bucket array as
 * max_lam + max_row_s + 1 (C_amg1/src/rs_classical.c:410-424) while a point's
 * measure can grow to twice its initial value, so bucket_head[] is indexed
 * past its end on vessel networks (a heap overflow: undefined behaviour that
 * crashed the reference on 1M- and 2M-node inputs).  The reference sources
 * are compiled unchanged with malloc renamed to ref_padded_malloc, which
 * returns a block followed by a tail as long as the block plus 4 KiB, filled
 * with 0xFF bytes: an out-of-range bucket then reads as -1, the empty list
 * that the reference's initialisation loop gives every in-range bucket.
 * free() is unaffected (the block starts where malloc's block starts).
 */
#include <stdlib.h>
#include <string.h>

#undef malloc /* this file is built with the same -Dmalloc flag as the reference */

void* ref_padded_malloc(size_t n) {
  size_t pad = n + 4096;
  unsigned char* p = (unsigned char*)malloc(n + pad);
  if (p) memset(p + n, 0xff, pad);
  return p;
}
