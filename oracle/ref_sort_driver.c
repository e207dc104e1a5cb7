/*
 * ref_sort_driver.c -- calls the reference's own local key sort
 * (treecode/sl_pepc/src/core/sort_radix.c, pepckeys_sort_radix) exactly as
 * slsort_keys does at one rank (treecode/sl_pepc/mpi_pepckeys.c:151-167):
 * elements = (key, 1-based index, work), radix parameters -1/-1/-1.
 *
 * TEST INFRASTRUCTURE ONLY: built by oracle/Makefile together with the
 * reference's sort sources into oracle/_ref/libslref.so, used to pin the
 * oracle's restated sort order.
 */
#include <stdint.h>
#include <stdlib.h>
#include "sl_pepckeys.h"

int ref_sort_keys(int64_t n, int64_t* keys, int64_t* idx0) {
  pepckeys_elements_t s;
  pepckeys_slindex_t* ix = (pepckeys_slindex_t*)malloc(sizeof(pepckeys_slindex_t) * (size_t)n);
  double* work = (double*)malloc(sizeof(double) * (size_t)n);
  if (!ix || !work) { free(ix); free(work); return -1; }
  for (int64_t i = 0; i < n; ++i) { ix[i] = (pepckeys_slindex_t)(i + 1); work[i] = 1.0; }
  pepckeys_elem_set_size(&s, n);
  pepckeys_elem_set_max_size(&s, n);
  pepckeys_elem_set_keys(&s, (pepckeys_slkey_t*)keys);
  pepckeys_elem_set_indices(&s, ix);
  pepckeys_elem_set_data(&s, work);
  pepckeys_sort_radix(&s, NULL, -1, -1, -1);
  for (int64_t i = 0; i < n; ++i) idx0[i] = (int64_t)ix[i] - 1;
  free(ix);
  free(work);
  return 0;
}
