/* Prints the sizes and a few field offsets of the structs of include/kks.h, so
 * that tests/test_abi.py can check the Python ctypes mirror against the C
 * compiler's layout. */
#include <stddef.h>
#include <stdio.h>

#include "kks.h"

int main(void) {
  printf("kks_params %zu %zu %zu %zu\n", sizeof(kks_params), offsetof(kks_params, n_sched),
         offsetof(kks_params, sched_time), offsetof(kks_params, table));
  printf("kks_record %zu %zu %zu\n", sizeof(kks_record), offsetof(kks_record, T), offsetof(kks_record, energy_s));
  printf("kks_step_row %zu\n", sizeof(kks_step_row));
  printf("kks_run_state %zu %zu %zu\n", sizeof(kks_run_state), offsetof(kks_run_state, t),
         offsetof(kks_run_state, error_dtime_s));
  printf("kks_gen_args %zu %zu %zu %zu\n", sizeof(kks_gen_args), offsetof(kks_gen_args, w),
         offsetof(kks_gen_args, rng_state), offsetof(kks_gen_args, pc_ratio));
  return 0;
}
