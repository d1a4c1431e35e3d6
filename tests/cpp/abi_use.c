/* Compiled as C and as C++ by tests/test_abi_compile.py: includes the public
 * header the way a host driver would, links against liblu_b200.so, and
 * calls the entry points that need no GPU. */
#include <stdio.h>
#include "lu_b200.h"

int main(void) {
  lu_config cfg;
  if (lu_config_default(&cfg, 2048, 128) != LU_OK) return 1;
  double b[4];
  if (lu_matgen_host(b, 4, 9934835, 0) != LU_OK) return 2;
  printf("n=%lld b=%d batch=%d layout=%d target=%g ws=%zu\n", (long long)cfg.n, (int)cfg.block_size,
         (int)cfg.pivot_batch, (int)cfg.layout, cfg.ir_target, lu_workspace_bytes(&cfg));
  printf("status(0)=%s status(-8)=%s\n", lu_status_string(LU_OK), lu_status_string(LU_ERR_UNSUPPORTED));
  printf("b0=%.17g\n", b[0]);
  /* an invalid layout is rejected before any device work */
  lu_handle h;
  cfg.layout = 7;
  printf("bad_layout=%d\n", lu_create(&cfg, &h));
  return 0;
}
