/* The C ABI from plain C (C99, -pedantic): the header compiles as C and the library links and
 * answers.  Without a GPU the context cannot be created (NOT_GPU_BUILD); the calls that need no
 * device (status numbering, argument checks, the .hdr header probe of a missing file) answer all
 * the same.  Exit status 0 when every check holds. */
#include <stdio.h>
#include <string.h>

#include "../../include/nova_b200.h"

int main(void) {
  int bad = 0;
  nova_b200_ctx *ctx = NULL;
  const nova_b200_status st = nova_b200_create(&ctx, 0);
  if (st == NOVA_B200_SUCCESS) {
    nova_b200_destroy(ctx);
  } else {
    bad += st != NOVA_B200_NOT_GPU_BUILD;
    bad += ctx != NULL;
  }
  bad += NOVA_B200_SUCCESS != 0 || NOVA_B200_RENDERER_EXCEPTION != 16; /* nova::ERROR_STATE values */
  bad += nova_b200_create(NULL, 0) == NOVA_B200_SUCCESS;               /* no place for the handle */
  {
    int32_t w = -1, h = -1;
    bad += nova_b200_hdr_info(NULL, "/nonexistent/missing.hdr", &w, &h) != NOVA_B200_INVALID_ARGUMENT;
    bad += w != -1 || h != -1;
  }
  printf("c abi caller: %d failed checks\n", bad);
  return bad ? 1 : 0;
}
