/* A plain C99 host program against include/deltamic_b200.h and the shared library:
 * version, status strings, workspace queries and host-side argument checks (no
 * device call).  Prints "ok" and exits 0 when every check holds. */
#include <stdio.h>
#include <string.h>

#include "deltamic_b200.h"

#define CHECK(c)                                         \
  do {                                                   \
    if (!(c)) {                                          \
      fprintf(stderr, "failed: %s (line %d)\n", #c, __LINE__); \
      return 1;                                          \
    }                                                    \
  } while (0)

int main(void) {
  CHECK(dm_abi_version() == 2);
  CHECK(strcmp(dm_status_string(DM_OK), "ok") == 0);
  CHECK(dm_meshft_forward_workspace_size(10, 16, 100) > 0);
  CHECK(dm_meshft_backward_workspace_size(642, 1280, 24464) <
        dm_meshft_backward_workspace_size(10242, 20480, 14064));
  CHECK(dm_conv3d_s2_workspace_size(2, 16, 16, 16, 16, 32) > 0);
  CHECK(dm_conv3d_s2_workspace_size(2, 16, 16, 16, 16, 24) == 0);
  dm_box box;
  memset(&box, 0, sizeof(box));
  for (int d = 0; d < 3; ++d) {
    box.lo[d] = 0.0;
    box.hi[d] = 1.0;
    box.shape[d] = 8;
  }
  CHECK(dm_mask_workspace_size(100, 2, &box) > 256);
  /* null arguments are refused before any device work */
  CHECK(dm_meshft_forward(NULL, 3, NULL, 1, NULL, &box, NULL, 0, NULL, NULL, NULL, NULL, 0,
                          NULL) & DM_ERR_INVALID_ARG);
  CHECK(dm_conv3d_s2_device_error(NULL, NULL) == DM_ERR_INVALID_ARG);
  printf("ok\n");
  return 0;
}
