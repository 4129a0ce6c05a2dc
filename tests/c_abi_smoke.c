/* Plain C client of the C ABI (no torch): sizes a batched workspace, checks
 * argument validation and the per-view superblock layout.  Needs no GPU. */
#include <stdio.h>
#include <string.h>

#include "dsplat.h"

int main(void) {
  printf("%s\n", dsplat_version());
  dsplat_view views[2];
  memset(views, 0, sizeof(views));
  views[0].width = 1920;
  views[0].height = 1080;
  views[1].width = 320;
  views[1].height = 240;
  dsplat_batch_layout lay;
  int rc = dsplat_gauss_batch_layout(1 << 20, 2, views, 8, 0, 1u << 26, &lay);
  if (rc != DSPLAT_OK) {
    printf("layout failed: %s\n", dsplat_last_error());
    return 1;
  }
  printf("items %u pix %u sb %u sb_log2 %d %d bytes %zu\n", lay.num_items, lay.num_pix, lay.num_sb, lay.sb_log2[0],
         lay.sb_log2[1], lay.total_bytes);
  if (lay.num_items != 240u * 135u + 40u * 30u || lay.sb_log2[0] != 3 || lay.sb_log2[1] != 1) return 2;
  rc = dsplat_gauss_batch_layout(1 << 20, 2, views, 12, 0, 1u << 26, &lay);
  if (rc != DSPLAT_ERR_UNSUPPORTED) return 3;
  printf("rejected: %s\n", dsplat_last_error());
  if (dsplat_tile2idx_workspace_size(1000, 16, 16, 5000) <= dsplat_tile2idx_workspace_size(1000, 16, 16, 0)) return 4;
  return 0;
}
