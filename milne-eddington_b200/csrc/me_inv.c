/* me_inv.c -- the command-line inversion, in place of the reference's MEINV
 * (Src/ME_INV.c:64-295): reads the control file (default ./input), inverts
 * the sol_box of data_path on the GPU(s) and writes result_path (and
 * fit_path, and the Cache_inv checkpoint) as the reference does.
 *
 *   me_inv [control_file] [--gpus N] [--batch PIXELS]
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/me_b200.h"

int main(int argc, char **argv) {
  const char *ctl = "./input";
  me_run_options opt;
  me_run_options_default(&opt);
  for (int i = 1; i < argc; i++) {
    if (!strcmp(argv[i], "--gpus") && i + 1 < argc) {
      opt.ndevices = atoi(argv[++i]);
    } else if (!strcmp(argv[i], "--batch") && i + 1 < argc) {
      opt.batch_pixels = atol(argv[++i]);
    } else if (argv[i][0] == '-') {
      fprintf(stderr, "usage: %s [control_file] [--gpus N] [--batch PIXELS]\n", argv[0]);
      return 2;
    } else {
      ctl = argv[i];
    }
  }
  me_run_report rep;
  const int st = me_run(ctl, &opt, &rep);
  if (st != ME_OK) {
    fprintf(stderr, "me_inv: %s: %s\n", me_strerror(st), me_last_error());
    return 1;
  }
  printf("me_inv: %ld pixels in %ld chunks of %ld (%ld done before), %.3f s\n",
         rep.pixels_inverted, rep.chunks_done, rep.chunk_pixels, rep.chunks_skipped, rep.seconds);
  return 0;
}
