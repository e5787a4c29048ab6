/* Links a plain C program against libmbd_b200.so through include/mbd_b200.h
 * and calls the entry points that need no GPU: a Fortran or C host binds the
 * same declarations.  Prints one line per check; exit status 0 when all pass. */
#include <math.h>
#include <stdio.h>
#include <string.h>

#include "mbd_b200.h"

int main(void) {
  int bad = 0;
  if (mbd_rsscs_element_z("C") != 6 || mbd_rsscs_element_z("H") != 1 || mbd_rsscs_element_z("Xx") != 0) {
    puts("element_z: FAIL");
    bad = 1;
  }
  double w[MBD_N_FREQ], wt[MBD_N_FREQ];
  if (mbd_rsscs_frequency_grid(w, wt, MBD_N_FREQ) != MBD_OK || w[0] != 0.0 || !(w[1] > 0.0) || wt[0] != 0.0) {
    puts("frequency_grid: FAIL");
    bad = 1;
  }
  if (mbd_rsscs_frequency_grid(w, NULL, MBD_N_FREQ - 1) != MBD_ERR_ARG) {
    puts("frequency_grid size check: FAIL");
    bad = 1;
  }
  double a0, c6, r0;
  if (mbd_rsscs_vdw_params(6, &a0, &c6, &r0) != MBD_OK || !(a0 > 0.0 && c6 > 0.0 && r0 > 0.0) ||
      mbd_rsscs_vdw_params(0, &a0, &c6, &r0) != MBD_ERR_UNKNOWN_ELEMENT) {
    puts("vdw_params: FAIL");
    bad = 1;
  }
  const char* msg = mbd_rsscs_strerror(MBD_ERR_TIMEOUT);
  if (!msg || strlen(msg) == 0) {
    puts("strerror: FAIL");
    bad = 1;
  }
  double v = 0.0;
  if (mbd_rsscs_set_option(NULL, MBD_OPT_RESIDUAL_GATE, 0.0) != MBD_ERR_ARG ||
      mbd_rsscs_get_option(NULL, MBD_OPT_WAIT_LIMIT_S, &v) != MBD_ERR_ARG) {
    puts("options without a context: FAIL");
    bad = 1;
  }
  /* without a GPU the context cannot be created; with one it must be */
  mbd_ctx* ctx = NULL;
  const int st = mbd_rsscs_create(&ctx, 0);
  if (st == MBD_OK) {
    mbd_rsscs_destroy(ctx);
  } else if (st != MBD_ERR_DEVICE) {
    printf("create: unexpected status %d\n", st);
    bad = 1;
  }
  printf("abi_check %s\n", bad ? "FAIL" : "ok");
  return bad;
}
