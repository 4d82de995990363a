/* A plain C host of the library: compiled against include/msg123_gpu.h and linked with
 * libmsg123gpu.so by tests/test_c_host.py.  It calls the entry points that need no GPU --
 * the restart reader, the argument checks of msg_gpu_create and the error string -- the way
 * a Fortran or C caller would, and prints what it got.  Usage: abi_host <restart file> <ncalc> */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "msg123_gpu.h"

int main(int argc, char **argv) {
  if (argc != 3) return 2;
  const int n = atoi(argv[2]);
  double *head = malloc(sizeof(double) * (size_t)n), t = -1.0;
  int rc = msg_gpu_read_restart(argv[1], n, 10.0, head, &t);
  double sum = 0.0;
  for (int i = 0; i < n && rc == MSG_OK; ++i) sum += head[i];
  printf("read_restart rc=%d time=%.1f sum=%.17g\n", rc, t, sum);
  rc = msg_gpu_read_restart(argv[1], n + 1, 10.0, head, &t);
  printf("read_restart(wrong n) rc=%d msg=%s\n", rc, msg_gpu_last_error());

  msg_grid_t g;
  msg_params_t p;
  memset(&g, 0, sizeof g);
  memset(&p, 0, sizeof p);
  g.nx = g.ny = g.nz = 2;
  p.len_scal = 1.0; p.ini_step = 1.0; p.maxout_iter = 5; p.maxinn_iter = 5; p.vg_form = 7;
  msg_ctx_t *ctx = NULL;
  rc = msg_gpu_create(&g, &p, &ctx);
  printf("create(vg_form=7) rc=%d ctx=%s msg=%s\n", rc, ctx ? "set" : "null", msg_gpu_last_error());
  p.vg_form = 0;
  rc = msg_gpu_create(&g, &p, &ctx);   /* grid arrays are NULL */
  printf("create(null arrays) rc=%d msg=%s\n", rc, msg_gpu_last_error());
  msg_gpu_destroy(NULL);
  free(head);
  return 0;
}
