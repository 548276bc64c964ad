/* Host-side checks of the XLA custom-call handler core (include/dmpc_xla.h), in C against the
 * shared library: operand lists, workspace size, and the validation that turns every malformed
 * operand list into an error before any CUDA call.  No device memory is touched: every call
 * here returns before its first CUDA call (the buffers are host placeholders). */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "dmpc_xla.h"

static int failures = 0;
#define CHECK(cond)                                                 \
  do {                                                              \
    if (!(cond)) {                                                  \
      fprintf(stderr, "%s:%d: check failed: %s\n", __FILE__, __LINE__, #cond); \
      ++failures;                                                   \
    }                                                               \
  } while (0)

static int count_names(const char* list, const char* section) {
  const char* s = strstr(list, section);
  if (!s) return -1;
  s += strlen(section);
  int n = 1;
  for (; *s && *s != ';'; ++s) n += (*s == ',');
  return n;
}

static char arena[1 << 16];
static dmpc_xla_buffer buf(size_t bytes) {
  dmpc_xla_buffer b;
  b.data = bytes ? (void*)arena : NULL;
  b.bytes = bytes;
  return b;
}

int main(void) {
  CHECK(count_names(dmpc_xla_fwd_operands(), "args: ") == DMPC_XLA_FWD_ARGS);
  CHECK(count_names(dmpc_xla_fwd_operands(), "rets: ") == DMPC_XLA_FWD_RETS);
  CHECK(count_names(dmpc_xla_adj_operands(), "args: ") == DMPC_XLA_ADJ_ARGS);
  CHECK(count_names(dmpc_xla_adj_operands(), "rets: ") == DMPC_XLA_ADJ_RETS);

  /* linear MPC, nx=6, nu=3, N=20, batch 4: model parameters A (36), B (18), b (6) */
  dmpc_xla_problem q = {DMPC_MODEL_LINEAR, 6, 3, 20, 4, DMPC_EULER, 0, 60};
  dmpc_solver_params p;
  dmpc_default_params(&p);
  const size_t B = 4, K = 21, nx = 6, nu = 3, P = 60, mi = (size_t)p.num_scp_iteration_max;
  const size_t ws = dmpc_xla_workspace_size(&q, &p);
  CHECK(ws > 256);

  dmpc_xla_buffer a[DMPC_XLA_FWD_ARGS], r[DMPC_XLA_FWD_RETS];
  a[0] = buf(B * 8);
  a[1] = buf(B * nx * 8);
  a[2] = buf(B * nx * 8);
  a[3] = buf(B * K * nx * 8);
  a[4] = buf(B * K * nu * 8);
  a[5] = buf(B * nx * 8);
  a[6] = buf(B * nu * 8);
  a[7] = buf(B * nx * 8);
  a[8] = buf(B * P * 8);
  a[9] = buf(0);
  a[10] = buf(B * K * nx * 8);
  a[11] = buf(B * K * nu * 8);
  a[12] = buf(B * K * nx * 8);
  r[0] = buf(B * K * nx * 8);
  r[1] = buf(B * K * nu * 8);
  r[2] = buf(B * K * nx * 8);
  r[3] = buf(B * 8);
  r[4] = buf(B * 4);
  r[5] = buf(B * 4);
  r[6] = buf(B * mi * 8);
  r[7] = buf(B * mi * 8);
  r[8] = buf(B * mi * 4);
  r[9] = buf(B * K * nx * 8);
  r[10] = buf(B * K * nu * 8);
  r[11] = buf(64); /* far below ws: refused before any CUDA call */

  CHECK(dmpc_xla_solve_fwd(&q, &p, a, DMPC_XLA_FWD_ARGS, r, DMPC_XLA_FWD_RETS, NULL) == DMPC_ERR_WORKSPACE);
  CHECK(dmpc_xla_solve_fwd(&q, &p, a, DMPC_XLA_FWD_ARGS - 1, r, DMPC_XLA_FWD_RETS, NULL) == DMPC_ERR_INVALID);
  CHECK(dmpc_xla_solve_fwd(&q, &p, a, DMPC_XLA_FWD_ARGS, r, DMPC_XLA_FWD_RETS - 1, NULL) == DMPC_ERR_INVALID);
  /* each wrong-sized operand is refused */
  for (int i = 0; i < DMPC_XLA_FWD_ARGS; ++i) {
    const dmpc_xla_buffer keep = a[i];
    a[i].bytes += 8;
    if (!a[i].data) a[i].data = arena;
    CHECK(dmpc_xla_solve_fwd(&q, &p, a, DMPC_XLA_FWD_ARGS, r, DMPC_XLA_FWD_RETS, NULL) == DMPC_ERR_INVALID);
    a[i] = keep;
  }
  for (int i = 0; i < DMPC_XLA_FWD_RETS - 1; ++i) {
    const dmpc_xla_buffer keep = r[i];
    r[i].bytes -= 4;
    CHECK(dmpc_xla_solve_fwd(&q, &p, a, DMPC_XLA_FWD_ARGS, r, DMPC_XLA_FWD_RETS, NULL) == DMPC_ERR_INVALID);
    r[i] = keep;
  }
  /* a required buffer with a null pointer; ragged horizons of the right size pass validation */
  a[1].data = NULL;
  CHECK(dmpc_xla_solve_fwd(&q, &p, a, DMPC_XLA_FWD_ARGS, r, DMPC_XLA_FWD_RETS, NULL) == DMPC_ERR_INVALID);
  a[1].data = arena;
  a[9] = buf(B * 4);
  CHECK(dmpc_xla_solve_fwd(&q, &p, a, DMPC_XLA_FWD_ARGS, r, DMPC_XLA_FWD_RETS, NULL) == DMPC_ERR_WORKSPACE);
  a[9] = buf(0);
  /* an unsupported problem: the model's parameter count is wrong */
  dmpc_xla_problem bad = q;
  bad.n_model_params = 59;
  a[8] = buf(B * 59 * 8);
  CHECK(dmpc_xla_solve_fwd(&bad, &p, a, DMPC_XLA_FWD_ARGS, r, DMPC_XLA_FWD_RETS, NULL) == DMPC_ERR_INVALID);
  CHECK(dmpc_xla_workspace_size(&bad, &p) == 0);
  a[8] = buf(B * P * 8);
  /* an empty batch does nothing and succeeds */
  {
    dmpc_xla_problem e = q;
    e.batch = 0;
    dmpc_xla_buffer z[DMPC_XLA_FWD_RETS > DMPC_XLA_FWD_ARGS ? DMPC_XLA_FWD_RETS : DMPC_XLA_FWD_ARGS];
    for (int i = 0; i < (int)(sizeof(z) / sizeof(z[0])); ++i) z[i] = buf(0);
    CHECK(dmpc_xla_solve_fwd(&e, &p, z, DMPC_XLA_FWD_ARGS, z, DMPC_XLA_FWD_RETS, NULL) == DMPC_OK);
  }

  /* adjoint */
  dmpc_xla_buffer aa[DMPC_XLA_ADJ_ARGS], ra[DMPC_XLA_ADJ_RETS];
  for (int i = 0; i < 10; ++i) aa[i] = a[i];
  aa[10] = buf(B * K * nx * 8);
  aa[11] = buf(B * K * nu * 8);
  aa[12] = buf(B * K * nx * 8);
  aa[13] = buf(B * K * nx * 8);
  aa[14] = buf(B * K * nu * 8);
  aa[15] = buf(B * K * nx * 8);
  aa[16] = buf(B * K * nu * 8);
  aa[17] = buf(0);
  ra[0] = buf(B * K * nx * 8);
  for (int i = 1; i < DMPC_XLA_ADJ_RETS; ++i) ra[i] = buf(0);
  ra[3] = buf(B * nx * 8); /* g_w_x only */
  ra[10] = buf(64);
  const int32_t idx[2] = {36, 37};
  CHECK(dmpc_xla_solve_adj(&q, &p, NULL, 0, aa, DMPC_XLA_ADJ_ARGS, ra, DMPC_XLA_ADJ_RETS, NULL) == DMPC_ERR_WORKSPACE);
  /* model-parameter gradients asked for without their result buffer, or with a wrong one */
  CHECK(dmpc_xla_solve_adj(&q, &p, idx, 2, aa, DMPC_XLA_ADJ_ARGS, ra, DMPC_XLA_ADJ_RETS, NULL) == DMPC_ERR_INVALID);
  ra[8] = buf(B * 3 * 8);
  CHECK(dmpc_xla_solve_adj(&q, &p, idx, 2, aa, DMPC_XLA_ADJ_ARGS, ra, DMPC_XLA_ADJ_RETS, NULL) == DMPC_ERR_INVALID);
  ra[8] = buf(B * 2 * 8);
  CHECK(dmpc_xla_solve_adj(&q, &p, idx, 2, aa, DMPC_XLA_ADJ_ARGS, ra, DMPC_XLA_ADJ_RETS, NULL) == DMPC_ERR_WORKSPACE);
  CHECK(dmpc_xla_solve_adj(&q, &p, NULL, 2, aa, DMPC_XLA_ADJ_ARGS, ra, DMPC_XLA_ADJ_RETS, NULL) == DMPC_ERR_INVALID);
  aa[17] = buf(B * K * nx * 8 - 8);
  CHECK(dmpc_xla_solve_adj(&q, &p, idx, 2, aa, DMPC_XLA_ADJ_ARGS, ra, DMPC_XLA_ADJ_RETS, NULL) == DMPC_ERR_INVALID);
  aa[17] = buf(0);
  CHECK(dmpc_xla_solve_adj(&q, &p, idx, 2, aa, DMPC_XLA_ADJ_ARGS - 1, ra, DMPC_XLA_ADJ_RETS, NULL) == DMPC_ERR_INVALID);

  if (failures) {
    fprintf(stderr, "%d check(s) failed\n", failures);
    return 1;
  }
  printf("ok\n");
  return 0;
}
