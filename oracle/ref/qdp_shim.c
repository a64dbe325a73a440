/* qdp_shim.c -- lattice, subsets, shifts and precision conversions of the
   single-process QDP interface in qdp.h (test infrastructure for building
   the reference's asqtad path).  Sites are in QOP raw order: even sites
   first, index lex/2 within a parity, lex = ((x0 L1 + x1) L2 + x2) L3 + x3
   (lib/layout_user.c:237-258). */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>
#include "qdp.h"

int QDP_this_node = 0;
int QDP_shim_V = 0;
int (*QDP_shim_coords)[4] = 0;
static int g_L[4], g_inited = 0;
static struct QDP_Subset_s s_all, s_even, s_odd;
QDP_Subset QDP_all = &s_all, QDP_even = &s_even, QDP_odd = &s_odd;
QDP_Subset QDP_even_and_odd[2] = {&s_even, &s_odd};
QDP_Shift QDP_neighbor[4];
QDP_Layout *QOP_layout_user = 0;   /* the reference's layout object: this shim has one fixed layout */

int QDP_is_initialized(void) { return g_inited; }
int QDP_initialize(int *argc, char ***argv) { (void)argc; (void)argv; g_inited = 1; return 0; }
void QDP_abort(int status) { fprintf(stderr, "QDP_abort(%d)\n", status); exit(status); }
void QDP_set_default_layout(QDP_Layout *layout) { (void)layout; }
void QDP_set_block_size(int bs) { (void)bs; }
int QDP_profcontrol(int level) { (void)level; return 0; }
int QDP_verbose(int level) { (void)level; return 0; }
QDP_Lattice *QDP_get_default_lattice(void) { return 0; }
int QDP_ndim(void) { return 4; }
void QDP_latsize(int *ls) { memcpy(ls, g_L, sizeof g_L); }
int QDP_coord_size(int i) { return g_L[i]; }
int QDP_volume(void) { return QDP_shim_V; }
int QDP_sites_on_node_fn(void) { return QDP_shim_V; }
int QDP_subset_len(QDP_Subset s) { return s->len; }
int QDP_node_number(const int x[]) { (void)x; return 0; }

int QDP_index(const int x[]) {
  const int lex = ((x[0] * g_L[1] + x[1]) * g_L[2] + x[2]) * g_L[3] + x[3];
  return ((x[0] + x[1] + x[2] + x[3]) & 1) ? (lex + QDP_shim_V) / 2 : lex / 2;
}

void QDP_get_coords(int x[], int node, int index) {
  (void)node;
  memcpy(x, QDP_shim_coords[index], sizeof(int) * 4);
}

void QDP_set_latsize(int nd, int *size) {
  if (nd != 4) QDP_abort(1);
  memcpy(g_L, size, sizeof g_L);
}

QDP_Shift QDP_create_shift(int disp[]) {
  const int V = QDP_shim_V;
  QDP_Shift s = (QDP_Shift)calloc(1, sizeof(*s));
  memcpy(s->disp, disp, sizeof(s->disp));
  s->fwd = (int *)malloc(sizeof(int) * V);
  s->bck = (int *)malloc(sizeof(int) * V);
  for (int i = 0; i < V; i++) {
    int y[4], z[4];
    for (int mu = 0; mu < 4; mu++) {
      y[mu] = ((QDP_shim_coords[i][mu] + disp[mu]) % g_L[mu] + g_L[mu]) % g_L[mu];
      z[mu] = ((QDP_shim_coords[i][mu] - disp[mu]) % g_L[mu] + g_L[mu]) % g_L[mu];
    }
    s->fwd[i] = QDP_index(y);
    s->bck[i] = QDP_index(z);
  }
  return s;
}

void QDP_destroy_shift(QDP_Shift s) {
  if (!s) return;
  free(s->fwd);
  free(s->bck);
  free(s);
}

void QDP_create_layout(void) {
  const int V = g_L[0] * g_L[1] * g_L[2] * g_L[3];
  QDP_shim_V = V;
  free(QDP_shim_coords);
  QDP_shim_coords = (int (*)[4])malloc(sizeof(int[4]) * V);
  int x[4];
  for (x[0] = 0; x[0] < g_L[0]; x[0]++)
    for (x[1] = 0; x[1] < g_L[1]; x[1]++)
      for (x[2] = 0; x[2] < g_L[2]; x[2]++)
        for (x[3] = 0; x[3] < g_L[3]; x[3]++) memcpy(QDP_shim_coords[QDP_index(x)], x, sizeof x);
  s_all.start = 0; s_all.len = V;
  s_even.start = 0; s_even.len = V / 2;
  s_odd.start = V / 2; s_odd.len = V / 2;
  for (int mu = 0; mu < 4; mu++) {
    int d[4] = {0, 0, 0, 0};
    d[mu] = 1;
    QDP_destroy_shift(QDP_neighbor[mu]);
    QDP_neighbor[mu] = QDP_create_shift(d);
  }
}

void QDP_finalize(void) {
  for (int mu = 0; mu < 4; mu++) {
    QDP_destroy_shift(QDP_neighbor[mu]);
    QDP_neighbor[mu] = 0;
  }
  g_inited = 0;
}

double QDP_time(void) {
  struct timeval tv;
  gettimeofday(&tv, 0);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

QDP_Subset *QDP_create_subset_L(QDP_Lattice *lat, int (*func)(QDP_Lattice *, int x[], void *), void *args,
                                int argsize, int n) {
  (void)lat; (void)func; (void)args; (void)argsize; (void)n;
  fprintf(stderr, "qdp_shim: QDP_create_subset_L is not provided\n");
  QDP_abort(1);
  return 0;
}

/* conversions between precisions (rounding to float, widening to double) */
#define SHIM_CONV(NAME, TD, TS, N, FIELD)                                                 \
  void NAME(TD *d, TS *s, QDP_Subset sub) {                                              \
    for (int i = sub->start; i < sub->start + sub->len; i++)                             \
      for (int k = 0; k < N; k++) {                                                      \
        d->d[i].FIELD[k].real = s->d[i].FIELD[k].real;                                   \
        d->d[i].FIELD[k].imag = s->d[i].FIELD[k].imag;                                   \
      }                                                                                  \
  }
SHIM_CONV(QDP_FD_V_eq_V, QDP_F3_ColorVector, QDP_D3_ColorVector, 3, c)
SHIM_CONV(QDP_DF_V_eq_V, QDP_D3_ColorVector, QDP_F3_ColorVector, 3, c)

void QDP_FD_M_eq_M(QDP_F3_ColorMatrix *d, QDP_D3_ColorMatrix *s, QDP_Subset sub) {
  for (int i = sub->start; i < sub->start + sub->len; i++)
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) {
        d->d[i].e[a][b].real = s->d[i].e[a][b].real;
        d->d[i].e[a][b].imag = s->d[i].e[a][b].imag;
      }
}
void QDP_DF_M_eq_M(QDP_D3_ColorMatrix *d, QDP_F3_ColorMatrix *s, QDP_Subset sub) {
  for (int i = sub->start; i < sub->start + sub->len; i++)
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) {
        d->d[i].e[a][b].real = s->d[i].e[a][b].real;
        d->d[i].e[a][b].imag = s->d[i].e[a][b].imag;
      }
}
