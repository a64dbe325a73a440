/* qmp.h -- the single-process QMP calls the reference's asqtad path makes
   (global sums, topology queries, error printing), for building it against
   qdp_shim (test infrastructure).  One process: sums are identities. */
#ifndef QMP_SHIM_H
#define QMP_SHIM_H
#include <stdarg.h>
#include <stdio.h>

typedef int QMP_status_t;
#define QMP_SUCCESS 0
#define QMP_GRID 0
#define QMP_SWITCH 1
static inline QMP_status_t QMP_sum_double(double *x) { (void)x; return QMP_SUCCESS; }
static inline QMP_status_t QMP_sum_int(int *x) { (void)x; return QMP_SUCCESS; }
static inline QMP_status_t QMP_sum_double_array(double *x, int n) { (void)x; (void)n; return QMP_SUCCESS; }
static inline QMP_status_t QMP_barrier(void) { return QMP_SUCCESS; }
static inline int QMP_logical_topology_is_declared(void) { return 0; }
static inline int QMP_get_logical_number_of_dimensions(void) { return 0; }
static inline const int *QMP_get_logical_dimensions(void) { return 0; }
static inline int QMP_get_number_of_nodes(void) { return 1; }
static inline int QMP_get_node_number(void) { return 0; }
static inline int QMP_get_msg_passing_type(void) { return QMP_SWITCH; }
static inline int QMP_error(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vfprintf(stderr, fmt, ap);
  va_end(ap);
  return 0;
}
#endif
