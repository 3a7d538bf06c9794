/*
 * Implementations behind oracle/shim/glib.h and oracle/shim/blaswrap.h.
 * Test infrastructure only: links into oracle/_ref/libwbfmm_ref.so, never
 * into the wbfmm_b200 product library.
 */
#include <pthread.h>
#include <stdarg.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include "glib.h"
#include "blaswrap.h"

void wbfmm_oracle_fatal(const char *file, int line, const char *fmt, ...)
{
  va_list ap;
  fprintf(stderr, "wbfmm oracle fatal (%s:%d): ", file, line);
  va_start(ap, fmt);
  vfprintf(stderr, fmt, ap);
  va_end(ap);
  fprintf(stderr, "\n");
  abort();
}

gpointer g_malloc(gsize n)
{
  gpointer p = malloc(n ? n : 1);
  if (p == NULL) wbfmm_oracle_fatal(__FILE__, __LINE__, "out of memory");
  return p;
}

gpointer g_malloc0(gsize n)
{
  gpointer p = calloc(n ? n : 1, 1);
  if (p == NULL) wbfmm_oracle_fatal(__FILE__, __LINE__, "out of memory");
  return p;
}

void g_free(gpointer p) { free(p); }

gchar *g_strdup(const gchar *s)
{
  size_t n;
  gchar *d;
  if (s == NULL) return NULL;
  n = strlen(s) + 1;
  d = g_malloc(n);
  memcpy(d, s, n);
  return d;
}

gchar *g_path_get_basename(const gchar *s)
{
  const gchar *b = strrchr(s, '/');
  return g_strdup(b ? b + 1 : s);
}

/* top-down merge sort: stable, as GLib's g_qsort_with_data is */
static void merge_sort(char *a, char *tmp, size_t n, size_t size,
                       GCompareDataFunc cmp, gpointer data)
{
  size_t h, i, j, k;
  if (n < 2) return;
  h = n / 2;
  merge_sort(a, tmp, h, size, cmp, data);
  merge_sort(a + h * size, tmp, n - h, size, cmp, data);
  i = 0; j = h; k = 0;
  while (i < h && j < n) {
    if (cmp(a + j * size, a + i * size, data) < 0) {
      memcpy(tmp + k * size, a + j * size, size); j++;
    } else {
      memcpy(tmp + k * size, a + i * size, size); i++;
    }
    k++;
  }
  while (i < h) { memcpy(tmp + k * size, a + i * size, size); i++; k++; }
  while (j < n) { memcpy(tmp + k * size, a + j * size, size); j++; k++; }
  memcpy(a, tmp, n * size);
}

void g_qsort_with_data(gpointer pbase, gint total_elems, gsize size,
                       GCompareDataFunc compare_func, gpointer user_data)
{
  char *tmp;
  if (total_elems < 2) return;
  tmp = g_malloc((gsize)total_elems * size);
  merge_sort((char *)pbase, tmp, (size_t)total_elems, size, compare_func,
             user_data);
  free(tmp);
}

guint g_get_num_processors(void)
{
  long n = sysconf(_SC_NPROCESSORS_ONLN);
  return n > 0 ? (guint)n : 1;
}

struct _GThread {
  pthread_t th;
  GThreadFunc func;
  gpointer data;
  gpointer ret;
};

static void *thread_trampoline(void *p)
{
  GThread *t = p;
  t->ret = t->func(t->data);
  return NULL;
}

GThread *g_thread_new(const gchar *name, GThreadFunc func, gpointer data)
{
  GThread *t = g_malloc0(sizeof(GThread));
  (void)name;
  t->func = func;
  t->data = data;
  if (pthread_create(&t->th, NULL, thread_trampoline, t) != 0)
    wbfmm_oracle_fatal(__FILE__, __LINE__, "pthread_create failed");
  return t;
}

gpointer g_thread_join(GThread *t)
{
  gpointer r;
  pthread_join(t->th, NULL);
  r = t->ret;
  free(t);
  return r;
}

struct _GTimer {
  struct timespec t0;
};

GTimer *g_timer_new(void)
{
  GTimer *t = g_malloc0(sizeof(GTimer));
  clock_gettime(CLOCK_MONOTONIC, &t->t0);
  return t;
}

void g_timer_start(GTimer *t) { clock_gettime(CLOCK_MONOTONIC, &t->t0); }

gdouble g_timer_elapsed(GTimer *t, gsize *us)
{
  struct timespec t1;
  double s;
  clock_gettime(CLOCK_MONOTONIC, &t1);
  s = (double)(t1.tv_sec - t->t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t->t0.tv_nsec);
  if (us) *us = (gsize)(s * 1e6);
  return s;
}

guint g_log_set_handler(const gchar *domain, GLogLevelFlags levels,
                        GLogFunc func, gpointer data)
{
  (void)domain; (void)levels; (void)func; (void)data;
  return 1;
}

void blaswrap_daxpy(int n, double a, double *x, int incx, double *y, int incy)
{
  int i;
  for (i = 0; i < n; i++) y[i * incy] += a * x[i * incx];
}

void blaswrap_saxpy(int n, float a, float *x, int incx, float *y, int incy)
{
  int i;
  for (i = 0; i < n; i++) y[i * incy] += a * x[i * incx];
}

/* naive column-major complex GEMM, C = al*op(A)*op(B) + bt*C, "N","N" only */
void zgemm_(const char *ta, const char *tb, int *m, int *n, int *k,
            double *al, double *A, int *lda, double *B, int *ldb,
            double *bt, double *C, int *ldc)
{
  int i, j, l;
  if (ta[0] != 'N' || tb[0] != 'N')
    wbfmm_oracle_fatal(__FILE__, __LINE__, "zgemm_ shim supports N,N only");
  for (j = 0; j < *n; j++)
    for (i = 0; i < *m; i++) {
      double sr = 0.0, si = 0.0, cr, ci;
      for (l = 0; l < *k; l++) {
        double ar = A[2 * (i + l * *lda)], ai = A[2 * (i + l * *lda) + 1];
        double br = B[2 * (l + j * *ldb)], bi = B[2 * (l + j * *ldb) + 1];
        sr += ar * br - ai * bi;
        si += ar * bi + ai * br;
      }
      cr = C[2 * (i + j * *ldc)]; ci = C[2 * (i + j * *ldc) + 1];
      C[2 * (i + j * *ldc)] = al[0] * sr - al[1] * si + bt[0] * cr - bt[1] * ci;
      C[2 * (i + j * *ldc) + 1] = al[0] * si + al[1] * sr + bt[0] * ci + bt[1] * cr;
    }
}

void cgemm_(const char *ta, const char *tb, int *m, int *n, int *k,
            float *al, float *A, int *lda, float *B, int *ldb,
            float *bt, float *C, int *ldc)
{
  int i, j, l;
  if (ta[0] != 'N' || tb[0] != 'N')
    wbfmm_oracle_fatal(__FILE__, __LINE__, "cgemm_ shim supports N,N only");
  for (j = 0; j < *n; j++)
    for (i = 0; i < *m; i++) {
      float sr = 0.0f, si = 0.0f, cr, ci;
      for (l = 0; l < *k; l++) {
        float ar = A[2 * (i + l * *lda)], ai = A[2 * (i + l * *lda) + 1];
        float br = B[2 * (l + j * *ldb)], bi = B[2 * (l + j * *ldb) + 1];
        sr += ar * br - ai * bi;
        si += ar * bi + ai * br;
      }
      cr = C[2 * (i + j * *ldc)]; ci = C[2 * (i + j * *ldc) + 1];
      C[2 * (i + j * *ldc)] = al[0] * sr - al[1] * si + bt[0] * cr - bt[1] * ci;
      C[2 * (i + j * *ldc) + 1] = al[0] * si + al[1] * sr + bt[0] * ci + bt[1] * cr;
    }
}
