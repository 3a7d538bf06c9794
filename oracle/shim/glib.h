/*
 * Minimal stand-in for the parts of GLib that the wbfmm reference sources
 * use, so that those sources compile unmodified into the test oracle
 * (oracle/_ref/libwbfmm_ref.so).  Test infrastructure only: nothing in the
 * wbfmm_b200 product links against this.
 *
 * Semantics kept from GLib where they matter for reproducibility:
 *  - g_qsort_with_data is a STABLE sort (GLib documents it as stable; the
 *    reference's point permutation t->ip depends on that);
 *  - g_error aborts, g_assert aborts when the condition is false.
 */
#ifndef WBFMM_ORACLE_GLIB_SHIM_H
#define WBFMM_ORACLE_GLIB_SHIM_H

#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <float.h>

typedef int gint;
typedef unsigned int guint;
typedef int gboolean;
typedef double gdouble;
typedef float gfloat;
typedef char gchar;
typedef size_t gsize;
typedef void *gpointer;
typedef const void *gconstpointer;
typedef uint32_t guint32;
typedef int32_t gint32;
typedef uint64_t guint64;
typedef int64_t gint64;

#ifndef TRUE
#define TRUE 1
#endif
#ifndef FALSE
#define FALSE 0
#endif

#ifndef MIN
#define MIN(a, b) (((a) < (b)) ? (a) : (b))
#endif
#ifndef MAX
#define MAX(a, b) (((a) > (b)) ? (a) : (b))
#endif
#ifndef ABS
#define ABS(a) (((a) < 0) ? -(a) : (a))
#endif

#define G_MAXFLOAT FLT_MAX
#define G_LOG_DOMAIN "WBFMM"

#define GINT_TO_POINTER(i) ((gpointer)(intptr_t)(i))
#define GPOINTER_TO_INT(p) ((gint)(intptr_t)(p))

typedef gint (*GCompareDataFunc)(gconstpointer a, gconstpointer b,
                                 gpointer user_data);
typedef gpointer (*GThreadFunc)(gpointer data);

typedef struct _GThread GThread;
typedef struct _GTimer GTimer;

typedef enum {
  G_LOG_FLAG_RECURSION = 1 << 0,
  G_LOG_FLAG_FATAL = 1 << 1,
  G_LOG_LEVEL_ERROR = 1 << 2,
  G_LOG_LEVEL_CRITICAL = 1 << 3,
  G_LOG_LEVEL_WARNING = 1 << 4,
  G_LOG_LEVEL_MESSAGE = 1 << 5,
  G_LOG_LEVEL_INFO = 1 << 6,
  G_LOG_LEVEL_DEBUG = 1 << 7
} GLogLevelFlags;
typedef void (*GLogFunc)(const gchar *log_domain, GLogLevelFlags log_level,
                         const gchar *message, gpointer user_data);

gpointer g_malloc(gsize n);
gpointer g_malloc0(gsize n);
void g_free(gpointer p);
gchar *g_strdup(const gchar *s);
gchar *g_path_get_basename(const gchar *s);
void g_qsort_with_data(gpointer pbase, gint total_elems, gsize size,
                       GCompareDataFunc compare_func, gpointer user_data);
guint g_get_num_processors(void);
GThread *g_thread_new(const gchar *name, GThreadFunc func, gpointer data);
gpointer g_thread_join(GThread *thread);
GTimer *g_timer_new(void);
void g_timer_start(GTimer *t);
gdouble g_timer_elapsed(GTimer *t, gsize *microseconds);
guint g_log_set_handler(const gchar *domain, GLogLevelFlags levels,
                        GLogFunc func, gpointer data);
void wbfmm_oracle_fatal(const char *file, int line, const char *fmt, ...);

#define g_error(...) wbfmm_oracle_fatal(__FILE__, __LINE__, __VA_ARGS__)
#define g_assert(expr)                                                    \
  do {                                                                    \
    if (!(expr))                                                          \
      wbfmm_oracle_fatal(__FILE__, __LINE__, "assertion failed: %s",      \
                         #expr);                                          \
  } while (0)
#define g_assert_not_reached()                                            \
  wbfmm_oracle_fatal(__FILE__, __LINE__, "code should not be reached")

#endif /* WBFMM_ORACLE_GLIB_SHIM_H */
