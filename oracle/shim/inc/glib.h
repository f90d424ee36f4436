/* glib.h -- the handful of GLib types, macros and calls that GSvit's CPU
 * solver files (yee.c, boundary.c, source.c, 1dpool.c, dline.c, farfield.c,
 * [dfi]cube.c, pool.c) use, written for this oracle build.  Test
 * infrastructure only; GLib itself is not installed in this image. */
#ifndef SHIM_GLIB_H
#define SHIM_GLIB_H
#include <stdlib.h>
#include <stdio.h>
#include <string.h>
#include <stdint.h>
#include <math.h>

typedef int gint;
typedef unsigned int guint;
typedef int gboolean;
typedef char gchar;
typedef unsigned char guchar;
typedef float gfloat;
typedef double gdouble;
typedef void *gpointer;
typedef const void *gconstpointer;
typedef long glong;
typedef unsigned long gulong;
typedef short gshort;
typedef unsigned short gushort;
typedef size_t gsize;
typedef int32_t gint32;
typedef uint32_t guint32;
typedef int64_t gint64;
typedef uint64_t guint64;
typedef int8_t gint8;
typedef uint8_t guint8;
typedef int16_t gint16;
typedef uint16_t guint16;

#ifndef TRUE
#define TRUE 1
#endif
#ifndef FALSE
#define FALSE 0
#endif
#undef MAX
#undef MIN
#define MAX(a, b) (((a) > (b)) ? (a) : (b))
#define MIN(a, b) (((a) < (b)) ? (a) : (b))
#define CLAMP(x, lo, hi) (((x) > (hi)) ? (hi) : (((x) < (lo)) ? (lo) : (x)))
#define ABS(a) (((a) < 0) ? -(a) : (a))
#define G_PI 3.1415926535897932384626433832795028841971693993751
#define G_GNUC_UNUSED __attribute__((unused))

typedef struct _GArray { gchar *data; guint len; } GArray;
typedef struct _GString { gchar *str; gsize len; gsize allocated_len; } GString;

static inline gpointer g_malloc(gsize n) { void *p = malloc(n ? n : 1); if (!p) abort(); return p; }
static inline gpointer g_malloc0(gsize n) { void *p = calloc(1, n ? n : 1); if (!p) abort(); return p; }
static inline gpointer g_realloc(gpointer p, gsize n) { void *q = realloc(p, n ? n : 1); if (!q) abort(); return q; }
static inline void g_free(gpointer p) { free(p); }
static inline gchar *g_strdup(const gchar *s) { if (!s) return NULL; size_t n = strlen(s) + 1; gchar *d = (gchar *)g_malloc(n); memcpy(d, s, n); return d; }
#define g_snprintf snprintf
#define g_new(T, n) ((T *)g_malloc(sizeof(T) * (n)))
#define g_new0(T, n) ((T *)g_malloc0(sizeof(T) * (n)))

/* local/random sources only (outside the path driven here) */
typedef struct _GRand { unsigned long long s; } GRand;
/* opaque thread-queue types named by gpu.h (compiled with UCUDA for the drop-in build only) */
typedef struct _GQueue GQueue;
typedef struct _GMutex GMutex;
/* the task queue and worker thread of src3d/gpu.c (sv_gpu_new, gpu_main),
 * for the build of GSvit's own CUDA path; implemented over pthreads in
 * oracle/shim/gthread.c */
typedef struct _GThread GThread;
typedef struct _GError { int code; gchar *message; } GError;
typedef void *(*GThreadFunc)(void *);
#define GINT_TO_POINTER(i) ((gpointer)(intptr_t)(i))
#define GPOINTER_TO_INT(p) ((gint)(intptr_t)(p))
GQueue *g_queue_new(void);
void g_queue_push_tail(GQueue *q, gpointer data);
gpointer g_queue_pop_tail(GQueue *q);
gpointer g_queue_peek_tail(GQueue *q);
gboolean g_queue_is_empty(GQueue *q);
GMutex *g_mutex_new(void);
GThread *g_thread_create(GThreadFunc func, gpointer data, gboolean joinable, GError **error);
static inline GRand *g_rand_new(void) { GRand *r = (GRand *)g_malloc(sizeof(GRand)); r->s = 88172645463325252ULL; return r; }
static inline GRand *g_rand_new_with_seed(guint32 seed) { GRand *r = g_rand_new(); r->s ^= seed; return r; }
static inline void g_rand_set_seed(GRand *r, guint32 seed) { r->s = 88172645463325252ULL ^ seed; }
static inline void g_rand_free(GRand *r) { free(r); }
static inline gdouble g_rand_double_range(GRand *r, gdouble lo, gdouble hi)
{ r->s ^= r->s << 13; r->s ^= r->s >> 7; r->s ^= r->s << 17; return lo + (hi - lo) * ((r->s >> 11) * (1.0 / 9007199254740992.0)); }
static inline guint32 g_random_int(void) { return (guint32)rand(); }

static inline void g_object_unref(gpointer p) { (void)p; }
#endif
