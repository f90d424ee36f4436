/* gthread.c -- the GLib queue, mutex and thread calls that GSvit's
 * src3d/gpu.c makes (g_queue_*, g_mutex_new, g_thread_create), over
 * pthreads.  Test infrastructure only: linked into
 * oracle/_ref/libgsvit_refcuda.so, the build of GSvit's own CUDA path that
 * serves as a measured context baseline.
 *
 * gpu.c drives one worker thread per device through a queue: the caller
 * pushes a task and spins until the queue is empty (sv_pool_sync,
 * gpu.c:787-802); the worker spins on the queue, runs the task it finds at
 * the tail and pops it only when the task is done (gpu_main,
 * gpu.c:1792-1955).  Both sides poll g_queue_is_empty, so the element
 * count is published with release stores and read with acquire loads; the
 * rest of the queue is under a mutex. */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>

#include "glib.h"

struct _GQueue {
    pthread_mutex_t lock;
    gpointer *items;
    int len, cap;
};

struct _GMutex {
    pthread_mutex_t lock;
};

GQueue *g_queue_new(void)
{
    GQueue *q = (GQueue *)g_malloc0(sizeof(GQueue));
    pthread_mutex_init(&q->lock, NULL);
    q->cap = 16;
    q->items = (gpointer *)g_malloc(sizeof(gpointer) * q->cap);
    return q;
}

void g_queue_push_tail(GQueue *q, gpointer data)
{
    pthread_mutex_lock(&q->lock);
    if (q->len == q->cap) {
        q->cap *= 2;
        q->items = (gpointer *)g_realloc(q->items, sizeof(gpointer) * q->cap);
    }
    q->items[q->len] = data;
    __atomic_store_n(&q->len, q->len + 1, __ATOMIC_RELEASE);
    pthread_mutex_unlock(&q->lock);
}

gpointer g_queue_pop_tail(GQueue *q)
{
    gpointer d = NULL;
    pthread_mutex_lock(&q->lock);
    if (q->len > 0) {
        d = q->items[q->len - 1];
        __atomic_store_n(&q->len, q->len - 1, __ATOMIC_RELEASE);
    }
    pthread_mutex_unlock(&q->lock);
    return d;
}

gpointer g_queue_peek_tail(GQueue *q)
{
    gpointer d = NULL;
    pthread_mutex_lock(&q->lock);
    if (q->len > 0) d = q->items[q->len - 1];
    pthread_mutex_unlock(&q->lock);
    return d;
}

gboolean g_queue_is_empty(GQueue *q) { return __atomic_load_n(&q->len, __ATOMIC_ACQUIRE) == 0; }

GMutex *g_mutex_new(void)
{
    GMutex *m = (GMutex *)g_malloc0(sizeof(GMutex));
    pthread_mutex_init(&m->lock, NULL);
    return m;
}

/* the worker runs until the process exits (gpu_main has no exit task) */
GThread *g_thread_create(GThreadFunc func, gpointer data, gboolean joinable, GError **error)
{
    pthread_t t;
    pthread_attr_t attr;
    (void)joinable;
    pthread_attr_init(&attr);
    pthread_attr_setdetachstate(&attr, PTHREAD_CREATE_DETACHED);
    if (pthread_create(&t, &attr, func, data) != 0) {
        pthread_attr_destroy(&attr);
        if (error) {
            *error = (GError *)g_malloc0(sizeof(GError));
            (*error)->code = 1;
        }
        return NULL;
    }
    pthread_attr_destroy(&attr);
    return (GThread *)(uintptr_t)1;
}
