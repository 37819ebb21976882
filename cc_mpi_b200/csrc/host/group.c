/*
 * cc_group: the partition group standing in for an MPI communicator
 * (include/cc_comm.h).  A group has `parts` partitions, all owned by this
 * process.  Per-rank views let code written rank by rank (the reference's
 * exchange_plan.c calls) run as one host thread per rank; the threads meet
 * in the group through a generation-counting barrier and a table of
 * per-rank published pointers.
 */
#include <errno.h>
#include <pthread.h>
#include <stdio.h>
#include <time.h>
#include <stdlib.h>
#include <string.h>

#include "cc_comm.h"
#include "host_common.h"

struct cc_group {
    int parts;
    int rank;
    struct cc_group *root; /* the group itself, or the group a view belongs to */
    int verbose;
    int has_last;
    ccgpu_dist_stats last;
    pthread_mutex_t mu;
    pthread_cond_t cv;
    int arrived;
    unsigned long gen;
    void *slots[CCGPU_MAX_PARTS];
    struct cc_group **views;
    /* pairwise mailboxes of the neighbourhood exchanges: what each rank
     * posted, how many of its readers are still to read it, and per
     * (reader, sender) how many posts the reader has taken */
    const void *box_buf[CCGPU_MAX_PARTS];
    const int *box_off[CCGPU_MAX_PARTS];
    const int *box_cnt[CCGPU_MAX_PARTS];
    unsigned long box_gen[CCGPU_MAX_PARTS];
    int box_left[CCGPU_MAX_PARTS];
    unsigned long *box_taken; /* [parts * parts], reader-major */
};

static cc_group *group_new(int parts)
{
    cc_group *g = (cc_group *)calloc(1, sizeof(cc_group));
    if (!g)
        return NULL;
    g->parts = parts;
    g->rank = 0;
    g->root = g;
    g->verbose = 1;
    pthread_mutex_init(&g->mu, NULL);
    pthread_cond_init(&g->cv, NULL);
    return g;
}

cc_group *cc_group_create(int parts)
{
    if (parts < 1 || parts > CCGPU_MAX_PARTS)
        return NULL;
    return group_new(parts);
}

static void free_views(cc_group *g)
{
    if (!g->views)
        return;
    for (int r = 0; r < g->parts; ++r)
        free(g->views[r]);
    free(g->views);
    g->views = NULL;
}

void cc_group_free(cc_group *g)
{
    if (!g || g->root != g || g == cc_group_world())
        return;
    free_views(g);
    free(g->box_taken);
    pthread_mutex_destroy(&g->mu);
    pthread_cond_destroy(&g->cv);
    free(g);
}

int cc_group_size(const cc_group *g)
{
    return g ? g->root->parts : 1;
}

int cc_group_rank(const cc_group *g)
{
    return g ? g->rank : 0;
}

static pthread_mutex_t g_world_mu = PTHREAD_MUTEX_INITIALIZER;
static cc_group *g_world = NULL;

cc_group *cc_group_world(void)
{
    pthread_mutex_lock(&g_world_mu);
    if (!g_world) {
        int parts = 1;
        const char *env = getenv("CCB200_PARTITIONS");
        if (env && *env) {
            int p = atoi(env);
            if (p >= 1 && p <= CCGPU_MAX_PARTS)
                parts = p;
        }
        g_world = group_new(parts);
    }
    cc_group *w = g_world;
    pthread_mutex_unlock(&g_world_mu);
    return w;
}

int cc_group_set_world_size(int parts)
{
    if (parts < 1 || parts > CCGPU_MAX_PARTS)
        return -1;
    cc_group *w = cc_group_world();
    if (!w)
        return -1;
    pthread_mutex_lock(&w->mu);
    free_views(w);
    free(w->box_taken);
    w->box_taken = NULL;
    memset(w->box_gen, 0, sizeof(w->box_gen));
    memset(w->box_left, 0, sizeof(w->box_left));
    w->parts = parts;
    pthread_mutex_unlock(&w->mu);
    return 0;
}

cc_group *cc_group_view(cc_group *g, int rank)
{
    if (!g)
        return NULL;
    g = g->root;
    if (rank < 0 || rank >= g->parts)
        return NULL;
    pthread_mutex_lock(&g->mu);
    if (!g->views) {
        g->views = (cc_group **)calloc((size_t)g->parts, sizeof(cc_group *));
        for (int r = 0; g->views && r < g->parts; ++r) {
            cc_group *v = (cc_group *)calloc(1, sizeof(cc_group));
            if (!v)
                continue;
            v->parts = g->parts;
            v->rank = r;
            v->root = g;
            v->verbose = g->verbose;
            g->views[r] = v;
        }
    }
    cc_group *v = g->views ? g->views[rank] : NULL;
    pthread_mutex_unlock(&g->mu);
    return v;
}

/* Waits on the group's condition variable with a limit: a rank that never
 * arrives turns into an error instead of a hang.  Called with g->mu held;
 * returns 0, or -1 once the limit has passed. */
static int group_wait(cc_group *g, const struct timespec *until)
{
    int rc = pthread_cond_timedwait(&g->cv, &g->mu, until);
    return rc == ETIMEDOUT ? -1 : 0;
}

static void wait_limit(struct timespec *until)
{
    double secs = 600.0;
    const char *env = getenv("CCB200_GROUP_TIMEOUT_S");
    if (env && *env && atof(env) > 0)
        secs = atof(env);
    clock_gettime(CLOCK_REALTIME, until);
    until->tv_sec += (time_t)secs;
    until->tv_nsec += (long)((secs - (double)(time_t)secs) * 1e9);
    if (until->tv_nsec >= 1000000000L) {
        until->tv_sec++;
        until->tv_nsec -= 1000000000L;
    }
}

int cc_group_barrier(cc_group *view)
{
    if (!view)
        return -1;
    cc_group *g = view->root;
    struct timespec until;
    wait_limit(&until);
    int rc = 0;
    pthread_mutex_lock(&g->mu);
    unsigned long gen = g->gen;
    if (++g->arrived == g->parts) {
        g->arrived = 0;
        g->gen++;
        pthread_cond_broadcast(&g->cv);
    } else {
        while (gen == g->gen && rc == 0)
            rc = group_wait(g, &until);
        if (rc)
            g->arrived--; /* leave the barrier: the others see the count drop */
    }
    pthread_mutex_unlock(&g->mu);
    if (rc)
        return ccb200_set_error(CCGPU_ERR_TIMEOUT, "cc_group_barrier: rank %d waited past the "
                                "limit for the other ranks", view->rank);
    return 0;
}

int cc_group_post(cc_group *view, const void *buf, const int *off, const int *cnt, int readers)
{
    if (!view)
        return -1;
    cc_group *g = view->root;
    const int r = view->rank;
    struct timespec until;
    wait_limit(&until);
    int rc = 0;
    pthread_mutex_lock(&g->mu);
    while (g->box_left[r] > 0 && rc == 0) /* the previous post is still being read */
        rc = group_wait(g, &until);
    if (rc == 0) {
        g->box_buf[r] = buf;
        g->box_off[r] = off;
        g->box_cnt[r] = cnt;
        g->box_left[r] = readers;
        g->box_gen[r]++;
        pthread_cond_broadcast(&g->cv);
    }
    pthread_mutex_unlock(&g->mu);
    if (rc)
        return ccb200_set_error(CCGPU_ERR_TIMEOUT, "cc_group_post: rank %d's readers did not "
                                "take its previous exchange", r);
    return 0;
}

int cc_group_take(cc_group *view, int src, void (*copy)(void *arg, const void *buf, int off,
                                                        int cnt),
                  void *arg)
{
    if (!view || src < 0 || src >= view->root->parts)
        return -1;
    cc_group *g = view->root;
    const int r = view->rank;
    struct timespec until;
    wait_limit(&until);
    int rc = 0;
    pthread_mutex_lock(&g->mu);
    if (!g->box_taken)
        g->box_taken = (unsigned long *)calloc((size_t)g->parts * g->parts, sizeof(unsigned long));
    if (!g->box_taken) {
        pthread_mutex_unlock(&g->mu);
        return ccb200_set_error(CCGPU_ERR_OOM, "cc_group_take: out of memory");
    }
    unsigned long *taken = g->box_taken + (size_t)r * g->parts + src;
    while (g->box_gen[src] <= *taken && rc == 0) /* src has not posted the next one */
        rc = group_wait(g, &until);
    if (rc == 0) {
        copy(arg, g->box_buf[src], g->box_off[src][r], g->box_cnt[src][r]);
        (*taken)++;
        g->box_left[src]--;
        pthread_cond_broadcast(&g->cv);
    }
    pthread_mutex_unlock(&g->mu);
    if (rc)
        return ccb200_set_error(CCGPU_ERR_TIMEOUT, "cc_group_take: rank %d waited past the "
                                "limit for rank %d's exchange", r, src);
    return 0;
}

int cc_group_drain(cc_group *view)
{
    if (!view)
        return -1;
    cc_group *g = view->root;
    const int r = view->rank;
    struct timespec until;
    wait_limit(&until);
    int rc = 0;
    pthread_mutex_lock(&g->mu);
    while (g->box_left[r] > 0 && rc == 0)
        rc = group_wait(g, &until);
    pthread_mutex_unlock(&g->mu);
    if (rc)
        return ccb200_set_error(CCGPU_ERR_TIMEOUT, "cc_group_drain: rank %d's readers did not "
                                "take its exchange", r);
    return 0;
}

void **cc_group_slots(cc_group *view)
{
    return view ? view->root->slots : NULL;
}

void cc_group_set_verbose(cc_group *g, int verbose)
{
    if (g)
        g->root->verbose = verbose;
}

int cc_group_verbose(const cc_group *g)
{
    return g ? g->root->verbose : 1;
}

void cc_group_store_stats(cc_group *g, const ccgpu_dist_stats *s)
{
    if (!g || !s)
        return;
    g = g->root;
    pthread_mutex_lock(&g->mu);
    g->last = *s;
    g->has_last = 1;
    pthread_mutex_unlock(&g->mu);
}

int cc_group_last_stats(const cc_group *g, ccgpu_dist_stats *out)
{
    if (!g || !out)
        return -1;
    g = g->root;
    if (!g->has_last)
        return -1;
    *out = g->last;
    return 0;
}
