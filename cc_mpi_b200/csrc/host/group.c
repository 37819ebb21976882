/*
 * cc_group: the partition group standing in for an MPI communicator
 * (include/cc_comm.h).  A group has `parts` partitions, all owned by this
 * process.  Per-rank views let code written rank by rank (the reference's
 * exchange_plan.c calls) run as one host thread per rank; the threads meet
 * in the group through a generation-counting barrier and a table of
 * per-rank published pointers.
 */
#include <pthread.h>
#include <stdio.h>
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

int cc_group_barrier(cc_group *view)
{
    if (!view)
        return -1;
    cc_group *g = view->root;
    pthread_mutex_lock(&g->mu);
    unsigned long gen = g->gen;
    if (++g->arrived == g->parts) {
        g->arrived = 0;
        g->gen++;
        pthread_cond_broadcast(&g->cv);
    } else {
        while (gen == g->gen)
            pthread_cond_wait(&g->cv, &g->mu);
    }
    pthread_mutex_unlock(&g->mu);
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
