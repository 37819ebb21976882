/*
 * CPU oracle for the connected-components hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: it is loaded by the
 * tests, by __graft_entry__.smoke() and by the cpu_baseline leg of bench.py,
 * and by nothing else.  The product (libccb200.so) never links or calls it.
 *
 * It restates, in plain single-threaded C, the algorithm of the CC_mpi
 * reference (paths are relative to the reference project):
 *
 *   - src/cc_pthreads.c:32-73,89-147,152-229   label propagation (orc_lp_labels)
 *   - src/graph_dist.c:22-51                    block vertex ranges
 *   - src/graph_dist.c:53-92                    edge+vertex weighted bounds
 *   - src/cc_mpi.c:41-76                        owner_of_vertex
 *   - src/boundary_sort.c:5-119                 boundary pair sort + dedup
 *   - src/cc_mpi.c:221-763                      distributed merge (orc_dist_cc)
 *   - src/exchange_plan.c:48-225,242-425        exchange plan + delta exchange
 *   - src/cc_mpi.c:765-792                      count_connected_components
 *
 * plus an independent union-find labelling (orc_uf_labels) that does not
 * follow the reference at all and serves as a second route to the same
 * labels (each label is the minimum vertex id of its component).
 *
 * Parity is pinned by running the reference's own cc_pthreads.c and
 * boundary_sort.c, compiled unmodified from the reference sources into
 * oracle/_ref/, over the fixtures in tests/golden/ (see
 * tests/golden/make_golden.py).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------ */
/* Union-find labelling: root of each tree is the minimum id.          */
/* ------------------------------------------------------------------ */

static uint32_t uf_find(uint32_t *p, uint32_t x)
{
    while (p[x] != x) {
        p[x] = p[p[x]]; /* path halving */
        x = p[x];
    }
    return x;
}

static void uf_union(uint32_t *p, uint32_t a, uint32_t b)
{
    uint32_t ra = uf_find(p, a), rb = uf_find(p, b);
    if (ra == rb)
        return;
    if (ra < rb)
        p[rb] = ra;
    else
        p[ra] = rb;
}

/* labels[v] = min vertex id of v's component.  Neighbour ids >= n are
 * ignored (the reference's merge path ignores them too, src/cc_mpi.c:269). */
ORC_EXPORT void orc_uf_labels(uint32_t n, const uint64_t *row_ptr,
                              const uint32_t *col, uint32_t *labels)
{
    for (uint32_t v = 0; v < n; ++v)
        labels[v] = v;
    for (uint32_t v = 0; v < n; ++v)
        for (uint64_t j = row_ptr[v]; j < row_ptr[v + 1]; ++j) {
            uint32_t u = col[j];
            if (u < n)
                uf_union(labels, v, u);
        }
    for (uint32_t v = 0; v < n; ++v)
        labels[v] = uf_find(labels, v);
}

/* ------------------------------------------------------------------ */
/* Label propagation as the reference runs it, one thread.             */
/* src/cc_pthreads.c:32-73 relax; :89-147 round loop; :169-170 init.   */
/* Returns the number of rounds (the last one changes nothing).        */
/* ------------------------------------------------------------------ */

ORC_EXPORT int orc_lp_labels(uint32_t n, const uint64_t *row_ptr,
                             const uint32_t *col, uint32_t *labels)
{
    for (uint32_t v = 0; v < n; ++v)
        labels[v] = v;
    int rounds = 0;
    for (;;) {
        int any = 0;
        rounds++;
        for (uint32_t u = 0; u < n; ++u) {
            uint32_t cur = labels[u], best = cur;
            for (uint64_t j = row_ptr[u]; j < row_ptr[u + 1]; ++j) {
                uint32_t w = labels[col[j]];
                if (w < best)
                    best = w;
            }
            if (best < cur) {
                labels[u] = best;
                for (uint64_t j = row_ptr[u]; j < row_ptr[u + 1]; ++j)
                    if (labels[col[j]] > best)
                        labels[col[j]] = best;
                any = 1;
            }
        }
        if (!any)
            break;
    }
    return rounds;
}

/* ------------------------------------------------------------------ */
/* Partitioning: src/graph_dist.c:22-51 and :53-92, src/cc_mpi.c:41-76 */
/* ------------------------------------------------------------------ */

ORC_EXPORT void orc_vertex_range(uint32_t n, int parts, int r,
                                 uint32_t *v_start, uint32_t *v_end)
{
    if (parts <= 0) {
        *v_start = *v_end = 0;
        return;
    }
    uint32_t base = n / (uint32_t)parts, rem = n % (uint32_t)parts;
    uint32_t ru = (uint32_t)r;
    if (ru < rem) {
        *v_start = ru * (base + 1u);
        *v_end = *v_start + base + 1u;
    } else {
        *v_start = rem * (base + 1u) + (ru - rem) * base;
        *v_end = *v_start + base;
    }
}

/* Weighted bounds: weight(v) = deg(v) + vertex_weight; cut r advances a
 * running cursor until the running weight reaches total*r/parts, then the
 * cursor is clamped to [bounds[r-1]+1, n-(parts-r)] and the clamped cursor
 * is where the next cut starts from (the running weight is not adjusted
 * for the clamp, exactly as in the reference). */
ORC_EXPORT void orc_weighted_bounds(const uint64_t *row_ptr, uint32_t n, int parts,
                                    uint32_t vertex_weight, uint32_t *bounds)
{
    if (parts <= 0)
        return;
    uint64_t total_w = row_ptr[n] + (uint64_t)vertex_weight * n;
    bounds[0] = 0;
    uint32_t v = 0;
    uint64_t cum = 0;
    for (int r = 1; r < parts; ++r) {
        uint64_t target = total_w * (uint64_t)r / (uint64_t)parts;
        while (v < n && cum < target) {
            cum += (row_ptr[v + 1] - row_ptr[v]) + vertex_weight;
            v++;
        }
        uint32_t lo = bounds[r - 1] + 1u;
        uint32_t hi = n - (uint32_t)(parts - r);
        if (v < lo)
            v = lo;
        if (v > hi)
            v = hi;
        bounds[r] = v;
    }
    bounds[parts] = n;
}

ORC_EXPORT int orc_owner_of_vertex(uint32_t v, uint32_t n, int parts, int kind,
                                   const uint32_t *bounds)
{
    if (kind != 0 && bounds && parts > 1) {
        int lo = 0, hi = parts - 1;
        while (lo <= hi) {
            int mid = lo + ((hi - lo) >> 1);
            if (v < bounds[mid])
                hi = mid - 1;
            else if (v >= bounds[mid + 1])
                lo = mid + 1;
            else
                return mid;
        }
        return (v >= bounds[parts]) ? parts - 1 : 0;
    }
    if (parts <= 1)
        return 0;
    uint32_t base = n / (uint32_t)parts, rem = n % (uint32_t)parts;
    uint64_t split = (uint64_t)(base + 1u) * rem;
    if ((uint64_t)v < split)
        return (int)(v / (base + 1u));
    if (base == 0)
        return (int)rem;
    return (int)(rem + (uint32_t)(((uint64_t)v - split) / base));
}

/* ------------------------------------------------------------------ */
/* Boundary pairs: src/boundary_sort.c.  Pairs are {rep, remote}; the  */
/* order is ascending on (remote << 32 | rep).  Any correct sort gives */
/* the same output because equal keys are equal pairs; this one is a   */
/* byte-wise LSD radix sort.                                           */
/* ------------------------------------------------------------------ */

typedef struct {
    uint32_t rep;
    uint32_t remote;
} orc_pair;

static inline uint64_t pair_key(orc_pair p)
{
    return ((uint64_t)p.remote << 32) | p.rep;
}

ORC_EXPORT int orc_boundary_sort(orc_pair *a, uint64_t n)
{
    if (!a || n <= 1)
        return 0;
    orc_pair *tmp = (orc_pair *)malloc(n * sizeof(orc_pair));
    if (!tmp)
        return -1;
    orc_pair *src = a, *dst = tmp;
    for (int shift = 0; shift < 64; shift += 8) {
        uint64_t cnt[257];
        memset(cnt, 0, sizeof(cnt));
        for (uint64_t i = 0; i < n; ++i)
            cnt[((pair_key(src[i]) >> shift) & 0xFF) + 1]++;
        if (cnt[((pair_key(src[0]) >> shift) & 0xFF) + 1] == n)
            continue; /* every key has the same digit here */
        for (int b = 0; b < 256; ++b)
            cnt[b + 1] += cnt[b];
        for (uint64_t i = 0; i < n; ++i)
            dst[cnt[(pair_key(src[i]) >> shift) & 0xFF]++] = src[i];
        orc_pair *t = src;
        src = dst;
        dst = t;
    }
    if (src != a)
        memcpy(a, src, n * sizeof(orc_pair));
    free(tmp);
    return 0;
}

ORC_EXPORT uint64_t orc_boundary_dedup(orc_pair *a, uint64_t n)
{
    if (!a || n <= 1)
        return n;
    uint64_t w = 1;
    for (uint64_t i = 1; i < n; ++i)
        if (a[i].rep != a[w - 1].rep || a[i].remote != a[w - 1].remote)
            a[w++] = a[i];
    return w;
}

/* ------------------------------------------------------------------ */
/* count_connected_components: src/cc_mpi.c:765-792                    */
/* ------------------------------------------------------------------ */

ORC_EXPORT uint32_t orc_count_components(const uint32_t *labels, uint32_t n)
{
    if (!labels || n == 0)
        return 0;
    unsigned char *seen = (unsigned char *)calloc(n, 1);
    if (!seen)
        return 0;
    uint32_t c = 0;
    for (uint32_t v = 0; v < n; ++v) {
        uint32_t r = labels[v];
        if (r < n && !seen[r]) {
            seen[r] = 1;
            c++;
        }
    }
    free(seen);
    return c;
}

/* ------------------------------------------------------------------ */
/* Distributed CC restated with all partitions in one process.         */
/* src/cc_mpi.c:221-763, src/exchange_plan.c:48-225,242-425.           */
/* ------------------------------------------------------------------ */

typedef struct {
    uint32_t v_start, v_end, n_local;
    uint32_t *comp_of;      /* [n_local] min local index of local comp */
    uint32_t rep_count;
    uint32_t *rep_list;     /* [rep_count] ascending                   */
    uint32_t *comp_label;   /* [n_local], valid at rep indices         */
    uint32_t *comp_next;    /* Jacobi double buffer                    */
    uint32_t *comp_min;     /* [n_local]                               */
    uint64_t boundary_raw;
    uint64_t pair_count;    /* after dedup                             */
    orc_pair *pairs;        /* {rep, gidx} after the ghost rewrite     */
    uint32_t ghost_count;
    uint32_t *ghost_vertices;
    uint32_t *ghost_labels;
    /* plan: ghosts owned by q are the contiguous ghost range
     * [seg[q], seg[q+1]) because ghosts are sorted and partitions are
     * contiguous vertex ranges; the reference's need_from lists
     * (src/exchange_plan.c:74-83) are exactly these ranges. */
    uint32_t *seg;          /* [parts+1] */
    uint32_t *prev_sent;    /* [ghost_count]: the owner's prev_sent for the
                             * entry that feeds ghost i of this partition */
    int has_neighbours;
} orc_part;

typedef struct {
    int rounds;
    int exchanges;
    uint64_t boundary_raw;   /* summed over partitions */
    uint64_t pair_count;     /* summed */
    uint64_t ghost_count;    /* summed */
    uint64_t rep_count;      /* summed */
    uint64_t roots;          /* number of components */
    uint64_t sent_pairs;     /* delta pairs moved over all exchanges */
} orc_dist_stats;

static uint32_t label_of(const orc_part *P, const uint32_t *lab, uint32_t x, int *missing)
{
    if (x >= P->v_start && x < P->v_end) {
        *missing = 0;
        return lab[P->comp_of[x - P->v_start]];
    }
    uint32_t lo = 0, hi = P->ghost_count;
    while (lo < hi) {
        uint32_t mid = lo + (hi - lo) / 2;
        if (P->ghost_vertices[mid] < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    if (lo < P->ghost_count && P->ghost_vertices[lo] == x) {
        *missing = 0;
        return P->ghost_labels[lo];
    }
    *missing = 1;
    return x;
}

static void free_part(orc_part *P)
{
    free(P->comp_of);
    free(P->rep_list);
    free(P->comp_label);
    free(P->comp_next);
    free(P->comp_min);
    free(P->pairs);
    free(P->ghost_vertices);
    free(P->ghost_labels);
    free(P->seg);
    free(P->prev_sent);
    memset(P, 0, sizeof(*P));
}

/* Steps a5..a12 for one partition (split, local CC, reps, boundary
 * pairs, sort, dedup, ghosts, plan ranges).  Returns 0 or -1 on OOM. */
static int build_part(orc_part *P, uint32_t n, const uint64_t *row_ptr,
                      const uint32_t *col, int parts, int kind,
                      const uint32_t *bounds)
{
    uint32_t nl = P->n_local, vs = P->v_start, ve = P->v_end;
    /* local CSR with local ids: src/cc_mpi.c:252-297 */
    uint64_t *lrow = (uint64_t *)calloc((size_t)nl + 1, sizeof(uint64_t));
    if (!lrow)
        return -1;
    uint64_t braw = 0;
    for (uint32_t li = 0; li < nl; ++li) {
        uint64_t c = 0;
        for (uint64_t j = row_ptr[vs + li]; j < row_ptr[vs + li + 1]; ++j) {
            uint32_t u = col[j];
            if (u >= vs && u < ve)
                c++;
            else if (u < n)
                braw++;
        }
        lrow[li + 1] = lrow[li] + c;
    }
    uint32_t *lcol = (uint32_t *)malloc((size_t)(lrow[nl] ? lrow[nl] : 1) * sizeof(uint32_t));
    P->comp_of = (uint32_t *)malloc((size_t)(nl ? nl : 1) * sizeof(uint32_t));
    if (!lcol || !P->comp_of) {
        free(lrow);
        free(lcol);
        return -1;
    }
    for (uint32_t li = 0; li < nl; ++li) {
        uint64_t w = lrow[li];
        for (uint64_t j = row_ptr[vs + li]; j < row_ptr[vs + li + 1]; ++j) {
            uint32_t u = col[j];
            if (u >= vs && u < ve)
                lcol[w++] = u - vs;
        }
    }
    /* local CC: the reference's pthreads LP yields the min local index */
    orc_uf_labels(nl, lrow, lcol, P->comp_of);
    free(lrow);
    free(lcol);

    /* reps: src/cc_mpi.c:326-362 (comp_of[r]==r marks exactly the reps) */
    P->rep_count = 0;
    for (uint32_t li = 0; li < nl; ++li)
        if (P->comp_of[li] == li)
            P->rep_count++;
    P->rep_list = (uint32_t *)malloc((size_t)(P->rep_count ? P->rep_count : 1) * sizeof(uint32_t));
    P->comp_label = (uint32_t *)malloc((size_t)(nl ? nl : 1) * sizeof(uint32_t));
    P->comp_next = (uint32_t *)malloc((size_t)(nl ? nl : 1) * sizeof(uint32_t));
    P->comp_min = (uint32_t *)malloc((size_t)(nl ? nl : 1) * sizeof(uint32_t));
    if (!P->rep_list || !P->comp_label || !P->comp_next || !P->comp_min)
        return -1;
    uint32_t w = 0;
    for (uint32_t li = 0; li < nl; ++li)
        if (P->comp_of[li] == li)
            P->rep_list[w++] = li;
    for (uint32_t i = 0; i < nl; ++i)
        P->comp_label[i] = P->comp_next[i] = vs + i;

    /* boundary pairs, sort, dedup: src/cc_mpi.c:364-413 */
    P->boundary_raw = braw;
    P->pairs = (orc_pair *)malloc((size_t)(braw ? braw : 1) * sizeof(orc_pair));
    if (!P->pairs)
        return -1;
    uint64_t wb = 0;
    for (uint32_t li = 0; li < nl; ++li)
        for (uint64_t j = row_ptr[vs + li]; j < row_ptr[vs + li + 1]; ++j) {
            uint32_t u = col[j];
            if ((u >= vs && u < ve) || u >= n)
                continue;
            P->pairs[wb].rep = P->comp_of[li];
            P->pairs[wb].remote = u;
            wb++;
        }
    if (orc_boundary_sort(P->pairs, wb) != 0)
        return -1;
    P->pair_count = orc_boundary_dedup(P->pairs, wb);

    /* ghosts: src/cc_mpi.c:425-461 */
    P->ghost_vertices = (uint32_t *)malloc((size_t)(P->pair_count ? P->pair_count : 1) * sizeof(uint32_t));
    if (!P->ghost_vertices)
        return -1;
    uint32_t gc = 0, prev = UINT32_MAX;
    for (uint64_t i = 0; i < P->pair_count; ++i) {
        uint32_t rv = P->pairs[i].remote;
        if (rv != prev) {
            P->ghost_vertices[gc++] = rv;
            prev = rv;
        }
        P->pairs[i].remote = gc - 1;
    }
    P->ghost_count = gc;
    P->ghost_labels = (uint32_t *)malloc((size_t)(gc ? gc : 1) * sizeof(uint32_t));
    P->prev_sent = (uint32_t *)malloc((size_t)(gc ? gc : 1) * sizeof(uint32_t));
    P->seg = (uint32_t *)calloc((size_t)parts + 1, sizeof(uint32_t));
    if (!P->ghost_labels || !P->prev_sent || !P->seg)
        return -1;
    for (uint32_t i = 0; i < gc; ++i) {
        P->ghost_labels[i] = P->ghost_vertices[i];
        P->prev_sent[i] = UINT32_MAX; /* src/cc_mpi.c:480-487 */
    }
    /* plan segments: owner of every ghost, ghosts grouped by owner */
    for (uint32_t i = 0; i < gc; ++i) {
        int q = orc_owner_of_vertex(P->ghost_vertices[i], n, parts, kind, bounds);
        P->seg[q + 1]++;
    }
    for (int q = 0; q < parts; ++q)
        P->seg[q + 1] += P->seg[q];
    return 0;
}

/*
 * Full distributed CC over `parts` in-process partitions.
 *   kind      1 = edge-balanced bounds (use_edge=1), 0 = block ranges
 *   interval  exchange interval (< 1 means 1), src/cc_mpi.c:228-229
 *   gauss_seidel  0: each round's UPD reads the labels of the previous
 *             round (the order the GPU path uses, deterministic);
 *             1: reps are updated in place in ascending order, as the
 *             reference does with one merge thread (src/cc_mpi.c:587-621).
 * labels_out may be NULL.  Returns 0, or -1 on OOM / bad arguments.
 */
ORC_EXPORT int orc_dist_cc(uint32_t n, const uint64_t *row_ptr, const uint32_t *col,
                           int parts, int kind, int interval, int gauss_seidel,
                           uint32_t *labels_out, uint32_t *bounds_out,
                           orc_dist_stats *st)
{
    if (parts < 1 || !row_ptr || (!col && row_ptr[n] > 0))
        return -1;
    if (interval < 1)
        interval = 1;
    memset(st, 0, sizeof(*st));
    uint32_t *bounds = (uint32_t *)malloc(((size_t)parts + 1) * sizeof(uint32_t));
    orc_part *P = (orc_part *)calloc((size_t)parts, sizeof(orc_part));
    if (!bounds || !P) {
        free(bounds);
        free(P);
        return -1;
    }
    /* src/graph_dist.c:183-210: bounds only exist for edge mode with >1 part */
    int eff_kind = (kind && parts > 1) ? 1 : 0;
    if (eff_kind)
        orc_weighted_bounds(row_ptr, n, parts, 1, bounds);
    else
        for (int p = 0; p < parts; ++p) {
            uint32_t s, e;
            orc_vertex_range(n, parts, p, &s, &e);
            bounds[p] = s;
            bounds[p + 1] = e;
        }
    if (bounds_out)
        memcpy(bounds_out, bounds, ((size_t)parts + 1) * sizeof(uint32_t));

    int rc = 0;
    int any_pending = 0;
    for (int p = 0; p < parts; ++p) {
        P[p].v_start = bounds[p];
        P[p].v_end = bounds[p + 1];
        P[p].n_local = bounds[p + 1] - bounds[p];
        if (build_part(&P[p], n, row_ptr, col, parts, eff_kind, bounds) != 0) {
            rc = -1;
            goto out;
        }
        st->boundary_raw += P[p].boundary_raw;
        st->pair_count += P[p].pair_count;
        st->ghost_count += P[p].ghost_count;
        st->rep_count += P[p].rep_count;
        if (P[p].ghost_count > 0 && P[p].pair_count > 0 && P[p].rep_count > 0)
            any_pending = 1;
    }
    /* a partition that sends to or receives from anyone joins exchanges */
    for (int p = 0; p < parts; ++p) {
        if (P[p].ghost_count > 0)
            P[p].has_neighbours = 1;
        for (int q = 0; q < parts; ++q)
            if (q != p && P[q].seg[p + 1] > P[q].seg[p])
                P[p].has_neighbours = 1;
    }

    /* merge loop: src/cc_mpi.c:535-710, all partitions in lock step */
    int *pending = (int *)calloc((size_t)parts, sizeof(int));
    if (!pending) {
        rc = -1;
        goto out;
    }
    for (int p = 0; p < parts; ++p)
        pending[p] = any_pending;
    int global_pending = any_pending, steps = 0;
    while (global_pending) {
        int changed_any = 0;
        global_pending = 0;
        for (int p = 0; p < parts; ++p) {
            orc_part *Q = &P[p];
            /* INIT :547-561 */
            for (uint32_t i = 0; i < Q->rep_count; ++i)
                Q->comp_min[Q->rep_list[i]] = Q->comp_label[Q->rep_list[i]];
            /* HOOK :564-573 */
            for (uint64_t e = 0; e < Q->pair_count; ++e) {
                uint32_t lbl = Q->ghost_labels[Q->pairs[e].remote];
                if (lbl < Q->comp_min[Q->pairs[e].rep])
                    Q->comp_min[Q->pairs[e].rep] = lbl;
            }
            /* UPD :575-622 (MAX_JUMPS = 4) */
            int changed = 0;
            uint32_t *dst = gauss_seidel ? Q->comp_label : Q->comp_next;
            for (uint32_t i = 0; i < Q->rep_count; ++i) {
                uint32_t r = Q->rep_list[i];
                uint32_t x = Q->comp_min[r];
                for (int t = 0; t < 4; ++t) {
                    int missing = 0;
                    uint32_t y = label_of(Q, Q->comp_label, x, &missing);
                    if (missing || y >= x)
                        break;
                    x = y;
                }
                if (x < Q->comp_min[r])
                    Q->comp_min[r] = x;
                uint32_t nl = Q->comp_label[r];
                if (Q->comp_min[r] < nl) {
                    nl = Q->comp_min[r];
                    changed = 1;
                }
                dst[r] = nl;
            }
            if (!gauss_seidel) {
                uint32_t *t = Q->comp_label;
                Q->comp_label = Q->comp_next;
                Q->comp_next = t;
            }
            if (changed)
                pending[p] = 1;
            changed_any |= changed;
        }
        for (int p = 0; p < parts; ++p)
            global_pending |= pending[p];
        st->rounds++;
        if (!global_pending)
            break;
        steps++;
        if (steps >= interval || !changed_any) {
            /* delta exchange: src/exchange_plan.c:325-412.  The owner q
             * of ghost i of partition p sends (i - seg, label) when the
             * label fell below what it sent last time. */
            for (int p = 0; p < parts; ++p) {
                orc_part *Q = &P[p];
                for (int q = 0; q < parts; ++q) {
                    if (q == p)
                        continue;
                    orc_part *O = &P[q];
                    for (uint32_t i = Q->seg[q]; i < Q->seg[q + 1]; ++i) {
                        uint32_t v = Q->ghost_vertices[i];
                        uint32_t lbl = v;
                        if (v >= O->v_start && v < O->v_end)
                            lbl = O->comp_label[O->comp_of[v - O->v_start]];
                        if (lbl < Q->prev_sent[i]) {
                            Q->prev_sent[i] = lbl;
                            Q->ghost_labels[i] = lbl;
                            st->sent_pairs++;
                        }
                    }
                }
            }
            st->exchanges++;
            for (int p = 0; p < parts; ++p)
                pending[p] = 0;
            steps = 0;
        }
    }
    free(pending);

    /* roots and labels: src/cc_mpi.c:730-742 */
    for (int p = 0; p < parts; ++p) {
        orc_part *Q = &P[p];
        for (uint32_t li = 0; li < Q->n_local; ++li) {
            uint32_t lbl = Q->comp_label[Q->comp_of[li]];
            if (lbl == Q->v_start + li)
                st->roots++;
            if (labels_out)
                labels_out[Q->v_start + li] = lbl;
        }
    }
out:
    for (int p = 0; p < parts; ++p)
        free_part(&P[p]);
    free(P);
    free(bounds);
    return rc;
}

/*
 * Intermediate artefacts of one partition, for kernel-level parity tests.
 * Buffers are caller-owned; each `*_cap` is its capacity in elements and
 * the actual sizes are returned through `sizes` = {rep_count, pair_count,
 * ghost_count, boundary_raw}.  Returns 0, 1 when a capacity is too small
 * (sizes still filled), -1 on OOM.
 */
ORC_EXPORT int orc_dist_partition(uint32_t n, const uint64_t *row_ptr, const uint32_t *col,
                                  int parts, int kind, int p,
                                  uint32_t *comp_of, uint32_t *rep_list, uint64_t rep_cap,
                                  orc_pair *pairs, uint64_t pair_cap,
                                  uint32_t *ghosts, uint64_t ghost_cap,
                                  uint32_t *seg, uint64_t *sizes)
{
    uint32_t *bounds = (uint32_t *)malloc(((size_t)parts + 1) * sizeof(uint32_t));
    if (!bounds)
        return -1;
    int eff_kind = (kind && parts > 1) ? 1 : 0;
    if (eff_kind)
        orc_weighted_bounds(row_ptr, n, parts, 1, bounds);
    else
        for (int r = 0; r < parts; ++r) {
            uint32_t s, e;
            orc_vertex_range(n, parts, r, &s, &e);
            bounds[r] = s;
            bounds[r + 1] = e;
        }
    orc_part P;
    memset(&P, 0, sizeof(P));
    P.v_start = bounds[p];
    P.v_end = bounds[p + 1];
    P.n_local = P.v_end - P.v_start;
    int rc = build_part(&P, n, row_ptr, col, parts, eff_kind, bounds);
    if (rc == 0) {
        sizes[0] = P.rep_count;
        sizes[1] = P.pair_count;
        sizes[2] = P.ghost_count;
        sizes[3] = P.boundary_raw;
        if (P.rep_count > rep_cap || P.pair_count > pair_cap || P.ghost_count > ghost_cap) {
            rc = 1;
        } else {
            memcpy(comp_of, P.comp_of, (size_t)P.n_local * sizeof(uint32_t));
            memcpy(rep_list, P.rep_list, (size_t)P.rep_count * sizeof(uint32_t));
            memcpy(pairs, P.pairs, (size_t)P.pair_count * sizeof(orc_pair));
            memcpy(ghosts, P.ghost_vertices, (size_t)P.ghost_count * sizeof(uint32_t));
            memcpy(seg, P.seg, ((size_t)parts + 1) * sizeof(uint32_t));
        }
    }
    free_part(&P);
    free(bounds);
    return rc;
}
