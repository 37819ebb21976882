/*
 * Partitioned connected components with every partition resident in HBM.
 *
 * Restates the reference's distributed path on one device:
 *   src/graph_dist.c:22-92      partition bounds           -> k_bounds
 *   src/cc_mpi.c:252-323        local subgraph + local CC  -> segmented
 *                               union-find with a same-partition edge filter
 *   src/cc_mpi.c:326-362        reps, comp_label init      -> k_reps
 *   src/cc_mpi.c:364-394        boundary pairs             -> k_emit*
 *   src/boundary_sort.c         sort + dedup               -> radix sort,
 *                                                             k_dedup_*
 *   src/cc_mpi.c:425-461        ghosts                     -> k_dedup_write
 *   src/exchange_plan.c:48-225  exchange plan              -> k_plan
 *   src/cc_mpi.c:541-710        merge rounds               -> k_hook_init,
 *                                                             k_upd
 *   src/exchange_plan.c:242-425 delta exchange             -> k_exchange,
 *                                                             k_delta_push /
 *                                                             k_hook_pull
 *   src/cc_mpi.c:730-742        roots / labels             -> k_final
 *
 * Layout in HBM: all per-vertex arrays are indexed by global vertex id (a
 * partition is a contiguous slice), so a partition's comp_label/comp_of of
 * the reference are slices of cur[] and label[].  Boundary keys pack
 * (partition, remote, rep) so one sort orders every partition's pairs at
 * once; after dedup, partition p's ghosts are the contiguous range
 * [gh_off[p], gh_off[p+1]) and the ghosts it needs from partition q are the
 * sub-range [seg[p][q], seg[p][q+1]) - the reference's need_from lists.
 *
 * The reference's HOOK (comp_min = min over cut pairs of the ghost labels)
 * only changes when ghost labels change, i.e. at exchanges; hook[] keeps that
 * minimum per rep and is lowered by each exchange for the pairs of every
 * ghost whose label it changed, which gives the same comp_min every round
 * without re-reading every pair.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "local_cc.h"
#include "primitives.h"

namespace {

constexpr int kB = 256;
constexpr int kW = kB / 32;
constexpr int kTileE = 16;              /* column entries per thread in a tile */
constexpr uint64_t kGhostMapBytes = 2ull << 30; /* direct ghost map budget  */

/* The direct ghost map's budget in bytes: kGhostMapBytes, or the value of
 * CCGPU_GHOST_MAP_BYTES when set (0 keeps every solve on the id buckets). */
static uint64_t ghost_map_budget()
{
    const char *e = getenv("CCGPU_GHOST_MAP_BYTES");
    if (!e || !*e)
        return kGhostMapBytes;
    char *end = nullptr;
    const unsigned long long v = strtoull(e, &end, 10);
    return end && *end == '\0' ? (uint64_t)v : kGhostMapBytes;
}
constexpr int kTile = kB * kTileE;      /* column entries per tile             */
constexpr int kDedupItems = 16;
constexpr uint64_t kDedupTile = kB * kDedupItems;

__device__ __forceinline__ int part_of(const uint32_t *__restrict__ b, int parts, uint32_t v)
{
    int lo = 0, hi = parts;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (b[mid] <= v)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

/* ------------------------------------------------------------- bounds */

/* One thread replays the reference's cursor loop (src/graph_dist.c:70-89)
 * with a binary search per cut: the running weight after advancing the
 * cursor from (v, cum) to v' is cum + row_ptr[v'] - row_ptr[v] + (v' - v),
 * strictly increasing in v'.  The clamp moves the cursor but not the
 * running weight, exactly as in the reference. */
__global__ void k_bounds(const uint64_t *__restrict__ row_ptr, uint32_t n, int parts, int kind,
                         uint32_t *bounds, uint64_t *seg)
{
    if (threadIdx.x != 0 || blockIdx.x != 0)
        return;
    if (kind == 0) {
        uint32_t base = n / (uint32_t)parts, rem = n % (uint32_t)parts;
        for (int r = 0; r < parts; ++r) {
            uint32_t ru = (uint32_t)r;
            bounds[r] = ru < rem ? ru * (base + 1u) : rem * (base + 1u) + (ru - rem) * base;
        }
        bounds[parts] = n;
    } else {
        const uint64_t rp0 = row_ptr[0];
        const uint64_t total_w = (row_ptr[n] - rp0) + (uint64_t)n;
        bounds[0] = 0;
        uint32_t v = 0;
        uint64_t cum = 0;
        for (int r = 1; r < parts; ++r) {
            uint64_t target = total_w * (uint64_t)r / (uint64_t)parts;
            if (v < n && cum < target) {
                const uint32_t v0 = v;
                const uint64_t base = cum - (row_ptr[v0] - rp0) - v0;
                /* smallest v' in (v0, n] with base + (row_ptr[v'] - rp0) + v' >= target */
                uint32_t lo = v0 + 1, hi = n;
                while (lo < hi) {
                    uint32_t mid = lo + (hi - lo) / 2;
                    if (base + (row_ptr[mid] - rp0) + mid >= target)
                        hi = mid;
                    else
                        lo = mid + 1;
                }
                v = lo;
                cum = base + (row_ptr[v] - rp0) + v;
            }
            uint32_t min_v = bounds[r - 1] + 1u;
            uint32_t max_v = n - (uint32_t)(parts - r);
            if (v < min_v)
                v = min_v;
            if (v > max_v)
                v = max_v;
            bounds[r] = v;
        }
        bounds[parts] = n;
    }
    for (int r = 0; r <= parts; ++r)
        seg[r] = bounds[r];
}

/* ---------------------------------------------------- boundary emission */

struct EmitParams {
    const uint64_t *row_ptr;
    const uint32_t *col;
    const uint32_t *label;   /* local CC labels (global min ids)          */
    const uint32_t *bounds;  /* [parts+1]                                  */
    uint32_t n;
    uint64_t m;
    int parts;
    int rb, gb;              /* key bit widths of rep and remote          */
    uint64_t *out;           /* keys, capacity m                          */
    unsigned long long *count;
    unsigned long long *raw; /* cut edges seen (the reference's raw count) */
    uint32_t *gflag;         /* [n/32] bit v: v's label is its partition's giant label */
    uint32_t *pmask;         /* [n] bit p: the vertex has a neighbour in p's giant tree */
    const uint32_t *giants;  /* [parts] giant root of each partition, NULL = no masks */
    uint64_t tiles;          /* column tiles of kTile entries     */
    const uint32_t *tile_first; /* [tiles+1] first row starting after each tile's first entry */
    int vec;                 /* col is 16-byte aligned: 16-byte loads */
    uint32_t *ngbits;        /* [m/32] bit j: entry j points to a vertex outside its
                              * partition's giant tree (sorted-row mode), NULL = gather gflag */
    unsigned long long *bad; /* set when a row is not strictly ascending or a
                              * mirror entry is missing: sorted-row mode invalid */
    const uint32_t *roff;    /* [n*parts] partition offsets of sorted rows
                              * (k_row_scan), NULL = not computed        */
};

/* Plain keys are rare (most cut entries fall in a giant tree), so a block
 * collects them in shared memory through a shared counter and writes them
 * out with one global reservation when the buffer is half full.  A key
 * arriving at a full buffer reserves its own slot. */
constexpr uint32_t kKeyBuf = 2048;

struct KeyBuf {
    uint64_t *keys;
    uint32_t *cnt;
    unsigned long long *base;
};

__device__ __forceinline__ void kb_put(const KeyBuf &kb, const EmitParams &E, uint64_t key)
{
    const uint32_t pos = atomicAdd(kb.cnt, 1u);
    if (pos < kKeyBuf)
        kb.keys[pos] = key;
    else
        E.out[atomicAdd(E.count, 1ull)] = key;
}

/* Block-uniform: every thread passes the count it read after a barrier. */
__device__ __noinline__ void kb_flush(const KeyBuf &kb, const EmitParams &E, uint32_t kc)
{
    const uint32_t nk = kc < kKeyBuf ? kc : kKeyBuf;
    if (threadIdx.x == 0)
        *kb.base = atomicAdd(E.count, (unsigned long long)nk);
    __syncthreads();
    const unsigned long long base = *kb.base;
    for (uint32_t i = threadIdx.x; i < nk; i += blockDim.x)
        E.out[base + i] = kb.keys[i];
    __syncthreads();
    if (threadIdx.x == 0)
        *kb.cnt = 0;
}

__device__ __forceinline__ uint64_t make_key(const EmitParams &E, int p, uint32_t u, uint32_t rep)
{
    return ((uint64_t)p << (E.gb + E.rb)) | ((uint64_t)u << E.rb) | rep;
}

/* Cut edges into the giant local component of a partition all carry that
 * partition's giant rep, so most raw pairs repeat the same (p, remote, giant)
 * key.  The pairs are emitted from the remote end: the graph is symmetric,
 * so the boundary pair (p, u, rep(v)) of a cut edge v-u with v in p is seen
 * as entry v of row u.  When v lies in p's giant tree (one bit per vertex,
 * gflag, small enough to stay in L2) the row only records partition p in a
 * mask it owns (pmask[u], one atomicOr per row segment of a thread);
 * k_mask_count / k_mask_write then write one (p, u, giant rep) key per
 * mask bit.  Every other cut edge emits its key, so the sorted,
 * deduplicated pair list is the reference's.  With strictly ascending rows
 * the giant test of each cut entry comes from mirror marks instead of gflag
 * gathers (k_ng_* and k_emit_sorted below). */

/* Giant label (global min id) of every partition, ~0 when it has none or the
 * mask path is off. */
__device__ __forceinline__ void load_giant_labels(const EmitParams &E, uint32_t *s_gl)
{
    for (int i = threadIdx.x; i < E.parts; i += blockDim.x) {
        uint32_t g = E.giants ? E.giants[i] : 0xffffffffu;
        s_gl[i] = g < E.n ? __ldg(E.label + g) : 0xffffffffu;
    }
}

/* Raw cut-edge count of the reference (src/cc_mpi.c:364-375), one atomic per
 * warp at the end of the kernel. */
__device__ __forceinline__ void add_raw(const EmitParams &E, unsigned long long raw, int lane)
{
    for (int o = 16; o > 0; o >>= 1)
        raw += __shfl_xor_sync(0xffffffffu, raw, o);
    if (lane == 0 && raw)
        atomicAdd(E.raw, raw);
}

/* Giant flags: bit v of gflag is set when label[v] is the giant label of
 * v's partition. */
__global__ void __launch_bounds__(kB) k_giant_flags(EmitParams E)
{
    __shared__ uint32_t s_b[CCGPU_MAX_PARTS + 1];
    __shared__ uint32_t s_gl[CCGPU_MAX_PARTS];
    for (int i = threadIdx.x; i <= E.parts; i += kB)
        s_b[i] = E.bounds[i];
    load_giant_labels(E, s_gl);
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * kB;
    for (uint64_t b0 = (uint64_t)blockIdx.x * kB; b0 < E.n; b0 += stride) {
        const uint64_t v = b0 + threadIdx.x;
        bool g = false;
        if (v < E.n) {
            const int p = part_of(s_b, E.parts, (uint32_t)v);
            g = __ldg(E.label + v) == s_gl[p];
        }
        const unsigned bal = __ballot_sync(0xffffffffu, g);
        if ((threadIdx.x & 31) == 0 && b0 + threadIdx.x < E.n)
            E.gflag[(b0 + threadIdx.x) >> 5] = bal;
    }
}

/* Boundary pairs (src/cc_mpi.c:364-394) from the remote end, streamed over
 * the column array in tiles of kTile entries (16 per thread, 16-byte
 * loads).  The row of each entry comes from a max-scan of the rows' start
 * marks over the tile (rows are laid out in vertex order, so the last row
 * start at or before a position is its row).  Long rows need no special
 * path. */
/* Partition of v < n: compares against bounds held in registers when
 * there are at most 8 partitions, else a binary search in shared memory. */
template <int PMAX>
__device__ __forceinline__ int part_fast(const uint32_t *s_b, const uint32_t *rb, int parts,
                                         uint32_t v)
{
    if (PMAX <= 8) { /* rb[parts] = n and rb[i > parts] = ~0: exact for v < n */
        int p = 0;
#pragma unroll
        for (int i = 1; i < PMAX; ++i)
            p += v >= rb[i];
        return p;
    }
    return part_of(s_b, parts, v);
}

/* ORs bits into a partition mask unless a (possibly stale) cached read
 * already shows them: bits are only ever added, so a stale value that has
 * them means the current one has them too. */
__device__ __forceinline__ void mask_or(uint32_t *w, uint32_t bits)
{
    uint32_t cur;
    asm("ld.global.ca.u32 %0, [%1];" : "=r"(cur) : "l"(w));
    if ((cur & bits) != bits)
        atomicOr(w, bits);
}

/* Position i of a tile's row-start array, padded by four words per 32 so
 * that thread t's 16 consecutive positions (t * 16 + k) start on a 16-byte
 * boundary and a quarter-warp's 16-byte reads cover 32 distinct banks. */
#define HP(i) ((i) + 4 * ((i) >> 5))
constexpr int kHeadWords = kTile + 4 * (kTile / 32);

/* Sorted-row mode, remote end: one warp per tile of kWarpTile entries (16
 * per lane), with no block barriers.  Row starts are marked in the warp's
 * slice of shared memory (stale marks from the warp's earlier tiles name
 * earlier rows and never raise the max-scan) and a warp max-scan gives
 * each entry its row.  Rows ascend, so along a row the entries' partition
 * is stepped forward against the next bound (entries >= n are clamped to
 * n, which steps to partition P: none); cutm has bit p set for every valid
 * partition other than the row's.  An unmarked cut entry sets bit pv in
 * the row's mask (marked ones had their keys written by the local end,
 * k_ng_*); a row that is not strictly ascending sets *bad.  Runs with
 * fewer than 32 partitions, so partition masks and shifts fit 32 bits. */
constexpr int kWarpTile = 32 * kTileE;
constexpr int kWarpHead = kWarpTile + 4 * (kWarpTile / 32);

template <int PMAX>
__global__ void __launch_bounds__(kB) k_emit_sorted(EmitParams E, const uint32_t *wt_first,
                                                    uint64_t wtiles)
{
    __shared__ __align__(16) uint32_t s_head[kW][kWarpHead];
    __shared__ uint32_t s_b[CCGPU_MAX_PARTS + 2]; /* bounds, then ~0 */
    for (int i = threadIdx.x; i < CCGPU_MAX_PARTS + 2; i += kB)
        s_b[i] = i <= E.parts ? E.bounds[i] : 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t *head = s_head[warp];
    uint4 *h4 = reinterpret_cast<uint4 *>(head);
    for (int i = lane; i < kWarpHead / 4; i += 32)
        h4[i] = make_uint4(0u, 0u, 0u, 0u);
    __syncthreads();
    uint32_t sb[8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
        sb[i] = s_b[i];
    const uint32_t allp = (1u << E.parts) - 1u; /* sorted-row mode: parts < 32 */
    const uint4 *mine = reinterpret_cast<const uint4 *>(head + HP(lane * kTileE));
    unsigned long long raw = 0;
    bool unsorted = false;
    const uint64_t nwarps = (uint64_t)gridDim.x * kW;
    for (uint64_t t = (uint64_t)blockIdx.x * kW + warp; t < wtiles; t += nwarps) {
        const uint64_t lo = t * kWarpTile;
        const uint32_t v0 = wt_first[t], v1 = wt_first[t + 1];
        const uint64_t j0 = lo + (uint64_t)lane * kTileE;
        uint32_t c[kTileE];
        if (E.vec && j0 + kTileE <= E.m) {
            const uint4 *c4 = reinterpret_cast<const uint4 *>(E.col + j0);
#pragma unroll
            for (int q = 0; q < kTileE / 4; ++q) {
                const uint4 x = __ldg(c4 + q);
                c[4 * q] = x.x;
                c[4 * q + 1] = x.y;
                c[4 * q + 2] = x.z;
                c[4 * q + 3] = x.w;
            }
        } else {
#pragma unroll
            for (int k = 0; k < kTileE; ++k)
                c[k] = j0 + k < E.m ? __ldg(E.col + j0 + k) : 0xffffffffu;
        }
        /* marks of the 16 entries (j0 is a multiple of 16) */
        const uint32_t ng = j0 < E.m ? __ldg(E.ngbits + (j0 >> 5)) >> (j0 & 31) : 0u;
        const int kv = j0 >= E.m ? 0 : (E.m - j0 < kTileE ? (int)(E.m - j0) : kTileE);
        __syncwarp(); /* the previous tile's reads of the slice are done */
        if (lane == 0)
            head[0] = v0 > 0 ? v0 - 1 : 0u; /* no row in [v0, v1) starts at 0 */
        for (uint64_t v = (uint64_t)v0 + lane; v < v1 && v < E.n; v += 32) {
            const uint64_t rp = __ldg(E.row_ptr + v);
            if (rp >= lo && rp < lo + kWarpTile)
                atomicMax(head + HP(rp - lo), (uint32_t)v);
        }
        __syncwarp();
        uint32_t run = 0;
#pragma unroll
        for (int q = 0; q < kTileE / 4; ++q) {
            const uint4 x = mine[q];
            run = max(max(run, max(x.x, x.y)), max(x.z, x.w));
        }
        uint32_t incl = run;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o)
                incl = y > incl ? y : incl;
        }
        uint32_t before = __shfl_up_sync(0xffffffffu, incl, 1);
        uint32_t prev = __shfl_up_sync(0xffffffffu, c[kTileE - 1], 1);
        uint32_t row = before; /* the row of entry j0 - 1 (lane 0: ~0 or the tile's first row) */
        if (lane == 0) {
            before = 0;
            row = 0xffffffffu;
            if (lo > 0 && v0 > 0 && __ldg(E.row_ptr + v0 - 1) < lo) {
                row = v0 - 1; /* the tile's first row began in an earlier tile */
                prev = __ldg(E.col + lo - 1);
            }
        }
        uint32_t bits = 0, rawc = 0, cur = before;
        int pu = row < E.n ? part_fast<PMAX>(s_b, sb, E.parts, row) : -1;
        uint32_t cutm = pu >= 0 ? allp & ~(1u << pu) : 0u;
        uint32_t v = c[0] < E.n ? c[0] : E.n;
        int pv = part_fast<PMAX>(s_b, sb, E.parts, v < E.n ? v : E.n - 1);
        uint32_t nb = s_b[pv + 1];
#pragma unroll
        for (int q = 0; q < kTileE / 4; ++q) {
            const uint4 x = mine[q];
            const uint32_t hs[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int k = 4 * q + e;
                cur = hs[e] > cur ? hs[e] : cur;
                v = c[k] < E.n ? c[k] : E.n;
                if (cur != row) {
                    if (bits)
                        mask_or(E.pmask + row, bits);
                    bits = 0;
                    row = cur;
                    pu = row < E.n ? part_fast<PMAX>(s_b, sb, E.parts, row) : -1;
                    cutm = pu >= 0 ? allp & ~(1u << pu) : 0u;
                    pv = part_fast<PMAX>(s_b, sb, E.parts, v < E.n ? v : E.n - 1);
                    nb = s_b[pv + 1];
                } else {
                    unsorted |= c[k] <= prev && k < kv;
                }
                while (v >= nb) {
                    ++pv;
                    nb = s_b[pv + 1];
                }
                prev = c[k];
                const uint32_t cut = (cutm >> pv) & 1u; /* pv <= parts < 32 */
                rawc += cut;
                bits |= (cut & ~(ng >> k)) << pv;
            }
        }
        if (bits)
            mask_or(E.pmask + row, bits);
        raw += rawc;
    }
    if (unsorted)
        *E.bad = 1ull;
    add_raw(E, raw, lane);
}

/* ---------------------------------------------- sorted-row ranges
 *
 * When every row is strictly ascending - what the reference's loader always
 * builds (the CSC to CSR transposition of src/graph.c:91-117 emits each row
 * in column order) - a row's entries inside partition q are one contiguous
 * run.  The local subgraph of each partition (src/cc_mpi.c:252-297) is then
 * the own run of every row, read in place by the local CC (rows as [lb, le)
 * sub-ranges), and the boundary pairs of a row's run in partition q come
 * from its mirror marks alone.  One streaming pass checks the row order and
 * finds every run. */

/* Row order check and partition offsets in one streaming pass over the
 * column array.  Each warp takes chunks of kChunk consecutive entries,
 * kTileE per lane (16-byte loads when aligned), and works on them alone:
 * no block barrier, so a warp with many events never holds up the others.
 *
 * With ascending rows the count of a row's entries below bound b_q is the
 * position of its first entry >= b_q, so a row's offsets change only at a
 * few entries: its first entry (S), the entries where the partition of the
 * column rises (C) and its last entry (E).  The per-entry path is the same
 * for every lane - the entry's partition, a rise bit (C), a below-its-
 * predecessor bit and the symmetry hash; S and E bits come from the row
 * starts as whole masks - and the events are resolved afterwards, the
 * warp's lanes spread evenly over the chunk's events, each re-reading its
 * entry and the one before it (in L1).
 *
 * Per chunk a bitmap marks where non-empty rows start (positions
 * 0..kChunk, the last one meaning that the chunk's last row ends with the
 * chunk; the array's end is marked too) and rowat[pos] names the row
 * starting at pos.  The row holding a position is the row of the last
 * start at or before it - found from the bitmap and a warp max-scan of each
 * lane's last start - or, before the chunk's first start, the row holding
 * the chunk's first entry (chunk_first, k_scan_prep).  Empty rows hold no
 * entry; the chunk where they start writes their offsets.
 *
 * roff[v*P + q-1] = entries of row v below bounds[q], q = 1..P (bounds[P] =
 * n, so the last is the count of valid ids); lb/le: v's own run, its local
 * entries.  flags[0] is set when some row descends (its partition runs are
 * not contiguous); repeated entries are allowed.  local_total counts the
 * entries inside their row's own partition, from the events: each own-run
 * segment adds its end and subtracts its start.  symsum checks symmetry:
 * each entry (r, c) with c < n adds r*B(c) - B(r)*c (mod 2^32) for
 * B(x) = x*x + K, i.e. (c - r)(r*c - K): antisymmetric in (r, c), so a
 * symmetric graph sums to zero; an entry without its mirror leaves a term
 * that cancels only by chance (self loops add zero). */
constexpr int kChunk = 32 * kTileE;           /* entries per warp chunk          */
constexpr int kChunkWords = kChunk / 32 + 2;  /* start bits 0..kChunk, one spare */
static_assert(kTileE == 16, "k_row_scan keeps a lane's start bits and the next lane's first in 17 bits");

__device__ __forceinline__ uint32_t sym_mix(uint32_t x)
{
    return x * x + 0x9E3779B9u;
}

/* The row holding each chunk's first entry (as k_tile_first, width
 * kChunk). */
__global__ void __launch_bounds__(kB) k_scan_prep(const uint64_t *__restrict__ row_ptr, uint32_t n,
                                                  uint64_t m, uint64_t chunks, uint32_t *first)
{
    const uint64_t stride = (uint64_t)gridDim.x * kB;
    for (uint64_t v = (uint64_t)blockIdx.x * kB + threadIdx.x; v <= n; v += stride) {
        if (v == 0) {
            first[chunks] = n + 1;
            uint64_t r0 = __ldg(row_ptr), rn = __ldg(row_ptr + n);
            r0 = r0 > m ? m : r0;
            rn = rn > m ? m : rn;
            for (uint64_t t = 0; t * kChunk < r0; ++t)
                first[t] = 0;
            for (uint64_t t = (rn + kChunk - 1) / kChunk; t < chunks; ++t)
                first[t] = n + 1;
            continue;
        }
        uint64_t a = __ldg(row_ptr + v - 1), b = __ldg(row_ptr + v);
        if (b > m)
            b = m;
        if (a > b)
            a = b;
        for (uint64_t t = (a + kChunk - 1) / kChunk; t * kChunk < b; ++t)
            first[t] = (uint32_t)v;
    }
}

template <int P>
__global__ void __launch_bounds__(kB, 4) k_row_scan(const uint64_t *__restrict__ row_ptr,
                                                 const uint32_t *__restrict__ col, uint32_t n,
                                                 uint64_t m, const uint32_t *bounds, int vec,
                                                 const uint32_t *__restrict__ chunk_first,
                                                 uint32_t *roff, uint64_t *lb, uint64_t *le,
                                                 unsigned *flags, unsigned long long *local_total,
                                                 unsigned long long *symsum)
{
    __shared__ uint32_t s_bits[kW][kChunkWords];
    __shared__ uint32_t s_rowat[kW][kChunk + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t *bits = s_bits[warp], *rowat = s_rowat[warp];
    /* cut[i] = bounds[i] below P, n at P: the partition of id x is the
     * number of cuts <= x (P for ids >= n) */
    uint32_t cut[P + 1];
#pragma unroll
    for (int i = 1; i < P; ++i)
        cut[i] = __ldg(bounds + i);
    cut[P] = n;
    auto part = [&](uint32_t x) {
        int p = 0;
#pragma unroll
        for (int i = 1; i <= P; ++i)
            p += (int)(x >= cut[i]);
        return p;
    };
    const uint64_t chunks = (m + kChunk - 1) / kChunk;
    bool desc = false;
    unsigned long long local = 0;
    uint32_t sym = 0;
    for (uint64_t t = (uint64_t)blockIdx.x * kW + warp; t < chunks; t += (uint64_t)gridDim.x * kW) {
        const uint64_t j0 = t * kChunk, jend = j0 + kChunk < m ? j0 + kChunk : m;
        const uint32_t tb = lane * kTileE; /* first position of this lane */
        const uint64_t jt = j0 + tb;
        const int kv = jt >= jend ? 0 : jend - jt < (uint64_t)kTileE ? (int)(jend - jt) : kTileE;
        uint32_t c[kTileE];
        if (vec && jt + kTileE <= m) {
            const uint4 *c4 = reinterpret_cast<const uint4 *>(col + jt);
#pragma unroll
            for (int q = 0; q < kTileE / 4; ++q) {
                const uint4 x = __ldg(c4 + q);
                c[4 * q] = x.x;
                c[4 * q + 1] = x.y;
                c[4 * q + 2] = x.z;
                c[4 * q + 3] = x.w;
            }
        } else {
#pragma unroll
            for (int k = 0; k < kTileE; ++k)
                c[k] = k < kv ? __ldg(col + jt + k) : 0u;
        }
        const uint32_t f0 = __ldg(chunk_first + t), f1 = __ldg(chunk_first + t + 1);
        const uint32_t r_lo = f0 ? f0 - 1 : 0u;
        const uint32_t r_hi = f1 < n ? f1 : n; /* row_ptr[r_hi] > jend - 1 */
        if (lane < kChunkWords)
            bits[lane] = 0u;
        __syncwarp();
        /* starts of the non-empty rows in [j0, jend]; the array's end.  The
         * empty rows starting in [j0, jend) (and, in the last chunk, at the
         * array's end) get their zero offsets and empty runs here, next to
         * the chunk's other rows, so their partial sectors are written
         * together */
        auto empty_row = [&](uint64_t r, uint64_t a) {
#pragma unroll
            for (int q = 0; q < P; ++q)
                roff[r * P + q] = 0u;
            lb[r] = a;
            le[r] = a;
        };
        for (uint32_t r = r_lo + lane; r < r_hi; r += 32) {
            const uint64_t a = __ldg(row_ptr + r), b = __ldg(row_ptr + r + 1);
            if (a < b) {
                if (a >= j0 && a <= jend) {
                    const uint32_t o = (uint32_t)(a - j0);
                    atomicOr(&bits[o >> 5], 1u << (o & 31));
                    rowat[o] = r;
                }
            } else if (a >= j0 && (a < jend || jend == m)) {
                empty_row(r, a);
            }
        }
        if (lane == 0) {
            if (jend == m) {
                const uint32_t o = (uint32_t)(jend - j0);
                atomicOr(&bits[o >> 5], 1u << (o & 31));
            }
            /* empty rows just before the row holding j0, starting at j0 */
            if (__ldg(row_ptr + r_lo) == j0)
                for (uint64_t e = r_lo; e > 0 && __ldg(row_ptr + e - 1) == j0; --e)
                    empty_row(e - 1, j0);
        }
        __syncwarp();
        /* this lane's start bits (and the one after them), and the last
         * start before its first entry: a warp max-scan */
        const uint32_t w0 = lane >> 1;
        const uint64_t ww = (uint64_t)bits[w0] | ((uint64_t)bits[w0 + 1] << 32);
        const uint32_t sb = kv ? (uint32_t)(ww >> (16 * (lane & 1))) & 0x1FFFFu : 0u;
        const uint32_t own = sb & 0xFFFFu;
        const int mylast = own ? (int)(tb + 31 - __clz(own)) : -1;
        int incl = mylast;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o)
                incl = y > incl ? y : incl;
        }
        int excl = __shfl_up_sync(0xffffffffu, incl, 1);
        if (lane == 0)
            excl = -1;
        /* evmask: the lane's events; dmask: its entries below their
         * predecessor (a descent unless the entry starts a row) */
        uint32_t evmask = 0, dmask = 0;
        const uint32_t up = __shfl_up_sync(0xffffffffu, c[kTileE - 1], 1);
        if (kv > 0) {
            uint32_t r = excl >= 0 ? rowat[excl] : r_lo;
            uint32_t br = sym_mix(r);
            /* the entry before jt: the previous lane's last, or a load (not
             * needed at a row start) */
            uint32_t prev = lane ? up : (!(own & 1u) && jt > 0 ? __ldg(col + jt - 1) : 0u);
            int pp = part(prev);
            auto entry = [&](int k) {
                const uint32_t x = c[k];
                const bool st = (sb >> k) & 1u;
                const int p = part(x);
                if (st) {
                    r = rowat[tb + k];
                    br = sym_mix(r);
                }
                dmask |= (uint32_t)(x < prev) << k;
                evmask |= (uint32_t)(p > pp) << k; /* C; S and E come from sb */
                if (p < P)
                    sym += r * sym_mix(x) - br * x;
                prev = x;
                pp = p;
            };
            if (kv == kTileE) {
#pragma unroll
                for (int k = 0; k < kTileE; ++k)
                    entry(k);
            } else {
#pragma unroll
                for (int k = 0; k < kTileE; ++k)
                    if (k < kv)
                        entry(k);
            }
            /* S at a start bit, E before one (bit kTileE: the next lane's
             * first entry); none past the lane's kv entries */
            evmask |= (sb | (sb >> 1)) & (0xFFFFu >> (kTileE - kv));
            desc |= (dmask & ~own) != 0u;
        }
        /* the chunk's events, spread over the lanes: event i is the
         * (i - before)-th set bit of the lane that holds it */
        const uint32_t cnt = __popc(evmask);
        uint32_t ci = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, ci, o);
            if (lane >= o)
                ci += y;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, ci, 31);
        for (uint32_t i0 = 0; i0 < total; i0 += 32) {
            const uint32_t i = i0 + lane;
            /* owner: the first lane whose inclusive count exceeds i */
            int ow = 0;
#pragma unroll
            for (int s = 16; s > 0; s >>= 1) {
                const uint32_t y = __shfl_sync(0xffffffffu, ci, ow + s - 1);
                if (y <= i)
                    ow += s;
            }
            const uint32_t om = __shfl_sync(0xffffffffu, evmask, ow);
            const uint32_t ob = __shfl_sync(0xffffffffu, ci - cnt, ow);
            const uint32_t osb = __shfl_sync(0xffffffffu, sb, ow);
            const int oex = __shfl_sync(0xffffffffu, excl, ow);
            if (i >= total)
                continue;
            /* k = the position of set bit number i - ob of om: a binary
             * search on the bit counts of the halves (fixed cost, where
             * dropping the lower bits one by one diverges) */
            uint32_t mm = om, dd = i - ob;
            int k = 0;
#pragma unroll
            for (int h = 8; h > 1; h >>= 1) {
                const uint32_t lo = __popc(mm & ((1u << h) - 1u));
                if (dd >= lo) {
                    dd -= lo;
                    mm >>= h;
                    k += h;
                }
            }
            k += (int)(dd >= (mm & 1u));
            const uint32_t o = (uint32_t)ow * kTileE + k;
            const uint64_t j = j0 + o;
            /* the row of j: the last start at or before it */
            const uint32_t below = osb & ((2u << k) - 1u) & 0xFFFFu;
            const int ls = below ? (int)(o - k + 31 - __clz(below)) : oex;
            const uint32_t r = ls >= 0 ? rowat[ls] : r_lo;
            const uint64_t rbase = ls >= 0 ? j0 + ls : __ldg(row_ptr + r_lo);
            const int pr = part(r);
            const bool st = (osb >> k) & 1u, en = (osb >> (k + 1)) & 1u;
            const int pj = part(__ldg(col + j));
            const int pp = st || j == 0 ? -1 : part(__ldg(col + j - 1));
            uint32_t *ro = roff + (uint64_t)r * P;
            /* S / C: bounds pp+1..pj are first reached at j; E: bounds
             * above pj are never reached, they take the row's end.  One
             * unrolled pass over the bounds, predicated, for every lane */
            const bool lo_ev = st || pj > pp;
            const uint32_t vlo = (uint32_t)(j - rbase);
#pragma unroll
            for (int q = 0; q <= P; ++q) {
                const bool wl = lo_ev && q > pp && q <= pj;
                const bool wh = en && q > pj;
                if (wl || wh) {
                    const uint64_t at = wh ? j + 1 : j;
                    if (q >= 1)
                        ro[q - 1] = wh ? vlo + 1u : vlo;
                    if (q == pr)
                        lb[r] = at;
                    if (q == pr + 1)
                        le[r] = at;
                }
            }
            if (lo_ev) {
                if (pj == pr)
                    local -= j;
                if (pp == pr)
                    local += j;
            }
            if (en && pj == pr)
                local += j + 1;
        }
        __syncwarp(); /* bits, rowat are rewritten by the next chunk */
    }
    for (int o = 16; o > 0; o >>= 1) {
        local += __shfl_xor_sync(0xffffffffu, local, o);
        sym += __shfl_xor_sync(0xffffffffu, sym, o);
    }
    const bool any_desc = __any_sync(0xffffffffu, desc);
    if (lane == 0 && local)
        atomicAdd(local_total, local);
    if (lane == 0 && sym)
        atomicAdd(symsum, (unsigned long long)sym);
    if (lane == 0 && any_desc)
        atomicOr(flags, 1u);
}

/* Sorted-row mode, remote end, from the partition offsets: every non-empty
 * run of row u in a partition q != u's own sets bit q of pmask[u]; the runs
 * that hold no neighbour in q's giant tree have their bit cleared after the
 * key sort (k_mask_fix).  The thread owning row u stores pmask[u] whole.
 * The raw cut count takes every valid entry outside u's own run. */
template <int PMAX>
__global__ void __launch_bounds__(kB) k_emit_ranges(EmitParams E)
{
    __shared__ uint32_t s_b[PMAX + 1];
    for (int i = threadIdx.x; i <= PMAX; i += kB)
        s_b[i] = i <= E.parts ? E.bounds[i] : 0xffffffffu;
    __syncthreads();
    const int P = E.parts;
    const uint64_t stride = (uint64_t)gridDim.x * kB;
    unsigned long long raw = 0;
    for (uint64_t u = (uint64_t)blockIdx.x * kB + threadIdx.x; u < E.n; u += stride) {
        int p = 0;
#pragma unroll
        for (int i = 1; i < PMAX; ++i)
            p += (int)((uint32_t)u >= s_b[i]);
        uint32_t o[PMAX + 1];
        o[0] = 0;
#pragma unroll
        for (int q = 0; q < PMAX; ++q)
            o[q + 1] = q < P ? __ldg(E.roff + u * (uint64_t)P + q) : 0u;
        uint32_t bits = 0, own = 0;
#pragma unroll
        for (int q = 0; q < PMAX; ++q) {
            if (q >= P || o[q + 1] <= o[q])
                continue;
            if (q == p) {
                own = o[q + 1] - o[q];
                continue;
            }
            bits |= 1u << q;
        }
        raw += (uint64_t)(o[P < PMAX ? P : PMAX] - own);
        E.pmask[u] = bits;
    }
    for (int off = 16; off > 0; off >>= 1)
        raw += __shfl_xor_sync(0xffffffffu, raw, off);
    if ((threadIdx.x & 31) == 0 && raw)
        atomicAdd(E.raw, raw);
}

/* Boundary pairs from the remote end over one column tile per block
 * iteration (the gather pass, used when rows are not strictly ascending or
 * the giant masks are off): each cut entry gathers its giant flag; giant
 * ones set bit pv in the row's mask, the others emit their key. */
template <int PMAX>
__global__ void __launch_bounds__(kB, 4) k_emit(EmitParams E)
{
    __shared__ uint64_t s_keys[kKeyBuf];
    __shared__ __align__(16) uint32_t s_head[kHeadWords];
    __shared__ uint32_t s_b[CCGPU_MAX_PARTS + 1];
    __shared__ uint32_t s_w[kW];
    __shared__ uint32_t s_kcnt;
    __shared__ unsigned long long s_kbase;
    for (int i = threadIdx.x; i <= E.parts; i += kB)
        s_b[i] = E.bounds[i];
    if (threadIdx.x == 0)
        s_kcnt = 0;
    /* Row-start marks are not cleared between tiles: a block's tiles come
     * in column order, so a stale mark names a row before the current
     * tile's first row (v0 - 1, stored at position 0) and never raises the
     * max-scan. */
    uint4 *h4 = reinterpret_cast<uint4 *>(s_head);
    for (int i = threadIdx.x; i < kHeadWords / 4; i += kB)
        h4[i] = make_uint4(0u, 0u, 0u, 0u);
    unsigned long long raw = 0;
    __syncthreads();
    uint32_t sb[8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
        sb[i] = i <= E.parts ? s_b[i] : 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const KeyBuf kbuf = {s_keys, &s_kcnt, &s_kbase};
    const uint4 *mine = reinterpret_cast<const uint4 *>(s_head + HP(threadIdx.x * kTileE));
    for (uint64_t t = blockIdx.x; t < E.tiles; t += gridDim.x) {
        const uint64_t lo = t * kTile;
        const uint32_t v0 = E.tile_first[t], v1 = E.tile_first[t + 1];
        /* this thread's 16 entries; positions past m read as no vertex */
        const uint64_t j0 = lo + (uint64_t)threadIdx.x * kTileE;
        uint32_t c[kTileE];
        if (E.vec && j0 + kTileE <= E.m) {
            const uint4 *c4 = reinterpret_cast<const uint4 *>(E.col + j0);
#pragma unroll
            for (int q = 0; q < kTileE / 4; ++q) {
                const uint4 x = __ldg(c4 + q);
                c[4 * q] = x.x;
                c[4 * q + 1] = x.y;
                c[4 * q + 2] = x.z;
                c[4 * q + 3] = x.w;
            }
        } else {
#pragma unroll
            for (int k = 0; k < kTileE; ++k)
                c[k] = j0 + k < E.m ? __ldg(E.col + j0 + k) : 0xffffffffu;
        }
        /* position 0 holds the row of the tile's first entry; no row in
         * [v0, v1) starts there */
        if (threadIdx.x == 0)
            s_head[0] = v0 > 0 ? v0 - 1 : 0u;
        for (uint64_t v = (uint64_t)v0 + threadIdx.x; v < v1 && v < E.n; v += kB) {
            const uint64_t rp = __ldg(E.row_ptr + v);
            if (rp >= lo && rp < lo + kTile)
                atomicMax(s_head + HP(rp - lo), (uint32_t)v);
        }
        __syncthreads();
        /* inclusive max-scan of the row starts: 16 positions per thread */
        uint32_t run = 0;
#pragma unroll
        for (int q = 0; q < kTileE / 4; ++q) {
            const uint4 x = mine[q];
            run = max(max(run, max(x.x, x.y)), max(x.z, x.w));
        }
        uint32_t incl = run;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o)
                incl = y > incl ? y : incl;
        }
        if (lane == 31)
            s_w[warp] = incl;
        __syncthreads();
        uint32_t pre = 0;
        for (int k = 0; k < warp; ++k)
            pre = s_w[k] > pre ? s_w[k] : pre;
        uint32_t before = __shfl_up_sync(0xffffffffu, incl, 1);
        if (lane == 0)
            before = 0;
        before = before > pre ? before : pre; /* max over earlier threads */
        uint32_t row = 0xffffffffu, bits = 0, rawc = 0;
        int pu = -1;
        uint32_t cur = before; /* running max of the row starts: the row of entry k */
#pragma unroll
        for (int q = 0; q < kTileE / 4; ++q) {
            const uint4 x = mine[q];
            const uint32_t hs[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int k = 4 * q + e;
                cur = hs[e] > cur ? hs[e] : cur;
                const uint32_t v = c[k];
                if (cur != row) {
                    if (bits)
                        mask_or(E.pmask + row, bits);
                    bits = 0;
                    row = cur;
                    pu = row < E.n ? part_fast<PMAX>(s_b, sb, E.parts, row) : -1;
                }
                const int pv = part_fast<PMAX>(s_b, sb, E.parts, v);
                if (pv != pu && v < E.n && pu >= 0) { /* a cut edge */
                    ++rawc;
                    bool gnt = false;
                    if (E.gflag)
                        gnt = (__ldg(E.gflag + (v >> 5)) >> (v & 31)) & 1u;
                    if (gnt)
                        bits |= 1u << pv;
                    else
                        kb_put(kbuf, E, make_key(E, pv, row, __ldg(E.label + v) - s_b[pv]));
                }
            }
        }
        if (bits)
            mask_or(E.pmask + row, bits);
        raw += rawc;
        __syncthreads();
        const uint32_t kc = s_kcnt;
        if (kc >= kKeyBuf / 2)
            kb_flush(kbuf, E, kc);
    }
    __syncthreads();
    const uint32_t kc = s_kcnt;
    if (kc)
        kb_flush(kbuf, E, kc);
    add_raw(E, raw, lane);
}

/* Sorted-row mode, local end: the rows of vertices outside their
 * partition's giant tree (few, mostly short).  For every cut entry u of
 * such a row v the key (p, u, rep(v)) is written here, and the mirror entry
 * v of row u is marked in ngbits, so the remote-end pass (k_emit) sends
 * every unmarked cut entry to the giant mask without reading gflag.  Three
 * passes: cut entries per such row (k_ng_count), after a scan their keys
 * and (u, v) work items at the row's offset (k_ng_emit), then one search
 * per item (k_ng_mark); a mirror that is not found sets *bad. */
template <int PMAX>
__device__ __forceinline__ bool ng_row(const EmitParams &E, const uint32_t *s_b,
                                       const uint32_t *sb, uint32_t v, uint64_t &b, uint64_t &e,
                                       int &pv)
{
    if ((__ldg(E.gflag + (v >> 5)) >> (v & 31)) & 1u)
        return false;
    b = __ldg(E.row_ptr + v);
    e = __ldg(E.row_ptr + v + 1);
    e = e > E.m ? E.m : e;
    b = b > e ? e : b;
    pv = part_fast<PMAX>(s_b, sb, E.parts, v);
    return b < e;
}

#define NG_PROLOGUE                                                    \
    __shared__ uint32_t s_b[CCGPU_MAX_PARTS + 1];                      \
    for (int i = threadIdx.x; i <= E.parts; i += kB)                   \
        s_b[i] = E.bounds[i];                                          \
    __syncthreads();                                                   \
    uint32_t sb[8];                                                    \
    _Pragma("unroll") for (int i = 0; i < 8; ++i) sb[i] =              \
        i <= E.parts ? s_b[i] : 0xffffffffu;                           \
    const uint64_t stride = (uint64_t)gridDim.x * kB

/* With partition offsets (sorted rows), row v's cut entries are the runs
 * before and after its own: [b, a1) and [c0, c1), c1 = the end of its
 * valid ids. */
__device__ __forceinline__ void cut_runs(const EmitParams &E, uint32_t v, int pv, uint64_t b,
                                         uint64_t &a1, uint64_t &c0, uint64_t &c1)
{
    const uint32_t *r = E.roff + (uint64_t)v * E.parts;
    a1 = b + (pv ? __ldg(r + pv - 1) : 0u);
    c0 = b + __ldg(r + pv);
    c1 = b + __ldg(r + E.parts - 1);
}

template <int PMAX>
__global__ void __launch_bounds__(kB) k_ng_count(EmitParams E, uint32_t *cnt)
{
    NG_PROLOGUE;
    for (uint64_t v = (uint64_t)blockIdx.x * kB + threadIdx.x; v < E.n; v += stride) {
        uint64_t b, e;
        int pv;
        uint32_t c = 0;
        if (ng_row<PMAX>(E, s_b, sb, (uint32_t)v, b, e, pv)) {
            if (E.roff) {
                uint64_t a1, c0, c1;
                cut_runs(E, (uint32_t)v, pv, b, a1, c0, c1);
                c = (uint32_t)((a1 - b) + (c1 - c0));
            } else {
                for (uint64_t j = b; j < e; ++j) {
                    const uint32_t u = __ldg(E.col + j);
                    c += u < E.n && part_fast<PMAX>(s_b, sb, E.parts, u) != pv;
                }
            }
        }
        cnt[v] = c;
    }
}

/* wcnt[w] = cnt[32w] + ... + cnt[32w + 31] (to n): the rows k_ng_emit_runs
 * gives one warp.  One warp per group, a coalesced 128-byte read each. */
__global__ void __launch_bounds__(kB) k_warp_sums(const uint32_t *__restrict__ cnt, uint64_t n,
                                                  uint32_t *wcnt)
{
    const int lane = threadIdx.x & 31;
    const uint64_t nw = (n + 31) / 32;
    const uint64_t wstride = (uint64_t)gridDim.x * kW;
    for (uint64_t w = (uint64_t)blockIdx.x * kW + (threadIdx.x >> 5); w < nw; w += wstride) {
        const uint64_t v = w * 32 + lane;
        uint32_t c = v < n ? __ldg(cnt + v) : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0)
            wcnt[w] = c;
    }
}

template <int PMAX>
__global__ void __launch_bounds__(kB) k_ng_emit(EmitParams E, const uint64_t *off,
                                                uint64_t *work)
{
    NG_PROLOGUE;
    for (uint64_t v = (uint64_t)blockIdx.x * kB + threadIdx.x; v < E.n; v += stride) {
        uint64_t b, e;
        int pv;
        if (!ng_row<PMAX>(E, s_b, sb, (uint32_t)v, b, e, pv))
            continue;
        uint64_t o = off[v];
        const uint64_t o_end = off[v + 1];
        const uint32_t rep = __ldg(E.label + v) - s_b[pv];
        for (uint64_t j = b; j < e && o < o_end; ++j) {
            const uint32_t u = __ldg(E.col + j);
            if (u >= E.n || part_fast<PMAX>(s_b, sb, E.parts, u) == pv)
                continue;
            E.out[o] = make_key(E, pv, u, rep);
            work[o] = ((uint64_t)u << 32) | (uint32_t)v;
            ++o;
        }
    }
}

/* Local end with partition runs: the cut entries of 32 consecutive rows
 * (counted by k_ng_count) are one flat list for their warp, each lane
 * taking every 32nd entry - the row of entry i is the first lane whose
 * inclusive count exceeds i - so short and long rows alike keep every lane
 * busy.  The warp's keys start at woff[warp's first row / 32], the scan of
 * the per-warp sums (k_warp_sums); once sorted, the keys of each
 * (partition, remote row) settle that row's mask bit (k_mask_fix). */
template <int PMAX>
__global__ void __launch_bounds__(kB) k_ng_emit_runs(EmitParams E, const uint32_t *cnt,
                                                     const uint64_t *woff)
{
    NG_PROLOGUE;
    (void)stride;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t wstride = (uint64_t)gridDim.x * kW * 32;
    for (uint64_t base = ((uint64_t)blockIdx.x * kW + warp) * 32; base < E.n; base += wstride) {
        const uint64_t v = base + lane;
        const uint32_t c = v < E.n ? __ldg(cnt + v) : 0u;
        if (!__any_sync(0xffffffffu, c != 0))
            continue;
        uint32_t incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o)
                incl += y;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        const uint64_t o0 = __ldg(woff + base / 32);
        uint64_t b = 0, a1 = 0, c0 = 0;
        int pv = 0;
        uint32_t rep = 0;
        if (c) {
            uint64_t c1;
            b = __ldg(E.row_ptr + v);
            pv = part_fast<PMAX>(s_b, sb, E.parts, (uint32_t)v);
            cut_runs(E, (uint32_t)v, pv, b, a1, c0, c1);
            rep = __ldg(E.label + v) - s_b[pv];
        }
        const uint32_t na = (uint32_t)(a1 - b);
        for (uint32_t i0 = 0; i0 < total; i0 += 32) {
            const uint32_t i = i0 + lane;
            int ow = 0;
#pragma unroll
            for (int st = 16; st > 0; st >>= 1) {
                const uint32_t y = __shfl_sync(0xffffffffu, incl, ow + st - 1);
                if (y <= i)
                    ow += st;
            }
            const uint32_t oex = __shfl_sync(0xffffffffu, incl - c, ow);
            const uint64_t ob = __shfl_sync(0xffffffffu, b, ow);
            const uint32_t ona = __shfl_sync(0xffffffffu, na, ow);
            const uint64_t oc0 = __shfl_sync(0xffffffffu, c0, ow);
            const int opv = __shfl_sync(0xffffffffu, pv, ow);
            const uint32_t orep = __shfl_sync(0xffffffffu, rep, ow);
            if (i < total) {
                const uint32_t t = i - oex;
                const uint32_t u = __ldg(E.col + (t < ona ? ob + t : oc0 + (t - ona)));
                E.out[o0 + i] = make_key(E, opv, u, orep);
            }
        }
    }
}

/* Clears bit p of pmask[u] when u's run in partition p holds no neighbour
 * in p's giant tree.  The local-end keys (p, u, rep) hold one key per entry
 * of u's run in p whose vertex lies outside that tree (the graph is
 * symmetric: v in p lists u, so u lists v), so there are never more keys
 * with (p, u) than the run has entries, and as many exactly when none of
 * them is in the tree.  The keys are sorted, so those with (p, u) sit
 * together: the first of them compares the key as many places on as the
 * run is long (from the offsets) - it still has (p, u) only then. */
__global__ void __launch_bounds__(kB) k_mask_fix(const uint64_t *__restrict__ keys,
                                                 uint64_t count, int rb, int gb, int parts,
                                                 const uint32_t *__restrict__ roff,
                                                 uint32_t *pmask)
{
    const int lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * kB;
    const uint64_t umask = (1ull << gb) - 1ull;
    for (uint64_t base = (uint64_t)blockIdx.x * kB + (threadIdx.x & ~31u); base < count;
         base += stride) {
        const uint64_t i = base + lane;
        const bool ok = i < count;
        const uint64_t pu = ok ? __ldg(keys + i) >> rb : ~0ull;
        uint64_t before = __shfl_up_sync(0xffffffffu, pu, 1);
        if (lane == 0)
            before = ok && i > 0 ? __ldg(keys + i - 1) >> rb : ~0ull;
        if (!ok || pu == before)
            continue;
        const uint32_t u = (uint32_t)(pu & umask);
        const int p = (int)(pu >> gb);
        const uint32_t *r = roff + (uint64_t)u * parts;
        const uint32_t len = __ldg(r + p) - (p ? __ldg(r + p - 1) : 0u);
        const uint64_t last = i + len - 1;
        if (len > 0 && last < count && (__ldg(keys + last) >> rb) == pu)
            atomicAnd(pmask + u, ~(1u << p));
    }
}

/* Position of v in the strictly ascending col[lo, hi), or ~0.  Up to four
 * interpolation probes (ids spread evenly, so each lands close to v), then
 * a binary search of what is left.  Probes differ from search to search,
 * where plain bisection would send every search of a long row through the
 * same few middle entries. */
__device__ __forceinline__ uint64_t find_sorted(const uint32_t *col, uint64_t lo, uint64_t hi,
                                                uint32_t v)
{
    constexpr uint64_t kNone = ~0ull;
    if (lo >= hi)
        return kNone;
    uint32_t a = __ldg(col + lo), z = __ldg(col + hi - 1);
    if (v == a)
        return lo;
    if (v == z)
        return hi - 1;
    if (v < a || v > z)
        return kNone;
    /* col[lo] = a < v < z = col[hi - 1] */
    for (int it = 0; it < 4 && hi - lo > 16; ++it) {
        const uint64_t span = hi - 1 - lo;
        uint64_t p = lo + (uint64_t)((double)(v - a) / (double)(z - a) * (double)span);
        p = p <= lo ? lo + 1 : (p >= hi - 1 ? hi - 2 : p);
        const uint32_t x = __ldg(col + p);
        if (x == v)
            return p;
        if (x < v) {
            lo = p;
            a = x;
        } else {
            hi = p + 1;
            z = x;
        }
    }
    uint64_t l = lo + 1, h = hi - 1; /* first entry >= v in (lo, hi - 1) */
    while (l < h) {
        const uint64_t mid = l + (h - l) / 2;
        if (__ldg(col + mid) < v)
            l = mid + 1;
        else
            h = mid;
    }
    return l < hi - 1 && __ldg(col + l) == v ? l : kNone;
}

/* Marks the mirror entry v of row u for every plain key (u, v) of the
 * local end (the sorted-row mode over a built local CSR). */
__global__ void __launch_bounds__(kB) k_ng_mark(EmitParams E, const uint64_t *work,
                                                const uint64_t *total)
{
    const uint64_t items = *total;
    const uint64_t stride = (uint64_t)gridDim.x * kB;
    bool missing = false;
    for (uint64_t i = (uint64_t)blockIdx.x * kB + threadIdx.x; i < items; i += stride) {
        const uint64_t w = work[i];
        const uint32_t u = (uint32_t)(w >> 32), v = (uint32_t)w;
        uint64_t lo = __ldg(E.row_ptr + u), hi = __ldg(E.row_ptr + u + 1);
        hi = hi > E.m ? E.m : hi;
        lo = lo > hi ? hi : lo;
        const uint64_t pos = find_sorted(E.col, lo, hi, v);
        if (pos != ~0ull)
            atomicOr(E.ngbits + (pos >> 5), 1u << (pos & 31));
        else
            missing = true;
    }
    if (missing)
        *E.bad = 1ull;
}

/* The mask keys in sorted order: key (p, u, giant rep of p) for every bit
 * p of pmask[u], partition-major and ascending in u - already the sort
 * order, so they skip the radix sort and are merged with the sorted plain
 * keys.  A block step covers kMaskBlock vertices, kMaskV consecutive ones
 * per thread (two 16-byte loads).  Pass 1 counts the bits of each
 * partition per block step (counts stored partition-major); after a scan,
 * pass 2 places each thread's keys of partition p after those of the lower
 * threads (one block scan for all partitions) and writes them in vertex
 * order. */
constexpr int kMaskV = 8;
constexpr int kMaskBlock = kB * kMaskV;

/* pmask of the thread's kMaskV vertices starting at u0 (0 past n). */
__device__ __forceinline__ void mask_load(const EmitParams &E, uint64_t u0, uint32_t (&bits)[kMaskV])
{
    if (u0 + kMaskV <= E.n) {
        const uint4 *p4 = reinterpret_cast<const uint4 *>(E.pmask + u0);
        const uint4 x = __ldg(p4), y = __ldg(p4 + 1);
        bits[0] = x.x; bits[1] = x.y; bits[2] = x.z; bits[3] = x.w;
        bits[4] = y.x; bits[5] = y.y; bits[6] = y.z; bits[7] = y.w;
    } else {
#pragma unroll
        for (int k = 0; k < kMaskV; ++k)
            bits[k] = u0 + k < E.n ? __ldg(E.pmask + u0 + k) : 0u;
    }
}

template <int PMAX>
__global__ void __launch_bounds__(kB) k_mask_count(EmitParams E, uint32_t nblk, uint32_t *cnt)
{
    __shared__ uint32_t s_c[kW][PMAX];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
        uint32_t bits[kMaskV];
        mask_load(E, (uint64_t)blk * kMaskBlock + (uint64_t)threadIdx.x * kMaskV, bits);
#pragma unroll
        for (int p = 0; p < PMAX; ++p) {
            if (p < E.parts) {
                uint32_t c = 0;
#pragma unroll
                for (int k = 0; k < kMaskV; ++k)
                    c += (bits[k] >> p) & 1u;
                c = __reduce_add_sync(0xffffffffu, c);
                if (lane == 0)
                    s_c[warp][p] = c;
            }
        }
        __syncthreads();
        if (threadIdx.x < (unsigned)E.parts) {
            uint32_t t = 0;
#pragma unroll
            for (int w = 0; w < kW; ++w)
                t += s_c[w][threadIdx.x];
            cnt[(uint64_t)threadIdx.x * nblk + blk] = t;
        }
        __syncthreads();
    }
}

template <int PMAX>
__global__ void __launch_bounds__(kB) k_mask_write(EmitParams E, uint32_t nblk,
                                                   const uint64_t *off, uint64_t *out)
{
    __shared__ uint32_t s_b[CCGPU_MAX_PARTS + 1];
    __shared__ uint32_t s_gl[CCGPU_MAX_PARTS];
    __shared__ uint32_t s_w[kW][PMAX];
    for (int i = threadIdx.x; i <= E.parts; i += kB)
        s_b[i] = E.bounds[i];
    load_giant_labels(E, s_gl);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
        const uint64_t u0 = (uint64_t)blk * kMaskBlock + (uint64_t)threadIdx.x * kMaskV;
        uint32_t bits[kMaskV];
        mask_load(E, u0, bits);
        uint32_t excl[PMAX];
#pragma unroll
        for (int p = 0; p < PMAX; ++p) {
            excl[p] = 0;
            if (p < E.parts) {
                uint32_t c = 0;
#pragma unroll
                for (int k = 0; k < kMaskV; ++k)
                    c += (bits[k] >> p) & 1u;
                uint32_t incl = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o)
                        incl += y;
                }
                if (lane == 31)
                    s_w[warp][p] = incl;
                excl[p] = incl - c;
            }
        }
        __syncthreads();
#pragma unroll
        for (int p = 0; p < PMAX; ++p) {
            if (p < E.parts) {
                uint64_t at = off[(uint64_t)p * nblk + blk] + excl[p];
#pragma unroll
                for (int w = 0; w < kW; ++w)
                    at += w < warp ? s_w[w][p] : 0u;
                const uint32_t rep = s_gl[p] - s_b[p];
#pragma unroll
                for (int k = 0; k < kMaskV; ++k)
                    if ((bits[k] >> p) & 1u)
                        out[at++] = make_key(E, p, (uint32_t)(u0 + k), rep);
            }
        }
        __syncthreads(); /* s_w is rewritten by the next step */
    }
}

/* Stable merge of two ascending key arrays (ties take a first): where each
 * tile of kMergeTile outputs starts on the merge path is found first, all
 * tiles' binary searches at once (k_merge_splits); each block then stages
 * its tile's inputs in shared memory, and each thread merges kMergeItems
 * outputs from its own split point. */
constexpr int kMergeItems = 8;
constexpr int kMergeTile = kB * kMergeItems;

__device__ __forceinline__ uint64_t merge_split(const uint64_t *a, uint64_t na, const uint64_t *b,
                                                uint64_t nb, uint64_t d)
{
    uint64_t lo = d > nb ? d - nb : 0, hi = d < na ? d : na;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (a[mid] <= b[d - mid - 1])
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

/* split[t] = merge_split(min(t * kMergeTile, na + nb)), t = 0..tiles. */
__global__ void __launch_bounds__(kB) k_merge_splits(const uint64_t *__restrict__ a, uint64_t na,
                                                     const uint64_t *__restrict__ b, uint64_t nb,
                                                     uint64_t tiles, uint64_t *split)
{
    const uint64_t total = na + nb;
    const uint64_t stride = (uint64_t)gridDim.x * kB;
    for (uint64_t t = (uint64_t)blockIdx.x * kB + threadIdx.x; t <= tiles; t += stride) {
        const uint64_t d = t * kMergeTile < total ? t * kMergeTile : total;
        split[t] = merge_split(a, na, b, nb, d);
    }
}

__global__ void __launch_bounds__(kB) k_merge(const uint64_t *__restrict__ a, uint64_t na,
                                              const uint64_t *__restrict__ b, uint64_t nb,
                                              const uint64_t *__restrict__ split,
                                              uint64_t *__restrict__ out)
{
    __shared__ uint64_t s_k[kMergeTile];
    __shared__ uint64_t s_o[kMergeTile];
    const uint64_t total = na + nb;
    for (uint64_t d0 = (uint64_t)blockIdx.x * kMergeTile; d0 < total;
         d0 += (uint64_t)gridDim.x * kMergeTile) {
        const uint64_t d1 = d0 + kMergeTile < total ? d0 + kMergeTile : total;
        const uint64_t t = d0 / kMergeTile;
        const uint64_t ia0 = __ldg(split + t), ia1 = __ldg(split + t + 1);
        const uint64_t ib0 = d0 - ia0, ib1 = d1 - ia1;
        const uint32_t la = (uint32_t)(ia1 - ia0), lb = (uint32_t)(ib1 - ib0);
        for (uint32_t i = threadIdx.x; i < la + lb; i += kB)
            s_k[i] = i < la ? a[ia0 + i] : b[ib0 + (i - la)];
        __syncthreads();
        const uint32_t dt = threadIdx.x * kMergeItems;
        if (dt < la + lb) {
            /* split of this thread's diagonal inside the tile */
            uint32_t lo = dt > lb ? dt - lb : 0, hi = dt < la ? dt : la;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (s_k[mid] <= s_k[la + (dt - mid - 1)])
                    lo = mid + 1;
                else
                    hi = mid;
            }
            uint32_t ia = lo, ib = dt - lo;
            const uint32_t end = dt + kMergeItems < la + lb ? dt + kMergeItems : la + lb;
            for (uint32_t o = dt; o < end; ++o) {
                const bool take_a = ib >= lb || (ia < la && s_k[ia] <= s_k[la + ib]);
                s_o[o] = take_a ? s_k[ia++] : s_k[la + ib++];
            }
        }
        __syncthreads();
        /* the tile's outputs leave in order, coalesced */
        for (uint32_t i = threadIdx.x; i < la + lb; i += kB)
            out[d0 + i] = s_o[i];
        __syncthreads();
    }
}

/* ------------------------------------------------------ local subgraph */

/* The local CSR of every partition (src/cc_mpi.c:252-297: the entries of a
 * vertex whose other end lies in the same partition), built by streaming
 * the column array in tiles of kTile entries.  Partitions are contiguous
 * vertex ranges, so partition p's rows fill the contiguous column range
 * [pcol[p], pcol[p+1]) with pcol[p] = row_ptr[bounds[p]]: whether an entry
 * is kept depends only on its position, and the stream needs no row
 * lookup.  Pass 1 counts kept entries per tile; after a scan of the tile
 * counts, pass 2 compacts each tile in order and gives every row whose start
 * falls in the tile its local row pointer.  Ids stay global; one CSR over
 * all n vertices holds every partition's subgraph.  Both passes read the
 * columns with 16-byte loads, fully coalesced. */

struct LocalParams {
    const uint64_t *row_ptr;
    const uint32_t *col;
    uint32_t n;
    uint64_t m;
    const uint32_t *bounds;     /* [parts+1] vertex bounds            */
    const uint64_t *pcol;       /* [parts+1] column bounds            */
    int parts;
    uint64_t tiles;
    uint32_t *tile_cnt;         /* [tiles] kept entries per tile      */
    const uint64_t *tile_off;   /* [tiles+1] scanned                  */
    uint32_t *tile_first;       /* [tiles+1] first row starting after the tile's first entry */
    uint64_t *lrp;              /* [n+1] local row pointers           */
    uint32_t *lcol;             /* [tile_off[tiles]] kept entries     */
    int vec;                    /* col is 16-byte aligned: 16-byte loads */
};

/* first[t] = smallest v with row_ptr[v] > t * width (v in [0, n]),
 * first[tiles] = n + 1. */
__global__ void __launch_bounds__(kB) k_tile_first(LocalParams L, uint64_t width,
                                                   uint64_t tiles, uint32_t *first)
{
    const uint64_t stride = (uint64_t)gridDim.x * kB;
    for (uint64_t v = (uint64_t)blockIdx.x * kB + threadIdx.x; v <= L.n; v += stride) {
        if (v == 0) {
            /* tiles before the first row or after the last one hold no row
             * start (only for a row_ptr that does not span [0, m]) */
            first[tiles] = L.n + 1;
            uint64_t r0 = __ldg(L.row_ptr), rn = __ldg(L.row_ptr + L.n);
            r0 = r0 > L.m ? L.m : r0;
            rn = rn > L.m ? L.m : rn;
            for (uint64_t t = 0; t * width < r0; ++t)
                first[t] = 0;
            for (uint64_t t = (rn + width - 1) / width; t < tiles; ++t)
                first[t] = L.n + 1;
            continue;
        }
        uint64_t a = __ldg(L.row_ptr + v - 1), b = __ldg(L.row_ptr + v);
        if (b > L.m)
            b = L.m;
        if (a > b)
            a = b;
        /* tiles whose first entry t*width lies in [a, b) */
        for (uint64_t t = (a + width - 1) / width; t * width < b; ++t)
            first[t] = (uint32_t)v;
    }
}

/* Partition whose column range holds position j (pcol ascending). */
__device__ __forceinline__ int part_at(const uint64_t *s_pcol, int parts, uint64_t j)
{
    int lo = 0, hi = parts;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (s_pcol[mid] <= j)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

/* The kTileE entries of thread t of tile `tile`: kept mask (bit k = entry k)
 * and values. */
__device__ __forceinline__ uint32_t tile_keep(const LocalParams &L, const uint32_t *s_b,
                                              const uint64_t *s_pcol, uint64_t tile,
                                              uint32_t *u)
{
    const uint64_t j0 = tile * kTile + (uint64_t)threadIdx.x * kTileE;
    if (L.vec && j0 + kTileE <= L.m) {
        const uint4 *c4 = reinterpret_cast<const uint4 *>(L.col + j0);
#pragma unroll
        for (int q = 0; q < kTileE / 4; ++q) {
            const uint4 x = __ldg(c4 + q);
            u[4 * q] = x.x;
            u[4 * q + 1] = x.y;
            u[4 * q + 2] = x.z;
            u[4 * q + 3] = x.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < kTileE; ++k)
            u[k] = j0 + k < L.m ? __ldg(L.col + j0 + k) : 0u;
    }
    if (j0 >= L.m)
        return 0u;
    const int kn = L.m - j0 < kTileE ? (int)(L.m - j0) : kTileE; /* entries before m */
    /* The partition of entry k is p until entry kc, where the next
     * partition's columns begin (rare inside 16 entries); its vertex range
     * [lo_b, hi_b) stays in registers. */
    int p = part_at(s_pcol, L.parts, j0);
    uint64_t pend = s_pcol[p + 1];
    int kc = pend <= j0 || pend - j0 >= kTileE ? kTileE : (int)(pend - j0);
    uint32_t lo_b = s_b[p], hi_b = s_b[p + 1];
    uint32_t mask = 0;
#pragma unroll
    for (int k = 0; k < kTileE; ++k) {
        if (k == kc) {
            const uint64_t j = j0 + k;
            while (j >= pend && p < L.parts - 1) {
                ++p;
                pend = s_pcol[p + 1];
            }
            kc = pend <= j || pend - j0 >= kTileE ? kTileE : (int)(pend - j0);
            lo_b = s_b[p];
            hi_b = s_b[p + 1];
        }
        const bool keep = k < kn && u[k] - lo_b < hi_b - lo_b; /* lo_b <= u < hi_b */
        mask |= (uint32_t)keep << k;
    }
    return mask;
}

__global__ void __launch_bounds__(kB) k_local_count(LocalParams L)
{
    __shared__ uint32_t s_b[CCGPU_MAX_PARTS + 1];
    __shared__ uint64_t s_pcol[CCGPU_MAX_PARTS + 1];
    __shared__ uint32_t s_w[kW];
    for (int i = threadIdx.x; i <= L.parts; i += kB) {
        s_b[i] = L.bounds[i];
        s_pcol[i] = L.pcol[i];
    }
    __syncthreads();
    for (uint64_t t = blockIdx.x; t < L.tiles; t += gridDim.x) {
        uint32_t u[kTileE];
        uint32_t c = __popc(tile_keep(L, s_b, s_pcol, t, u));
        c = __reduce_add_sync(0xffffffffu, c);
        if ((threadIdx.x & 31) == 0)
            s_w[threadIdx.x >> 5] = c;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t sum = 0;
            for (int k = 0; k < kW; ++k)
                sum += s_w[k];
            L.tile_cnt[t] = sum;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kB) k_local_fill(LocalParams L)
{
    __shared__ uint32_t s_b[CCGPU_MAX_PARTS + 1];
    __shared__ uint64_t s_pcol[CCGPU_MAX_PARTS + 1];
    __shared__ uint32_t s_excl[kB + 1];
    __shared__ uint32_t s_mask[kB];
    __shared__ uint32_t s_w[kW];
    __shared__ uint32_t s_out[kTile]; /* the tile's kept entries, compacted */
    for (int i = threadIdx.x; i <= L.parts; i += kB) {
        s_b[i] = L.bounds[i];
        s_pcol[i] = L.pcol[i];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint64_t t = blockIdx.x; t < L.tiles; t += gridDim.x) {
        uint32_t u[kTileE];
        const uint32_t mask = tile_keep(L, s_b, s_pcol, t, u);
        const uint32_t c = __popc(mask);
        uint32_t incl = c;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o)
                incl += y;
        }
        if (lane == 31)
            s_w[warp] = incl;
        __syncthreads();
        uint32_t pre = 0, total = 0;
#pragma unroll
        for (int k = 0; k < kW; ++k) {
            const uint32_t y = s_w[k];
            pre += k < warp ? y : 0u;
            total += y;
        }
        const uint32_t excl = pre + incl - c;
        s_excl[threadIdx.x] = excl;
        s_mask[threadIdx.x] = mask;
        if (threadIdx.x == 0)
            s_excl[kB] = total;
        const uint64_t base = L.tile_off[t];
        uint32_t k = excl;
#pragma unroll
        for (int q = 0; q < kTileE; ++q)
            if (mask & (1u << q))
                s_out[k++] = u[q];
        __syncthreads();
        /* coalesced write-out of the compacted tile */
        for (uint32_t i = threadIdx.x; i < total; i += kB)
            L.lcol[base + i] = s_out[i];
        /* local row pointers of the rows starting in (tile start, tile end] */
        const uint64_t lo = t * kTile;
        const uint32_t v0 = L.tile_first[t], v1 = L.tile_first[t + 1];
        for (uint64_t v = (uint64_t)v0 + threadIdx.x; v < v1; v += kB) {
            uint64_t rp = __ldg(L.row_ptr + v);
            if (rp > L.m)
                rp = L.m;
            const uint32_t pos = (uint32_t)(rp - lo); /* in (0, kTile] */
            uint32_t kb;
            if (pos >= kTile) {
                kb = total;
            } else {
                const uint32_t q = pos / kTileE, bit = pos % kTileE;
                kb = s_excl[q] + __popc(s_mask[q] & ((1u << bit) - 1u));
            }
            L.lrp[v] = base + kb;
        }
        /* rows that start at position 0 (no entries before them) */
        if (t == 0)
            for (uint32_t v = threadIdx.x; v < v0; v += kB)
                L.lrp[v] = 0;
        __syncthreads();
    }
}

/* pcol[p] = row_ptr[bounds[p]] (clamped to m): the column range of each
 * partition's rows. */
__global__ void k_part_cols(const uint64_t *row_ptr, uint64_t m, const uint32_t *bounds,
                            int parts, uint64_t *pcol)
{
    for (int p = threadIdx.x; p <= parts; p += blockDim.x) {
        uint64_t x = row_ptr[bounds[p]];
        pcol[p] = x > m ? m : x;
    }
}

/* --------------------------------------------------------------- reps */

/* Reps (src/cc_mpi.c:326-362): a vertex whose local label is itself.  Each
 * rep's comp_label starts as its own id (cur and nxt, so reps no round
 * updates keep it in both buffers) and its hook minimum as none.  The
 * count is reduced per block, one atomic per block. */
__global__ void __launch_bounds__(kB) k_reps(const uint32_t *__restrict__ label, uint32_t n,
                                             unsigned long long *rep_count, uint32_t *cur,
                                             uint32_t *nxt, uint32_t *hook)
{
    __shared__ unsigned long long s_w[kW];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t stride = (uint64_t)gridDim.x * kB;
    unsigned long long c = 0;
    for (uint64_t v = (uint64_t)blockIdx.x * kB + threadIdx.x; v < n; v += stride) {
        if (__ldg(label + v) == (uint32_t)v) {
            cur[v] = (uint32_t)v; /* comp_label[i] = v_start + i, src/cc_mpi.c:361-362 */
            nxt[v] = (uint32_t)v;
            hook[v] = 0xffffffffu;
            ++c;
        }
    }
    for (int o = 16; o > 0; o >>= 1)
        c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0)
        s_w[warp] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < kW; ++w)
            t += s_w[w];
        if (t)
            atomicAdd(rep_count, t);
    }
}

/* Reps that own at least one boundary pair (their hook minimum is set).  A
 * rep without one has no hook and its own label as its only jump target,
 * so a merge round never changes it (src/cc_mpi.c:575-622): the rounds
 * walk only the others.  kActiveV consecutive vertices per thread; the
 * block scans its counts and reserves its slots with one atomic per
 * step. */
constexpr int kActiveV = 8;

__global__ void __launch_bounds__(kB) k_active_reps(const uint32_t *__restrict__ label, uint32_t n,
                                                    const uint32_t *hook, uint32_t *act,
                                                    unsigned long long *act_count)
{
    __shared__ uint32_t s_warp[kW];
    __shared__ unsigned long long s_base;
    const uint64_t step = (uint64_t)kB * kActiveV;
    for (uint64_t base = (uint64_t)blockIdx.x * step; base < n; base += (uint64_t)gridDim.x * step) {
        const uint64_t v0 = base + (uint64_t)threadIdx.x * kActiveV;
        uint32_t bits = 0;
#pragma unroll
        for (int k = 0; k < kActiveV; ++k) {
            const uint64_t v = v0 + k;
            if (v < n && __ldg(label + v) == (uint32_t)v && hook[v] != 0xffffffffu)
                bits |= 1u << k;
        }
        const uint32_t mine = __popc(bits);
        uint32_t total = 0;
        const uint32_t incl = cc_block_incl_scan256<uint32_t>(mine, s_warp, &total);
        if (threadIdx.x == 0)
            s_base = total ? atomicAdd(act_count, (unsigned long long)total) : 0ull;
        __syncthreads();
        uint64_t o = s_base + incl - mine;
        while (bits) {
            const int k = __ffs(bits) - 1;
            bits &= bits - 1;
            act[o++] = (uint32_t)(v0 + k);
        }
        __syncthreads(); /* s_base is rewritten by the next step */
    }
}

/* -------------------------------------------------------------- dedup */

struct DedupParams {
    const uint64_t *keys;   /* sorted */
    uint64_t count;
    int rb, gb;
    const uint32_t *bounds;
    int parts;
    uint32_t *tile_u, *tile_g;         /* per tile counts   */
    const uint64_t *u_off, *g_off;     /* scanned, [T+1]    */
    uint32_t *pair_rep, *pair_g;       /* [U]               */
    uint32_t *ghost_v;                 /* [G]               */
    uint64_t *ghost_pairs;             /* [G+1] first pair  */
    uint32_t *ghost_labels;
    uint64_t *gh_first;                /* [parts] first ghost of each partition, ~0 if none */
};

/* A tile of sorted keys staged in shared memory with one pad slot per 16
 * keys, so that thread t's 16 consecutive keys sit in distinct banks. */
#define DD_PAD(i) ((i) + ((i) >> 4))
constexpr int kDedupSmem = kDedupTile + kDedupTile / 16;

__device__ __forceinline__ void dedup_stage(const DedupParams &D, uint64_t *s_keys,
                                            uint64_t *s_prev)
{
    const uint64_t tile = (uint64_t)blockIdx.x * kDedupTile;
    for (int i = threadIdx.x; i < (int)kDedupTile; i += kB) {
        uint64_t gi = tile + i;
        s_keys[DD_PAD(i)] = gi < D.count ? D.keys[gi] : 0ull;
    }
    if (threadIdx.x == 0)
        *s_prev = tile > 0 ? D.keys[tile - 1] : 0ull;
    __syncthreads();
}

/* Flags of the key at tile position li (global index gi): a new pair
 * (unique) and a new ghost (partition or remote changed). */
__device__ __forceinline__ void dedup_flags(const DedupParams &D, const uint64_t *s_keys,
                                            uint64_t s_prev, int li, uint64_t gi, uint64_t &k,
                                            bool &uniq, bool &gst)
{
    k = s_keys[DD_PAD(li)];
    if (gi == 0) {
        uniq = gst = true;
        return;
    }
    uint64_t prev = li > 0 ? s_keys[DD_PAD(li - 1)] : s_prev;
    uniq = k != prev;
    gst = (k >> D.rb) != (prev >> D.rb);
}

__global__ void __launch_bounds__(kB) k_dedup_count(DedupParams D)
{
    __shared__ uint64_t s_keys[kDedupSmem];
    __shared__ uint64_t s_prev;
    __shared__ uint32_t s_w[2][kW];
    dedup_stage(D, s_keys, &s_prev);
    const uint64_t tile = (uint64_t)blockIdx.x * kDedupTile;
    uint32_t cu = 0, cg = 0;
    for (int j = 0; j < kDedupItems; ++j) {
        int li = threadIdx.x * kDedupItems + j;
        if (tile + li < D.count) {
            uint64_t k;
            bool u, g;
            dedup_flags(D, s_keys, s_prev, li, tile + li, k, u, g);
            cu += u;
            cg += g;
        }
    }
    cu = __reduce_add_sync(0xffffffffu, cu);
    cg = __reduce_add_sync(0xffffffffu, cg);
    if ((threadIdx.x & 31) == 0) {
        s_w[0][threadIdx.x >> 5] = cu;
        s_w[1][threadIdx.x >> 5] = cg;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t a = 0, b = 0;
        for (int w = 0; w < kW; ++w) {
            a += s_w[0][w];
            b += s_w[1][w];
        }
        D.tile_u[blockIdx.x] = a;
        D.tile_g[blockIdx.x] = b;
    }
}

/* Writes pairs and ghosts with coalesced stores: warp w walks tile
 * positions [w * 512, (w + 1) * 512) 32 consecutive keys per step, and a
 * step's new pairs (and new ghosts) go to consecutive slots found by
 * ballots.  A first sweep counts each warp's pairs and ghosts for the
 * block's offsets. */
__global__ void __launch_bounds__(kB) k_dedup_write(DedupParams D)
{
    __shared__ uint64_t s_keys[kDedupSmem];
    __shared__ uint64_t s_prev;
    __shared__ uint32_t s_wu[kW], s_wg[kW];
    __shared__ uint32_t s_b[CCGPU_MAX_PARTS + 1];
    for (int i = threadIdx.x; i <= D.parts; i += kB)
        s_b[i] = D.bounds[i];
    dedup_stage(D, s_keys, &s_prev);
    const uint64_t tile = (uint64_t)blockIdx.x * kDedupTile;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wbase = warp * 32 * kDedupItems;
    uint32_t cu = 0, cg = 0;
    for (int j = 0; j < kDedupItems; ++j) {
        const int li = wbase + j * 32 + lane;
        bool u = false, g = false;
        if (tile + li < D.count) {
            uint64_t k;
            dedup_flags(D, s_keys, s_prev, li, tile + li, k, u, g);
        }
        cu += __popc(__ballot_sync(0xffffffffu, u));
        cg += __popc(__ballot_sync(0xffffffffu, g));
    }
    if (lane == 0) {
        s_wu[warp] = cu;
        s_wg[warp] = cg;
    }
    __syncthreads();
    uint64_t up = D.u_off[blockIdx.x], gp = D.g_off[blockIdx.x]; /* before this warp */
    for (int w = 0; w < warp; ++w) {
        up += s_wu[w];
        gp += s_wg[w];
    }
    const uint64_t pmask = (1ull << D.gb) - 1ull;
    const uint64_t rmask = (1ull << D.rb) - 1ull;
    const int pshift = D.rb + D.gb;
    const uint32_t lt = (1u << lane) - 1u, le = (lt << 1) | 1u;
    for (int j = 0; j < kDedupItems; ++j) {
        const int li = wbase + j * 32 + lane;
        const uint64_t gi = tile + li;
        uint64_t k = 0;
        bool u = false, g = false;
        if (gi < D.count)
            dedup_flags(D, s_keys, s_prev, li, gi, k, u, g);
        const uint32_t bu = __ballot_sync(0xffffffffu, u), bg = __ballot_sync(0xffffffffu, g);
        const int p = (int)(k >> pshift);
        if (g) {
            const uint64_t my = gp + __popc(bg & lt);
            const uint32_t remote = (uint32_t)((k >> D.rb) & pmask);
            const uint64_t prev = gi == 0 ? ~0ull : (li > 0 ? s_keys[DD_PAD(li - 1)] : s_prev);
            if (gi == 0 || (int)(prev >> pshift) != p)
                D.gh_first[p] = my; /* first ghost of partition p */
            D.ghost_v[my] = remote;
            D.ghost_pairs[my] = up + __popc(bu & lt);
            D.ghost_labels[my] = remote; /* src/cc_mpi.c:456-457 */
        }
        if (u) {
            const uint64_t my = up + __popc(bu & lt);
            D.pair_rep[my] = s_b[p] + (uint32_t)(k & rmask);
            D.pair_g[my] = (uint32_t)(gp + __popc(bg & le) - 1); /* the latest ghost */
        }
        up += __popc(bu);
        gp += __popc(bg);
    }
}

/* --------------------------------------------------------------- plan */

/* seg[p*(parts+1)+q] = first ghost of partition p owned by partition >= q
 * (src/exchange_plan.c:74-83: need_from lists grouped by owner). */
__global__ void k_plan(const uint32_t *__restrict__ ghost_v, const uint64_t *__restrict__ gh_off,
                       const uint32_t *__restrict__ bounds, int parts, uint64_t *seg)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= parts * (parts + 1))
        return;
    int p = t / (parts + 1), q = t % (parts + 1);
    uint64_t lo = gh_off[p], hi = gh_off[p + 1];
    uint32_t key = bounds[q];
    if (q == parts) {
        seg[t] = hi;
        return;
    }
    while (lo < hi) {
        uint64_t mid = lo + (hi - lo) / 2;
        if (ghost_v[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    seg[t] = lo;
}

/* Id buckets of every partition's ghost list: gbucket[p*(nb+1) + b] = the
 * first of p's ghosts with id >= b << shift (p's ghosts ascend), for
 * b = 0..nb; one binary search per bucket. */
__global__ void __launch_bounds__(kB) k_ghost_buckets(const uint32_t *__restrict__ ghost_v,
                                                      const uint64_t *__restrict__ gh_off,
                                                      int parts, uint32_t nb, int shift,
                                                      uint32_t *gbucket)
{
    const uint64_t total = (uint64_t)parts * (nb + 1);
    const uint64_t stride = (uint64_t)gridDim.x * kB;
    for (uint64_t i = (uint64_t)blockIdx.x * kB + threadIdx.x; i < total; i += stride) {
        const int p = (int)(i / (nb + 1));
        const uint64_t key = (uint64_t)(i % (nb + 1)) << shift;
        uint64_t lo = gh_off[p], hi = gh_off[p + 1];
        while (lo < hi) {
            const uint64_t mid = lo + (hi - lo) / 2;
            if (__ldg(ghost_v + mid) < key)
                lo = mid + 1;
            else
                hi = mid;
        }
        gbucket[i] = (uint32_t)lo;
    }
}

/* Direct ghost map, for graphs where parts * n words fit the budget:
 * gmap[p*n + v] = the index of ghost v in p's list.  Only ghosts' slots are
 * written (one write per ghost; p's ghosts ascend, so a warp's writes fall
 * in a few lines); the others keep whatever the memory held, and a lookup
 * accepts a slot only when its index lies in p's list and that ghost is
 * the id looked up (label_of). */
__global__ void __launch_bounds__(kB) k_ghost_map(const uint32_t *__restrict__ ghost_v,
                                                  const uint64_t *__restrict__ gh_off, int parts,
                                                  uint64_t n, uint32_t *gmap)
{
    __shared__ uint64_t s_off[CCGPU_MAX_PARTS + 1];
    for (int i = threadIdx.x; i <= parts; i += kB)
        s_off[i] = gh_off[i];
    __syncthreads();
    const uint64_t G = s_off[parts];
    const uint64_t stride = (uint64_t)gridDim.x * kB;
    for (uint64_t g = (uint64_t)blockIdx.x * kB + threadIdx.x; g < G; g += stride) {
        int p = 0;
        while (p + 1 < parts && s_off[p + 1] <= g)
            ++p;
        gmap[(uint64_t)p * n + __ldg(ghost_v + g)] = (uint32_t)g;
    }
}

/* ------------------------------------------------------------- merge */

/* Round state of a merge driven on the device (k_merge_ctl, one graph
 * launch for all rounds); NULL in MergeParams when the host drives it. */
struct MergeCtl {
    uint32_t *cur, *next;         /* labels before / after the round     */
    int pending[CCGPU_MAX_PARTS];
    int steps, done, do_exch, rep_ready;
    int rounds, exchanges, launch_rounds;
};

struct MergeParams {
    const uint32_t *label;        /* comp_of as global rep ids          */
    const uint32_t *bounds;
    int parts;
    const uint32_t *rep_list;
    uint64_t rep_count;
    const uint32_t *cur;
    uint32_t *next;
    uint32_t *hook;
    const uint32_t *pair_rep, *pair_g;
    uint64_t pairs;
    const uint32_t *ghost_v;
    const uint64_t *ghost_pairs;
    uint32_t *ghost_labels;
    uint64_t ghosts;
    const uint64_t *gh_off;       /* [parts+1] */
    const uint64_t *seg;          /* [parts*(parts+1)] */
    uint32_t *delta;              /* [ghosts] ghosts whose label an exchange lowered */
    uint32_t *delta_count;        /* entries of delta in the current exchange */
    int *changed;                 /* [parts] */
    unsigned long long *sent;
    uint32_t *ghost_rep;          /* [ghosts] local rep of each ghost vertex */
    int ghost_rep_ready;          /* 0: k_exchange fills ghost_rep from label[] */
    const uint32_t *gmap;         /* [parts*n] ghost index per (p, id), ~0u: none;
                                   * NULL: the buckets below are used      */
    const uint32_t *gbucket;      /* [parts*(gnb+1)] first ghost of each id bucket */
    uint32_t gnb;                 /* id buckets per partition                      */
    int gshift;                   /* bucket = id >> gshift                         */
    uint8_t *dirty;               /* [n] 1: the rep's label fell since the last
                                   * exchange (set by k_upd, cleared after an
                                   * exchange); read from the second exchange on */
    uint64_t n;                   /* vertices (the dirty bytes)                    */
    MergeCtl *ctl;                /* device-driven rounds, or NULL                 */
};

/* Labels before the round (cur) and after it (next): the host's pointers,
 * or the device-driven merge's current pair. */
__device__ __forceinline__ const uint32_t *merge_cur(const MergeParams &M)
{
    return M.ctl ? M.ctl->cur : M.cur;
}

__device__ __forceinline__ uint32_t *merge_next(const MergeParams &M)
{
    return M.ctl ? M.ctl->next : M.next;
}

/* Whether this round's exchange runs (always when the host drives the
 * rounds: it launches the exchange only when one is due). */
__device__ __forceinline__ bool merge_exchanges(const MergeParams &M)
{
    return !M.ctl || M.ctl->do_exch;
}

/* An exchange lowers the hook minima by one pass over every pair (pull)
 * when it changes more than one ghost label per 8 pairs; below that, the
 * pairs of each changed ghost are walked (push). */
__device__ __forceinline__ bool pull_hooks(const MergeParams &M, uint64_t messages)
{
    return messages * 8 > M.pairs;
}

/* hook[r] lowered to the minimum ghost label over r's pairs, every pair:
 * kHookRounds pairs per thread per step, loaded in phases (reps and ghost
 * ids, then labels, then the hook values) so the loads of a step overlap.
 * Lanes whose pairs share a rep (consecutive pairs of a rep are
 * contiguous) combine first and one of them issues the atomicMin; a hook
 * already <= the minimum needs no atomic. */
constexpr int kHookRounds = 4;

__device__ __forceinline__ void hook_all_pairs(const MergeParams &M)
{
    const int lane = threadIdx.x & 31;
    const uint64_t span = (uint64_t)kB * kHookRounds;
    for (uint64_t base = (uint64_t)blockIdx.x * span; base < M.pairs;
         base += (uint64_t)gridDim.x * span) {
        uint32_t r[kHookRounds], g[kHookRounds], l[kHookRounds], h[kHookRounds];
#pragma unroll
        for (int i = 0; i < kHookRounds; ++i) {
            const uint64_t k = base + (uint64_t)i * kB + threadIdx.x;
            const bool ok = k < M.pairs;
            r[i] = ok ? __ldg(M.pair_rep + k) : 0xffffffffu;
            g[i] = ok ? __ldg(M.pair_g + k) : 0xffffffffu;
        }
#pragma unroll
        for (int i = 0; i < kHookRounds; ++i)
            l[i] = g[i] != 0xffffffffu ? M.ghost_labels[g[i]] : 0xffffffffu;
#pragma unroll
        for (int i = 0; i < kHookRounds; ++i)
            h[i] = r[i] != 0xffffffffu ? M.hook[r[i]] : 0u;
#pragma unroll
        for (int i = 0; i < kHookRounds; ++i) {
            const unsigned peers = __match_any_sync(0xffffffffu, r[i]);
            const uint32_t mn = __reduce_min_sync(peers, l[i]);
            if (r[i] != 0xffffffffu && (__ffs(peers) - 1) == lane && mn < h[i])
                atomicMin(M.hook + r[i], mn);
        }
    }
}

/* hook[rep] = min over the rep's cut pairs of the ghost labels. */
__global__ void __launch_bounds__(kB) k_hook_init(MergeParams M)
{
    hook_all_pairs(M);
}

__device__ __forceinline__ bool label_of(const MergeParams &M, const uint32_t *cur,
                                         const uint32_t *s_b, int p, uint32_t x, uint32_t &y)
{
    if (x >= s_b[p] && x < s_b[p + 1]) {
        y = cur[__ldg(M.label + x)];
        return true;
    }
    if (M.gmap) {
        /* the map is not cleared: a slot of an id that is not p's ghost
         * holds anything, so the index must fall in p's list and name x */
        const uint32_t gi = x < M.n ? __ldg(M.gmap + (uint64_t)p * M.n + x) : 0xffffffffu;
        if (gi < M.gh_off[p] || gi >= M.gh_off[p + 1])
            return false;
        const uint32_t gv = __ldg(M.ghost_v + gi);
        y = M.ghost_labels[gi];
        return gv == x;
    }
    /* p's ghosts are ascending; the bucket of x narrows the search */
    const uint32_t *bk = M.gbucket + (uint64_t)p * (M.gnb + 1) + (x >> M.gshift);
    uint64_t lo = __ldg(bk), hi = __ldg(bk + 1);
    while (lo < hi) {
        uint64_t mid = lo + (hi - lo) / 2;
        if (__ldg(M.ghost_v + mid) < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    if (lo < M.gh_off[p + 1] && __ldg(M.ghost_v + lo) == x) {
        y = M.ghost_labels[lo];
        return true;
    }
    return false;
}

/* One merge round over every rep (src/cc_mpi.c:547-622, MAX_JUMPS = 4),
 * reading cur and writing next. */
__global__ void __launch_bounds__(kB) k_upd(MergeParams M)
{
    __shared__ uint32_t s_b[CCGPU_MAX_PARTS + 1];
    for (int i = threadIdx.x; i <= M.parts; i += kB)
        s_b[i] = M.bounds[i];
    __syncthreads();
    const uint32_t *cur = merge_cur(M);
    uint32_t *next = merge_next(M);
    const uint64_t stride = (uint64_t)gridDim.x * kB;
    for (uint64_t i = (uint64_t)blockIdx.x * kB + threadIdx.x; i < M.rep_count; i += stride) {
        uint32_t r = M.rep_list[i];
        int p = part_of(s_b, M.parts, r);
        uint32_t c = cur[r], h = M.hook[r];
        uint32_t x = h < c ? h : c;
        for (int t = 0; t < 4; ++t) {
            uint32_t y;
            if (!label_of(M, cur, s_b, p, x, y) || y >= x)
                break;
            x = y;
        }
        next[r] = x;
        if (x < c) {
            M.changed[p] = 1;
            M.dirty[r] = 1;
        }
    }
}

/* Delta exchange (src/exchange_plan.c:242-425) on one device.  The
 * reference's (owner q -> reader p) message region is p's need-from range
 * for q, which is the index range of p's ghosts owned by q, so a message's
 * slot at the reader is its ghost.  One pass therefore does the sender's
 * pack and the reader's scatter: for every ghost g whose owner's current
 * label fell below what was last sent the label goes straight into
 * ghost_labels[g], and g is appended
 * to the exchange's delta list - the in-HBM compaction of the changed
 * boundary labels - with one slot reservation per block step of
 * kExchRounds * kB ghosts (a counter taken once per 256 ghosts was the
 * kernel's bottleneck).  The delta list
 * drives the hook update (k_delta_push) and its length is the reference's
 * count of sent pairs.  The reference's prev_sent (src/cc_mpi.c:480-487,
 * ~0 at first) needs no array here: the first exchange sends every label
 * (each is below ~0), and from then on a slot's last sent label and its
 * ghost label change together, so ghost_labels[g] is the last sent label. */
constexpr int kExchRounds = 8; /* ghosts per thread per block step */

__global__ void __launch_bounds__(kB) k_exchange(MergeParams M)
{
    __shared__ uint32_t s_wcnt[kB / 32];
    __shared__ uint32_t s_base;
    if (!merge_exchanges(M))
        return;
    const int ready = M.ctl ? M.ctl->rep_ready : M.ghost_rep_ready;
    const uint32_t *cur = merge_cur(M);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t span = (uint64_t)kB * kExchRounds;
    for (uint64_t base = (uint64_t)blockIdx.x * span; base < M.ghosts;
         base += (uint64_t)gridDim.x * span) {
        /* the step's loads in phases (reps, then dirty bytes, then labels
         * and last-sent values), so each thread keeps kExchRounds loads in
         * flight instead of one dependent chain per ghost */
        uint32_t rep[kExchRounds];
        bool look[kExchRounds];
#pragma unroll
        for (int i = 0; i < kExchRounds; ++i) {
            const uint64_t g = base + (uint64_t)i * kB + threadIdx.x;
            look[i] = g < M.ghosts;
            rep[i] = 0;
            if (look[i])
                rep[i] = ready ? __ldg(M.ghost_rep + g) : __ldg(M.label + __ldg(M.ghost_v + g));
        }
        if (ready) {
            /* a rep whose label did not fall since the last exchange still
             * has the label last sent: nothing to send */
#pragma unroll
            for (int i = 0; i < kExchRounds; ++i)
                look[i] = look[i] && M.dirty[rep[i]] != 0;
        } else {
#pragma unroll
            for (int i = 0; i < kExchRounds; ++i)
                if (look[i]) /* fixed by the local solve */
                    M.ghost_rep[base + (uint64_t)i * kB + threadIdx.x] = rep[i];
        }
        uint32_t lbl[kExchRounds], ps[kExchRounds];
#pragma unroll
        for (int i = 0; i < kExchRounds; ++i) {
            const uint64_t g = base + (uint64_t)i * kB + threadIdx.x;
            lbl[i] = look[i] ? cur[rep[i]] : 0xffffffffu;
            ps[i] = look[i] ? (ready ? M.ghost_labels[g] : 0xffffffffu) : 0u;
        }
        uint32_t sendmask = 0;
#pragma unroll
        for (int i = 0; i < kExchRounds; ++i) {
            if (look[i] && lbl[i] < ps[i]) {
                const uint64_t g = base + (uint64_t)i * kB + threadIdx.x;
                M.ghost_labels[g] = lbl[i];
                sendmask |= 1u << i;
            }
        }
        /* one slot reservation for the block's step */
        const uint32_t cnt = __popc(sendmask);
        uint32_t incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o)
                incl += y;
        }
        if (lane == 31)
            s_wcnt[warp] = incl;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t acc = 0;
            for (int w = 0; w < kB / 32; ++w) {
                const uint32_t c = s_wcnt[w];
                s_wcnt[w] = acc;
                acc += c;
            }
            s_base = acc ? atomicAdd(M.delta_count, acc) : 0u;
        }
        __syncthreads();
        uint32_t pos = s_base + s_wcnt[warp] + incl - cnt;
        while (sendmask) {
            const int i = __ffs(sendmask) - 1;
            sendmask &= sendmask - 1u;
            M.delta[pos++] = (uint32_t)(base + (uint64_t)i * kB + threadIdx.x);
        }
        __syncthreads(); /* s_wcnt / s_base are rewritten by the next step */
    }
}

/* Hook update of an exchange with few changed ghosts (push side): every
 * ghost on the delta list lowers the hook minimum of each rep it is paired
 * with (its pairs are contiguous, [ghost_pairs[g], ghost_pairs[g+1])).
 * One ghost per lane, one pair per lane per step: lanes whose pairs share a
 * rep (most cut pairs of a partition carry its giant rep) combine their
 * labels first and one of them issues the atomicMin.  Hook values only
 * decrease, so a plain read that is already <= the minimum means the atomic
 * would change nothing.  Does nothing when the exchange takes the pull
 * side. */
__global__ void __launch_bounds__(kB) k_delta_push(MergeParams M)
{
    if (!merge_exchanges(M))
        return;
    const uint32_t total = *M.delta_count;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (total)
            atomicAdd(M.sent, (unsigned long long)total); /* the exchange's sent pairs */
        if (M.ctl)
            M.ctl->rep_ready = 1; /* k_exchange has filled ghost_rep */
    }
    if (pull_hooks(M, total))
        return;
    const int lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * kB;
    for (uint64_t base = (uint64_t)blockIdx.x * kB; base < total; base += stride) {
        const uint64_t i = base + threadIdx.x;
        uint64_t k0 = 0, k1 = 0;
        uint32_t lbl = 0;
        if (i < total) {
            const uint32_t g = M.delta[i];
            lbl = M.ghost_labels[g];
            k0 = M.ghost_pairs[g];
            k1 = M.ghost_pairs[g + 1];
        }
        const uint64_t nk = k1 - k0;
        uint64_t steps = nk;
        for (int o = 16; o > 0; o >>= 1) {
            const uint64_t y = __shfl_xor_sync(0xffffffffu, steps, o);
            steps = y > steps ? y : steps;
        }
        for (uint64_t t = 0; t < steps; ++t) {
            const bool act = t < nk;
            const uint32_t r = act ? M.pair_rep[k0 + t] : 0xffffffffu;
            const unsigned peers = __match_any_sync(0xffffffffu, r);
            const uint32_t mn = __reduce_min_sync(peers, act ? lbl : 0xffffffffu);
            if (act && (__ffs(peers) - 1) == lane && mn < M.hook[r])
                atomicMin(M.hook + r, mn);
        }
    }
}

/* Hook update of an exchange with many changed ghosts (pull side): after
 * k_exchange wrote the new ghost labels, one pass over every pair lowers
 * the hook minima.  Ghost labels only decrease and hook[r] already bounds
 * the old labels of r's ghosts, so the minima equal the push side's.  Does
 * nothing when the exchange takes the push side. */
__global__ void __launch_bounds__(kB) k_hook_pull(MergeParams M)
{
    if (!merge_exchanges(M) || !pull_hooks(M, *M.delta_count))
        return;
    hook_all_pairs(M);
}

/* dirty[] cleared after an exchange. */
__global__ void __launch_bounds__(kB) k_dirty_clear(MergeParams M)
{
    if (!merge_exchanges(M))
        return;
    const uint64_t words = M.n / 16, stride = (uint64_t)gridDim.x * kB;
    uint4 *d4 = reinterpret_cast<uint4 *>(M.dirty);
    for (uint64_t i = (uint64_t)blockIdx.x * kB + threadIdx.x; i < words; i += stride)
        d4[i] = make_uint4(0u, 0u, 0u, 0u);
    for (uint64_t i = words * 16 + (uint64_t)blockIdx.x * kB + threadIdx.x; i < M.n; i += stride)
        M.dirty[i] = 0;
}

/* The round bookkeeping of the reference's merge loop (src/cc_mpi.c:
 * 624-710) on the device, one thread, after each k_upd: partitions whose
 * labels changed become pending, the labels swap, the loop ends when
 * nothing is pending, and an exchange is due after `interval` rounds or a
 * round that changed nothing.  The graph's while node repeats the round
 * while this sets its condition: until the merge ends, or after
 * kLaunchRounds rounds, when the host reads the state and launches again. */
constexpr int kLaunchRounds = 4096;

__global__ void k_merge_ctl(MergeCtl *ctl, int *changed, int parts, int interval,
                            cudaGraphConditionalHandle loop)
{
    if (threadIdx.x != 0 || blockIdx.x != 0)
        return;
    int any = 0, pending = 0;
    for (int p = 0; p < parts; ++p) {
        const int c = changed[p];
        if (c)
            ctl->pending[p] = 1;
        any |= c;
        pending |= ctl->pending[p];
    }
    ctl->rounds++;
    ctl->launch_rounds++;
    uint32_t *t = ctl->cur;
    ctl->cur = ctl->next;
    ctl->next = t;
    ctl->do_exch = 0;
    if (!pending) {
        ctl->done = 1;
        cudaGraphSetConditional(loop, 0u);
        return;
    }
    if (++ctl->steps >= interval || !any) {
        ctl->do_exch = 1;
        ctl->exchanges++;
        for (int p = 0; p < parts; ++p)
            ctl->pending[p] = 0;
        ctl->steps = 0;
    }
    cudaGraphSetConditional(loop, ctl->launch_rounds < kLaunchRounds ? 1u : 0u);
}

__global__ void __launch_bounds__(kB) k_final(const uint32_t *__restrict__ label,
                                              const uint32_t *__restrict__ cur, uint32_t n,
                                              uint32_t *out, unsigned long long *roots)
{
    const uint64_t stride = (uint64_t)gridDim.x * kB;
    uint32_t c = 0;
    for (uint64_t v = (uint64_t)blockIdx.x * kB + threadIdx.x; v < n; v += stride) {
        uint32_t l = cur[__ldg(label + v)];
        if (out)
            out[v] = l;
        c += (l == (uint32_t)v);
    }
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0 && c)
        atomicAdd(roots, (unsigned long long)c);
}

int bits_for(uint64_t max_value)
{
    int b = 0;
    while (b < 64 && (max_value >> b) != 0)
        ++b;
    return b < 1 ? 1 : b;
}

struct PhaseClock {
    cudaEvent_t ev[8];
    int n = 0;
    bool on = false;
};

int clock_mark(PhaseClock &c, cudaStream_t st)
{
    if (!c.on)
        return CCGPU_OK;
    CC_CUDA(cudaEventRecord(c.ev[c.n++], st));
    return CCGPU_OK;
}

} // namespace

/* ------------------------------------------------------------------ API */

extern "C" void ccgpu_dist_opts_default(ccgpu_dist_opts *o)
{
    if (!o)
        return;
    o->parts = 1;
    o->use_edge = 1;
    o->chunk_size = 2048; /* the reference CLI's default -c, src/mpi_cc_benchmark.c:40 */
    o->exchange_interval = 1;
    o->verbose = 0;
}

extern "C" int ccgpu_partition_bounds(const uint64_t *d_row_ptr, uint32_t n, int parts,
                                      int use_edge, uint32_t *h_bounds, void *stream)
{
    if (!d_row_ptr || !h_bounds || parts < 1 || parts > CCGPU_MAX_PARTS)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_partition_bounds: bad arguments");
    if ((uint32_t)parts > n && n > 0)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_partition_bounds: %d parts > %u vertices",
                               parts, n);
    cudaStream_t st = (cudaStream_t)stream;
    DevBufs b;
    CC_TRY(cc_bufs_init(&b, st));
    uint32_t *d_b = nullptr;
    uint64_t *d_s = nullptr;
    int rc = cc_bufs_get(&b, (void **)&d_b, (parts + 1) * sizeof(uint32_t));
    if (rc == CCGPU_OK)
        rc = cc_bufs_get(&b, (void **)&d_s, (parts + 1) * sizeof(uint64_t));
    if (rc == CCGPU_OK) {
        k_bounds<<<1, 32, 0, st>>>(d_row_ptr, n, parts, (use_edge && parts > 1) ? 1 : 0, d_b, d_s);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(h_bounds, d_b, (parts + 1) * sizeof(uint32_t),
                                cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(st);
        if (e != cudaSuccess)
            rc = ccgpu_cuda_fail(e, "partition bounds", __FILE__, __LINE__);
    }
    cc_bufs_release(&b);
    return rc;
}

/* The rest of a merge driven on the device (see k_merge_ctl), from the
 * host loop's state: labels cur / nxt, pending flags, rounds since the last
 * exchange, whether ghost_rep is filled.  Sets *used to false, with nothing
 * launched, when conditional graph nodes are not available; the caller
 * then goes on driving the rounds from the host. */
static int merge_on_device(ccgpu_ctx *ctx, const MergeParams &M0, uint32_t *cur, uint32_t *nxt,
                           const std::vector<int> &pending, int steps, int P, int interval,
                           uint64_t act_count, uint64_t G, uint64_t U, uint32_t n, DevBufs *B,
                           cudaStream_t st, uint32_t **final_labels, ccgpu_dist_stats *S,
                           bool *used)
{
    *used = false;
    MergeCtl h;
    memset(&h, 0, sizeof(h));
    h.cur = cur;
    h.next = nxt;
    for (int p = 0; p < P; ++p)
        h.pending[p] = pending[p];
    h.steps = steps;
    h.rep_ready = M0.ghost_rep_ready;
    MergeCtl *d_ctl = nullptr;
    CC_TRY(cc_bufs_get(B, (void **)&d_ctl, sizeof(MergeCtl)));
    CC_CUDA(cudaMemcpyAsync(d_ctl, &h, sizeof(h), cudaMemcpyHostToDevice, st));
    MergeParams M = M0;
    M.ctl = d_ctl;
    M.cur = nullptr;
    M.next = nullptr;
    const unsigned gbk = (unsigned)ctx->sm_count * 8;

    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    cudaStream_t cs = nullptr;
    int rc = CCGPU_OK;
    auto fail = [&](cudaError_t e, int line) {
        if (rc == CCGPU_OK && e != cudaSuccess)
            rc = ccgpu_cuda_fail(e, "merge rounds graph", __FILE__, line);
    };
    cudaGraphConditionalHandle loop = 0;
    if (cudaGraphCreate(&g, 0) != cudaSuccess ||
        cudaGraphConditionalHandleCreate(&loop, g, 1u, cudaGraphCondAssignDefault) !=
            cudaSuccess) {
        cudaGetLastError();
        if (g)
            cudaGraphDestroy(g);
        return CCGPU_OK; /* not available: the host drives the rounds */
    }
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = loop;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t wn = nullptr;
    fail(cudaGraphAddNode(&wn, g, nullptr, 0, &cp), __LINE__);
    if (rc == CCGPU_OK)
        fail(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), __LINE__);
    if (rc == CCGPU_OK) {
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        fail(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal),
             __LINE__);
        if (rc == CCGPU_OK) {
            const cudaStream_t st = cs; /* CC_* macros launch on `st` */
            int lrc = [&]() -> int {
                CC_CUDA(cudaMemsetAsync(M.changed, 0, P * sizeof(int), st));
                CC_KLAUNCH(ctx, CCK_MERGE_UPD, k_upd, cc_blocks(act_count, kB, gbk), kB, 0, st, M);
                CC_KLAUNCH(ctx, CCK_MERGE_UPD, k_merge_ctl, 1, 32, 0, st, d_ctl, M.changed, P,
                           interval, loop);
                CC_CUDA(cudaMemsetAsync(M.delta_count, 0, sizeof(uint32_t), st));
                CC_KLAUNCH(ctx, CCK_MERGE_EXCH_PACK, k_exchange,
                           cc_blocks(G, (unsigned)(kB * kExchRounds), gbk), kB, 0, st, M);
                CC_KLAUNCH(ctx, CCK_MERGE_EXCH_SCATTER, k_delta_push, cc_blocks(G, kB, gbk), kB,
                           0, st, M);
                CC_KLAUNCH(ctx, CCK_MERGE_EXCH_PULL, k_hook_pull,
                           cc_blocks(U, (unsigned)(kB * kHookRounds), gbk), kB, 0, st, M);
                CC_KLAUNCH(ctx, CCK_MERGE_EXCH_PULL, k_dirty_clear,
                           cc_blocks((uint64_t)n / 16 + 1, kB, gbk), kB, 0, st, M);
                return CCGPU_OK;
            }();
            cudaGraph_t out = nullptr;
            fail(cudaStreamEndCapture(cs, &out), __LINE__);
            if (rc == CCGPU_OK)
                rc = lrc;
        }
    }
    if (rc == CCGPU_OK)
        fail(cudaGraphInstantiate(&ge, g, 0), __LINE__);
    for (int launch = 0; rc == CCGPU_OK; ++launch) {
        if (launch)
            fail(cudaMemsetAsync(&d_ctl->launch_rounds, 0, sizeof(int), st), __LINE__);
        fail(cudaGraphLaunch(ge, st), __LINE__);
        fail(cudaMemcpyAsync(&h, d_ctl, sizeof(h), cudaMemcpyDeviceToHost, st), __LINE__);
        fail(cudaStreamSynchronize(st), __LINE__);
        if (h.done)
            break;
        if (rc == CCGPU_OK && h.rounds >= (1 << 22))
            rc = ccgpu_set_error(CCGPU_ERR_LIMIT, "merge rounds: no end after %d rounds",
                                 h.rounds);
    }
    if (ge)
        cudaGraphExecDestroy(ge);
    cudaGraphDestroy(g);
    if (cs)
        cudaStreamDestroy(cs);
    if (rc != CCGPU_OK)
        return rc;
    S->rounds += h.rounds;
    S->exchanges += h.exchanges;
    *final_labels = h.cur;
    *used = true;
    return CCGPU_OK;
}

static int dist_run(ccgpu_ctx *ctx, const uint64_t *d_row_ptr, const uint32_t *d_col, uint32_t n,
                    uint64_t m, const ccgpu_dist_opts &o, uint32_t *d_labels, uint32_t *h_bounds,
                    ccgpu_dist_stats *st_out, cudaStream_t st, DevBufs &B)
{
    const int P = o.parts;
    const int interval = o.exchange_interval < 1 ? 1 : o.exchange_interval;
    ccgpu_dist_stats S;
    memset(&S, 0, sizeof(S));
    PhaseClock clk;
    clk.on = st_out != nullptr || o.verbose;
    for (int i = 0; clk.on && i < 8; ++i)
        CC_CUDA(cudaEventCreate(&clk.ev[i]));
    struct EvGuard {
        PhaseClock &c;
        ~EvGuard()
        {
            for (int i = 0; c.on && i < 8; ++i)
                cudaEventDestroy(c.ev[i]);
        }
    } guard{clk};
    CC_TRY(clock_mark(clk, st)); /* 0 */

    /* 1. bounds */
    uint32_t *bounds = nullptr;
    uint64_t *seg64 = nullptr;
    CC_TRY(cc_bufs_get(&B, (void **)&bounds, (P + 1) * sizeof(uint32_t)));
    CC_TRY(cc_bufs_get(&B, (void **)&seg64, (P + 1) * sizeof(uint64_t)));
    const int kind = (o.use_edge && P > 1) ? 1 : 0;
    CC_KLAUNCH(ctx, CCK_DIST_BOUNDS, k_bounds, 1, 32, 0, st, d_row_ptr, n, P, kind, bounds, seg64);
    std::vector<uint32_t> hb(P + 1);
    CC_CUDA(cudaMemcpyAsync(hb.data(), bounds, (P + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                            st));
    CC_CUDA(cudaStreamSynchronize(st));
    if (h_bounds)
        memcpy(h_bounds, hb.data(), (P + 1) * sizeof(uint32_t));
    uint32_t max_local = 1;
    for (int p = 0; p < P; ++p)
        if (hb[p + 1] - hb[p] > max_local)
            max_local = hb[p + 1] - hb[p];
    CC_TRY(clock_mark(clk, st)); /* 1 */

    /* 2. local subgraph of every partition, then local CC on it.
     * Ranges mode (2 to 8 partitions): the row order is checked in one
     * streaming pass and each row's partition runs are found in place; the
     * local CC reads every row's own run.  If some row turns out to descend
     * (known after step 3), steps 2-3 run again with the local CSR built
     * (count + fill), as they do for more partitions. */
    uint32_t *label = nullptr;
    CC_TRY(cc_bufs_get(&B, (void **)&label, (size_t)n * sizeof(uint32_t)));
    ccgpu_cc_opts lo;
    ccgpu_cc_opts_default(&lo);
    lo.chunk_size = o.chunk_size;
    ccgpu_cc_opts ro;
    CC_TRY(cc_local_resolve_opts(&lo, &ro));
    const bool use_mask = P > 1 && P <= 32 && ro.sample_rounds > 0 && ro.skip_giant;
    bool ranges = use_mask && P <= 8 && m > 0;
    LocalParams Lp;
    Lp.row_ptr = d_row_ptr;
    Lp.col = d_col;
    Lp.vec = ((uintptr_t)d_col & 15) == 0;
    Lp.n = n;
    Lp.m = m;
    Lp.bounds = bounds;
    Lp.parts = P;
    Lp.tiles = (m + kTile - 1) / kTile;
    const unsigned vb = cc_blocks((uint64_t)n + 1, kB, (unsigned)ctx->sm_count * 8);
    uint32_t *tile_first = nullptr, *wt_first = nullptr;
    uint64_t col_tiles = 0, wtiles = 0;
    /* first row starting after each column tile's first entry (the gather
     * pass and the local CSR build) */
    auto tiles_of = [&]() -> int {
        if (tile_first || !(P > 1 && m > 0))
            return CCGPU_OK;
        CC_TRY(cc_bufs_get(&B, (void **)&tile_first, (Lp.tiles + 1) * sizeof(uint32_t)));
        CC_KLAUNCH(ctx, CCK_DIST_TILES, k_tile_first, vb, kB, 0, st, Lp, (uint64_t)kTile, Lp.tiles,
                   tile_first);
        col_tiles = Lp.tiles;
        return CCGPU_OK;
    };
    uint64_t l_m = m;
    unsigned *rflags = nullptr;                     /* [0] a row descends, [1] repeats */
    unsigned long long *local_total = nullptr;
    uint32_t *roff = nullptr;
    uint64_t *rlb = nullptr, *rle = nullptr;
    LocalCCScratch ls;
    uint32_t *cur = nullptr, *nxt = nullptr, *hook = nullptr;
    unsigned long long *counters = nullptr; /* [0] keys [1] reps [2] roots [3] sent [4] raw [5] active reps [6] bad */
    CC_TRY(cc_bufs_get(&B, (void **)&cur, (size_t)n * sizeof(uint32_t)));
    CC_TRY(cc_bufs_get(&B, (void **)&nxt, (size_t)n * sizeof(uint32_t)));
    CC_TRY(cc_bufs_get(&B, (void **)&hook, (size_t)n * sizeof(uint32_t)));
    CC_TRY(cc_bufs_get(&B, (void **)&counters, 8 * sizeof(unsigned long long)));
    CC_TRY(cc_bufs_get(&B, (void **)&rflags, 2 * sizeof(unsigned)));
    uint64_t *keys = nullptr, *alt = nullptr;
    CC_TRY(cc_bufs_get(&B, (void **)&keys, (size_t)(m ? m : 1) * sizeof(uint64_t)));
    const int rb = bits_for(max_local - 1 ? max_local - 1 : 1);
    const int gb = bits_for(n - 1 ? n - 1 : 1);
    const int pb = P > 1 ? bits_for((uint64_t)P - 1) : 0;
    if (rb + gb + pb > 64)
        return ccgpu_set_error(CCGPU_ERR_LIMIT, "boundary key needs %d bits", rb + gb + pb);
    const unsigned sb = cc_blocks(n, kB, (unsigned)ctx->sm_count * 8);
    EmitParams E;
    unsigned long long hc[7];
    bool sorted_mode = false;
    bool run_masks = false; /* remote-end masks from the row runs, settled
                             * after the key sort by k_mask_fix */
    for (int pass = 0;; ++pass) {
        clk.n = 2 < clk.n ? 2 : clk.n; /* a second pass re-records phases 2-3 */
        const uint64_t *l_rp = d_row_ptr, *l_end = nullptr;
        const uint32_t *l_col = d_col;
        l_m = m;
        CC_CUDA(cudaMemsetAsync(rflags, 0, 2 * sizeof(unsigned), st));
        if (ranges) {
            if (!roff) {
                CC_TRY(cc_bufs_get(&B, (void **)&roff, (size_t)n * P * sizeof(uint32_t)));
                CC_TRY(cc_bufs_get(&B, (void **)&rlb, (size_t)n * sizeof(uint64_t)));
                CC_TRY(cc_bufs_get(&B, (void **)&rle, (size_t)n * sizeof(uint64_t)));
                /* [0] local entries, [1] symmetry sum */
                CC_TRY(cc_bufs_get(&B, (void **)&local_total, 2 * sizeof(unsigned long long)));
                CC_CUDA(cudaMemsetAsync(local_total, 0, 2 * sizeof(unsigned long long), st));
                /* the row holding each warp chunk's first entry */
                const uint64_t chunks = (m + kChunk - 1) / kChunk;
                uint32_t *chunk_first = nullptr;
                CC_TRY(cc_bufs_get(&B, (void **)&chunk_first, (chunks + 1) * sizeof(uint32_t)));
                CC_KLAUNCH(ctx, CCK_DIST_TILES, k_scan_prep, vb, kB, 0, st, d_row_ptr, n, m,
                           chunks, chunk_first);
                const unsigned scan_b = cc_blocks(chunks, kW, (unsigned)ctx->sm_count * 16);
#define CC_ROW_SCAN(PP)                                                                    \
    CC_KLAUNCH(ctx, CCK_DIST_LOCAL_COUNT, k_row_scan<PP>, scan_b, kB, 0, st, d_row_ptr, d_col, n, \
               m, bounds, Lp.vec, chunk_first, roff, rlb, rle, rflags, local_total,           \
               local_total + 1)
                switch (P) {
                case 2: CC_ROW_SCAN(2); break;
                case 3: CC_ROW_SCAN(3); break;
                case 4: CC_ROW_SCAN(4); break;
                case 5: CC_ROW_SCAN(5); break;
                case 6: CC_ROW_SCAN(6); break;
                case 7: CC_ROW_SCAN(7); break;
                default: CC_ROW_SCAN(8); break;
                }
#undef CC_ROW_SCAN
            }
            l_rp = rlb;
            l_end = rle;
        } else if (P > 1 && m > 0) {
            uint64_t *pcol = nullptr, *tile_off = nullptr;
            CC_TRY(cc_bufs_get(&B, (void **)&pcol, (P + 1) * sizeof(uint64_t)));
            CC_TRY(cc_bufs_get(&B, (void **)&Lp.tile_cnt, Lp.tiles * sizeof(uint32_t)));
            CC_TRY(cc_bufs_get(&B, (void **)&tile_off, (Lp.tiles + 1) * sizeof(uint64_t)));
            CC_TRY(cc_bufs_get(&B, (void **)&Lp.lrp, ((size_t)n + 1) * sizeof(uint64_t)));
            CC_KLAUNCH(ctx, CCK_DIST_TILES, k_part_cols, 1, 32, 0, st, d_row_ptr, m, bounds, P,
                       pcol);
            Lp.pcol = pcol;
            Lp.tile_off = tile_off;
            Lp.lcol = nullptr;
            const unsigned tb = cc_blocks(Lp.tiles, 1, (unsigned)ctx->sm_count * 8);
            CC_KLAUNCH(ctx, CCK_DIST_LOCAL_COUNT, k_local_count, tb, kB, 0, st, Lp);
            CC_TRY(tiles_of());
            Lp.tile_first = tile_first;
            wtiles = (m + kWarpTile - 1) / kWarpTile;
            CC_TRY(cc_bufs_get(&B, (void **)&wt_first, (wtiles + 1) * sizeof(uint32_t)));
            CC_KLAUNCH(ctx, CCK_DIST_TILES, k_tile_first, vb, kB, 0, st, Lp, (uint64_t)kWarpTile,
                       wtiles, wt_first);
            CC_TRY(cc_scan_u32(ctx, Lp.tile_cnt, tile_off, Lp.tiles, &B, st));
            CC_CUDA(cudaMemcpyAsync(&l_m, tile_off + Lp.tiles, sizeof(uint64_t),
                                    cudaMemcpyDeviceToHost, st));
            CC_CUDA(cudaStreamSynchronize(st));
            CC_TRY(cc_bufs_get(&B, (void **)&Lp.lcol,
                               (size_t)(l_m ? l_m : 1) * sizeof(uint32_t)));
            CC_KLAUNCH(ctx, CCK_DIST_LOCAL_FILL, k_local_fill, tb, kB, 0, st, Lp);
            l_rp = Lp.lrp;
            l_col = Lp.lcol;
        }
        LocalCCArgs a = {l_rp, l_col, n, ranges ? m : l_m, label, seg64, (uint32_t)P, ro, 0, 1,
                         l_end};
        {
            cc_carve c = {nullptr, 0};
            cc_local_carve(&c, &ls, a);
            void *base = nullptr;
            CC_TRY(cc_bufs_get(&B, &base, c.off));
            c = {(char *)base, 0};
            cc_local_carve(&c, &ls, a);
        }
        CC_TRY(cc_local_run(ctx, a, ls, st, 0, 0));
        CC_TRY(clock_mark(clk, st)); /* 2 */

        /* 3. reps and boundary keys */
        CC_CUDA(cudaMemsetAsync(counters, 0, 8 * sizeof(unsigned long long), st));
        CC_KLAUNCH(ctx, CCK_DIST_REPS, k_reps, sb, kB, 0, st, label, n, counters + 1,
                   cur, nxt, hook);
        E.row_ptr = d_row_ptr;
        E.col = d_col;
        E.vec = ((uintptr_t)d_col & 15) == 0;
        E.label = label;
        E.bounds = bounds;
        E.n = n;
        E.m = m;
        E.parts = P;
        E.rb = rb;
        E.gb = gb;
        E.out = keys;
        E.count = counters;
        E.tiles = col_tiles;
        E.tile_first = tile_first;
        E.raw = counters + 4;
        E.roff = ranges ? roff : nullptr;
        /* giant flags and per-vertex partition masks (P <= 32) */
        E.gflag = nullptr;
        E.pmask = nullptr;
        E.giants = nullptr;
        if (use_mask) {
            CC_TRY(cc_bufs_get(&B, (void **)&E.gflag, (((size_t)n + 31) / 32) * 4));
            CC_TRY(cc_bufs_get(&B, (void **)&E.pmask, (size_t)n * 4));
            if (!(ranges && P > 1 && P < 32)) /* else k_emit_ranges writes every word */
                CC_CUDA(cudaMemsetAsync(E.pmask, 0, (size_t)n * 4, st));
            E.giants = ls.giants;
            CC_KLAUNCH(ctx, CCK_DIST_GFLAG, k_giant_flags,
                       cc_blocks(n, kB, (unsigned)ctx->sm_count * 8), kB, 0, st, E);
        }
        /* Sorted-row mode (giant masks on): the local end writes the plain
         * keys and marks their mirror entries, the remote end reads the
         * marks instead of gathering gflag - from the partition runs
         * (k_emit_ranges) or by streaming the columns (k_emit_sorted).  The
         * rows must be strictly ascending and symmetric: the row check (or
         * k_emit_sorted) and the mirror search report it, and if not, the
         * pairs are made again by the gather pass alone. */
        E.ngbits = nullptr;
        E.bad = counters + 6;
        sorted_mode = use_mask && P > 1 && P < 32 && (ranges || col_tiles > 0);
        auto emit = [&]() -> int {
            const unsigned lb = cc_blocks(n, kB, (unsigned)ctx->sm_count * 8);
            if (E.roff) {
                /* row-run mode: the cut entries of every row, their sums
                 * per warp's 32 rows, a scan over the warps only (2M entries
                 * on C3 rather than one per row), and the emit pass; the remote
                 * end (k_emit_ranges, k_mask_fix) runs once the keys are
                 * sorted */
                const uint64_t nw = ((uint64_t)n + 31) / 32;
                uint32_t *cnt = nullptr, *wcnt = nullptr;
                uint64_t *woff = nullptr;
                CC_TRY(cc_bufs_get(&B, (void **)&cnt, (size_t)n * sizeof(uint32_t)));
                CC_TRY(cc_bufs_get(&B, (void **)&wcnt, (size_t)nw * sizeof(uint32_t)));
                CC_TRY(cc_bufs_get(&B, (void **)&woff, ((size_t)nw + 1) * sizeof(uint64_t)));
                if (P <= 4)
                    CC_KLAUNCH(ctx, CCK_DIST_PAIRS_LOCAL, k_ng_count<4>, lb, kB, 0, st, E, cnt);
                else
                    CC_KLAUNCH(ctx, CCK_DIST_PAIRS_LOCAL, k_ng_count<8>, lb, kB, 0, st, E, cnt);
                const unsigned wlb = cc_blocks(nw, kW, (unsigned)ctx->sm_count * 8);
                CC_KLAUNCH(ctx, CCK_DIST_PAIRS_LOCAL, k_warp_sums, wlb, kB, 0, st,
                           (const uint32_t *)cnt, (uint64_t)n, wcnt);
                CC_TRY(cc_scan_u32(ctx, wcnt, woff, nw, &B, st));
                if (P <= 4)
                    CC_KLAUNCH(ctx, CCK_DIST_PAIRS_LOCAL, k_ng_emit_runs<4>, wlb, kB, 0, st, E,
                               (const uint32_t *)cnt, (const uint64_t *)woff);
                else
                    CC_KLAUNCH(ctx, CCK_DIST_PAIRS_LOCAL, k_ng_emit_runs<8>, wlb, kB, 0, st, E,
                               (const uint32_t *)cnt, (const uint64_t *)woff);
                CC_CUDA(cudaMemcpyAsync(E.count, woff + nw, sizeof(unsigned long long),
                                        cudaMemcpyDeviceToDevice, st));
            } else if (E.ngbits) {
                uint32_t *cnt = nullptr;
                uint64_t *off = nullptr, *work = nullptr;
                CC_TRY(cc_bufs_get(&B, (void **)&cnt, (size_t)n * sizeof(uint32_t)));
                CC_TRY(cc_bufs_get(&B, (void **)&off, ((size_t)n + 1) * sizeof(uint64_t)));
                if (P <= 4)
                    CC_KLAUNCH(ctx, CCK_DIST_PAIRS_LOCAL, k_ng_count<4>, lb, kB, 0, st, E, cnt);
                else if (P <= 8)
                    CC_KLAUNCH(ctx, CCK_DIST_PAIRS_LOCAL, k_ng_count<8>, lb, kB, 0, st, E, cnt);
                else
                    CC_KLAUNCH(ctx, CCK_DIST_PAIRS_LOCAL, k_ng_count<CCGPU_MAX_PARTS>, lb, kB, 0,
                               st, E, cnt);
                CC_TRY(cc_scan_u32(ctx, cnt, off, n, &B, st));
                unsigned long long items = 0;
                CC_CUDA(cudaMemcpyAsync(&items, off + n, sizeof(items), cudaMemcpyDeviceToHost,
                                        st));
                CC_CUDA(cudaStreamSynchronize(st));
                CC_TRY(cc_bufs_get(&B, (void **)&work,
                                   (size_t)(items ? items : 1) * sizeof(uint64_t)));
                if (P <= 4)
                    CC_KLAUNCH(ctx, CCK_DIST_PAIRS_LOCAL, k_ng_emit<4>, lb, kB, 0, st, E, off,
                               work);
                else if (P <= 8)
                    CC_KLAUNCH(ctx, CCK_DIST_PAIRS_LOCAL, k_ng_emit<8>, lb, kB, 0, st, E, off,
                               work);
                else
                    CC_KLAUNCH(ctx, CCK_DIST_PAIRS_LOCAL, k_ng_emit<CCGPU_MAX_PARTS>, lb, kB, 0,
                               st, E, off, work);
                CC_CUDA(cudaMemcpyAsync(E.count, off + n, sizeof(unsigned long long),
                                        cudaMemcpyDeviceToDevice, st));
                CC_KLAUNCH(ctx, CCK_DIST_PAIRS_LOCAL, k_ng_mark, lb, kB, 0, st, E, work, off + n);
                const unsigned wb = cc_blocks(wtiles, kW, (unsigned)ctx->sm_count * 8);
                if (P <= 4)
                    CC_KLAUNCH(ctx, CCK_DIST_PAIRS, k_emit_sorted<4>, wb, kB, 0, st, E, wt_first,
                               wtiles);
                else if (P <= 8)
                    CC_KLAUNCH(ctx, CCK_DIST_PAIRS, k_emit_sorted<8>, wb, kB, 0, st, E, wt_first,
                               wtiles);
                else
                    CC_KLAUNCH(ctx, CCK_DIST_PAIRS, k_emit_sorted<CCGPU_MAX_PARTS>, wb, kB, 0,
                               st, E, wt_first, wtiles);
            } else {
                CC_TRY(tiles_of());
                E.tiles = col_tiles;
                E.tile_first = tile_first;
                const unsigned eb = cc_blocks(col_tiles, 1, (unsigned)ctx->sm_count * 4);
                if (P <= 4)
                    CC_KLAUNCH(ctx, CCK_DIST_PAIRS, k_emit<4>, eb, kB, 0, st, E);
                else if (P <= 8)
                    CC_KLAUNCH(ctx, CCK_DIST_PAIRS, k_emit<8>, eb, kB, 0, st, E);
                else
                    CC_KLAUNCH(ctx, CCK_DIST_PAIRS, k_emit<CCGPU_MAX_PARTS>, eb, kB, 0, st, E);
            }
            return CCGPU_OK;
        };
        run_masks = sorted_mode && ranges;
        if (sorted_mode && !ranges) {
            const size_t words = (size_t)((m + 31) / 32);
            CC_TRY(cc_bufs_get(&B, (void **)&E.ngbits, words * 4));
            CC_CUDA(cudaMemsetAsync(E.ngbits, 0, words * 4, st));
        }
        if (P > 1 && m > 0)
            CC_TRY(emit());
        unsigned hf[2] = {0, 0};
        unsigned long long hl[2] = {m, 0};
        CC_CUDA(cudaMemcpyAsync(hc, counters, 7 * sizeof(unsigned long long),
                                cudaMemcpyDeviceToHost, st));
        CC_CUDA(cudaMemcpyAsync(hf, rflags, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        if (ranges)
            CC_CUDA(cudaMemcpyAsync(hl, local_total, sizeof(hl), cudaMemcpyDeviceToHost, st));
        CC_CUDA(cudaStreamSynchronize(st));
        if (ranges)
            l_m = hl[0];
        if (ranges && hf[0]) {
            /* some row descends: its partition runs are not contiguous */
            ranges = false;
            continue;
        }
        /* the run counts need a symmetric graph, the mirror marks strictly
         * ascending rows with every mirror present */
        const bool redo = ranges ? (uint32_t)hl[1] != 0u : (hc[6] || hf[1]);
        if (sorted_mode && redo) {
            E.ngbits = nullptr;
            E.roff = nullptr;
            run_masks = false;
            CC_CUDA(cudaMemsetAsync(counters, 0, sizeof(unsigned long long), st));
            CC_CUDA(cudaMemsetAsync(counters + 4, 0, sizeof(unsigned long long), st));
            CC_CUDA(cudaMemsetAsync(counters + 6, 0, sizeof(unsigned long long), st));
            CC_CUDA(cudaMemsetAsync(E.pmask, 0, (size_t)n * 4, st));
            CC_TRY(emit());
            CC_CUDA(cudaMemcpyAsync(hc, counters, 7 * sizeof(unsigned long long),
                                    cudaMemcpyDeviceToHost, st));
            CC_CUDA(cudaStreamSynchronize(st));
            sorted_mode = false;
        }
        break;
    }
    S.sorted_rows = sorted_mode;
    S.row_runs = ranges;
    const uint64_t R = hc[0];
    S.boundary_raw = hc[4];
    S.sorted_keys = R;
    S.local_entries = l_m;
    S.rep_count = hc[1];
    CC_TRY(clock_mark(clk, st)); /* 3 */

    /* 4. sort the plain keys; the mask keys come out sorted and are merged
     * in */
    uint64_t *sorted = keys;
    if (R > 1) {
        CC_TRY(cc_bufs_get(&B, (void **)&alt, (size_t)R * sizeof(uint64_t)));
        CC_TRY(cc_radix_sort_u64(ctx, keys, alt, R, rb + gb + pb, &sorted, &S.sort_passes, &B,
                                 st));
    }
    uint64_t R_all = R;
    if (E.roff && run_masks) {
        /* row-run mode: a mask bit for every foreign run, cleared where the
         * sorted local-end keys cover the whole run */
        const unsigned lb = cc_blocks(n, kB, (unsigned)ctx->sm_count * 8);
        if (P <= 4)
            CC_KLAUNCH(ctx, CCK_DIST_PAIRS, k_emit_ranges<4>, lb, kB, 0, st, E);
        else
            CC_KLAUNCH(ctx, CCK_DIST_PAIRS, k_emit_ranges<8>, lb, kB, 0, st, E);
        if (R > 0)
            CC_KLAUNCH(ctx, CCK_DIST_PAIRS, k_mask_fix,
                       cc_blocks(R, kB, (unsigned)ctx->sm_count * 8), kB, 0, st,
                       (const uint64_t *)sorted, R, rb, gb, P, E.roff, E.pmask);
        unsigned long long raw = 0;
        CC_CUDA(cudaMemcpyAsync(&raw, counters + 4, sizeof(raw), cudaMemcpyDeviceToHost, st));
        CC_CUDA(cudaStreamSynchronize(st));
        S.boundary_raw = raw;
    }
    if (use_mask) {
        const uint32_t nblk = (uint32_t)(((uint64_t)n + kMaskBlock - 1) / kMaskBlock);
        uint32_t *mcnt = nullptr;
        uint64_t *moff = nullptr, *mkeys = nullptr, *merged = nullptr;
        CC_TRY(cc_bufs_get(&B, (void **)&mcnt, (size_t)P * nblk * sizeof(uint32_t)));
        CC_TRY(cc_bufs_get(&B, (void **)&moff, ((size_t)P * nblk + 1) * sizeof(uint64_t)));
        const unsigned mb = cc_blocks(nblk, 1, (unsigned)ctx->sm_count * 8);
        if (P <= 4)
            CC_KLAUNCH(ctx, CCK_DIST_PAIRS_BITMAP, k_mask_count<4>, mb, kB, 0, st, E, nblk, mcnt);
        else if (P <= 8)
            CC_KLAUNCH(ctx, CCK_DIST_PAIRS_BITMAP, k_mask_count<8>, mb, kB, 0, st, E, nblk, mcnt);
        else
            CC_KLAUNCH(ctx, CCK_DIST_PAIRS_BITMAP, k_mask_count<32>, mb, kB, 0, st, E, nblk,
                       mcnt);
        CC_TRY(cc_scan_u32(ctx, mcnt, moff, (uint64_t)P * nblk, &B, st));
        uint64_t M_keys = 0;
        CC_CUDA(cudaMemcpyAsync(&M_keys, moff + (uint64_t)P * nblk, sizeof(uint64_t),
                                cudaMemcpyDeviceToHost, st));
        CC_CUDA(cudaStreamSynchronize(st));
        if (M_keys) {
            CC_TRY(cc_bufs_get(&B, (void **)&mkeys, (size_t)M_keys * sizeof(uint64_t)));
            if (P <= 4)
                CC_KLAUNCH(ctx, CCK_DIST_PAIRS_BITMAP, k_mask_write<4>, mb, kB, 0, st, E, nblk,
                           (const uint64_t *)moff, mkeys);
            else if (P <= 8)
                CC_KLAUNCH(ctx, CCK_DIST_PAIRS_BITMAP, k_mask_write<8>, mb, kB, 0, st, E, nblk,
                           (const uint64_t *)moff, mkeys);
            else
                CC_KLAUNCH(ctx, CCK_DIST_PAIRS_BITMAP, k_mask_write<32>, mb, kB, 0, st, E, nblk,
                           (const uint64_t *)moff, mkeys);
            if (R > 0) {
                CC_TRY(cc_bufs_get(&B, (void **)&merged, (size_t)(R + M_keys) * sizeof(uint64_t)));
                const uint64_t tiles = (R + M_keys + kMergeTile - 1) / kMergeTile;
                uint64_t *split = nullptr;
                CC_TRY(cc_bufs_get(&B, (void **)&split, (tiles + 1) * sizeof(uint64_t)));
                CC_KLAUNCH(ctx, CCK_DIST_MERGE_KEYS, k_merge_splits,
                           cc_blocks(tiles + 1, kB, (unsigned)ctx->sm_count * 8), kB, 0, st, sorted,
                           R, mkeys, M_keys, tiles, split);
                CC_KLAUNCH(ctx, CCK_DIST_MERGE_KEYS, k_merge,
                           cc_blocks(tiles, 1, (unsigned)ctx->sm_count * 8), kB, 0, st, sorted, R,
                           mkeys, M_keys, (const uint64_t *)split, merged);
                sorted = merged;
            } else {
                sorted = mkeys;
            }
            R_all = R + M_keys;
        }
    }
    CC_TRY(clock_mark(clk, st)); /* 4 */

    /* 5. dedup, ghosts, plan */
    DedupParams D;
    memset(&D, 0, sizeof(D));
    D.keys = sorted;
    D.count = R_all;
    D.rb = rb;
    D.gb = gb;
    D.bounds = bounds;
    D.parts = P;
    uint64_t U = 0, G = 0;
    std::vector<uint64_t> gfirst(P, ~0ull);
    const uint64_t T = (R_all + kDedupTile - 1) / kDedupTile;
    uint64_t *gh_off = nullptr, *segs = nullptr;
    CC_TRY(cc_bufs_get(&B, (void **)&gh_off, (P + 1) * sizeof(uint64_t)));
    CC_TRY(cc_bufs_get(&B, (void **)&segs, (size_t)P * (P + 1) * sizeof(uint64_t)));
    CC_TRY(cc_bufs_get(&B, (void **)&D.gh_first, P * sizeof(uint64_t)));
    CC_CUDA(cudaMemsetAsync(D.gh_first, 0xff, P * sizeof(uint64_t), st));
    if (R_all > 0) {
        uint64_t *u_off = nullptr, *g_off = nullptr;
        CC_TRY(cc_bufs_get(&B, (void **)&D.tile_u, T * sizeof(uint32_t)));
        CC_TRY(cc_bufs_get(&B, (void **)&D.tile_g, T * sizeof(uint32_t)));
        CC_TRY(cc_bufs_get(&B, (void **)&u_off, (T + 1) * sizeof(uint64_t)));
        CC_TRY(cc_bufs_get(&B, (void **)&g_off, (T + 1) * sizeof(uint64_t)));
        CC_KLAUNCH(ctx, CCK_DIST_DEDUP, k_dedup_count, (unsigned)T, kB, 0, st, D);
        CC_TRY(cc_scan_u32(ctx, D.tile_u, u_off, T, &B, st));
        CC_TRY(cc_scan_u32(ctx, D.tile_g, g_off, T, &B, st));
        uint64_t tot[2];
        CC_CUDA(cudaMemcpyAsync(&tot[0], u_off + T, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
        CC_CUDA(cudaMemcpyAsync(&tot[1], g_off + T, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
        CC_CUDA(cudaStreamSynchronize(st));
        U = tot[0];
        G = tot[1];
        D.u_off = u_off;
        D.g_off = g_off;
    }
    S.pair_count = U;
    S.ghost_count = G;
    CC_TRY(cc_bufs_get(&B, (void **)&D.pair_rep, (size_t)(U ? U : 1) * sizeof(uint32_t)));
    CC_TRY(cc_bufs_get(&B, (void **)&D.pair_g, (size_t)(U ? U : 1) * sizeof(uint32_t)));
    CC_TRY(cc_bufs_get(&B, (void **)&D.ghost_v, (size_t)(G ? G : 1) * sizeof(uint32_t)));
    CC_TRY(cc_bufs_get(&B, (void **)&D.ghost_pairs, (size_t)(G + 1) * sizeof(uint64_t)));
    CC_TRY(cc_bufs_get(&B, (void **)&D.ghost_labels, (size_t)(G ? G : 1) * sizeof(uint32_t)));
    if (R_all > 0) {
        CC_KLAUNCH(ctx, CCK_DIST_GHOSTS, k_dedup_write, (unsigned)T, kB, 0, st, D);
        CC_CUDA(cudaMemcpyAsync(D.ghost_pairs + G, &U, sizeof(uint64_t), cudaMemcpyHostToDevice,
                                st));
    }
    CC_CUDA(cudaMemcpyAsync(gfirst.data(), D.gh_first, P * sizeof(uint64_t),
                            cudaMemcpyDeviceToHost, st));
    CC_CUDA(cudaStreamSynchronize(st));
    /* partition p's ghosts: [first ghost of p, first ghost of the next
     * partition that has any) */
    std::vector<uint64_t> hoff(P + 1, G);
    for (int p = P - 1; p >= 0; --p)
        hoff[p] = gfirst[p] != ~0ull ? gfirst[p] : hoff[p + 1];
    CC_CUDA(cudaMemcpyAsync(gh_off, hoff.data(), (P + 1) * sizeof(uint64_t),
                            cudaMemcpyHostToDevice, st));
    {
        int tot = P * (P + 1);
        CC_KLAUNCH(ctx, CCK_DIST_PLAN, k_plan, (tot + kB - 1) / kB, kB, 0, st, D.ghost_v, gh_off,
                   bounds, P, segs);
    }
    /* the merge's ghost lookups: a direct map when parts * n words fit in
     * the budget (one load per lookup, then the ghost's id and label
     * together), else id buckets of the ghost
     * lists (about 16 ids per bucket, at most ~64 MB in all) and a short
     * binary search */
    uint32_t *gmap = nullptr, *gbucket = nullptr;
    int gshift = 4;
    uint32_t gnb = 0;
    const uint64_t map_bytes = (uint64_t)P * n * sizeof(uint32_t);
    if (map_bytes <= ghost_map_budget()) {
        CC_TRY(cc_bufs_get(&B, (void **)&gmap, (size_t)map_bytes));
        if (G)
            CC_KLAUNCH(ctx, CCK_DIST_PLAN, k_ghost_map,
                       cc_blocks(G, kB, (unsigned)ctx->sm_count * 8), kB, 0, st, D.ghost_v,
                       gh_off, P, (uint64_t)n, gmap);
    } else {
        while (gshift < 31 && (uint64_t)P * ((n >> gshift) + 2) * 4 > (64ull << 20))
            ++gshift;
        gnb = (uint32_t)((n >> gshift) + 1);
        CC_TRY(cc_bufs_get(&B, (void **)&gbucket, (size_t)P * (gnb + 1) * sizeof(uint32_t)));
        CC_KLAUNCH(ctx, CCK_DIST_PLAN, k_ghost_buckets,
                   cc_blocks((uint64_t)P * (gnb + 1), kB, (unsigned)ctx->sm_count * 8), kB, 0,
                   st, D.ghost_v, gh_off, P, gnb, gshift, gbucket);
    }
    CC_TRY(clock_mark(clk, st)); /* 5 */
    if (o.verbose >= 2) {
        for (int p = 0; p < P; ++p)
            printf("[part %d] ghost_count=%llu\n", p, (unsigned long long)(hoff[p + 1] - hoff[p]));
        printf("[all] boundary_edges raw=%llu dedup=%llu reps=%llu sort_passes=%d\n",
               (unsigned long long)S.boundary_raw, (unsigned long long)U,
               (unsigned long long)S.rep_count,
               S.sort_passes);
    }

    /* 6. merge rounds, over the reps that own boundary pairs */
    MergeParams M;
    M.label = label;
    M.bounds = bounds;
    M.parts = P;
    M.rep_list = nullptr;
    M.rep_count = 0;
    M.hook = hook;
    M.pair_rep = D.pair_rep;
    M.pair_g = D.pair_g;
    M.pairs = U;
    M.ghost_v = D.ghost_v;
    M.ghost_pairs = D.ghost_pairs;
    M.ghost_labels = D.ghost_labels;
    M.ghosts = G;
    M.gh_off = gh_off;
    M.gmap = gmap;
    M.gbucket = gbucket;
    M.gnb = gnb;
    M.gshift = gshift;
    M.seg = segs;
    M.sent = counters + 3;
    CC_TRY(cc_bufs_get(&B, (void **)&M.delta, (size_t)(G ? G : 1) * sizeof(uint32_t)));
    CC_TRY(cc_bufs_get(&B, (void **)&M.delta_count, sizeof(uint32_t)));
    CC_TRY(cc_bufs_get(&B, (void **)&M.changed, P * sizeof(int)));
    CC_TRY(cc_bufs_get(&B, (void **)&M.ghost_rep, (size_t)(G ? G : 1) * sizeof(uint32_t)));
    M.ghost_rep_ready = 0;
    M.n = n;
    M.ctl = nullptr;
    CC_TRY(cc_bufs_get(&B, (void **)&M.dirty, (size_t)n));
    CC_CUDA(cudaMemsetAsync(M.dirty, 0, (size_t)n, st));
    const unsigned gbk = (unsigned)ctx->sm_count * 8;
    uint64_t act_count = 0;
    if (U > 0) {
        /* hook minima first: a rep owns a pair exactly when its hook left ~0
         * (ghost labels start as vertex ids) */
        M.cur = cur;
        M.next = nxt;
        CC_KLAUNCH(ctx, CCK_MERGE_HOOK, k_hook_init,
                   cc_blocks(U, (unsigned)(kB * kHookRounds), gbk), kB, 0, st, M);
        uint32_t *act = nullptr;
        CC_TRY(cc_bufs_get(&B, (void **)&act, (size_t)S.rep_count * sizeof(uint32_t) + 4));
        CC_CUDA(cudaMemsetAsync(counters + 5, 0, sizeof(unsigned long long), st));
        CC_KLAUNCH(ctx, CCK_MERGE_INIT, k_active_reps,
                   cc_blocks((n + kActiveV - 1) / kActiveV, kB, gbk), kB, 0, st, label, n, hook,
                   act, counters + 5);
        unsigned long long ac = 0;
        CC_CUDA(cudaMemcpyAsync(&ac, counters + 5, sizeof(ac), cudaMemcpyDeviceToHost, st));
        CC_CUDA(cudaStreamSynchronize(st));
        act_count = ac;
        M.rep_list = act;
        M.rep_count = act_count;
    }
    /* src/cc_mpi.c:538: merge only when some partition has ghosts, pairs
     * and reps; a partition with none joins the rounds and exchanges
     * without effect (the reference would stall there). */
    std::vector<int> pending(P, 0), changed(P, 0);
    int global_pending = (G > 0 && U > 0 && act_count > 0) ? 1 : 0;
    for (int p = 0; p < P; ++p)
        pending[p] = global_pending;
    int steps = 0;
    uint32_t *pc = cur, *pn = nxt;
    /* The host drives the first kHostRounds rounds (most merges end within
     * them, and a round costs the host one small read); a longer merge goes
     * on as one CUDA graph: a while node repeats k_upd, k_merge_ctl and the
     * exchange kernels (which return at once in a round without an
     * exchange) until the merge ends, the host reading the round state once
     * per launch of kLaunchRounds rounds at most. */
    constexpr int kHostRounds = 8;
    bool device_rounds = !ctx->prof && o.verbose < 2;
    while (global_pending) {
        if (device_rounds && S.rounds >= kHostRounds) {
            bool used = false;
            CC_TRY(merge_on_device(ctx, M, pc, pn, pending, steps, P, interval, act_count, G, U,
                                   n, &B, st, &pc, &S, &used));
            if (used)
                break;
            device_rounds = false;
        }
        M.cur = pc;
        M.next = pn;
        CC_CUDA(cudaMemsetAsync(M.changed, 0, P * sizeof(int), st));
        CC_KLAUNCH(ctx, CCK_MERGE_UPD, k_upd, cc_blocks(act_count, kB, gbk), kB, 0, st, M);
        CC_CUDA(cudaMemcpyAsync(changed.data(), M.changed, P * sizeof(int),
                                cudaMemcpyDeviceToHost, st));
        CC_CUDA(cudaStreamSynchronize(st));
        uint32_t *t = pc;
        pc = pn;
        pn = t;
        int any_changed = 0;
        global_pending = 0;
        for (int p = 0; p < P; ++p) {
            if (changed[p])
                pending[p] = 1;
            any_changed |= changed[p];
            global_pending |= pending[p];
        }
        S.rounds++;
        if (o.verbose >= 2 && (S.rounds <= 3 || S.rounds % 10 == 0))
            printf("[all] iter=%d pending=%d changed=%d\n", S.rounds, global_pending,
                   any_changed);
        if (!global_pending)
            break;
        steps++;
        if (steps >= interval || !any_changed) {
            M.cur = pc;
            CC_CUDA(cudaMemsetAsync(M.delta_count, 0, sizeof(uint32_t), st));
            CC_KLAUNCH(ctx, CCK_MERGE_EXCH_PACK, k_exchange,
                       cc_blocks(G, (unsigned)(kB * kExchRounds), gbk), kB, 0, st, M);
            M.ghost_rep_ready = 1;
            CC_KLAUNCH(ctx, CCK_MERGE_EXCH_SCATTER, k_delta_push, cc_blocks(G, kB, gbk), kB, 0,
                       st, M);
            CC_KLAUNCH(ctx, CCK_MERGE_EXCH_PULL, k_hook_pull,
                       cc_blocks(U, (unsigned)(kB * kHookRounds), gbk), kB, 0, st, M);
            CC_CUDA(cudaMemsetAsync(M.dirty, 0, (size_t)n, st));
            S.exchanges++;
            for (int p = 0; p < P; ++p)
                pending[p] = 0;
            steps = 0;
        }
    }
    CC_TRY(clock_mark(clk, st)); /* 6 */

    /* 7. labels and roots */
    CC_KLAUNCH(ctx, CCK_DIST_LABELS, k_final, sb, kB, 0, st, label, pc, n, d_labels, counters + 2);
    unsigned long long hr[2];
    CC_CUDA(cudaMemcpyAsync(hr, counters + 2, 2 * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, st));
    CC_TRY(clock_mark(clk, st)); /* 7 */
    CC_CUDA(cudaStreamSynchronize(st));
    S.roots = hr[0];
    S.sent_pairs = hr[1];
    if (clk.on) {
        float t[7] = {0};
        for (int i = 0; i < 7; ++i)
            CC_CUDA(cudaEventElapsedTime(&t[i], clk.ev[i], clk.ev[i + 1]));
        S.ms_bounds = t[0];
        S.ms_local = t[1];
        S.ms_pairs = t[2];
        S.ms_sort = t[3];
        S.ms_ghosts = t[4];
        S.ms_merge = t[5];
        float tot = 0;
        CC_CUDA(cudaEventElapsedTime(&tot, clk.ev[0], clk.ev[7]));
        S.ms_total = tot;
    }
    if (o.verbose >= 2)
        printf("[all] phases ms: bounds=%.3f local=%.3f pairs=%.3f sort=%.3f ghosts=%.3f "
               "merge=%.3f total=%.3f\n",
               S.ms_bounds, S.ms_local, S.ms_pairs, S.ms_sort, S.ms_ghosts, S.ms_merge,
               S.ms_total);
    if (o.verbose >= 1) { /* src/cc_mpi.c:712-713,741-742 */
        printf("CC merge converged in %d rounds\n", S.rounds);
        printf("Number of connected components: %llu\n", (unsigned long long)S.roots);
        fflush(stdout);
    }
    if (st_out)
        *st_out = S;
    return CCGPU_OK;
}

extern "C" int ccgpu_dist_cc(ccgpu_ctx *ctx, const uint64_t *d_row_ptr, const uint32_t *d_col_idx,
                             uint32_t n, uint64_t m, const ccgpu_dist_opts *opts,
                             uint32_t *d_labels, uint32_t *h_bounds, ccgpu_dist_stats *stats,
                             void *stream)
{
    ccgpu_dist_opts o;
    ccgpu_dist_opts_default(&o);
    if (opts)
        o = *opts;
    if (stats)
        memset(stats, 0, sizeof(*stats));
    if (o.parts < 1 || o.parts > CCGPU_MAX_PARTS)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_dist_cc: parts %d outside [1, %d]",
                               o.parts, CCGPU_MAX_PARTS);
    if (n == 0)
        return CCGPU_OK;
    if (!d_row_ptr || (m && !d_col_idx))
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_dist_cc: NULL row_ptr/col_idx");
    if ((uint32_t)o.parts > n)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_dist_cc: %d parts > %u vertices",
                               o.parts, n);
    if (n == 0xffffffffu)
        return ccgpu_set_error(CCGPU_ERR_LIMIT, "ccgpu_dist_cc: n must be below 2^32-1");
    CC_TRY(ccgpu_ctx_resolve(&ctx));
    cudaStream_t st = (cudaStream_t)stream;
    DevBufs B;
    CC_TRY(cc_bufs_init(&B, st));
    int rc = dist_run(ctx, d_row_ptr, d_col_idx, n, m, o, d_labels, h_bounds, stats, st, B);
    if (rc != CCGPU_OK)
        cudaStreamSynchronize(st);
    cc_bufs_release(&B);
    return rc;
}

/* ----------------------------------------------------- pair sort / dedup */

namespace {

/* {rep, remote} as one little-endian u64 is remote << 32 | rep: the
 * reference's key.  Compact it to (remote << rb | rep) for the sort and
 * back afterwards. */
__global__ void k_pairs_pack(uint64_t *p, uint64_t count, int rb)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        uint64_t x = p[i];
        p[i] = ((x >> 32) << rb) | (x & 0xffffffffull);
    }
}

__global__ void k_pairs_unpack(const uint64_t *src, uint64_t *dst, uint64_t count, int rb)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t rmask = (1ull << rb) - 1ull;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        uint64_t x = src[i];
        dst[i] = ((x >> rb) << 32) | (x & rmask);
    }
}

__global__ void k_flag_new(const uint64_t *p, uint64_t count, uint32_t *flag)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride)
        flag[i] = (i == 0 || p[i] != p[i - 1]) ? 1u : 0u;
}

__global__ void k_compact(const uint64_t *src, const uint64_t *pos, uint64_t count, uint64_t *dst)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride)
        if (pos[i + 1] != pos[i])
            dst[pos[i]] = src[i];
}

} // namespace

extern "C" int ccgpu_boundary_sort(ccgpu_ctx *ctx, uint32_t *d_pairs, uint64_t count,
                                   uint32_t max_rep, uint32_t max_remote, void *stream)
{
    if (count <= 1)
        return CCGPU_OK;
    if (!d_pairs)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_boundary_sort: NULL pairs");
    if (((uintptr_t)d_pairs & 7) != 0)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_boundary_sort: pairs not 8-byte aligned");
    CC_TRY(ccgpu_ctx_resolve(&ctx));
    cudaStream_t st = (cudaStream_t)stream;
    const int rb = bits_for(max_rep), gb = bits_for(max_remote);
    uint64_t *p = (uint64_t *)d_pairs;
    DevBufs B;
    CC_TRY(cc_bufs_init(&B, st));
    int rc = CCGPU_OK;
    do {
        uint64_t *alt = nullptr, *sorted = nullptr;
        if ((rc = cc_bufs_get(&B, (void **)&alt, count * sizeof(uint64_t))) != CCGPU_OK)
            break;
        const unsigned blocks = cc_blocks(count, 256, (unsigned)ctx->sm_count * 8);
        k_pairs_pack<<<blocks, 256, 0, st>>>(p, count, rb);
        ctx->launches++;
        if ((rc = cc_radix_sort_u64(ctx, p, alt, count, rb + gb, &sorted, nullptr, &B, st)) !=
            CCGPU_OK)
            break;
        k_pairs_unpack<<<blocks, 256, 0, st>>>(sorted, p, count, rb);
        ctx->launches++;
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(st);
        if (e != cudaSuccess)
            rc = ccgpu_cuda_fail(e, "boundary sort", __FILE__, __LINE__);
    } while (0);
    cc_bufs_release(&B);
    return rc;
}

extern "C" int ccgpu_sort_keys(ccgpu_ctx *ctx, uint64_t *d_keys, uint64_t *d_alt, uint64_t count,
                               int bits, int *in_alt, void *stream)
{
    if (in_alt)
        *in_alt = 0;
    if (count <= 1)
        return CCGPU_OK;
    if (!d_keys || !d_alt)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_sort_keys: NULL buffer");
    CC_TRY(ccgpu_ctx_resolve(&ctx));
    cudaStream_t st = (cudaStream_t)stream;
    DevBufs B;
    CC_TRY(cc_bufs_init(&B, st));
    uint64_t *sorted = d_keys;
    int rc = cc_radix_sort_u64(ctx, d_keys, d_alt, count, bits, &sorted, nullptr, &B, st);
    cc_bufs_release(&B);
    if (in_alt)
        *in_alt = sorted == d_alt;
    return rc;
}

extern "C" int ccgpu_unique_keys(ccgpu_ctx *ctx, const uint64_t *d_keys, uint64_t count,
                                 uint64_t *d_out, uint64_t *out_count, void *stream)
{
    if (!out_count)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_unique_keys: out_count is NULL");
    *out_count = 0;
    if (count == 0)
        return CCGPU_OK;
    if (!d_keys || !d_out)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_unique_keys: NULL buffer");
    CC_TRY(ccgpu_ctx_resolve(&ctx));
    cudaStream_t st = (cudaStream_t)stream;
    DevBufs B;
    CC_TRY(cc_bufs_init(&B, st));
    int rc = CCGPU_OK;
    do {
        uint32_t *flag = nullptr;
        uint64_t *pos = nullptr;
        if ((rc = cc_bufs_get(&B, (void **)&flag, count * sizeof(uint32_t))) != CCGPU_OK ||
            (rc = cc_bufs_get(&B, (void **)&pos, (count + 1) * sizeof(uint64_t))) != CCGPU_OK)
            break;
        const unsigned blocks = cc_blocks(count, 256, (unsigned)ctx->sm_count * 8);
        k_flag_new<<<blocks, 256, 0, st>>>(d_keys, count, flag);
        ctx->launches++;
        if ((rc = cc_scan_u32(ctx, flag, pos, count, &B, st)) != CCGPU_OK)
            break;
        k_compact<<<blocks, 256, 0, st>>>(d_keys, pos, count, d_out);
        ctx->launches++;
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(out_count, pos + count, sizeof(uint64_t), cudaMemcpyDeviceToHost,
                                st);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(st);
        if (e != cudaSuccess)
            rc = ccgpu_cuda_fail(e, "ccgpu_unique_keys", __FILE__, __LINE__);
    } while (0);
    cc_bufs_release(&B);
    return rc;
}

extern "C" int ccgpu_boundary_dedup(ccgpu_ctx *ctx, uint32_t *d_pairs, uint64_t count,
                                    uint64_t *new_count, void *stream)
{
    if (!new_count)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_boundary_dedup: new_count is NULL");
    *new_count = count;
    if (count <= 1)
        return CCGPU_OK;
    if (!d_pairs)
        return ccgpu_set_error(CCGPU_ERR_INVALID, "ccgpu_boundary_dedup: NULL pairs");
    CC_TRY(ccgpu_ctx_resolve(&ctx));
    cudaStream_t st = (cudaStream_t)stream;
    uint64_t *p = (uint64_t *)d_pairs;
    DevBufs B;
    CC_TRY(cc_bufs_init(&B, st));
    int rc = CCGPU_OK;
    do {
        uint32_t *flag = nullptr;
        uint64_t *pos = nullptr, *tmp = nullptr;
        if ((rc = cc_bufs_get(&B, (void **)&flag, count * sizeof(uint32_t))) != CCGPU_OK ||
            (rc = cc_bufs_get(&B, (void **)&pos, (count + 1) * sizeof(uint64_t))) != CCGPU_OK ||
            (rc = cc_bufs_get(&B, (void **)&tmp, count * sizeof(uint64_t))) != CCGPU_OK)
            break;
        const unsigned blocks = cc_blocks(count, 256, (unsigned)ctx->sm_count * 8);
        k_flag_new<<<blocks, 256, 0, st>>>(p, count, flag);
        ctx->launches++;
        if ((rc = cc_scan_u32(ctx, flag, pos, count, &B, st)) != CCGPU_OK)
            break;
        k_compact<<<blocks, 256, 0, st>>>(p, pos, count, tmp);
        ctx->launches++;
        uint64_t kept = 0;
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&kept, pos + count, sizeof(uint64_t), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(p, tmp, kept * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            rc = ccgpu_cuda_fail(e, "boundary dedup", __FILE__, __LINE__);
            break;
        }
        *new_count = kept;
    } while (0);
    cc_bufs_release(&B);
    return rc;
}
