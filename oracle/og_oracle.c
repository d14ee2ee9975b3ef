/*
 * og_oracle.c -- CPU restatement of the OpenGraph CSR hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see og_oracle.h).  Written from the reference's
 * algorithm, not its code: sequential, one pass per digit-free counting sort,
 * explicit integer types.  Built with -ffp-contract=off semantics kept by
 * hand (every float product and sum is a separate statement).
 */
#include "og_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ sort -- */

/* Stable counting sort by one u32 key (keys need not be dense: a 16-bit LSD
 * two-pass counting sort keeps memory bounded). */
static void sort_by_key(uint32_t E, const uint32_t *key, const uint32_t *pa, const uint32_t *pb,
                        uint32_t *okey, uint32_t *oa, uint32_t *ob)
{
    uint32_t *k1 = malloc((size_t)E * 4 + 4), *a1 = malloc((size_t)E * 4 + 4), *b1 = malloc((size_t)E * 4 + 4);
    uint64_t *cnt = malloc(sizeof(uint64_t) * 65537);
    const uint32_t *ik = key, *ia = pa, *ib = pb;
    uint32_t *tk = k1, *ta = a1, *tb = b1;
    for (int pass = 0; pass < 2; pass++)
    {
        const int sh = pass * 16;
        if (pass == 1)
        {
            tk = okey; ta = oa; tb = ob;
        }
        memset(cnt, 0, sizeof(uint64_t) * 65537);
        for (uint32_t i = 0; i < E; i++) cnt[((ik[i] >> sh) & 0xFFFF) + 1]++;
        for (int d = 0; d < 65536; d++) cnt[d + 1] += cnt[d];
        for (uint32_t i = 0; i < E; i++)
        {
            const uint64_t p = cnt[(ik[i] >> sh) & 0xFFFF]++;
            tk[p] = ik[i];
            ta[p] = ia[i];
            if (ib) tb[p] = ib[i];
        }
        ik = k1; ia = a1; ib = pb ? b1 : NULL;
    }
    free(k1); free(a1); free(b1); free(cnt);
}

void orc_sort(uint32_t E, const uint32_t *src, const uint32_t *dst, const float *w, int mode,
              uint32_t *osrc, uint32_t *odst, float *ow)
{
    const uint32_t *wb = (const uint32_t *)w;
    uint32_t *owb = (uint32_t *)ow;
    if (mode == 0)
    {
        sort_by_key(E, src, dst, wb, osrc, odst, owb);
    }
    else if (mode == 2)
    {
        sort_by_key(E, dst, src, wb, odst, osrc, owb);
    }
    else
    {
        /* by dst first, then stably by src: lexicographic (src, dst) */
        uint32_t *ts = malloc((size_t)E * 4 + 4), *td = malloc((size_t)E * 4 + 4), *tw = w ? malloc((size_t)E * 4 + 4) : NULL;
        sort_by_key(E, dst, src, wb, td, ts, tw);
        sort_by_key(E, ts, td, tw, osrc, odst, owb);
        free(ts); free(td); free(tw);
    }
}

int orc_csr_map(uint32_t E, uint32_t V, const uint32_t *s, uint32_t *out_degree, uint32_t *edges_idx)
{
    memset(out_degree, 0, (size_t)V * 4);
    memset(edges_idx, 0, (size_t)V * 4);
    for (uint32_t i = 0; i < E; i++)
    {
        if (s[i] >= V) return -1;
        if (i == 0 || s[i] != s[i - 1]) edges_idx[s[i]] = i;
        out_degree[s[i]]++;
    }
    return 0;
}

int orc_build(uint32_t E, uint32_t V, const uint32_t *src, const uint32_t *dst, const float *w, int sort_type,
              uint32_t *f_src, uint32_t *f_dst, float *f_w, uint32_t *f_outdeg, uint32_t *f_indeg, uint32_t *f_idx,
              uint32_t *i_src, uint32_t *i_dst, float *i_w, uint32_t *i_outdeg, uint32_t *i_indeg, uint32_t *i_idx)
{
    const int mode = (sort_type == 1 || sort_type == 3) ? 1 : 0;
    orc_sort(E, src, dst, w, mode, f_src, f_dst, w ? f_w : NULL);
    if (orc_csr_map(E, V, f_src, f_outdeg, f_idx)) return -1;
    /* inverse list = sorted forward list with src/dst swapped, sorted again */
    orc_sort(E, f_dst, f_src, w ? f_w : NULL, mode, i_src, i_dst, w ? i_w : NULL);
    if (orc_csr_map(E, V, i_src, i_outdeg, i_idx)) return -1;
    memcpy(i_indeg, f_outdeg, (size_t)V * 4);
    memcpy(f_indeg, i_outdeg, (size_t)V * 4);
    return 0;
}

uint32_t orc_dedup(uint32_t E, const uint32_t *s, const uint32_t *d, const float *w, uint32_t *os, uint32_t *od,
                   float *ow, int truncate_w)
{
    uint32_t n = 0;
    for (uint32_t i = 0; i < E; i++)
    {
        if (s[i] == d[i]) continue;
        if (n > 0 && os[n - 1] == s[i] && od[n - 1] == d[i]) continue;
        os[n] = s[i];
        od[n] = d[i];
        if (w) ow[n] = truncate_w ? (float)(uint32_t)w[i] : w[i];
        n++;
    }
    return n;
}

/* ------------------------------------------------------------------- BFS -- */

int orc_bfs(uint32_t V, uint32_t E, const uint32_t *f_outdeg, const uint32_t *f_idx, const uint32_t *f_dst,
            const uint32_t *i_outdeg, const uint32_t *i_idx, const uint32_t *i_dst, uint32_t root, int mode,
            int bu_entry_nf_frontier, int32_t *parents, uint32_t *dist, orc_bfs_stats *st, uint8_t *dirs,
            uint32_t max_dirs)
{
    if (root >= V) return -1;
    for (uint32_t v = 0; v < V; v++)
    {
        parents[v] = f_outdeg[v] ? -(int32_t)f_outdeg[v] : -1;
        dist[v] = 0;
    }
    uint32_t *q = malloc((size_t)V * 4 + 4), *nq = malloc((size_t)V * 4 + 4);
    uint8_t *cur = calloc(V + 1, 1), *nxt = calloc(V + 1, 1);
    uint32_t qn = 1, step = 0;
    q[0] = root;
    parents[root] = (int32_t)root;
    uint32_t mu = E, mf = f_outdeg[root], nf = 0, nf_prev = 0;
    const uint32_t alpha = 15, beta = 18;
    orc_bfs_stats s = {1, 1, 0, 0, 0, 0};
    while (qn > 0)
    {
        const int bu = (mode == 0) || (mode == 2 && mf > mu / alpha);
        if (bu)
        {
            memset(cur, 0, V);
            for (uint32_t i = 0; i < qn; i++) cur[q[i]] = 1;
            nf = bu_entry_nf_frontier ? qn : 0;
            do
            {
                nf_prev = nf;
                nf = 0;
                memset(nxt, 0, V);
                for (uint32_t v = 0; v < V; v++)
                {
                    if (parents[v] >= 0) continue;
                    for (uint32_t j = i_idx[v]; j < i_idx[v] + i_outdeg[v]; j++)
                    {
                        const uint32_t u = i_dst[j] & 0x3FFFFFFFu;
                        if (cur[u])
                        {
                            parents[v] = (int32_t)u;
                            dist[v] = dist[u] + 1;
                            nxt[v] = 1;
                            nf++;
                            break;
                        }
                    }
                }
                uint8_t *t = cur; cur = nxt; nxt = t;
                s.iteration++;
                s.processed_nodes += nf;
                s.bu_steps++;
                if (dirs && step < max_dirs) dirs[step] = 1;
                step++;
            } while (mode == 0 ? (nf > 0) : ((nf > nf_prev) || (nf > V / beta)));
            qn = 0;
            for (uint32_t v = 0; v < V; v++)
                if (cur[v]) q[qn++] = v;
            mf = 1;
        }
        else
        {
            mu -= mf;
            mf = 0;
            uint32_t nn = 0;
            for (uint32_t i = 0; i < qn; i++)
            {
                const uint32_t v = q[i];
                for (uint32_t j = f_idx[v]; j < f_idx[v] + f_outdeg[v]; j++)
                {
                    const uint32_t u = f_dst[j] & 0x3FFFFFFFu;
                    if (parents[u] < 0)
                    {
                        mf += (uint32_t)(-parents[u]);
                        parents[u] = (int32_t)v;
                        dist[u] = dist[v] + 1;
                        nq[nn++] = u;
                    }
                }
            }
            uint32_t *t = q; q = nq; nq = t;
            qn = nn;
            s.iteration++;
            s.processed_nodes += nn;
            s.td_steps++;
            if (dirs && step < max_dirs) dirs[step] = 0;
            step++;
        }
    }
    for (uint32_t v = 0; v < V; v++)
        if (parents[v] >= 0)
        {
            s.reached++;
            s.reached_out_edges += f_outdeg[v];
        }
    if (st) *st = s;
    free(q); free(nq); free(cur); free(nxt);
    return 0;
}

/* -------------------------------------------------------------- PageRank -- */

/* Reduction order of the GPU pull kernel (mode 2 of orc_pagerank): rows with
 * in-degree <= warp_thr are summed sequentially; rows above it by 32 lanes
 * (lane l sums edges l, l+32, ... in order) folded by the butterfly
 * s_l + s_(l^o), o = 16..1; rows above cta_thr are cut into chunks of `chunk`
 * edges, each chunk summed by cta_threads threads (each warp folded the same
 * way, then the warp results summed in warp order), and the chunk sums added
 * in chunk order. */
static uint32_t g_warp_thr = 32, g_cta_thr = 2048, g_cta_threads = 256, g_chunk = 8192;

void orc_set_gpu_order(uint32_t warp_thr, uint32_t cta_thr, uint32_t cta_threads, uint32_t chunk)
{
    g_warp_thr = warp_thr;
    g_cta_thr = cta_thr;
    g_cta_threads = cta_threads;
    g_chunk = chunk ? chunk : 0xFFFFFFFFu;
}

static float tree_sum(const float *c, const uint32_t *nbr, uint32_t a, uint32_t d, uint32_t T)
{
    float part[1024];
    for (uint32_t t = 0; t < T; t++)
    {
        float s = 0.0f;
        for (uint32_t j = a + t; j < a + d; j += T) s += c[nbr[j] & 0x3FFFFFFFu];
        part[t] = s;
    }
    for (uint32_t w = 0; w < T / 32; w++)
    {
        float *p = part + w * 32;
        for (uint32_t o = 16; o; o >>= 1)
        {
            float q[32];
            for (uint32_t l = 0; l < 32; l++) q[l] = p[l] + p[l ^ o];
            memcpy(p, q, sizeof(q));
        }
    }
    if (T == 32) return part[0];
    float tot = 0.0f;
    for (uint32_t w = 0; w < T / 32; w++) tot += part[w * 32];
    return tot;
}

uint32_t orc_pagerank(uint32_t V, const uint32_t *f_outdeg, const uint32_t *f_idx, const uint32_t *f_dst,
                      const uint32_t *i_outdeg, const uint32_t *i_idx, const uint32_t *i_dst, int mode,
                      uint32_t max_iters, double epsilon, const float *init, float *pr,
                      uint32_t *iterations_out, double *error_out, double *err_hist, uint32_t *active_hist)
{
    const float damp = 0.85f;
    const float base_pr = 1.0f - damp;
    float *contrib = malloc((size_t)V * 4 + 4), *next = calloc((size_t)V + 1, 4);
    for (uint32_t v = 0; v < V; v++) pr[v] = init ? init[v] : base_pr;
    uint32_t it, executed = 0;
    double error_total = 0.0;
    for (it = 0; it < max_iters; it++)
    {
        error_total = 0.0;
        uint32_t active = 0;
        for (uint32_t v = 0; v < V; v++)
            contrib[v] = f_outdeg[v] ? pr[v] / (float)f_outdeg[v] : 0.0f;
        if (mode == 0)
        {
            for (uint32_t v = 0; v < V; v++)
            {
                float s = 0.0f;
                for (uint32_t j = i_idx[v]; j < i_idx[v] + i_outdeg[v]; j++) s += contrib[i_dst[j] & 0x3FFFFFFFu];
                next[v] = s;
            }
        }
        else if (mode == 2)
        {
            for (uint32_t v = 0; v < V; v++)
            {
                const uint32_t d = i_outdeg[v];
                if (d > g_cta_thr)
                {
                    float tot = 0.0f;
                    for (uint32_t c = 0; c < d; c += g_chunk)
                    {
                        const uint32_t len = (d - c < g_chunk) ? d - c : g_chunk;
                        tot += tree_sum(contrib, i_dst, i_idx[v] + c, len, g_cta_threads);
                    }
                    next[v] = tot;
                }
                else if (d > g_warp_thr)
                    next[v] = tree_sum(contrib, i_dst, i_idx[v], d, 32);
                else
                {
                    float s = 0.0f;
                    for (uint32_t j = i_idx[v]; j < i_idx[v] + d; j++) s += contrib[i_dst[j] & 0x3FFFFFFFu];
                    next[v] = s;
                }
            }
        }
        else
        {
            for (uint32_t v = 0; v < V; v++)
                for (uint32_t j = f_idx[v]; j < f_idx[v] + f_outdeg[v]; j++) next[f_dst[j] & 0x3FFFFFFFu] += contrib[v];
        }
        for (uint32_t v = 0; v < V; v++)
        {
            const float prev = pr[v];
            const float scaled = damp * next[v];
            const float nv = base_pr + scaled;
            pr[v] = nv;
            next[v] = 0.0f;
            const float diff = nv - prev;
            const double e = fabs((double)diff);
            error_total += e / V;
            if (e >= epsilon) active++;
        }
        if (err_hist) err_hist[executed] = error_total;
        if (active_hist) active_hist[executed] = active;
        executed++;
        if (active == 0) break;
    }
    for (uint32_t v = 0; v < V; v++) pr[v] = pr[v] / (float)V;
    if (iterations_out) *iterations_out = it;
    if (error_out) *error_out = error_total;
    free(contrib);
    free(next);
    return executed;
}

void orc_pagerank_f64(uint32_t V, const uint32_t *f_outdeg, const uint32_t *i_outdeg, const uint32_t *i_idx,
                      const uint32_t *i_dst, uint32_t iters, const double *init, double *pr)
{
    const double damp = 0.85, base_pr = 1.0 - damp;
    double *contrib = malloc((size_t)V * 8 + 8);
    for (uint32_t v = 0; v < V; v++) pr[v] = init ? init[v] : base_pr;
    for (uint32_t it = 0; it < iters; it++)
    {
        for (uint32_t v = 0; v < V; v++) contrib[v] = f_outdeg[v] ? pr[v] / f_outdeg[v] : 0.0;
        for (uint32_t v = 0; v < V; v++)
        {
            double s = 0.0;
            for (uint32_t j = i_idx[v]; j < i_idx[v] + i_outdeg[v]; j++) s += contrib[i_dst[j] & 0x3FFFFFFFu];
            pr[v] = base_pr + damp * s;
        }
    }
    for (uint32_t v = 0; v < V; v++) pr[v] /= V;
    free(contrib);
}

/* ------------------------------------------------------------------ roots -- */

/* MT19937 (Matsumoto & Nishimura 1998) with the LCG seeding x -> 69069x + 1. */
typedef struct { uint32_t mt[624]; int mti; } orc_mt;

static void orc_mt_seed(orc_mt *m, uint32_t seed)
{
    uint64_t x = seed; /* the reference keeps 64-bit state; only the low 32 bits matter */
    for (int i = 0; i < 624; i++)
    {
        uint32_t hi = (uint32_t)(x & 0xffff0000u);
        x = 69069u * x + 1u;
        uint32_t lo = (uint32_t)((x & 0xffff0000u) >> 16);
        x = 69069u * x + 1u;
        m->mt[i] = hi | lo;
    }
    m->mti = 624;
}

static uint32_t orc_mt_next(orc_mt *m)
{
    if (m->mti >= 624)
    {
        for (int k = 0; k < 624; k++)
        {
            uint32_t y = (m->mt[k] & 0x80000000u) | (m->mt[(k + 1) % 624] & 0x7fffffffu);
            m->mt[k] = m->mt[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        m->mti = 0;
    }
    uint32_t y = m->mt[m->mti++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

void orc_random_roots(uint32_t seed, uint32_t V, uint32_t avg_degree, const uint32_t *out_degree, uint32_t n,
                      uint32_t *roots)
{
    orc_mt m;
    orc_mt_seed(&m, seed);
    for (uint32_t k = 0; k < n; k++)
    {
        for (;;)
        {
            const uint32_t s = orc_mt_next(&m);
            if (s < V && out_degree[s] > avg_degree)
            {
                roots[k] = s;
                break;
            }
        }
    }
}

/* ------------------------------------------------------------- inputs -- */

/* The benchmark's synthetic RMAT input, restated here so that the timed
 * reference arm can make its .wbin file without loading the product library.
 * Every draw is SplitMix64's finalizer (Steele, Lea, Flood 2014) of (seed,
 * edge index, level); quadrant a/b/c/d per level from a 53-bit uniform; ids
 * relabelled by a seeded Fisher-Yates permutation; weights uniform in
 * [1, 256).  Must equal the product's generator bit for bit (tested). */
static uint64_t orc_mix64(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static uint64_t orc_draw(uint64_t seed, uint64_t index, uint64_t k)
{
    return orc_mix64(orc_mix64(seed ^ (k * 0xD1B54A32D192ED03ull)) ^ index);
}

int orc_generate_rmat(uint32_t scale, uint32_t edge_factor, uint64_t seed, double a, double b, double c,
                      int permute, uint32_t *src, uint32_t *dst, float *w)
{
    if (scale == 0 || scale > 30) return -1;
    const uint64_t V = 1ull << scale, E = V * edge_factor;
    if (E > 0xFFFFFFFFull) return -1;
    uint32_t *perm = NULL;
    if (permute)
    {
        perm = malloc(V * 4);
        for (uint64_t i = 0; i < V; i++) perm[i] = (uint32_t)i;
        uint64_t state = orc_mix64(seed ^ 0xA5A5A5A5ull);
        for (uint64_t i = V; i > 1; i--)
        {
            state = orc_mix64(state);
            const uint32_t j = (uint32_t)(((unsigned __int128)state * i) >> 64);
            const uint32_t t = perm[i - 1];
            perm[i - 1] = perm[j];
            perm[j] = t;
        }
    }
    /* per-level keys do not depend on the edge: hoist them */
    uint64_t key[32];
    for (uint32_t l = 0; l < scale; l++) key[l] = orc_mix64(seed ^ ((uint64_t)l * 0xD1B54A32D192ED03ull));
    const double ab = a + b, abc = a + b + c;
    /* edges are independent draws: the only parallel loop of the oracle */
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < E; i++)
    {
        uint32_t u = 0, v = 0;
        for (uint32_t l = 0; l < scale; l++)
        {
            const double r = (double)(orc_mix64(key[l] ^ i) >> 11) * (1.0 / 9007199254740992.0);
            const uint32_t bu = r >= ab;
            const uint32_t bv = (r >= a && r < ab) || r >= abc;
            u = (u << 1) | bu;
            v = (v << 1) | bv;
        }
        if (perm)
        {
            u = perm[u];
            v = perm[v];
        }
        src[i] = u;
        dst[i] = v;
        if (w)
        {
            const double x = (double)(orc_draw(seed ^ 0x5713ull, i, 0xFFFF) >> 40) * (1.0 / 16777216.0);
            w[i] = (float)(1.0 + 255.0 * x);
        }
    }
    free(perm);
    return 0;
}

/* ------------------------------------------------ data-driven PageRank -- */

/* Row sum of c[] over in-row [a, a + d) in the GPU kernels' order (the
 * split of orc_set_gpu_order), or sequentially in CSR order. */
static float row_sum(const float *c, const uint32_t *nbr, uint32_t a, uint32_t d, int gpu_order)
{
    if (gpu_order && d > g_cta_thr)
    {
        float tot = 0.0f;
        for (uint32_t k = 0; k < d; k += g_chunk)
        {
            const uint32_t len = (d - k < g_chunk) ? d - k : g_chunk;
            tot += tree_sum(c, nbr, a + k, len, g_cta_threads);
        }
        return tot;
    }
    if (gpu_order && d > g_warp_thr) return tree_sum(c, nbr, a, d, 32);
    float s = 0.0f;
    for (uint32_t j = a; j < a + d; j++) s += c[nbr[j] & 0x3FFFFFFFu];
    return s;
}

/* pageRankDataDrivenPullGraphCSR (pageRank.c:2405-2564, mode 6),
 * pageRankDataDrivenPushGraphCSR (:2566-2721, mode 7) and
 * pageRankDataDrivenPullPushGraphCSR (:2723-2919, mode 8), run
 * sequentially in vertex order (the reference's loops with one thread).
 * gpu_order (mode 6 only) sums long in-rows in the GPU kernels' order. */
uint32_t orc_pagerank_dd(uint32_t V, const uint32_t *f_outdeg, const uint32_t *f_idx, const uint32_t *f_dst,
                         const uint32_t *i_outdeg, const uint32_t *i_idx, const uint32_t *i_dst, int mode,
                         int gpu_order, uint32_t max_iters, double epsilon, float *pr, uint32_t *iterations_out,
                         double *error_out, uint32_t *active_hist)
{
    const float damp = 0.85f;
    const float base_pr = 1.0f - damp;
    uint8_t *cur = malloc((size_t)V + 1), *next = malloc((size_t)V + 1);
    float *c = malloc((size_t)V * 4 + 4), *res = malloc((size_t)V * 4 + 4);
    for (uint32_t v = 0; v < V; v++)
    {
        pr[v] = base_pr;
        cur[v] = 1;
        next[v] = 0;
    }
    if (mode != 6)
    {
        /* residuals: (1 - d) d * sum over in-neighbours of 1 / out_degree */
        for (uint32_t v = 0; v < V; v++) c[v] = f_outdeg[v] ? 1.0f / (float)f_outdeg[v] : 0.0f;
        const float coef = (1.0f - damp) * damp;
        for (uint32_t v = 0; v < V; v++)
        {
            const float s = row_sum(c, i_dst, i_idx[v], i_outdeg[v], gpu_order);
            res[v] = coef * s;
        }
    }
    uint32_t it, executed = 0;
    double error_total = 0.0;
    for (it = 0; it < max_iters; it++)
    {
        error_total = 0.0;
        uint32_t active = 0;
        if (mode == 6)
        {
            for (uint32_t v = 0; v < V; v++) c[v] = f_outdeg[v] ? pr[v] / (float)f_outdeg[v] : 0.0f;
            for (uint32_t v = 0; v < V; v++)
            {
                if (!cur[v]) continue;
                const float s = row_sum(c, i_dst, i_idx[v], i_outdeg[v], gpu_order);
                const float scaled = damp * s;
                const float nv = base_pr + scaled;
                const float diff = nv - pr[v];
                const double e = fabs((double)diff);
                error_total += e / V;
                if (e >= epsilon)
                {
                    pr[v] = nv;
                    for (uint32_t j = f_idx[v]; j < f_idx[v] + f_outdeg[v]; j++) next[f_dst[j] & 0x3FFFFFFFu] = 1;
                    active++;
                }
            }
        }
        else
        {
            for (uint32_t v = 0; v < V; v++)
            {
                if (!cur[v]) continue;
                float nv;
                const float old = pr[v];
                if (mode == 7)
                {
                    nv = res[v] + old;
                }
                else
                {
                    float s = 0.0f;
                    for (uint32_t j = i_idx[v]; j < i_idx[v] + i_outdeg[v]; j++)
                    {
                        const uint32_t u = i_dst[j] & 0x3FFFFFFFu;
                        s += pr[u] / (float)f_outdeg[u];
                    }
                    const float scaled = damp * s;
                    nv = base_pr + scaled;
                }
                const float a = nv / (float)V, b = old / (float)V;
                const float diff = a - b;
                error_total += fabs((double)diff);
                pr[v] = nv;
                const uint32_t d = f_outdeg[v];
                if (d)
                {
                    const float q = res[v] / (float)d;
                    const float delta = damp * q;
                    for (uint32_t j = f_idx[v]; j < f_idx[v] + d; j++)
                    {
                        const uint32_t u = f_dst[j] & 0x3FFFFFFFu;
                        const float prev = res[u];
                        res[u] = prev + delta;
                        const float sum = prev + delta;
                        if (fabs((double)sum) >= epsilon && (double)prev <= epsilon)
                        {
                            active++;
                            if (mode == 8) res[u] = res[u] + delta;
                            next[u] = 1;
                        }
                    }
                }
                res[v] = 0.0f;
            }
        }
        if (active_hist) active_hist[executed] = active;
        executed++;
        uint8_t *t = cur;
        cur = next;
        next = t;
        memset(next, 0, V);
        if (active == 0) break;
    }
    for (uint32_t v = 0; v < V; v++) pr[v] = pr[v] / (float)V;
    if (iterations_out) *iterations_out = it;
    if (error_out) *error_out = error_total;
    free(cur);
    free(next);
    free(c);
    free(res);
    return executed;
}

/* ------------------------------------------------------------------ SPMV -- */

/* SPMVPullGraphCSR (SPMV.c:616-713, mode 0) and SPMVPushGraphCSR
 * (:715-810, mode 1), sequential.  w (in the direction the mode reads:
 * inverse for pull, forward for push) may be NULL: every weight 0.0001.
 * gpu_order (pull) adds long rows' sums, in the GPU kernels' order, to y
 * once per iteration. */
void orc_spmv(uint32_t V, const uint32_t *f_outdeg, const uint32_t *f_idx, const uint32_t *f_dst,
              const uint32_t *i_outdeg, const uint32_t *i_idx, const uint32_t *i_dst, const float *w, int mode,
              int gpu_order, uint32_t iters, float *x, float *y)
{
    for (uint32_t v = 0; v < V; v++)
    {
        x[v] = f_outdeg[v] ? 1.0f / (float)f_outdeg[v] : 0.001f;
        y[v] = 0.0f;
    }
    float *t = NULL;
    const uint32_t E = V ? (mode == 0 ? i_idx[V - 1] + i_outdeg[V - 1] : f_idx[V - 1] + f_outdeg[V - 1]) : 0;
    (void)E;
    if (mode == 0 && gpu_order)
    {
        /* the per-edge terms as a gather array for tree_sum: t[j] = w_j * x[src] */
        uint32_t Et = 0;
        for (uint32_t v = 0; v < V; v++)
            if (i_idx[v] + i_outdeg[v] > Et) Et = i_idx[v] + i_outdeg[v];
        t = malloc((size_t)Et * 4 + 4);
        uint32_t *ident = malloc((size_t)Et * 4 + 4);
        for (uint32_t j = 0; j < Et; j++)
        {
            const float wj = w ? w[j] : 0.0001f;
            t[j] = wj * x[i_dst[j] & 0x3FFFFFFFu];
            ident[j] = j;
        }
        for (uint32_t it = 0; it < iters; it++)
            for (uint32_t v = 0; v < V; v++)
            {
                const uint32_t d = i_outdeg[v];
                if (d > g_warp_thr)
                    y[v] += row_sum(t, ident, i_idx[v], d, 1);
                else
                    for (uint32_t j = i_idx[v]; j < i_idx[v] + d; j++) y[v] += t[j];
            }
        free(ident);
        free(t);
        return;
    }
    for (uint32_t it = 0; it < iters; it++)
    {
        if (mode == 0)
        {
            for (uint32_t v = 0; v < V; v++)
                for (uint32_t j = i_idx[v]; j < i_idx[v] + i_outdeg[v]; j++)
                {
                    const float wj = w ? w[j] : 0.0001f;
                    const float p = wj * x[i_dst[j] & 0x3FFFFFFFu];
                    y[v] += p;
                }
        }
        else
        {
            for (uint32_t v = 0; v < V; v++)
                for (uint32_t j = f_idx[v]; j < f_idx[v] + f_outdeg[v]; j++)
                {
                    const float wj = w ? w[j] : 0.0001f;
                    const float p = wj * x[v];
                    y[f_dst[j] & 0x3FFFFFFFu] += p;
                }
        }
    }
}

/* radixSortEdgesByPageRank (reorder.c:165-221): labels stably sorted by the
 * key (uint32_t)(rank * 2^20 + 0.5f) (FloatToFixed32SORT, fixedPoint.h:33),
 * in place. */
void orc_rank_sort(uint32_t n, const float *ranks, uint32_t *labels)
{
    uint32_t *key = malloc((size_t)n * 4 + 4), *ok = malloc((size_t)n * 4 + 4), *ol = malloc((size_t)n * 4 + 4);
    for (uint32_t i = 0; i < n; i++)
    {
        const float scaled = ranks[i] * 1048576.0f;
        const float r = scaled + (ranks[i] >= 0 ? 0.5f : -0.5f);
        key[i] = r > 0.0f ? (uint32_t)r : 0u;
    }
    sort_by_key(n, key, labels, NULL, ok, ol, NULL);
    memcpy(labels, ol, (size_t)n * 4);
    free(key);
    free(ok);
    free(ol);
}

/* One pull PageRank iteration over the destination vertices [lo, hi) of a
 * 1-D partition (the iteration of pageRank.c:984-1044 restricted to a
 * range): rows summed as row_sum (gpu_order: the GPU kernels' order),
 * ranks and contrib_next written on [lo, hi); the range's error and active
 * count added to *err / *active. */
void orc_pull_range_step(uint32_t V, const uint32_t *f_outdeg, const uint32_t *i_outdeg, const uint32_t *i_idx,
                         const uint32_t *i_dst, uint32_t lo, uint32_t hi, const float *contrib, float *pr,
                         float *contrib_next, double epsilon, int gpu_order, double *err, uint32_t *active)
{
    const float damp = 0.85f;
    const float base_pr = 1.0f - damp;
    for (uint32_t v = lo; v < hi; v++)
    {
        const float s = row_sum(contrib, i_dst, i_idx[v], i_outdeg[v], gpu_order);
        const float scaled = damp * s;
        const float nv = base_pr + scaled;
        const float prev = pr[v];
        pr[v] = nv;
        contrib_next[v] = f_outdeg[v] ? nv / (float)f_outdeg[v] : 0.0f;
        const float diff = nv - prev;
        const double e = fabs((double)diff);
        *err += e / V;
        if (e >= epsilon) (*active)++;
    }
}

/* ------------------------------------------------- partitioned DO-BFS -- */

#define ORC_NO_CAND 0x7F7F7F7F /* cand of a vertex no frontier vertex reached */

/* The first in-neighbour of v in the frontier, in CSR order; -1 if none.
 * *examined grows by the in-edges read (BFS.c:736-748's early break). */
static int64_t first_frontier_in(const uint32_t *i_outdeg, const uint32_t *i_idx, const uint32_t *i_dst, uint32_t v,
                                 const uint8_t *frontier, uint64_t *examined)
{
    for (uint32_t j = i_idx[v]; j < i_idx[v] + i_outdeg[v]; j++)
    {
        const uint32_t u = i_dst[j] & 0x3FFFFFFFu;
        if (frontier[u])
        {
            *examined += j + 1 - i_idx[v];
            return u;
        }
    }
    *examined += i_outdeg[v];
    return -1;
}

void orc_bfs_range_init(uint32_t V, const uint32_t *f_outdeg, uint32_t lo, uint32_t hi, uint32_t root,
                        int32_t *parents, uint32_t *dist, uint8_t *frontier, uint8_t *visited, int32_t *cand)
{
    for (uint32_t v = 0; v < V; v++) cand[v] = ORC_NO_CAND;
    for (uint32_t v = lo; v < hi; v++)
    {
        parents[v] = f_outdeg[v] ? -(int32_t)f_outdeg[v] : -1;
        dist[v] = 0;
    }
    if (root >= lo && root < hi) parents[root] = (int32_t)root;
    memset(frontier, 0, V);
    memset(visited, 0, V);
    frontier[root] = 1;
    visited[root] = 1;
}

void orc_bfs_range_expand(uint32_t V, const uint32_t *f_outdeg, const uint32_t *f_idx, const uint32_t *f_dst,
                          const uint32_t *i_outdeg, const uint32_t *i_idx, const uint32_t *i_dst, uint32_t lo,
                          uint32_t hi, int direction, uint32_t depth, const uint8_t *frontier, const uint8_t *visited,
                          uint8_t *next, int32_t *cand, int32_t *parents, uint32_t *dist, uint64_t *counts)
{
    memset(counts, 0, 4 * sizeof(uint64_t));
    if (direction != 0) memset(next, 0, V);
    for (uint32_t v = lo; v < hi; v++)
    {
        if (direction == 0)
        {
            if (!frontier[v]) continue;
            for (uint32_t j = f_idx[v]; j < f_idx[v] + f_outdeg[v]; j++)
            {
                const uint32_t w = f_dst[j] & 0x3FFFFFFFu;
                if (!visited[w] && (int32_t)v < cand[w]) cand[w] = (int32_t)v;
            }
        }
        else
        {
            if (visited[v]) continue;
            const int64_t p = first_frontier_in(i_outdeg, i_idx, i_dst, v, frontier, &counts[2]);
            if (p < 0) continue;
            parents[v] = (int32_t)p;
            dist[v] = depth;
            next[v] = 1;
            counts[0]++;
        }
    }
}

void orc_bfs_range_settle(uint32_t V, const uint32_t *f_outdeg, uint32_t lo, uint32_t hi, int direction,
                          uint32_t depth, int32_t *cand, uint8_t *next, uint8_t *visited, int32_t *parents,
                          uint32_t *dist, uint64_t *counts)
{
    for (uint32_t v = 0; v < V; v++)
    {
        if (direction == 0)
        {
            next[v] = cand[v] != ORC_NO_CAND;
            if (next[v] && v >= lo && v < hi)
            {
                parents[v] = cand[v];
                dist[v] = depth;
                counts[0]++;
                counts[1] += f_outdeg[v] ? f_outdeg[v] : 1u;
            }
            cand[v] = ORC_NO_CAND;
        }
        if (next[v]) visited[v] = 1;
    }
}
