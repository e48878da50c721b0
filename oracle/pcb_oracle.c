/* CPU oracle for the pcbroute search back end -- TEST INFRASTRUCTURE ONLY (see pcb_oracle.h).
 *
 * Built with -ffp-contract=off: every float product below is one IEEE single-precision multiply, exactly as the
 * kernels compute it (__fmul_rn), so the fixed-point weights agree bit for bit.
 */
#include "pcb_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>

#define CINF 1e30f

/* moves in the order of the CPU search's move codes (src/router.cpp:1230, src/gpu.cu:488-489):
 * 0 +x, 1 -x, 2 +y, 3 -y, 4 (+,+), 5 (+,-), 6 (-,+), 7 (-,-) */
static const int MDX[8] = {1, -1, 0, 0, 1, 1, -1, -1};
static const int MDY[8] = {0, 0, 1, -1, 1, -1, 1, -1};

uint64_t pcbo_weight(float cf, float fac) {
    if (!(cf < CINF)) return PCBO_INF64;
    float x = cf * fac;
    float y = x * 16.0f;
    if (!(y < PCBO_WLIM)) return PCBO_INF64;
    if (!(y > 0.0f)) return 0;
    return (uint64_t)rintf(y);
}

uint64_t pcbo_start_d(float g0) {
    float y = g0 * 16.0f;
    if (!(y > 0.0f)) return 0;
    if (!(y < PCBO_WLIM)) return PCBO_INF64;
    return (uint64_t)ceilf(y);
}

void pcbo_factors(float step, const float dirf[8][8], float fac[8][8]) {
    float len[8];
    for (int m = 0; m < 8; ++m) len[m] = m < 4 ? step : (float)((double)step * sqrt(2.0));
    for (int l = 0; l < 8; ++l)
        for (int m = 0; m < 8; ++m) fac[l][m] = len[m] * dirf[l][m];
}

/* src/gpu.cu:78-105 (prep_cf) and 107-115 (prep_v), after the own-copper scatters of src/gpu.cu:460-476 */
void pcbo_resolve(const pcbg_query* q, int rx0, int ry0, int rw, int rh, float* cf, uint8_t* flags, float* vcf) {
    const size_t RN = (size_t)rw * rh, N = RN * (size_t)q->nl, FWN = (size_t)q->ww * q->wh;
    float* ovr = (float*)malloc(N * sizeof(float));
    uint8_t* has = (uint8_t*)calloc(N, 1);
    for (int64_t k = 0; k < q->n_own_cf; ++k) {
        size_t w = q->own_cf_idx[k], l = w / FWN, c = w % FWN;
        int i = (int)(c % q->ww) - rx0, j = (int)(c / q->ww) - ry0;
        if (i < 0 || j < 0 || i >= rw || j >= rh || l >= (size_t)q->nl) continue;
        size_t s = l * RN + (size_t)j * rw + i;
        ovr[s] = q->own_cf_val[k];
        has[s] = 1;
    }
    for (int l = 0; l < q->nl; ++l)
        for (int j = 0; j < rh; ++j)
            for (int i = 0; i < rw; ++i) {
                const int gx = q->wi0 + rx0 + i, gy = q->wj0 + ry0 + j;
                const size_t h = (size_t)gy * q->nx + gx, s = (size_t)l * RN + (size_t)j * rw + i;
                const size_t ws = ((size_t)l * q->wh + (size_t)(ry0 + j)) * q->ww + (size_t)(rx0 + i);
                const int tg = (int)((q->tbit[ws >> 6] >> (ws & 63)) & 1);
                const float v = has[s] ? ovr[s] : q->cst[l][h];
                const uint16_t o = q->st[l][h];
                float r;
                if (!q->lay[l] || !(v < CINF)) r = CINF;
                else if (v < 0) r = o == q->me ? -v : CINF;
                else r = v;
                int pv = 255;
                if (q->prior && q->lay[l]) {
                    const int pl = q->play[l];
                    if (pl >= 0) {
                        const int x = q->pcol[gx] - q->pi0, y = q->prow[gy] - q->pj0;
                        pv = (x < 0 || y < 0 || x >= q->pw || y >= q->ph) ? 0 : q->prior[((size_t)pl * q->ph + y) * q->pw + x];
                    }
                    if (q->corridor && pv < q->mthr && !tg) r = CINF;
                    else if (r < CINF) r = r * q->mlf[pv];
                }
                cf[s] = r;
                int vok;
                if (q->lay[l]) vok = (o == 0 || o == q->me) && (!q->corridor || tg || pv >= q->mthr);
                else vok = tg;
                flags[s] = (uint8_t)((vok ? 1 : 0) | (tg ? 2 : 0));
            }
    if (vcf) {
        float* vo = (float*)malloc(RN * sizeof(float));
        uint8_t* vh = (uint8_t*)calloc(RN, 1);
        for (int64_t k = 0; k < q->n_own_vcf; ++k) {
            size_t c = q->own_vcf_idx[k] % FWN;
            int i = (int)(c % q->ww) - rx0, j = (int)(c / q->ww) - ry0;
            if (i < 0 || j < 0 || i >= rw || j >= rh) continue;
            vo[(size_t)j * rw + i] = q->own_vcf_val[k];
            vh[(size_t)j * rw + i] = 1;
        }
        for (int j = 0; j < rh; ++j)
            for (int i = 0; i < rw; ++i) {
                const size_t h = (size_t)(q->wj0 + ry0 + j) * q->nx + (q->wi0 + rx0 + i), c = (size_t)j * rw + i;
                const float v = vh[c] ? vo[c] : q->vcst[h];
                const uint16_t o = q->vst[h];
                float r = !(v < CINF) ? CINF : v < 0 ? (o == q->me ? -v : CINF) : v;
                vcf[c] = r < CINF ? r * q->via_cost : CINF;
            }
        free(vo);
        free(vh);
    }
    free(ovr);
    free(has);
}

/* ---- exact solve: Dijkstra with a binary heap of (distance, state) ---- */

typedef struct { uint64_t d; uint32_t s; } hitem;
typedef struct { hitem* a; size_t n, cap; } heap;

static int hless(const hitem* x, const hitem* y) { return x->d < y->d || (x->d == y->d && x->s < y->s); }
static void hpush(heap* h, uint64_t d, uint32_t s) {
    if (h->n == h->cap) { h->cap = h->cap ? h->cap * 2 : 1024; h->a = (hitem*)realloc(h->a, h->cap * sizeof(hitem)); }
    size_t k = h->n++;
    hitem it = {d, s};
    while (k > 0) {
        size_t p = (k - 1) / 2;
        if (!hless(&it, &h->a[p])) break;
        h->a[k] = h->a[p];
        k = p;
    }
    h->a[k] = it;
}
static hitem hpop(heap* h) {
    hitem top = h->a[0], last = h->a[--h->n];
    size_t k = 0;
    for (;;) {
        size_t c = 2 * k + 1;
        if (c >= h->n) break;
        if (c + 1 < h->n && hless(&h->a[c + 1], &h->a[c])) ++c;
        if (!hless(&h->a[c], &last)) break;
        h->a[k] = h->a[c];
        k = c;
    }
    if (h->n) h->a[k] = last;
    return top;
}

static inline uint64_t sat_add(uint64_t a, uint64_t b) { return a > PCBO_INF64 - b ? PCBO_INF64 : a + b; }

int64_t pcbo_dijkstra(int rw, int rh, int nl, const float fac[8][8], const float* cf, const uint8_t* flags,
                      const float* vcf, int64_t n_starts, const uint32_t* start_idx, const uint64_t* start_d,
                      uint64_t* dist, uint64_t* best_d) {
    const size_t RN = (size_t)rw * rh, N = RN * (size_t)nl;
    for (size_t s = 0; s < N; ++s) dist[s] = PCBO_INF64;
    heap h = {0, 0, 0};
    for (int64_t k = 0; k < n_starts; ++k) {
        uint32_t s = start_idx[k];
        if (s >= N) continue;
        if (start_d[k] < dist[s]) { dist[s] = start_d[k]; hpush(&h, start_d[k], s); }
    }
    /* Early exit at the best target, as the device solve: once a target is popped at distance D, every state at or
     * below D is exact when the pops pass D (ties included), and nothing above D is reported. States above D keep
     * their tentative distances (upper bounds, never below the exact ones). */
    uint64_t bound = PCBO_INF64;
    while (h.n) {
        hitem it = hpop(&h);
        if (it.d != dist[it.s]) continue;
        if (it.d > bound) break;
        if ((flags[it.s] & 2) && bound == PCBO_INF64) bound = it.d;
        const uint32_t s = it.s;
        const int l = (int)(s / RN);
        const size_t c = s % RN;
        const int j = (int)(c / rw), i = (int)(c % rw);
        for (int m = 0; m < 8; ++m) {
            const int ni = i + MDX[m], nj = j + MDY[m];
            if (ni < 0 || nj < 0 || ni >= rw || nj >= rh) continue;
            const size_t t = (size_t)l * RN + (size_t)nj * rw + ni;
            const uint64_t w = pcbo_weight(cf[t], fac[l][m]);
            if (w == PCBO_INF64) continue;
            const uint64_t nd = sat_add(it.d, w);
            if (nd < dist[t]) { dist[t] = nd; hpush(&h, nd, (uint32_t)t); }
        }
        if (vcf) {
            const uint64_t wv = pcbo_weight(vcf[c], 1.0f);
            if (wv != PCBO_INF64)
                for (int l2 = 0; l2 < nl; ++l2) {
                    if (l2 == l) continue;
                    const size_t t = (size_t)l2 * RN + c;
                    if (!(flags[t] & 1)) continue;
                    const uint64_t nd = sat_add(it.d, wv);
                    if (nd < dist[t]) { dist[t] = nd; hpush(&h, nd, (uint32_t)t); }
                }
        }
    }
    free(h.a);
    int64_t best = -1;
    uint64_t bd = PCBO_INF64;
    for (size_t s = 0; s < N; ++s)
        if ((flags[s] & 2) && dist[s] < bd) { bd = dist[s]; best = (int64_t)s; }
    *best_d = bd;
    return best;
}

int64_t pcbo_walkback(int rw, int rh, int nl, const float fac[8][8], const float* cf, const uint8_t* flags,
                      const float* vcf, int64_t n_starts, const uint32_t* start_idx, const uint64_t* start_d,
                      const uint64_t* dist, int64_t best, uint32_t* path, int64_t cap) {
    if (best < 0) return 0;
    const size_t RN = (size_t)rw * rh;
    size_t q = (size_t)best;
    for (int64_t n = 0; n < cap; ++n) {
        const int l = (int)(q / RN);
        const size_t c = q % RN;
        const int j = (int)(c / rw), i = (int)(c % rw);
        const uint64_t dq = dist[q];
        path[n] = (uint32_t)q;
        for (int64_t k = 0; k < n_starts; ++k)
            if (start_idx[k] == (uint32_t)q && start_d[k] < PCBO_INF64 && start_d[k] == dq) return n + 1;
        int found = 0;
        for (int m = 0; m < 8 && !found; ++m) {           /* p -> q by move m: p = q - (MDX[m], MDY[m]) */
            const int pi = i - MDX[m], pj = j - MDY[m];
            if (pi < 0 || pj < 0 || pi >= rw || pj >= rh) continue;
            const size_t p = (size_t)l * RN + (size_t)pj * rw + pi;
            const uint64_t w = pcbo_weight(cf[q], fac[l][m]);
            if (w != PCBO_INF64 && dist[p] != PCBO_INF64 && dist[p] + w == dq) { q = p; found = 1; }
        }
        if (!found && vcf && (flags[q] & 1)) {
            const uint64_t w = pcbo_weight(vcf[c], 1.0f);
            for (int l2 = 0; l2 < nl && !found && w != PCBO_INF64; ++l2) {
                if (l2 == l) continue;
                const size_t p = (size_t)l2 * RN + c;
                if (dist[p] != PCBO_INF64 && dist[p] + w == dq) { q = p; found = 1; }
            }
        }
        if (!found) return -1;
    }
    return -1;
}

void pcbo_report(int64_t n, const uint64_t* dist, int64_t best, uint64_t best_d, float* out) {
    for (int64_t s = 0; s < n; ++s) {
        const uint64_t d = dist[s];
        out[s] = (d < PCBO_INF64 && (best < 0 || d <= best_d)) ? (float)d * 0.0625f : CINF;
    }
}

static void solve_rect(const pcbg_query* q, int rx0, int ry0, int rw, int rh, float** field, int64_t* best,
                       float* ub) {
    const size_t RN = (size_t)rw * rh, N = RN * (size_t)q->nl, FWN = (size_t)q->ww * q->wh;
    float* cf = (float*)malloc(N * sizeof(float));
    uint8_t* fl = (uint8_t*)malloc(N);
    float* vcf = q->via_cost >= 0 ? (float*)malloc(RN * sizeof(float)) : NULL;
    pcbo_resolve(q, rx0, ry0, rw, rh, cf, fl, vcf);
    uint32_t* si = (uint32_t*)malloc((size_t)(q->n_starts + 1) * sizeof(uint32_t));
    uint64_t* sd = (uint64_t*)malloc((size_t)(q->n_starts + 1) * sizeof(uint64_t));
    int64_t ns = 0;
    for (int64_t k = 0; k < q->n_starts; ++k) {
        size_t w = q->start_idx[k], l = w / FWN, c = w % FWN;
        int i = (int)(c % q->ww) - rx0, j = (int)(c / q->ww) - ry0;
        if (i < 0 || j < 0 || i >= rw || j >= rh || l >= (size_t)q->nl) continue;
        si[ns] = (uint32_t)(l * RN + (size_t)j * rw + i);
        sd[ns] = pcbo_start_d(q->start_val[k]);
        ++ns;
    }
    float fac[8][8];
    pcbo_factors(q->step, q->dirf, fac);
    uint64_t* dist = (uint64_t*)malloc(N * sizeof(uint64_t));
    uint64_t bd;
    int64_t b = pcbo_dijkstra(rw, rh, q->nl, fac, cf, fl, vcf, ns, si, sd, dist, &bd);
    float* out = (float*)malloc(N * sizeof(float));
    pcbo_report((int64_t)N, dist, b, bd, out);
    *field = out;
    if (b >= 0) {
        size_t l = (size_t)b / RN, c = (size_t)b % RN;
        *best = (int64_t)((l * q->wh + (c / rw + ry0)) * q->ww + (c % rw + rx0));
        *ub = (float)bd * 0.0625f;
    } else {
        *best = -1;
        *ub = CINF;
    }
    free(cf); free(fl); free(vcf); free(si); free(sd); free(dist);
}

static double dmax3(double a, double b, double c) { double m = a > b ? a : b; return m > c ? m : c; }

static size_t g_max_states = (size_t)48 << 20;
void pcbo_set_max_states(size_t n) { if (n) g_max_states = n; }

int pcbo_solve(const pcbg_query* q, pcbg_result* out) {
    const size_t FWN = (size_t)q->ww * q->wh, WS = FWN * (size_t)q->nl, WB = WS / 64 + 1;
    int sx0 = 1 << 30, sy0 = 1 << 30, sx1 = -1, sy1 = -1, tx0 = 1 << 30, ty0 = 1 << 30, tx1 = -1, ty1 = -1;
    for (int64_t k = 0; k < q->n_starts; ++k) {
        size_t c = q->start_idx[k] % FWN;
        int i = (int)(c % q->ww), j = (int)(c / q->ww);
        if (i < sx0) sx0 = i; if (i > sx1) sx1 = i; if (j < sy0) sy0 = j; if (j > sy1) sy1 = j;
    }
    for (size_t w = 0; w < WB; ++w) {
        uint64_t b = q->tbit[w];
        while (b) {
            int k = __builtin_ctzll(b);
            b &= b - 1;
            size_t st = w * 64 + (size_t)k;
            if (st >= WS) continue;
            size_t c = st % FWN;
            int i = (int)(c % q->ww), j = (int)(c / q->ww);
            if (i < tx0) tx0 = i; if (i > tx1) tx1 = i; if (j < ty0) ty0 = j; if (j > ty1) ty1 = j;
        }
    }
    if (sx1 < 0 || tx1 < 0) return -1;
    float minfac = 1.f;
    for (int l = 0; l < q->nl; ++l)
        if (q->lay[l])
            for (int m = 0; m < 8; ++m)
                if (q->dirf[l][m] < minfac) minfac = q->dirf[l][m];
    const double unit = (double)q->step * minfac;
#define OCT(i, j, x0, y0, x1, y1)                                                                     \
    (unit * (fmax(dmax3(0, (double)(x0) - (i), (double)(i) - (x1)), dmax3(0, (double)(y0) - (j), (double)(j) - (y1))) + \
             0.41421356 * fmin(dmax3(0, (double)(x0) - (i), (double)(i) - (x1)), dmax3(0, (double)(y0) - (j), (double)(j) - (y1)))))
#define LB(i, j) (OCT(i, j, sx0, sy0, sx1, sy1) + OCT(i, j, tx0, ty0, tx1, ty1))
    const int hx0 = sx0 < tx0 ? sx0 : tx0, hy0 = sy0 < ty0 ? sy0 : ty0;
    const int hx1 = sx1 > tx1 ? sx1 : tx1, hy1 = sy1 > ty1 ? sy1 : ty1;
    int M = 80, tries = 0;
    float* field = NULL;
    for (;; M *= 3, ++tries) {
        int rx0 = hx0 - M > 0 ? hx0 - M : 0, ry0 = hy0 - M > 0 ? hy0 - M : 0;
        int rx1 = hx1 + M + 1 < q->ww ? hx1 + M + 1 : q->ww, ry1 = hy1 + M + 1 < q->wh ? hy1 + M + 1 : q->wh;
        if (tries == 0 && (double)(rx1 - rx0) * (ry1 - ry0) > 0.5 * (double)q->ww * q->wh) {
            rx0 = ry0 = 0;
            rx1 = q->ww;
            ry1 = q->wh;
        }
        const int full = rx0 == 0 && ry0 == 0 && rx1 == q->ww && ry1 == q->wh;
        free(field);
        field = NULL;
        if ((size_t)(rx1 - rx0) * (size_t)(ry1 - ry0) * (size_t)q->nl > g_max_states) return -1;
        int64_t best;
        float ub;
        solve_rect(q, rx0, ry0, rx1 - rx0, ry1 - ry0, &field, &best, &ub);
        out->rx0 = rx0; out->ry0 = ry0; out->rw = rx1 - rx0; out->rh = ry1 - ry0;
        out->nl = q->nl; out->ww = q->ww; out->wh = q->wh;
        out->best = best;
        out->ub = ub;
        if (full) break;
        if (ub < CINF * 0.5f) {
            const double lim = (double)ub * 1.0001 + 1e-3;
            double mn = 1e300;
            if (rx0 > 0) for (int j = 0; j < q->wh; ++j) mn = fmin(mn, LB(rx0 - 1, j));
            if (rx1 < q->ww) for (int j = 0; j < q->wh; ++j) mn = fmin(mn, LB(rx1, j));
            if (ry0 > 0) for (int i = 0; i < q->ww; ++i) mn = fmin(mn, LB(i, ry0 - 1));
            if (ry1 < q->wh) for (int i = 0; i < q->ww; ++i) mn = fmin(mn, LB(i, ry1));
            if (mn > lim) break;
        }
    }
#undef LB
#undef OCT
    out->d = field;
    out->cap = (size_t)out->rw * out->rh * out->nl;
    out->tries = tries + 1;
    out->rounds = 1;
    out->wide = 0;
    out->tile_visits = 0;
    return tries + 1;
}

void pcbo_free(float* p) { free(p); }

/* ---- many searches on host threads (the CPU baseline) ---- */

typedef struct { pcbo_search* s; int n; atomic_int next; } many_ctx;

static void* many_worker(void* arg) {
    many_ctx* c = (many_ctx*)arg;
    for (;;) {
        int k = atomic_fetch_add(&c->next, 1);
        if (k >= c->n) break;
        pcbo_search* s = &c->s[k];
        size_t N = (size_t)s->rw * s->rh * s->nl;
        uint64_t* dist = (uint64_t*)malloc(N * sizeof(uint64_t));
        s->best = pcbo_dijkstra(s->rw, s->rh, s->nl, (const float(*)[8])s->fac, s->cf, s->flags, s->vcf, s->n_starts,
                                s->start_idx, s->start_d, dist, &s->best_d);
        /* the states a solve reports: at or below the best target's cost (every reached state when none) */
        const uint64_t lim = s->best >= 0 ? s->best_d : PCBO_INF64 - 1;
        int64_t settled = 0;
        for (size_t q = 0; q < N; ++q) settled += dist[q] <= lim;
        s->settled = settled;
        free(dist);
    }
    return NULL;
}

void pcbo_solve_many(pcbo_search* s, int n, int threads) {
    many_ctx c;
    c.s = s;
    c.n = n;
    atomic_init(&c.next, 0);
    if (threads < 1) threads = 1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)threads);
    for (int t = 0; t < threads; ++t) pthread_create(&th[t], NULL, many_worker, &c);
    for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
    free(th);
}

/* ---- congestion cost maps: cost_xp / vcost_xp with own = 0 (src/router.cpp:386-405), over whole grids ---- */

void pcbo_costs_rebuild(int n, int nl, int nclasses, const uint16_t* st, const uint8_t* oc, const uint8_t* ov,
                        const uint16_t* vst, const float* hist, const float* const* gnd, float pres, int hard,
                        float* cst, float* vcst) {
    for (int k = 0; k < nclasses; ++k) {
        for (int l = 0; l < nl; ++l)
            for (int c = 0; c < n; ++c) {
                const size_t id = ((size_t)k * nl + l) * n + c;
                const uint16_t s = st[id];
                float v;
                if (s == 0xFFFF) v = CINF;
                else {
                    const int occ = oc[id];
                    if (hard && occ > 0) v = CINF;
                    else {
                        v = (1.f + hist[(size_t)l * n + c]) * (1.f + pres * (float)(occ > 0 ? occ : 0));
                        if (gnd && gnd[l]) v *= gnd[l][c];
                        if (s != 0) v = -v;
                    }
                }
                cst[id] = v;
            }
        for (int c = 0; c < n; ++c) {
            const uint16_t s = vst[(size_t)k * n + c];
            float v;
            if (s == 0xFFFF) v = CINF;
            else {
                int occ = 0;
                float hs = 0;
                for (int l = 0; l < nl; ++l) {
                    occ += ov[((size_t)k * nl + l) * n + c];
                    hs += hist[(size_t)l * n + c];
                }
                if (hard && occ > 0) v = CINF;
                else {
                    v = (1.f + hs / (float)nl) * (1.f + pres * (float)(occ > 0 ? occ : 0));
                    if (s != 0) v = -v;
                }
            }
            vcst[(size_t)k * n + c] = v;
        }
    }
}
