/*
 * CPU oracle for the no-three-in-line population search hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is a plain-C restatement of the
 * reference's CPU algorithms (MilliganCo/no-three-in-line, package
 * src/no_three_75).  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline / reference arm may load it, and only as the checker or as the
 * timed CPU baseline.  The product path (the CUDA library) never calls it.
 *
 * Parity is pinned: tests/test_oracle_golden.py checks every function here
 * against golden vectors produced by the reference itself
 * (tests/golden/make_golden.py imports the reference and records its
 * outputs), including the reference's own fixture
 * results/best-near-solution-E10.json (E = 10).
 *
 * Slot layout used throughout (the reference's interleave,
 * src/no_three_75/accelerated.py:18-24 and src/no_three_75/tempering.py:38):
 *   slot s = 2*row + layer,  row(s) = s >> 1,  col[2r] = P[r], col[2r+1] = Q[r].
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <pthread.h>
#include <unistd.h>

#define N3O_SENTINEL64 (((int64_t)1) << 60)

/* Minimal static-split parallel-for over [0, count) on `threads` pthreads
 * (threads < 1: every online CPU). */
typedef void (*n3o_body_fn)(int index, void* ctx);
typedef struct {
    n3o_body_fn body;
    void* ctx;
    int begin, end;
} n3o_span;

static void* n3o_run_span(void* arg) {
    n3o_span* s = (n3o_span*)arg;
    for (int i = s->begin; i < s->end; ++i) s->body(i, s->ctx);
    return NULL;
}

int n3o_max_threads(void) {
    const long c = sysconf(_SC_NPROCESSORS_ONLN);
    return c > 0 ? (int)c : 1;
}

static void n3o_parallel_for(int count, int threads, n3o_body_fn body, void* ctx) {
    if (threads < 1) threads = n3o_max_threads();
    if (threads > count) threads = count;
    if (threads <= 1) {
        for (int i = 0; i < count; ++i) body(i, ctx);
        return;
    }
    pthread_t tid[256];
    n3o_span spans[256];
    if (threads > 256) threads = 256;
    for (int t = 0; t < threads; ++t) {
        spans[t].body = body;
        spans[t].ctx = ctx;
        spans[t].begin = (int)((long long)count * t / threads);
        spans[t].end = (int)((long long)count * (t + 1) / threads);
        pthread_create(&tid[t], NULL, n3o_run_span, &spans[t]);
    }
    for (int t = 0; t < threads; ++t) pthread_join(tid[t], NULL);
}

static void interleave(const int32_t* p, const int32_t* q, int n, int32_t* rows, int32_t* cols) {
    for (int r = 0; r < n; ++r) {
        rows[2 * r] = r;
        cols[2 * r] = p[r];
        rows[2 * r + 1] = r;
        cols[2 * r + 1] = q[r];
    }
}

/* Restates src/no_three_75/accelerated.py:14-37 (score_and_badness): the
 * i<j<k triple loop with the hoisted (dx1, dy1) of the pair (i, j) and the
 * cross-product test dx1*(c_k-c_i) == dy1*(r_k-r_i). */
int64_t n3o_score_and_badness(const int32_t* p, const int32_t* q, int n, int64_t* badness) {
    const int m = 2 * n;
    int32_t rows[512], cols[512];
    if (m > 512) return -1;
    interleave(p, q, n, rows, cols);
    if (badness) memset(badness, 0, sizeof(int64_t) * (size_t)m);
    int64_t score = 0;
    for (int i = 0; i < m - 2; ++i) {
        for (int j = i + 1; j < m - 1; ++j) {
            const int32_t dx1 = rows[j] - rows[i];
            const int32_t dy1 = cols[j] - cols[i];
            for (int k = j + 1; k < m; ++k) {
                if (dx1 * (cols[k] - cols[i]) == dy1 * (rows[k] - rows[i])) {
                    ++score;
                    if (badness) {
                        ++badness[i];
                        ++badness[j];
                        ++badness[k];
                    }
                }
            }
        }
    }
    return score;
}

typedef struct {
    const int32_t *p, *q;
    int n;
    int32_t *scores, *badness;
    int slope;
} n3o_pop_ctx;

int64_t n3o_slope_score_points(const int32_t* rows, const int32_t* cols, int m, int64_t* badness);

static void n3o_pop_body(int b, void* arg) {
    const n3o_pop_ctx* c = (const n3o_pop_ctx*)arg;
    const int n = c->n;
    int64_t bad[512];
    int64_t s;
    if (c->slope) {
        int32_t rows[512], cols[512];
        interleave(c->p + (size_t)b * n, c->q + (size_t)b * n, n, rows, cols);
        s = n3o_slope_score_points(rows, cols, 2 * n, bad);
    } else {
        s = n3o_score_and_badness(c->p + (size_t)b * n, c->q + (size_t)b * n, n, bad);
    }
    c->scores[b] = (int32_t)s;
    if (c->badness)
        for (int t = 0; t < 2 * n; ++t) c->badness[(size_t)b * 2 * n + t] = (int32_t)bad[t];
}

/* Batched form of the above over a population of P/Q states, the CPU side of
 * src/no_three_75/gpu.py:99-109 (benchmark_gpu's serial loop), optionally
 * spread over `threads` threads (< 1: all CPUs).  badness may be NULL. */
void n3o_score_population(const int32_t* p, const int32_t* q, int B, int n, int32_t* scores,
                          int32_t* badness, int threads) {
    n3o_pop_ctx c = {p, q, n, scores, badness, 0};
    n3o_parallel_for(B, threads, n3o_pop_body, &c);
}

static int igcd(int a, int b) {
    if (a < 0) a = -a;
    if (b < 0) b = -b;
    while (b) {
        const int t = a % b;
        a = b;
        b = t;
    }
    return a;
}

/* Primitive undirected direction of b - a: src/no_three_75/verifier_b.py:8-19
 * (gcd-reduced, dx >= 0, and dy > 0 when dx == 0).  Packed into one int. */
static int direction_key(int ra, int ca, int rb, int cb) {
    int dx = rb - ra, dy = cb - ca;
    const int g = igcd(dx, dy);
    dx /= g;
    dy /= g;
    if (dx < 0 || (dx == 0 && dy < 0)) {
        dx = -dx;
        dy = -dy;
    }
    return (dx + 1024) * 4096 + (dy + 1024);
}

static int cmp_int(const void* a, const void* b) {
    const int x = *(const int*)a, y = *(const int*)b;
    return (x > y) - (x < y);
}

/* Normalised-slope line count over an arbitrary point list.  For each anchor a
 * the other points are grouped by primitive direction (verifier_b.py:22-33
 * stops at the first repeat; here every repeat is counted).  A line holding k
 * points gives each member C(k-1,2) equal-direction pairs, so
 *   badness[a] = sum_dir C(c_dir, 2)           (conflicts.py:376-378)
 *   E          = (1/3) sum_a badness[a]        (= sum_lines C(k,3), conflicts.py:373)
 * Returns E, or -1 when the points are not distinct or m is too large. */
int64_t n3o_slope_score_points(const int32_t* rows, const int32_t* cols, int m, int64_t* badness) {
    int keys[512];
    if (m > 512) return -1;
    int64_t total = 0;
    for (int a = 0; a < m; ++a) {
        int c = 0;
        for (int b = 0; b < m; ++b) {
            if (b == a) continue;
            if (rows[a] == rows[b] && cols[a] == cols[b]) return -1;
            keys[c++] = direction_key(rows[a], cols[a], rows[b], cols[b]);
        }
        qsort(keys, (size_t)c, sizeof(int), cmp_int);
        int64_t pairs = 0;
        int run = 1;
        for (int t = 1; t <= c; ++t) {
            if (t < c && keys[t] == keys[t - 1]) {
                ++run;
            } else {
                pairs += (int64_t)run * (run - 1) / 2;
                run = 1;
            }
        }
        if (badness) badness[a] = pairs;
        total += pairs;
    }
    if (total % 3) return -2;
    return total / 3;
}

/* Batched slope line count over P/Q states (threads as above). */
void n3o_slope_population(const int32_t* p, const int32_t* q, int B, int n, int32_t* scores,
                          int32_t* badness, int threads) {
    n3o_pop_ctx c = {p, q, n, scores, badness, 1};
    n3o_parallel_for(B, threads, n3o_pop_body, &c);
}

/* Restates src/no_three_75/accelerated.py:122-195 (evaluate_two_switches):
 * for the selected slot u, the full score after exchanging its column with
 * every legal partner slot v, via current - (bad[u]+bad[v]-joint_old) +
 * new_affected.  Illegal partners keep the sentinel 1<<60. */
void n3o_two_switches(const int32_t* p, const int32_t* q, int n, int u, int64_t current,
                      const int64_t* badness, int64_t* out) {
    const int m = 2 * n;
    int32_t rows[512], cols[512];
    interleave(p, q, n, rows, cols);
    for (int v = 0; v < m; ++v) out[v] = N3O_SENTINEL64;
    const int srow = rows[u];
    const int sother = 2 * srow + (1 - (u & 1));
    for (int v = 0; v < m; ++v) {
        if (v == u || rows[v] == srow) continue;
        const int prow = rows[v];
        const int pother = 2 * prow + (1 - (v & 1));
        if (cols[v] == cols[sother] || cols[u] == cols[pother]) continue;
        int64_t joint = 0;
        for (int o = 0; o < m; ++o) {
            if (o == u || o == v) continue;
            if ((rows[v] - rows[u]) * (cols[o] - cols[u]) == (cols[v] - cols[u]) * (rows[o] - rows[u])) ++joint;
        }
        const int64_t old_aff = badness[u] + badness[v] - joint;
        const int nur = rows[u], nuc = cols[v], nvr = rows[v], nvc = cols[u];
        int64_t aff = 0;
        for (int i = 0; i < m - 1; ++i) {
            if (i == u) continue;
            const int ir = rows[i], ic = (i == v) ? nvc : cols[i];
            for (int j = i + 1; j < m; ++j) {
                if (j == u) continue;
                const int jr = rows[j], jc = (j == v) ? nvc : cols[j];
                if ((ir - nur) * (jc - nuc) == (ic - nuc) * (jr - nur)) ++aff;
            }
        }
        for (int i = 0; i < m - 1; ++i) {
            if (i == u || i == v) continue;
            for (int j = i + 1; j < m; ++j) {
                if (j == u || j == v) continue;
                if ((rows[i] - nvr) * (cols[j] - nvc) == (cols[i] - nvc) * (rows[j] - nvr)) ++aff;
            }
        }
        out[v] = current - old_aff + aff;
    }
}

/* Restates src/no_three_75/accelerated.py:40-119 (evaluate_transpositions):
 * same-layer row transpositions of the selected (layer, row). */
void n3o_transpositions(const int32_t* p, const int32_t* q, int n, int layer, int row, int64_t current,
                        const int64_t* badness, int64_t* out) {
    const int m = 2 * n;
    int32_t rows[512], cols[512];
    interleave(p, q, n, rows, cols);
    for (int r = 0; r < n; ++r) out[r] = N3O_SENTINEL64;
    const int u = 2 * row + layer;
    for (int pr = 0; pr < n; ++pr) {
        if (pr == row) continue;
        if (layer == 0) {
            if (p[pr] == q[row] || p[row] == q[pr]) continue;
        } else {
            if (q[pr] == p[row] || q[row] == p[pr]) continue;
        }
        const int v = 2 * pr + layer;
        int64_t joint = 0;
        for (int o = 0; o < m; ++o) {
            if (o == u || o == v) continue;
            if ((rows[v] - rows[u]) * (cols[o] - cols[u]) == (cols[v] - cols[u]) * (rows[o] - rows[u])) ++joint;
        }
        const int64_t old_aff = badness[u] + badness[v] - joint;
        const int nur = rows[u], nuc = cols[v], nvr = rows[v], nvc = cols[u];
        int64_t aff = 0;
        for (int i = 0; i < m - 1; ++i) {
            if (i == u) continue;
            const int ir = rows[i], ic = (i == v) ? nvc : cols[i];
            for (int j = i + 1; j < m; ++j) {
                if (j == u) continue;
                const int jr = rows[j], jc = (j == v) ? nvc : cols[j];
                if ((ir - nur) * (jc - nuc) == (ic - nuc) * (jr - nur)) ++aff;
            }
        }
        for (int i = 0; i < m - 1; ++i) {
            if (i == u || i == v) continue;
            for (int j = i + 1; j < m; ++j) {
                if (j == u || j == v) continue;
                if ((rows[i] - nvr) * (cols[j] - nvc) == (cols[i] - nvc) * (rows[j] - nvr)) ++aff;
            }
        }
        out[pr] = current - old_aff + aff;
    }
}

static int aligned3(int a, int ca, int b, int cb, int c, int cc) {
    return (b - a) * (cc - ca) == (cb - ca) * (c - a);
}

/* Restates the exact move delta of the reference's persistent walk kernel,
 * src/no_three_75/tempering.py:58 (legality) and :68-89 (delta): slot u takes
 * column c_v and slot v takes c_u.  Every pair (i<j) outside {u,v} adds
 * aligned(u',i,j)-aligned(u,i,j) + aligned(v',i,j)-aligned(v,i,j); every k
 * outside {u,v} adds aligned(u',v',k)-aligned(u,v,k).  Each changed triple
 * also moves the badness of its three members by the same +-1.
 * cols is the slot-layout column array of one state (length 2n).
 * Returns 1 for a legal move (dE / dbad written), 0 otherwise. */
int n3o_walk_delta(const int32_t* cols, int n, int u, int v, int32_t* dE, int32_t* dbad) {
    const int m = 2 * n;
    if (dbad) memset(dbad, 0, sizeof(int32_t) * (size_t)m);
    *dE = 0;
    const int cu = cols[u], cv = cols[v];
    if (!((u >> 1) != (v >> 1) && cu != cv && cols[u ^ 1] != cv && cols[v ^ 1] != cu)) return 0;
    const int ru = u >> 1, rv = v >> 1;
    int32_t delta = 0;
    for (int i = 0; i < m - 1; ++i) {
        if (i == u || i == v) continue;
        const int ri = i >> 1, ci = cols[i];
        for (int j = i + 1; j < m; ++j) {
            if (j == u || j == v) continue;
            const int rj = j >> 1, cj = cols[j];
            int d = aligned3(ru, cv, ri, ci, rj, cj) - aligned3(ru, cu, ri, ci, rj, cj);
            if (d) {
                delta += d;
                if (dbad) { dbad[u] += d; dbad[i] += d; dbad[j] += d; }
            }
            d = aligned3(rv, cu, ri, ci, rj, cj) - aligned3(rv, cv, ri, ci, rj, cj);
            if (d) {
                delta += d;
                if (dbad) { dbad[v] += d; dbad[i] += d; dbad[j] += d; }
            }
        }
    }
    for (int k = 0; k < m; ++k) {
        if (k == u || k == v) continue;
        const int d = aligned3(ru, cv, rv, cu, k >> 1, cols[k]) - aligned3(ru, cu, rv, cv, k >> 1, cols[k]);
        if (d) {
            delta += d;
            if (dbad) { dbad[u] += d; dbad[v] += d; dbad[k] += d; }
        }
    }
    *dE = delta;
    return 1;
}

/* Score + badness of one slot-layout column array (rows implicit). */
int32_t n3o_score_columns(const int32_t* cols, int n, int32_t* badness) {
    const int m = 2 * n;
    int32_t p[256] = {0}, q[256] = {0};
    int64_t bad[512];
    if (n > 256) return -1;
    for (int r = 0; r < n; ++r) {
        p[r] = cols[2 * r];
        q[r] = cols[2 * r + 1];
    }
    const int64_t s = n3o_score_and_badness(p, q, n, bad);
    if (badness)
        for (int t = 0; t < m; ++t) badness[t] = (int32_t)bad[t];
    return (int32_t)s;
}


/* Determinant count over an arbitrary point list (the test of
 * src/no_three_75/verifier_a.py:8-16, counted over all triples instead of
 * stopping at the first witness).  badness may be NULL. */
int64_t n3o_det_score_points(const int32_t* rows, const int32_t* cols, int m, int64_t* badness) {
    if (badness) memset(badness, 0, sizeof(int64_t) * (size_t)m);
    int64_t score = 0;
    for (int i = 0; i < m - 2; ++i)
        for (int j = i + 1; j < m - 1; ++j)
            for (int k = j + 1; k < m; ++k)
                if ((rows[j] - rows[i]) * (cols[k] - cols[i]) == (cols[j] - cols[i]) * (rows[k] - rows[i])) {
                    ++score;
                    if (badness) {
                        ++badness[i];
                        ++badness[j];
                        ++badness[k];
                    }
                }
    return score;
}

/* ---------------------------------------------------------------------------
 * Tempering replay (ladder_rounds, when given, is each ladder's round count).  Philox4x32-10 restated from Salmon et al., SC'11 (the
 * paper's multipliers and Weyl constants), and the tempering schedule of the
 * device kernel: per round, every chain makes `per_round` proposals (slots
 * u = floor(r0*m/2^32), v = floor(r1*m/2^32) of the Philox block with counter
 * (proposal index lo, hi, chain, 0x50000000) and key = seed), each scored by
 * the reference's pair formulation (n3o_walk_delta, tempering.py:68-89) and
 * accepted iff dE <= 0 or (dE < W and r2 < acc[temp][dE]).  With bad_bias,
 * when floor(r3*100/2^32) < bad_bias, u is instead the reference's
 * badness-weighted slot (tempering.py:51-55) for the target floor(r*3E/2^32),
 * r the first word of the Philox block (proposal index lo, hi, chain,
 * 0xB0000000).  No proposal moves a chain at E = 0 (tempering.py:58).  An
 * umbrella adds s_q (2 removed dd + dd^2) - c2s_q dd (units of 2^-24) to the
 * acceptance energy (tempering.py:59-63, 93-94).  Then each ladder
 * exchanges neighbours (t, t+1) for t = round%2, round%2+2, ... with the
 * reference's rule (tempering.py:178-184): swap when E(lower T) >= E(higher T),
 * else iff the Philox word for (round, t, ladder, 0xE0000000) is below
 * exch[t][E(higher T) - E(lower T)].
 * ------------------------------------------------------------------------- */
static void n3o_philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t y0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0, y1 = (uint32_t)p1;
        const uint32_t y2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1, y3 = (uint32_t)p0;
        c[0] = y0;
        c[1] = y1;
        c[2] = y2;
        c[3] = y3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

void n3o_philox4x32_10(const uint32_t* ctr, uint32_t k0, uint32_t k1, uint32_t* out) {
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    n3o_philox(c, k0, k1);
    memcpy(out, c, sizeof(c));
}

typedef struct {
    int C, L, stride;
    int32_t *cols, *bad, *E, *bestE, *best_cols, *temp_of, *chain_at;
    uint64_t* counter;
    uint32_t* accepted;
    const int32_t* ladder_n;
    uint32_t *ladder_round, *ladder_exch;
    const uint32_t* acc;
    int W;
    const uint32_t* exch;
    int XW;
    uint64_t seed;
    int rounds, round_sweeps, round_proposals, exchange;
    const int32_t* ladder_rounds;
    int round;
    int bad_bias;
    const int32_t* reference; /* umbrella: reference slot columns, or NULL */
    int32_t* removed;
    const int64_t* umbrella;  /* [C][2] per replica position */
    const uint32_t* frac;     /* [L][768] */
} n3o_temper_ctx;

static uint32_t n3o_mulhi(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) >> 32); }

/* The reference's badness-weighted slot (tempering.py:52-54), literally. */
static int n3o_bias_slot(const int32_t* bad, int m, int32_t target) {
    int u = 0;
    while (u < m - 1 && target >= bad[u]) {
        target -= bad[u];
        ++u;
    }
    return u;
}

/* distance_delta of tempering.py:59-63. */
static int n3o_distance_delta(const int32_t* ref, int u, int v, int cu, int cv) {
    const int ur = (u >> 1) * 2, vr = (v >> 1) * 2;
    return (cu == ref[ur] || cu == ref[ur + 1]) + (cv == ref[vr] || cv == ref[vr + 1]) -
           (cv == ref[ur] || cv == ref[ur + 1]) - (cu == ref[vr] || cu == ref[vr + 1]);
}

/* Acceptance with the umbrella term in units of 2^-24 (see the device's
 * umbrella_accept): thresholds thr[a] x three 8-bit fraction factors. */
static int n3o_umbrella_accept(int32_t dE, int64_t umb, uint32_t z, const uint32_t* thr, int W,
                               const uint32_t* frac) {
    const int64_t e = ((int64_t)dE << 24) + umb;
    if (e <= 0) return 1;
    const int64_t a = e >> 24;
    if (a >= W) return 0;
    uint32_t t = thr[a];
    const int b = (int)(e & 0xFFFFFF);
    if (b >> 16) t = n3o_mulhi(t, frac[b >> 16]);
    if ((b >> 8) & 255) t = n3o_mulhi(t, frac[256 + ((b >> 8) & 255)]);
    if (b & 255) t = n3o_mulhi(t, frac[512 + (b & 255)]);
    return z < t;
}

static void n3o_temper_chain_round(int c, void* arg) {
    n3o_temper_ctx* T = (n3o_temper_ctx*)arg;
    if (T->ladder_rounds && T->round >= T->ladder_rounds[c / T->L]) return;
    const int n = T->ladder_n[c / T->L], m = 2 * n;
    int32_t* cols = T->cols + (size_t)c * T->stride;
    int32_t* bad = T->bad + (size_t)c * T->stride;
    const int per = T->round_proposals > 0 ? T->round_proposals : T->round_sweeps * m;
    const int temp = T->temp_of[c];
    const uint32_t* thr = T->acc + (size_t)temp * T->W;
    const size_t pos = (size_t)(c / T->L) * T->L + temp;
    int32_t dbad[512];
    for (int p = 0; p < per; ++p) {
        const uint64_t k = T->counter[c]++;
        if (T->E[c] <= 0) continue; /* tempering.py:58: no move once score == 0 */
        uint32_t r[4] = {(uint32_t)k, (uint32_t)(k >> 32), (uint32_t)c, 0x50000000u};
        n3o_philox(r, (uint32_t)T->seed, (uint32_t)(T->seed >> 32));
        int u = (int)n3o_mulhi(r[0], (uint32_t)m);
        const int v = (int)n3o_mulhi(r[1], (uint32_t)m);
        if (T->bad_bias > 0 && (int)n3o_mulhi(r[3], 100u) < T->bad_bias) {
            uint32_t r2[4] = {(uint32_t)k, (uint32_t)(k >> 32), (uint32_t)c, 0xB0000000u};
            n3o_philox(r2, (uint32_t)T->seed, (uint32_t)(T->seed >> 32));
            u = n3o_bias_slot(bad, m, (int32_t)n3o_mulhi(r2[0], 3u * (uint32_t)T->E[c]));
        }
        int32_t dE = 0;
        if (!n3o_walk_delta(cols, n, u, v, &dE, dbad)) continue;
        int dd = 0;
        if (T->umbrella) {
            dd = n3o_distance_delta(T->reference, u, v, cols[u], cols[v]);
            const int64_t sq = T->umbrella[2 * pos], c2 = T->umbrella[2 * pos + 1];
            const int64_t umb = sq * (int64_t)(2 * T->removed[c] * dd + dd * dd) - c2 * (int64_t)dd;
            if (!n3o_umbrella_accept(dE, umb, r[2], thr, T->W, T->frac + (size_t)temp * 768)) continue;
        } else if (!(dE <= 0 || (dE < T->W && r[2] < thr[dE]))) {
            continue;
        }
        const int32_t t = cols[u];
        cols[u] = cols[v];
        cols[v] = t;
        for (int s = 0; s < m; ++s) bad[s] += dbad[s];
        T->E[c] += dE;
        if (T->umbrella) T->removed[c] += dd;
        T->accepted[c] += 1;
        if (T->E[c] < T->bestE[c]) {
            T->bestE[c] = T->E[c];
            memcpy(T->best_cols + (size_t)c * T->stride, cols, sizeof(int32_t) * (size_t)m);
        }
    }
}

static void n3o_temper_exchange(n3o_temper_ctx* T, int lad) {
    const int L = T->L;
    int32_t* at = T->chain_at + (size_t)lad * L;
    int32_t* tof = T->temp_of + (size_t)lad * L;
    const int32_t* e = T->E + (size_t)lad * L;
    const uint32_t round = T->ladder_round[lad];
    for (int t = (int)(round & 1u); t < L - 1; t += 2) {
        const int a = at[t], b = at[t + 1];
        const int D = e[a] - e[b];
        int swap = D >= 0;
        if (!swap) {
            uint32_t r[4] = {round, (uint32_t)t, (uint32_t)lad, 0xE0000000u};
            n3o_philox(r, (uint32_t)T->seed, (uint32_t)(T->seed >> 32));
            swap = -D < T->XW && r[0] < T->exch[(size_t)t * T->XW + (-D)];
        }
        if (swap) {
            at[t] = b;
            at[t + 1] = a;
            tof[a] = t + 1;
            tof[b] = t;
            T->ladder_exch[lad] += 1;
        }
    }
    T->ladder_round[lad] = round + 1;
}

/* Replays `rounds` rounds of the device tempering kernel on the CPU.  Arrays
 * follow the n3_chains layout (columns widened to int32, row stride `stride`).
 * bad_bias, reference/removed/umbrella/frac: see n3o_temper_chain_round
 * (umbrella NULL: no restraint). */
void n3o_temper_run(int C, int L, int stride, int32_t* cols, int32_t* bad, int32_t* E, int32_t* bestE,
                    int32_t* best_cols, int32_t* temp_of, int32_t* chain_at, uint64_t* counter, uint32_t* accepted,
                    const int32_t* ladder_n, uint32_t* ladder_round, uint32_t* ladder_exch, const uint32_t* acc,
                    int W, const uint32_t* exch, int XW, uint64_t seed, int rounds, int round_sweeps,
                    int round_proposals, int exchange, const int32_t* ladder_rounds, int threads, int bad_bias,
                    const int32_t* reference, int32_t* removed, const int64_t* umbrella, const uint32_t* frac) {
    n3o_temper_ctx T = {C, L, stride, cols, bad, E, bestE, best_cols, temp_of, chain_at, counter, accepted,
                        ladder_n, ladder_round, ladder_exch, acc, W, exch, XW, seed, rounds, round_sweeps,
                        round_proposals, exchange, ladder_rounds, 0, bad_bias, reference, removed, umbrella, frac};
    int max_rounds = rounds;
    if (ladder_rounds)
        for (int lad = 0; lad < C / L; ++lad)
            if (ladder_rounds[lad] > max_rounds) max_rounds = ladder_rounds[lad];
    for (int r = 0; r < max_rounds; ++r) {
        T.round = r;
        n3o_parallel_for(C, threads, n3o_temper_chain_round, &T);
        if (exchange)
            for (int lad = 0; lad < C / L; ++lad)
                if (!ladder_rounds || r < ladder_rounds[lad]) n3o_temper_exchange(&T, lad);
    }
}

/* ------------------------------------------------------------------------
 * Device beam search mutation (gpu_device_search.py:17-114, the CUDA kernel
 * `mutate_population`), one child at a time.  The RNG is xorshift64* (Vigna)
 * seeded per child and generation (gpu_device_search.py:18-25, 44-46): the
 * multiplier and the two seed-mixing constants are the kernel's.
 * ---------------------------------------------------------------------- */
static uint64_t n3o_xs64(uint64_t* s) {
  uint64_t x = *s;
  x ^= x >> 12;
  x ^= x << 25;
  x ^= x >> 27;
  *s = x;
  return x * 2685821657736338717ULL;
}

void n3o_beam_mutate(const int32_t* pp, const int32_t* pq, const int32_t* pbad, int elite_count, int quality_count,
                     int n, int population, int active_strength, int max_strength, int bad_bias, uint64_t seed,
                     int generation, int32_t* cp, int32_t* cq) {
  const int m = 2 * n;
  for (int child = 0; child < population; ++child) {
    uint64_t rng = seed ^ (0x9e3779b97f4a7c15ULL * (uint64_t)(child + 1)) ^
                   (0xbf58476d1ce4e5b9ULL * (uint64_t)(generation + 1));
    int parent = child;
    if (child >= elite_count) {
      const uint64_t pick = n3o_xs64(&rng);
      const int pool = (pick & 255ULL) < 160ULL ? quality_count : elite_count;
      parent = (int)(n3o_xs64(&rng) % (uint64_t)pool);
    }
    int32_t* P = cp + (size_t)child * n;
    int32_t* Q = cq + (size_t)child * n;
    for (int r = 0; r < n; ++r) {
      P[r] = pp[(size_t)parent * n + r];
      Q[r] = pq[(size_t)parent * n + r];
    }
    if (child < elite_count) continue;
    const int32_t* bad = pbad + (size_t)parent * m;
    int strength;
    if ((n3o_xs64(&rng) & 31ULL) == 0ULL)
      strength = 1 + (int)(n3o_xs64(&rng) % (uint64_t)max_strength);
    else
      strength = 1 + (int)(n3o_xs64(&rng) % (uint64_t)active_strength);
    for (int step = 0; step < strength; ++step) {
      for (int attempt = 0; attempt < 32; ++attempt) {
        int u;
        if ((int)(n3o_xs64(&rng) % 100ULL) < bad_bias) {
          int total = 0;
          for (int e = 0; e < m; ++e) total += bad[e];
          if (total) {
            int t = (int)(n3o_xs64(&rng) % (uint64_t)total);
            for (u = 0; u < m - 1; ++u) {
              t -= bad[u];
              if (t < 0) break;
            }
          } else {
            u = (int)(n3o_xs64(&rng) % (uint64_t)m);
          }
        } else {
          u = (int)(n3o_xs64(&rng) % (uint64_t)m);
        }
        const int v = (int)(n3o_xs64(&rng) % (uint64_t)m);
        const int ru = u >> 1, rv = v >> 1;
        if (ru == rv) continue;
        int32_t* su = (u & 1) ? &Q[ru] : &P[ru];
        int32_t* sv = (v & 1) ? &Q[rv] : &P[rv];
        const int cu = *su, cv = *sv;
        if (cu == cv) continue;
        const int ou = (u & 1) ? P[ru] : Q[ru];
        const int ov = (v & 1) ? P[rv] : Q[rv];
        if (cv == ou || cu == ov) continue;
        *su = cv;
        *sv = cu;
        break;
      }
    }
  }
}

/* ------------------------------------------------------------------------
 * Three-cycle scores (accelerated.py:196-276): for each candidate
 * (u, v, w, orientation) the triples through the three slots before the move
 * (badness sum minus pair lines plus the triple itself) and after it, counted
 * literally over all pairs as the reference does.
 * ---------------------------------------------------------------------- */
static int col3(const int32_t* rows, const int32_t* cols, int a, int b, int c) {
  return (rows[b] - rows[a]) * (cols[c] - cols[a]) == (cols[b] - cols[a]) * (rows[c] - rows[a]);
}

void n3o_three_cycles(const int32_t* p, const int32_t* q, int n, const int32_t* cand, int count, int64_t current,
                      const int64_t* badness, int64_t* out) {
  const int m = 2 * n;
  int32_t rows[150], cols[150], nc[150];
  for (int r = 0; r < n; ++r) {
    rows[2 * r] = rows[2 * r + 1] = r;
    cols[2 * r] = p[r];
    cols[2 * r + 1] = q[r];
  }
  for (int k = 0; k < count; ++k) {
    const int u = cand[4 * k], v = cand[4 * k + 1], w = cand[4 * k + 2], o = cand[4 * k + 3];
    int64_t juv = 0, juw = 0, jvw = 0;
    for (int x = 0; x < m; ++x) {
      if (x != u && x != v) juv += col3(rows, cols, u, v, x);
      if (x != u && x != w) juw += col3(rows, cols, u, w, x);
      if (x != v && x != w) jvw += col3(rows, cols, v, w, x);
    }
    const int64_t tri = col3(rows, cols, u, v, w);
    const int64_t old_affected = badness[u] + badness[v] + badness[w] - juv - juw - jvw + tri;
    for (int x = 0; x < m; ++x) nc[x] = cols[x];
    if (o == 0) {
      nc[u] = cols[v];
      nc[v] = cols[w];
      nc[w] = cols[u];
    } else {
      nc[u] = cols[w];
      nc[w] = cols[v];
      nc[v] = cols[u];
    }
    int64_t na = 0;
    const int moved[3] = {u, v, w};
    for (int t = 0; t < 3; ++t) {
      const int c = moved[t];
      for (int i = 0; i < m - 1; ++i) {
        int skip = 0;
        for (int s = 0; s <= t; ++s) skip |= i == moved[s];
        if (skip) continue;
        for (int j = i + 1; j < m; ++j) {
          int sk = 0;
          for (int s = 0; s <= t; ++s) sk |= j == moved[s];
          if (sk) continue;
          na += (rows[i] - rows[c]) * (nc[j] - nc[c]) == (nc[i] - nc[c]) * (rows[j] - rows[c]);
        }
      }
    }
    out[k] = current - old_affected + na;
  }
}
