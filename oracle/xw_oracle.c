/* xw_oracle.c -- CPU restatement of the weighing-matrix annealer.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the parity tests, smoke() and the
 * bench's cpu_baseline leg.  The product never links or calls this file.
 *
 * Reference files cited as path:line inside flinty-mathematics/xtax:
 *   anneal.hpp = src/xweigh_anneal.hpp, cu = src/xweigh_cuda.cu.
 *
 * Pinning: tests/golden/ holds fixtures produced by the reference's own code
 * built here (oracle/_ref/ref_harness and oracle/_ref/xweigh); the reference
 * mode below reproduces them bit for bit (random starts, proposals, deltas,
 * calibration, whole annealing walks, solved CLI runs).  The device mode
 * shares the move arithmetic with the reference mode and replaces cuRAND by
 * the Philox draw layout documented at dev_word().
 *
 * Must be built with -ffp-contract=off (see Makefile): xwo_exp() has to round
 * exactly like the device's explicit __fma_rn/__dmul_rn sequence.
 */
#include "xw_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXN XWO_MAX_N

/* ======================================================================= */
/* Philox4x32-10, from the published description: Salmon, Moraes, Dror and
 * Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11.  Round:
 * (hi0,lo0)=M0*c0, (hi1,lo1)=M1*c2, c'=(hi1^c1^k0, lo1, hi0^c3^k1, lo0);
 * the key is bumped by the Weyl constants between rounds. */
void xwo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int round = 0; round < 10; ++round) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        const uint32_t n1 = (uint32_t)p1;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        const uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* ======================================================================= */
/* mt19937 (Matsumoto and Nishimura 1998) and the two libstdc++ adaptors the
 * reference draws through: uniform_int_distribution (Lemire's nearly
 * divisionless reduction, libstdc++ >= 11) and generate_canonical<double,53>
 * (two 32-bit draws, low word first). */
typedef struct { uint32_t mt[624]; int idx; } mt_t;

static void mt_seed(mt_t* s, uint32_t seed) {
    s->mt[0] = seed;
    for (int i = 1; i < 624; ++i)
        s->mt[i] = 1812433253u * (s->mt[i - 1] ^ (s->mt[i - 1] >> 30)) + (uint32_t)i;
    s->idx = 624;
}

static uint32_t mt_next(mt_t* s) {
    if (s->idx >= 624) {
        for (int i = 0; i < 624; ++i) {
            const uint32_t y = (s->mt[i] & 0x80000000u) | (s->mt[(i + 1) % 624] & 0x7fffffffu);
            uint32_t v = s->mt[(i + 397) % 624] ^ (y >> 1);
            if (y & 1u) v ^= 0x9908b0dfu;
            s->mt[i] = v;
        }
        s->idx = 0;
    }
    uint32_t y = s->mt[s->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

/* uniform in [0, range), range >= 1 */
static uint32_t mt_uniform(mt_t* s, uint32_t range) {
    uint64_t product = (uint64_t)mt_next(s) * range;
    uint32_t low = (uint32_t)product;
    if (low < range) {
        const uint32_t threshold = (uint32_t)(0u - range) % range;
        while (low < threshold) {
            product = (uint64_t)mt_next(s) * range;
            low = (uint32_t)product;
        }
    }
    return (uint32_t)(product >> 32);
}

static double mt_canonical(mt_t* s) {
    double sum = 0.0, tmp = 1.0;
    for (int k = 0; k < 2; ++k) {
        sum += (double)mt_next(s) * tmp;
        tmp *= 4294967296.0;
    }
    double ret = sum / tmp;
    if (ret >= 1.0) ret = nextafter(1.0, 0.0);
    return ret;
}

void xwo_mt_stream(uint32_t seed, int count, uint32_t* out) {
    mt_t s; mt_seed(&s, seed);
    for (int i = 0; i < count; ++i) out[i] = mt_next(&s);
}

void xwo_mt_uniform_stream(uint32_t seed, uint32_t range, int count, uint32_t* out) {
    mt_t s; mt_seed(&s, seed);
    for (int i = 0; i < count; ++i) out[i] = mt_uniform(&s, range);
}

void xwo_mt_canonical_stream(uint32_t seed, int count, double* out) {
    mt_t s; mt_seed(&s, seed);
    for (int i = 0; i < count; ++i) out[i] = mt_canonical(&s);
}

/* ======================================================================= */
/* Acceptance exponential, exp(x) for x <= 0, computed by Cody-Waite range
 * reduction (x = k ln2 + r, |r| <= ln2/2, ln2 split into a 32-bit head and a
 * tail) and the degree-14 Taylor polynomial of exp(r) in Horner form with
 * fused multiply-adds; 2^k is applied exactly.  Every step is a correctly
 * rounded IEEE operation, so the device (which issues the same operations as
 * __dmul_rn/__fma_rn) gets the same bits.  Below x = -40 the value only has
 * to be positive and below 2^-32 for the acceptance test u*2^-32 < exp(x)
 * (u a 32-bit integer); it is 0 below -745, where double exp underflows. */
static const double XW_INV_LN2 = 0x1.71547652b82fep+0;
static const double XW_LN2_HI = 0x1.62e42fee00000p-1;
static const double XW_LN2_LO = 0x1.a39ef35793c76p-33;
static const double XW_EXP_C[15] = {
    0x1.0000000000000p+0, 0x1.0000000000000p+0, 0x1.0000000000000p-1,
    0x1.5555555555555p-3, 0x1.5555555555555p-5, 0x1.1111111111111p-7,
    0x1.6c16c16c16c17p-10, 0x1.a01a01a01a01ap-13, 0x1.a01a01a01a01ap-16,
    0x1.71de3a556c734p-19, 0x1.27e4fb7789f5cp-22, 0x1.ae64567f544e4p-26,
    0x1.1eed8eff8d898p-29, 0x1.6124613a86d09p-33, 0x1.93974a8c07c9dp-37,
};

double xwo_exp(double x) {
    if (x >= 0.0) return 1.0;
    if (!(x > -40.0)) return (x > -745.0) ? 0x1p-60 : 0.0;
    const double k = rint(x * XW_INV_LN2);
    double r = fma(-k, XW_LN2_HI, x);
    r = fma(-k, XW_LN2_LO, r);
    double p = XW_EXP_C[14];
    for (int j = 13; j >= 0; --j) p = fma(p, r, XW_EXP_C[j]);
    const uint64_t bits = (uint64_t)(1023 + (int)k) << 52;
    double scale;
    memcpy(&scale, &bits, sizeof scale);
    return p * scale;
}

/* ======================================================================= */
/* Reference state (anneal.hpp:103-667): column-major int8 W, Gram, int64 row
 * residuals and the per-row minority list (nonzero columns when w <= n-w,
 * zero columns otherwise), kept in the reference's order. */
typedef struct {
    int n, w, m, sparse;
    int8_t W[MAXN * MAXN];
    int32_t G[MAXN * MAXN];
    int64_t res[MAXN];
    uint16_t mino[MAXN * MAXN];
    int64_t score, conflicts;
} rstate;

#define AT(s, r, c) ((s)->W[(size_t)(c) * (s)->n + (r)])
#define GR(s, r, c) ((s)->G[(size_t)(r) * (s)->n + (c)])
#define MINO(s, r, p) ((s)->mino[(size_t)(r) * (s)->m + (p)])

static void rs_init(rstate* s, int n, int w) {
    memset(s, 0, sizeof *s);
    s->n = n; s->w = w;
    s->sparse = w <= n - w;
    s->m = w < n - w ? w : n - w;
}

/* anneal.hpp:314-329 */
static int rs_rebuild_minority(rstate* s) {
    if (s->m == 0) return 0;
    for (int r = 0; r < s->n; ++r) {
        int pos = 0;
        for (int c = 0; c < s->n; ++c) {
            const int nz = AT(s, r, c) != 0;
            if (nz == s->sparse) {
                if (pos >= s->m) return -1;
                MINO(s, r, pos++) = (uint16_t)c;
            }
        }
        if (pos != s->m) return -1;
    }
    return 0;
}

/* anneal.hpp:455-475 (the sparse and bitset Gram builds give the same G) */
static void rs_rebuild(rstate* s) {
    const int n = s->n;
    for (int a = 0; a < n; ++a) {
        GR(s, a, a) = s->w;
        for (int b = a + 1; b < n; ++b) {
            int dot = 0;
            for (int c = 0; c < n; ++c) dot += AT(s, a, c) * AT(s, b, c);
            GR(s, a, b) = dot;
            GR(s, b, a) = dot;
        }
    }
    s->score = 0; s->conflicts = 0;
    for (int r = 0; r < n; ++r) s->res[r] = 0;
    for (int a = 0; a < n; ++a)
        for (int b = a + 1; b < n; ++b) {
            const int v = GR(s, a, b);
            const int64_t av = v < 0 ? -v : v;
            s->score += av;
            s->res[a] += av;
            s->res[b] += av;
            if (v != 0) ++s->conflicts;
        }
}

/* anneal.hpp:331-369 */
static int rs_raw_support_switch(rstate* s, mt_t* rng) {
    if (s->m == 0 || s->n < 2) return 0;
    const int r1 = (int)mt_uniform(rng, (uint32_t)s->n);
    int r2 = (int)mt_uniform(rng, (uint32_t)(s->n - 1));
    if (r2 >= r1) ++r2;
    const int p1 = (int)mt_uniform(rng, (uint32_t)s->m);
    const int p2 = (int)mt_uniform(rng, (uint32_t)s->m);
    int c1, c2;
    if (s->sparse) { c1 = MINO(s, r1, p1); c2 = MINO(s, r2, p2); }
    else { c2 = MINO(s, r1, p1); c1 = MINO(s, r2, p2); }
    if (c1 == c2 || AT(s, r1, c2) != 0 || AT(s, r2, c1) != 0) return 0;
    const int8_t v1 = AT(s, r1, c1), v2 = AT(s, r2, c2);
    if (v1 == 0 || v2 == 0) return 0;
    AT(s, r1, c1) = 0; AT(s, r2, c2) = 0;
    AT(s, r1, c2) = v1; AT(s, r2, c1) = v2;
    if (s->sparse) { MINO(s, r1, p1) = (uint16_t)c2; MINO(s, r2, p2) = (uint16_t)c1; }
    else { MINO(s, r1, p1) = (uint16_t)c1; MINO(s, r2, p2) = (uint16_t)c2; }
    return 1;
}

/* anneal.hpp:117-131, 371-381 */
static void rs_random_start(rstate* s, int n, int w, uint32_t seed) {
    rs_init(s, n, w);
    mt_t rng; mt_seed(&rng, seed);
    for (int r = 0; r < n; ++r)
        for (int k = 0; k < w; ++k)
            AT(s, r, (r + k) % n) = (mt_next(&rng) & 1u) ? 1 : -1;
    rs_rebuild_minority(s);
    if (s->m != 0) {
        const int per_row = s->m < 64 ? s->m : 64;
        const uint64_t target = (uint64_t)4 * (uint64_t)n * (uint64_t)per_row;
        uint64_t accepted = 0, attempts = 0;
        while (accepted < target && attempts < target * 12) {
            ++attempts;
            if (rs_raw_support_switch(s, &rng)) ++accepted;
        }
    }
    rs_rebuild(s);
}

void xwo_random_start(int n, int w, uint32_t seed, int8_t* W) {
    rstate* s = (rstate*)malloc(sizeof *s);
    rs_random_start(s, n, w, seed);
    memcpy(W, s->W, (size_t)n * n);
    free(s);
}

/* anneal.hpp:133-149 */
void xwo_sylvester(int n, int w, int8_t* W) {
    memset(W, 0, (size_t)n * n);
    for (int b = 0; b < n / w; ++b)
        for (int r = 0; r < w; ++r)
            for (int c = 0; c < w; ++c)
                W[(size_t)(b * w + c) * n + (b * w + r)] =
                    (__builtin_popcount((unsigned)(r & c)) & 1) ? -1 : 1;
}

void xwo_rescore(int n, int w, const int8_t* W, int64_t stats[4], int64_t* G, int64_t* residual) {
    (void)w;
    int64_t score = 0, conf = 0, sq = 0, par = 0;
    if (residual) for (int r = 0; r < n; ++r) residual[r] = 0;
    for (int a = 0; a < n; ++a) {
        if (G) {
            int64_t d = 0;
            for (int c = 0; c < n; ++c) d += (int64_t)W[(size_t)c * n + a] * W[(size_t)c * n + a];
            G[(size_t)a * n + a] = d;
        }
        for (int b = a + 1; b < n; ++b) {
            int64_t d = 0;
            for (int c = 0; c < n; ++c) d += (int64_t)W[(size_t)c * n + a] * W[(size_t)c * n + b];
            if (G) { G[(size_t)a * n + b] = d; G[(size_t)b * n + a] = d; }
            const int64_t ad = d < 0 ? -d : d;
            score += ad;
            conf += d != 0;
            sq += d * d;
            par += ad & 1;
            if (residual) { residual[a] += ad; residual[b] += ad; }
        }
    }
    stats[0] = score; stats[1] = conf; stats[2] = sq; stats[3] = par;
}

/* anneal.hpp:221-264 */
int xwo_verify(int n, int w, const int8_t* W) {
    int flags = 1;
    for (int r = 0; r < n && flags; ++r) {
        int rw = 0;
        for (int c = 0; c < n; ++c) {
            const int v = W[(size_t)c * n + r];
            if (v < -1 || v > 1) { flags = 0; break; }
            rw += v != 0;
        }
        if (rw != w) flags = 0;
    }
    for (int c = 0; c < n && flags; ++c) {
        int cw = 0;
        for (int r = 0; r < n; ++r) cw += W[(size_t)c * n + r] != 0;
        if (cw != w) flags = 0;
    }
    if (!flags) return 0;
    for (int a = 0; a < n; ++a)
        for (int b = a + 1; b < n; ++b) {
            int64_t d = 0;
            for (int c = 0; c < n; ++c) d += (int64_t)W[(size_t)c * n + a] * W[(size_t)c * n + b];
            if (d != 0) return 1;
        }
    return 3;
}

/* ======================================================================= */
/* Reference mode: the CPU engine's moves (anneal.hpp:192-219, 477-666). */
typedef struct { int kind, r1, r2, c1, c2, p1, p2; } rmove;
typedef struct { int64_t ds, dc; } reval;

void xwo_ref_params_default(xwo_ref_params* p) {
    p->sign_fraction = 0.5; p->greedy_fraction = 0.5; p->target_fraction = 0.7;
    p->candidate_samples = 4; p->target_samples = 8;
    p->t_init = 0.0; p->t_min = 0.25; p->cooling = 0.999; p->reheat = 1.0;
    p->reseed_factor = 1.25; p->moves_per_cool = 500; p->stuck_threshold = 50000;
}

static int rs_hot_row(const rstate* s, mt_t* rng, int samples) {
    int best = (int)mt_uniform(rng, (uint32_t)s->n);
    for (int k = 1; k < samples; ++k) {
        const int cand = (int)mt_uniform(rng, (uint32_t)s->n);
        if (s->res[cand] > s->res[best]) best = cand;
    }
    return best;
}

static int rs_propose_flip(const rstate* s, mt_t* rng, int row, rmove* mv) {
    int col;
    if (s->sparse && s->m > 0) {
        col = MINO(s, row, (int)mt_uniform(rng, (uint32_t)s->m));
    } else {
        const int start = (int)mt_uniform(rng, (uint32_t)s->n);
        col = start;
        while (AT(s, row, col) == 0) {
            if (++col == s->n) col = 0;
            if (col == start) return 0;
        }
    }
    mv->kind = 0; mv->r1 = row; mv->c1 = col;
    return 1;
}

static int rs_propose_switch(const rstate* s, mt_t* rng, int r1, rmove* mv) {
    if (s->m == 0 || s->n < 2) return 0;
    for (int a = 0; a < 24; ++a) {
        int r2 = (int)mt_uniform(rng, (uint32_t)(s->n - 1));
        if (r2 >= r1) ++r2;
        const int p1 = (int)mt_uniform(rng, (uint32_t)s->m);
        const int p2 = (int)mt_uniform(rng, (uint32_t)s->m);
        int c1, c2;
        if (s->sparse) { c1 = MINO(s, r1, p1); c2 = MINO(s, r2, p2); }
        else { c2 = MINO(s, r1, p1); c1 = MINO(s, r2, p2); }
        if (c1 == c2 || AT(s, r1, c2) != 0 || AT(s, r2, c1) != 0) continue;
        if (AT(s, r1, c1) == 0 || AT(s, r2, c2) == 0) continue;
        mv->kind = 1; mv->r1 = r1; mv->r2 = r2; mv->c1 = c1; mv->c2 = c2;
        mv->p1 = p1; mv->p2 = p2;
        return 1;
    }
    return 0;
}

static int rs_propose(const rstate* s, mt_t* rng, const xwo_ref_params* p, int targeted, rmove* mv) {
    const int row = targeted ? rs_hot_row(s, rng, p->target_samples)
                             : (int)mt_uniform(rng, (uint32_t)s->n);
    if (s->w == s->n || mt_canonical(rng) < p->sign_fraction)
        return rs_propose_flip(s, rng, row, mv);
    if (rs_propose_switch(s, rng, row, mv)) return 1;
    return rs_propose_flip(s, rng, row, mv);
}

static inline int64_t iabs64(int64_t v) { return v < 0 ? -v : v; }
static inline int64_t cdelta(int o, int nw) { return (int64_t)(nw != 0) - (int64_t)(o != 0); }

static reval rs_evaluate(const rstate* s, const rmove* mv) {
    reval e = {0, 0};
    const int n = s->n;
    if (mv->kind == 0) {
        const int change = -2 * AT(s, mv->r1, mv->c1);
        for (int o = 0; o < n; ++o) {
            if (o == mv->r1) continue;
            const int old = GR(s, mv->r1, o);
            const int nw = old + change * AT(s, o, mv->c1);
            e.ds += iabs64(nw) - iabs64(old);
            e.dc += cdelta(old, nw);
        }
    } else {
        const int v1 = AT(s, mv->r1, mv->c1), v2 = AT(s, mv->r2, mv->c2);
        for (int o = 0; o < n; ++o) {
            if (o == mv->r1 || o == mv->r2) continue;
            const int o1 = GR(s, mv->r1, o), o2 = GR(s, mv->r2, o);
            const int n1 = o1 + v1 * (AT(s, o, mv->c2) - AT(s, o, mv->c1));
            const int n2 = o2 + v2 * (AT(s, o, mv->c1) - AT(s, o, mv->c2));
            e.ds += iabs64(n1) - iabs64(o1) + iabs64(n2) - iabs64(o2);
            e.dc += cdelta(o1, n1) + cdelta(o2, n2);
        }
    }
    return e;
}

static void rs_commit(rstate* s, const rmove* mv, reval e) {
    const int n = s->n;
    if (mv->kind == 0) {
        const int r = mv->r1, c = mv->c1;
        const int change = -2 * AT(s, r, c);
        for (int o = 0; o < n; ++o) {
            if (o == r) continue;
            const int old = GR(s, r, o);
            const int nw = old + change * AT(s, o, c);
            const int64_t d = iabs64(nw) - iabs64(old);
            GR(s, r, o) = nw; GR(s, o, r) = nw;
            s->res[r] += d; s->res[o] += d;
        }
        AT(s, r, c) = (int8_t)-AT(s, r, c);
    } else {
        const int r1 = mv->r1, r2 = mv->r2, c1 = mv->c1, c2 = mv->c2;
        const int8_t v1 = AT(s, r1, c1), v2 = AT(s, r2, c2);
        for (int o = 0; o < n; ++o) {
            if (o == r1 || o == r2) continue;
            const int o1 = GR(s, r1, o), o2 = GR(s, r2, o);
            const int n1 = o1 + v1 * (AT(s, o, c2) - AT(s, o, c1));
            const int n2 = o2 + v2 * (AT(s, o, c1) - AT(s, o, c2));
            const int64_t d1 = iabs64(n1) - iabs64(o1), d2 = iabs64(n2) - iabs64(o2);
            GR(s, r1, o) = n1; GR(s, o, r1) = n1;
            GR(s, r2, o) = n2; GR(s, o, r2) = n2;
            s->res[r1] += d1; s->res[r2] += d2; s->res[o] += d1 + d2;
        }
        AT(s, r1, c1) = 0; AT(s, r2, c2) = 0;
        AT(s, r1, c2) = v1; AT(s, r2, c1) = v2;
        if (s->sparse) { MINO(s, r1, mv->p1) = (uint16_t)c2; MINO(s, r2, mv->p2) = (uint16_t)c1; }
        else { MINO(s, r1, mv->p1) = (uint16_t)c1; MINO(s, r2, mv->p2) = (uint16_t)c2; }
    }
    s->score += e.ds;
    s->conflicts += e.dc;
}

static int better_pair(int64_t sa, int64_t ca, int64_t sb, int64_t cb) {
    return sa < sb || (sa == sb && ca < cb);
}

/* anneal.hpp:881-899 */
static double rs_calibrate(const rstate* s, const xwo_ref_params* p, uint32_t seed) {
    if (p->t_init > 0.0) return p->t_init;
    mt_t rng; mt_seed(&rng, seed ^ 0xa511e9b3u);
    long double sum = 0.0L;
    int count = 0;
    for (int k = 0; k < 256; ++k) {
        rmove mv;
        if (!rs_propose(s, &rng, p, 0, &mv)) continue;
        const reval e = rs_evaluate(s, &mv);
        if (e.ds > 0) { sum += (long double)e.ds; ++count; }
    }
    if (count == 0) return 1.0;
    const double mean = (double)(sum / count);
    const double t = mean / log(2.0);
    return t > 1.0 ? t : 1.0;
}

double xwo_calibrate(int n, int w, uint32_t seed, const xwo_ref_params* p) {
    rstate* s = (rstate*)malloc(sizeof *s);
    rs_random_start(s, n, w, seed);
    const double t = rs_calibrate(s, p, seed);
    free(s);
    return t;
}

static uint64_t fnv1a(uint64_t h, uint64_t v) {
    for (int i = 0; i < 8; ++i) {
        h ^= (v >> (8 * i)) & 0xffu;
        h *= 1099511628211ull;
    }
    return h;
}

static void rs_apply_entries(int8_t* E, int n, const rmove* mv) {
    if (mv->kind == 0) {
        E[(size_t)mv->c1 * n + mv->r1] = (int8_t)-E[(size_t)mv->c1 * n + mv->r1];
        return;
    }
    const int8_t v1 = E[(size_t)mv->c1 * n + mv->r1], v2 = E[(size_t)mv->c2 * n + mv->r2];
    E[(size_t)mv->c1 * n + mv->r1] = 0;
    E[(size_t)mv->c2 * n + mv->r2] = 0;
    E[(size_t)mv->c2 * n + mv->r1] = v1;
    E[(size_t)mv->c1 * n + mv->r2] = v2;
}

static void rs_from_entries(rstate* s, int n, int w, const int8_t* E) {
    rs_init(s, n, w);
    memcpy(s->W, E, (size_t)n * n);
    rs_rebuild_minority(s);
    rs_rebuild(s);
}

/* run_annealer (anneal.hpp:1106-1170) with one worker, i.e. anneal_worker
 * (anneal.hpp:909-1104) with tempering off; bounded by max_moves. */
void xwo_ref_walk(int n, int w, uint32_t seed, int64_t max_moves, const xwo_ref_params* p,
                  xwo_walk_result* r, int8_t* start_out, int8_t* final_out, int8_t* best_out) {
    rstate* start = (rstate*)malloc(sizeof *start);
    rstate* cur = (rstate*)malloc(sizeof *cur);
    rs_random_start(start, n, w, seed);
    const double t0 = rs_calibrate(start, p, seed);
    mt_t seed_rng; mt_seed(&seed_rng, seed);
    const uint32_t worker_seed = mt_next(&seed_rng);
    memcpy(cur, start, sizeof *cur);
    mt_t rng; mt_seed(&rng, worker_seed);

    int8_t* best = (int8_t*)malloc((size_t)n * n);
    memcpy(best, start->W, (size_t)n * n);
    const size_t path_cap = 250000;
    rmove* path = (rmove*)malloc(sizeof(rmove) * path_cap);
    size_t path_len = 0;
    int64_t best_score = cur->score, best_conf = cur->conflicts;
    int msi = 0, cool = 0;
    int64_t moves = 0, accepted = 0;
    double T = t0;
    uint64_t h = 1469598103934665603ull;

    while (moves < max_moves && cur->score != 0) {
        rmove sel = {0}; reval se = {0, 0};
        int have = 0;
        const int greedy = mt_canonical(&rng) < p->greedy_fraction;
        const int samples = greedy ? p->candidate_samples : 1;
        for (int k = 0; k < samples; ++k) {
            rmove cand;
            const int targeted = mt_canonical(&rng) < p->target_fraction;
            if (!rs_propose(cur, &rng, p, targeted, &cand)) continue;
            const reval e = rs_evaluate(cur, &cand);
            if (!have || better_pair(e.ds, e.dc, se.ds, se.dc)) { sel = cand; se = e; have = 1; }
        }
        if (!have) continue;
        ++moves;
        const int accept = se.ds <= 0 ||
            mt_canonical(&rng) < exp(-(double)se.ds / (T > 1e-12 ? T : 1e-12));
        if (accept) {
            rs_commit(cur, &sel, se);
            path[path_len++] = sel;
            ++accepted;
        }
        if (better_pair(cur->score, cur->conflicts, best_score, best_conf)) {
            best_score = cur->score; best_conf = cur->conflicts; msi = 0;
            for (size_t i = 0; i < path_len; ++i) rs_apply_entries(best, n, &path[i]);
            path_len = 0;
        } else {
            ++msi;
        }
        if (++cool >= p->moves_per_cool) {
            cool = 0;
            const double t = T * p->cooling;
            T = p->t_min > t ? p->t_min : t;
        }
        if (msi >= p->stuck_threshold) {
            msi = 0;
            const double t = t0 * p->reheat;
            T = p->t_min > t ? p->t_min : t;
            const int64_t gb = best_score > 1 ? best_score : 1;
            if ((double)cur->score > p->reseed_factor * (double)gb) {
                rs_from_entries(cur, n, w, best);
                path_len = 0;
            }
        }
        if (path_len >= path_cap) {
            rs_from_entries(cur, n, w, best);
            path_len = 0;
            msi = 0;
        }
        h = fnv1a(h, (uint64_t)cur->score);
        h = fnv1a(h, (uint64_t)cur->conflicts);
        h = fnv1a(h, accept ? 1u : 0u);
    }
    r->moves = moves; r->accepted = accepted;
    r->score = cur->score; r->conflicts = cur->conflicts;
    r->best_score = best_score; r->best_conflicts = best_conf;
    r->initial_temperature = t0; r->temperature = T;
    r->worker_seed = worker_seed; r->hash = h;
    if (start_out) memcpy(start_out, start->W, (size_t)n * n);
    if (final_out) memcpy(final_out, cur->W, (size_t)n * n);
    if (best_out) memcpy(best_out, best, (size_t)n * n);
    free(path); free(best); free(cur); free(start);
}

/* ======================================================================= */
/* Device mode.
 *
 * Draw layout (shared with the CUDA kernel).  Every 32-bit draw of replica
 * `stream` of a job with key (key0,key1) is word j of
 *     Philox4x32-10(ctr = {slot, it_lo, it_hi, stream}, key)
 * where `it` is the replica's iteration number and `slot` names the use:
 *   slot 0                      move-level: word 0 greedy coin, word 1 accept
 *   slot 1 + 128*c + b          candidate c (0..31), block b:
 *     b=0   targeted coin, random row, double-flip coin, sign-flip coin
 *     b=1   flip index | switch attempt 0: row2, pos1, pos2
 *           (within-row swap: flip index, nonzero pick, zero pick, sign)
 *     b=2   switch attempt 0: sign1, sign2; fallback flip index; first flip
 *           index of a double flip
 *     b=3   double-flip attempt 0: same-row coin, row, flip index
 *     b=4+k/4, word k%4    hot-row tournament sample k (k < 64)
 *     b=20+(a-1)           double-flip attempt a (1..15): coin, row, index
 *     b=36+2(a-1), +1      switch attempt a (1..23): row2, pos1, pos2, sign1 | sign2
 * An index in [0,count) is Lemire's multiply-shift of the word; the rare
 * rejected word is replaced by word j of the same counter with slot
 * |= r<<24 for the r-th retry.  A coin "u < p" compares u with ceil(p*2^32).
 * Exchange draws use ctr = {pair/4, round_lo, round_hi, 0x80000000} (word
 * pair%4); the row-only start uses ctr = {b, row, 0, 0x40000000|stream}.
 */
struct xwo_replica {
    xwo_job job;
    uint32_t index;
    int n, w, m, sparse;
    uint64_t thr_greedy, thr_target, thr_double, thr_sign, thr_swsign;
    int8_t W[MAXN * MAXN];
    int8_t bestW[MAXN * MAXN];
    int32_t G[MAXN * MAXN];
    int64_t res[MAXN];
    uint16_t mino[MAXN * MAXN];
    xwo_replica_scalars s;
};

static uint64_t coin_threshold(double p) {
    if (!(p > 0.0)) return 0;
    if (p >= 1.0) return 4294967296ull;
    return (uint64_t)ceil(p * 4294967296.0);
}

static uint32_t dev_word(const xwo_replica* r, uint64_t it, uint32_t slot, int j) {
    const uint32_t ctr[4] = {slot, (uint32_t)it, (uint32_t)(it >> 32), r->index};
    const uint32_t key[2] = {r->job.key0, r->job.key1};
    uint32_t out[4];
    xwo_philox4x32_10(ctr, key, out);
    return out[j];
}

static uint32_t lemire_index(uint32_t key0, uint32_t key1, const uint32_t ctr_in[4], int j, uint32_t count) {
    uint32_t ctr[4] = {ctr_in[0], ctr_in[1], ctr_in[2], ctr_in[3]};
    const uint32_t key[2] = {key0, key1};
    uint32_t out[4];
    xwo_philox4x32_10(ctr, key, out);
    uint32_t v = out[j];
    for (uint32_t retry = 1;; ++retry) {
        const uint64_t prod = (uint64_t)v * count;
        const uint32_t low = (uint32_t)prod;
        if (low >= count || low >= (0u - count) % count || retry > 255)
            return (uint32_t)(prod >> 32);
        ctr[0] = (ctr_in[0] & 0x00ffffffu) | (retry << 24);
        xwo_philox4x32_10(ctr, key, out);
        v = out[j];
    }
}

static uint32_t dev_index(const xwo_replica* r, uint64_t it, uint32_t slot, int j, uint32_t count) {
    const uint32_t ctr[4] = {slot, (uint32_t)it, (uint32_t)(it >> 32), r->index};
    return lemire_index(r->job.key0, r->job.key1, ctr, j, count);
}

#define CSLOT(c, b) (1u + 128u * (uint32_t)(c) + (uint32_t)(b))
#define DW(r, W_) ((r)->W)
#define DAT(r, row, col) ((r)->W[(size_t)(col) * (r)->n + (row)])
#define DG(r, a, b) ((r)->G[(size_t)(a) * (r)->n + (b)])
#define DMINO(r, row, p) ((r)->mino[(size_t)(row) * (r)->m + (p)])

/* kinds: 0 sign flip, 1 support switch (new values v1,v2), 2 double flip,
 * 3 within-row swap (nonzero at c1 moves to the zero at c2 with value v1) */
typedef struct { int kind, r1, r2, c1, c2, p1, p2, v1, v2; } dmove;
typedef struct { int64_t ds, dc, dsq, dpar; } deval;

static int d_flip(const xwo_replica* r, uint64_t it, int c, int b, int j, int row, dmove* mv) {
    int col;
    if (r->sparse && r->m > 0) {
        col = DMINO(r, row, (int)dev_index(r, it, CSLOT(c, b), j, (uint32_t)r->m));
    } else {
        const int start = (int)dev_index(r, it, CSLOT(c, b), j, (uint32_t)r->n);
        col = start;
        while (DAT(r, row, col) == 0) {
            if (++col == r->n) col = 0;
            if (col == start) return 0;
        }
    }
    memset(mv, 0, sizeof *mv);
    mv->kind = 0; mv->r1 = row; mv->c1 = col;
    return 1;
}

static int d_hot_row(const xwo_replica* r, uint64_t it, int c) {
    int best = (int)dev_index(r, it, CSLOT(c, 4), 0, (uint32_t)r->n);
    for (int k = 1; k < r->job.target_samples; ++k) {
        const int cand = (int)dev_index(r, it, CSLOT(c, 4 + k / 4), k % 4, (uint32_t)r->n);
        if (r->res[cand] > r->res[best]) best = cand;
    }
    return best;
}

/* cu:389-421 */
static int d_double(const xwo_replica* r, uint64_t it, int c, int row1, dmove* mv) {
    dmove first;
    if (!d_flip(r, it, c, 2, 3, row1, &first)) return 0;
    for (int a = 0; a < 16; ++a) {
        const int b = a == 0 ? 3 : 20 + (a - 1);
        const int row2 = dev_word(r, it, CSLOT(c, b), 0) < 0x80000000u
                             ? row1 : (int)dev_index(r, it, CSLOT(c, b), 1, (uint32_t)r->n);
        dmove second;
        if (!d_flip(r, it, c, b, 2, row2, &second)) continue;
        if (first.r1 == second.r1 && first.c1 == second.c1) continue;
        memset(mv, 0, sizeof *mv);
        mv->kind = 2; mv->r1 = first.r1; mv->c1 = first.c1;
        mv->r2 = second.r1; mv->c2 = second.c1;
        return 1;
    }
    return 0;
}

/* cu:327-387 */
static int d_switch(const xwo_replica* r, uint64_t it, int c, int row1, dmove* mv) {
    if (r->m == 0 || r->n < 2) return 0;
    for (int a = 0; a < 24; ++a) {
        uint32_t sr, sp1, sp2, ss1, ss2;
        int jr, jp1, jp2, js1, js2;
        if (a == 0) {
            sr = sp1 = sp2 = CSLOT(c, 1); jr = 1; jp1 = 2; jp2 = 3;
            ss1 = ss2 = CSLOT(c, 2); js1 = 0; js2 = 1;
        } else {
            const int B = 36 + 2 * (a - 1);
            sr = sp1 = sp2 = ss1 = CSLOT(c, B); jr = 0; jp1 = 1; jp2 = 2; js1 = 3;
            ss2 = CSLOT(c, B + 1); js2 = 0;
        }
        int row2 = (int)dev_index(r, it, sr, jr, (uint32_t)(r->n - 1));
        if (row2 >= row1) ++row2;
        const int p1 = (int)dev_index(r, it, sp1, jp1, (uint32_t)r->m);
        const int p2 = (int)dev_index(r, it, sp2, jp2, (uint32_t)r->m);
        int c1, c2;
        if (r->sparse) { c1 = DMINO(r, row1, p1); c2 = DMINO(r, row2, p2); }
        else { c2 = DMINO(r, row1, p1); c1 = DMINO(r, row2, p2); }
        if (c1 == c2 || DAT(r, row1, c2) != 0 || DAT(r, row2, c1) != 0) continue;
        if (DAT(r, row1, c1) == 0 || DAT(r, row2, c2) == 0) continue;
        const int v1 = DAT(r, row1, c1), v2 = DAT(r, row2, c2);
        mv->kind = 1; mv->r1 = row1; mv->r2 = row2; mv->c1 = c1; mv->c2 = c2;
        mv->p1 = p1; mv->p2 = p2;
        mv->v1 = dev_word(r, it, ss1, js1) < r->thr_swsign ? -v1 : v1;
        mv->v2 = dev_word(r, it, ss2, js2) < r->thr_swsign ? -v2 : v2;
        return 1;
    }
    return 0;
}

/* within-row swap: a nonzero of the row moves to one of the row's zeros */
static int d_row_swap(const xwo_replica* r, uint64_t it, int c, int row, dmove* mv) {
    const int n = r->n;
    if (r->m == 0) return 0;
    int c1, c2, pos;
    if (r->sparse) {
        pos = (int)dev_index(r, it, CSLOT(c, 1), 1, (uint32_t)r->m);
        c1 = DMINO(r, row, pos);
        const int start = (int)dev_index(r, it, CSLOT(c, 1), 2, (uint32_t)n);
        c2 = start;
        while (DAT(r, row, c2) != 0) { if (++c2 == n) c2 = 0; if (c2 == start) return 0; }
    } else {
        pos = (int)dev_index(r, it, CSLOT(c, 1), 2, (uint32_t)r->m);
        c2 = DMINO(r, row, pos);
        const int start = (int)dev_index(r, it, CSLOT(c, 1), 1, (uint32_t)n);
        c1 = start;
        while (DAT(r, row, c1) == 0) { if (++c1 == n) c1 = 0; if (c1 == start) return 0; }
    }
    memset(mv, 0, sizeof *mv);
    mv->kind = 3; mv->r1 = row; mv->c1 = c1; mv->c2 = c2; mv->p1 = pos;
    mv->v1 = dev_word(r, it, CSLOT(c, 1), 3) < 0x80000000u ? 1 : -1;
    return 1;
}

/* cu:423-447 (move set 0); move set 1 replaces the switch by the
 * within-row swap and has no double flips */
static int d_propose(const xwo_replica* r, uint64_t it, int c, dmove* mv) {
    const int targeted = dev_word(r, it, CSLOT(c, 0), 0) < r->thr_target;
    const int row = targeted ? d_hot_row(r, it, c)
                             : (int)dev_index(r, it, CSLOT(c, 0), 1, (uint32_t)r->n);
    if (r->job.move_set == 1) {
        if (r->w == r->n || dev_word(r, it, CSLOT(c, 0), 3) < r->thr_sign)
            return d_flip(r, it, c, 1, 0, row, mv);
        if (d_row_swap(r, it, c, row, mv)) return 1;
        return d_flip(r, it, c, 2, 2, row, mv);
    }
    if (dev_word(r, it, CSLOT(c, 0), 2) < r->thr_double && d_double(r, it, c, row, mv)) return 1;
    if (r->w == r->n || dev_word(r, it, CSLOT(c, 0), 3) < r->thr_sign)
        return d_flip(r, it, c, 1, 0, row, mv);
    if (d_switch(r, it, c, row, mv)) return 1;
    return d_flip(r, it, c, 2, 2, row, mv);
}

static inline void acc(deval* e, int o, int nw) {
    const int64_t ao = o < 0 ? -o : o, an = nw < 0 ? -nw : nw;
    e->ds += an - ao;
    e->dc += (int64_t)(nw != 0) - (int64_t)(o != 0);
    e->dsq += (int64_t)nw * nw - (int64_t)o * o;
    e->dpar += (an & 1) - (ao & 1);
}

/* cu:449-599, plus the within-row swap */
static deval d_evaluate(const xwo_replica* r, const dmove* mv) {
    deval e = {0, 0, 0, 0};
    const int n = r->n;
    if (mv->kind == 0) {
        const int ch = -2 * DAT(r, mv->r1, mv->c1);
        for (int o = 0; o < n; ++o) {
            if (o == mv->r1) continue;
            const int old = DG(r, mv->r1, o);
            acc(&e, old, old + ch * DAT(r, o, mv->c1));
        }
    } else if (mv->kind == 1) {
        const int v1 = DAT(r, mv->r1, mv->c1), v2 = DAT(r, mv->r2, mv->c2);
        for (int o = 0; o < n; ++o) {
            if (o == mv->r1 || o == mv->r2) continue;
            const int o1 = DG(r, mv->r1, o), o2 = DG(r, mv->r2, o);
            acc(&e, o1, o1 + mv->v1 * DAT(r, o, mv->c2) - v1 * DAT(r, o, mv->c1));
            acc(&e, o2, o2 + mv->v2 * DAT(r, o, mv->c1) - v2 * DAT(r, o, mv->c2));
        }
    } else if (mv->kind == 2) {
        const int ch1 = -2 * DAT(r, mv->r1, mv->c1), ch2 = -2 * DAT(r, mv->r2, mv->c2);
        if (mv->r1 == mv->r2) {
            for (int o = 0; o < n; ++o) {
                if (o == mv->r1) continue;
                const int old = DG(r, mv->r1, o);
                acc(&e, old, old + ch1 * DAT(r, o, mv->c1) + ch2 * DAT(r, o, mv->c2));
            }
        } else {
            for (int o = 0; o < n; ++o) {
                if (o == mv->r1 || o == mv->r2) continue;
                const int o1 = DG(r, mv->r1, o), o2 = DG(r, mv->r2, o);
                acc(&e, o1, o1 + ch1 * DAT(r, o, mv->c1));
                acc(&e, o2, o2 + ch2 * DAT(r, o, mv->c2));
            }
            const int op = DG(r, mv->r1, mv->r2);
            acc(&e, op, op + ch1 * DAT(r, mv->r2, mv->c1) + ch2 * DAT(r, mv->r1, mv->c2) +
                            (mv->c1 == mv->c2 ? ch1 * ch2 : 0));
        }
    } else {
        const int v = DAT(r, mv->r1, mv->c1);
        for (int o = 0; o < n; ++o) {
            if (o == mv->r1) continue;
            const int old = DG(r, mv->r1, o);
            acc(&e, old, old + mv->v1 * DAT(r, o, mv->c2) - v * DAT(r, o, mv->c1));
        }
    }
    return e;
}

static int64_t primary(const deval* e, int kind) {
    return kind == 1 ? e->dsq : kind == 2 ? e->dpar : e->ds;
}

/* cu:227-244 */
static int d_better(const deval* a, const deval* b, int kind) {
    const int64_t pa = primary(a, kind), pb = primary(b, kind);
    if (pa != pb) return pa < pb;
    if (a->ds != b->ds) return a->ds < b->ds;
    return a->dc < b->dc;
}

static void set_pair(xwo_replica* r, int a, int b, int nw) {
    const int old = DG(r, a, b);
    const int64_t d = (int64_t)(nw < 0 ? -nw : nw) - (old < 0 ? -old : old);
    DG(r, a, b) = nw; DG(r, b, a) = nw;
    r->res[a] += d; r->res[b] += d;
}

/* cu:607-877, plus the within-row swap */
static void d_commit(xwo_replica* r, const dmove* mv, const deval* e) {
    const int n = r->n;
    if (mv->kind == 0) {
        const int ch = -2 * DAT(r, mv->r1, mv->c1);
        for (int o = 0; o < n; ++o)
            if (o != mv->r1) set_pair(r, mv->r1, o, DG(r, mv->r1, o) + ch * DAT(r, o, mv->c1));
        DAT(r, mv->r1, mv->c1) = (int8_t)-DAT(r, mv->r1, mv->c1);
    } else if (mv->kind == 1) {
        const int v1 = DAT(r, mv->r1, mv->c1), v2 = DAT(r, mv->r2, mv->c2);
        for (int o = 0; o < n; ++o) {
            if (o == mv->r1 || o == mv->r2) continue;
            const int n1 = DG(r, mv->r1, o) + mv->v1 * DAT(r, o, mv->c2) - v1 * DAT(r, o, mv->c1);
            const int n2 = DG(r, mv->r2, o) + mv->v2 * DAT(r, o, mv->c1) - v2 * DAT(r, o, mv->c2);
            set_pair(r, mv->r1, o, n1);
            set_pair(r, mv->r2, o, n2);
        }
        DAT(r, mv->r1, mv->c1) = 0; DAT(r, mv->r2, mv->c2) = 0;
        DAT(r, mv->r1, mv->c2) = (int8_t)mv->v1; DAT(r, mv->r2, mv->c1) = (int8_t)mv->v2;
        if (r->sparse) { DMINO(r, mv->r1, mv->p1) = (uint16_t)mv->c2; DMINO(r, mv->r2, mv->p2) = (uint16_t)mv->c1; }
        else { DMINO(r, mv->r1, mv->p1) = (uint16_t)mv->c1; DMINO(r, mv->r2, mv->p2) = (uint16_t)mv->c2; }
    } else if (mv->kind == 2) {
        const int ch1 = -2 * DAT(r, mv->r1, mv->c1), ch2 = -2 * DAT(r, mv->r2, mv->c2);
        if (mv->r1 == mv->r2) {
            for (int o = 0; o < n; ++o)
                if (o != mv->r1)
                    set_pair(r, mv->r1, o, DG(r, mv->r1, o) + ch1 * DAT(r, o, mv->c1) + ch2 * DAT(r, o, mv->c2));
        } else {
            const int np = DG(r, mv->r1, mv->r2) + ch1 * DAT(r, mv->r2, mv->c1) +
                           ch2 * DAT(r, mv->r1, mv->c2) + (mv->c1 == mv->c2 ? ch1 * ch2 : 0);
            for (int o = 0; o < n; ++o) {
                if (o == mv->r1 || o == mv->r2) continue;
                set_pair(r, mv->r1, o, DG(r, mv->r1, o) + ch1 * DAT(r, o, mv->c1));
                set_pair(r, mv->r2, o, DG(r, mv->r2, o) + ch2 * DAT(r, o, mv->c2));
            }
            set_pair(r, mv->r1, mv->r2, np);
        }
        DAT(r, mv->r1, mv->c1) = (int8_t)-DAT(r, mv->r1, mv->c1);
        DAT(r, mv->r2, mv->c2) = (int8_t)-DAT(r, mv->r2, mv->c2);
    } else {
        const int v = DAT(r, mv->r1, mv->c1);
        for (int o = 0; o < n; ++o)
            if (o != mv->r1)
                set_pair(r, mv->r1, o, DG(r, mv->r1, o) + mv->v1 * DAT(r, o, mv->c2) - v * DAT(r, o, mv->c1));
        DAT(r, mv->r1, mv->c1) = 0;
        DAT(r, mv->r1, mv->c2) = (int8_t)mv->v1;
        DMINO(r, mv->r1, mv->p1) = (uint16_t)(r->sparse ? mv->c2 : mv->c1);
    }
    r->s.score += e->ds;
    r->s.conflicts += e->dc;
    r->s.obj_total += primary(e, r->s.obj_kind);
}

static int rep_rebuild(xwo_replica* r) {
    const int n = r->n;
    if (r->m != 0) {
        for (int row = 0; row < n; ++row) {
            int pos = 0;
            for (int c = 0; c < n; ++c) {
                const int nz = DAT(r, row, c) != 0;
                if (nz == r->sparse) {
                    if (pos >= r->m) return -1;
                    DMINO(r, row, pos++) = (uint16_t)c;
                }
            }
            if (pos != r->m) return -1;
        }
    }
    int64_t st[4];
    int64_t* G64 = (int64_t*)malloc(sizeof(int64_t) * n * n);
    xwo_rescore(n, r->w, r->W, st, G64, r->res);
    for (int i = 0; i < n * n; ++i) r->G[i] = (int32_t)G64[i];
    free(G64);
    r->s.score = st[0]; r->s.conflicts = st[1];
    r->s.obj_total = r->s.obj_kind == 1 ? st[2] : r->s.obj_kind == 2 ? st[3] : st[0];
    return 0;
}

xwo_replica* xwo_rep_create(const xwo_job* job, uint32_t index, const int8_t* W0, double t0, int32_t rung) {
    if (job->n < 1 || job->n > MAXN || job->w < 1 || job->w > job->n) return NULL;
    xwo_replica* r = (xwo_replica*)calloc(1, sizeof *r);
    r->job = *job;
    r->index = index;
    r->n = job->n; r->w = job->w;
    r->sparse = job->w <= job->n - job->w;
    r->m = job->w < job->n - job->w ? job->w : job->n - job->w;
    r->thr_greedy = coin_threshold(job->greedy_fraction);
    r->thr_target = coin_threshold(job->target_fraction);
    r->thr_double = job->move_set == 0 ? coin_threshold(job->double_sign_fraction) : 0;
    r->thr_sign = coin_threshold(job->sign_fraction);
    r->thr_swsign = coin_threshold(job->switch_sign_fraction);
    memcpy(r->W, W0, (size_t)r->n * r->n);
    if (job->objective >= 0) {
        r->s.obj_kind = job->objective;
    } else {
        /* cu:969-981 */
        const uint32_t h = index * 0x9e3779b9u + 0x85ebca6bu;
        const double choice = (double)h * (1.0 / 4294967296.0);
        r->s.obj_kind = choice < job->squared_objective_fraction ? 1
            : choice < job->squared_objective_fraction + job->parity_objective_fraction ? 2 : 0;
    }
    if (rep_rebuild(r) != 0) { free(r); return NULL; }
    memcpy(r->bestW, r->W, (size_t)r->n * r->n);
    r->s.best_score = r->s.score;
    r->s.best_conflicts = r->s.conflicts;
    r->s.temperature = t0;
    r->s.reheat_temperature = t0;
    r->s.rung = rung;
    return r;
}

void xwo_rep_destroy(xwo_replica* r) { free(r); }

void xwo_rep_set_temperature(xwo_replica* r, double t, int32_t rung) {
    r->s.temperature = t;
    r->s.rung = rung;
}

/* the iteration loop of cu:988-1130 */
int64_t xwo_rep_run(xwo_replica* r, int64_t iters, int stop_on_solve) {
    const xwo_job* job = &r->job;
    int64_t done = 0;
    for (; done < iters; ++done) {
        if (stop_on_solve && r->s.best_score == 0) break;
        const uint64_t it = r->s.it;
        const int count = dev_word(r, it, 0, 0) < r->thr_greedy ? job->candidate_samples : 1;
        int have = 0;
        dmove sel; deval se;
        memset(&sel, 0, sizeof sel); memset(&se, 0, sizeof se);
        for (int c = 0; c < count; ++c) {
            dmove mv;
            if (!d_propose(r, it, c, &mv)) continue;
            const deval e = d_evaluate(r, &mv);
            ++r->s.cand_evals;
            if (!have || d_better(&e, &se, r->s.obj_kind)) { sel = mv; se = e; have = 1; }
        }
        r->s.it = it + 1;
        if (!have) continue;
        ++r->s.moves;
        const int64_t delta = primary(&se, r->s.obj_kind);
        int accept = delta <= 0;
        if (!accept) {
            const double t = r->s.temperature > 1.0e-12 ? r->s.temperature : 1.0e-12;
            const double x = -(double)delta / t;
            accept = (double)dev_word(r, it, 0, 1) * 0x1p-32 < xwo_exp(x);
        }
        if (accept) d_commit(r, &sel, &se);
        if (better_pair(r->s.score, r->s.conflicts, r->s.best_score, r->s.best_conflicts)) {
            r->s.best_score = r->s.score;
            r->s.best_conflicts = r->s.conflicts;
            r->s.msi = 0;
            memcpy(r->bestW, r->W, (size_t)r->n * r->n);
        } else {
            ++r->s.msi;
        }
        if (!job->tempering) {
            if (++r->s.cool_ctr >= job->moves_per_cool) {
                r->s.cool_ctr = 0;
                r->s.temperature *= job->cooling;
                if (r->s.temperature < job->t_min) r->s.temperature = job->t_min;
            }
            if (r->s.msi >= job->stuck_threshold) {
                r->s.msi = 0;
                r->s.temperature = r->s.reheat_temperature * job->reheat;
                if (r->s.temperature < job->t_min) r->s.temperature = job->t_min;
            }
        }
    }
    return done;
}

void xwo_rep_get(const xwo_replica* r, xwo_replica_scalars* s, int8_t* W, int8_t* best_W,
                 uint16_t* minority, int32_t* G, int32_t* residual) {
    const int n = r->n;
    if (s) *s = r->s;
    if (W) memcpy(W, r->W, (size_t)n * n);
    if (best_W) memcpy(best_W, r->bestW, (size_t)n * n);
    if (minority) memcpy(minority, r->mino, sizeof(uint16_t) * n * r->m);
    if (G) memcpy(G, r->G, sizeof(int32_t) * n * n);
    if (residual) for (int i = 0; i < n; ++i) residual[i] = (int32_t)r->res[i];
}

int xwo_rep_check(const xwo_replica* r) {
    const int n = r->n;
    int64_t st[4];
    int64_t* G64 = (int64_t*)malloc(sizeof(int64_t) * n * n);
    int64_t res[MAXN];
    xwo_rescore(n, r->w, r->W, st, G64, res);
    int bad = 0;
    for (int a = 0; a < n; ++a) {
        for (int b = 0; b < n; ++b)
            if (a != b && G64[a * n + b] != r->G[a * n + b]) bad |= 1;
        if (res[a] != r->res[a]) bad |= 2;
    }
    free(G64);
    if (st[0] != r->s.score || st[1] != r->s.conflicts) bad |= 4;
    const int64_t obj = r->s.obj_kind == 1 ? st[2] : r->s.obj_kind == 2 ? st[3] : st[0];
    if (obj != r->s.obj_total) bad |= 8;
    for (int row = 0; row < n && r->m; ++row)
        for (int p = 0; p < r->m; ++p) {
            const int col = r->mino[row * r->m + p];
            if ((DAT(r, row, col) != 0) != r->sparse) bad |= 16;
        }
    return bad;
}

/* adjacent-rung sweep of anneal.hpp:1187-1221 on the device draw stream */
int xwo_exchange(const xwo_job* job, xwo_replica** reps, int R, const double* ladder, uint64_t round) {
    int owner[1024];
    if (R > 1024) return -1;
    for (int k = 0; k < R; ++k) owner[reps[k]->s.rung] = k;
    int swaps = 0;
    const uint32_t key[2] = {job->key0, job->key1};
    for (int rung = 0; rung + 1 < R; ++rung) {
        const int a = owner[rung], b = owner[rung + 1];
        const double x = (1.0 / ladder[rung] - 1.0 / ladder[rung + 1]) *
                         (double)(reps[a]->s.obj_total - reps[b]->s.obj_total);
        int accept = x >= 0.0;
        if (!accept) {
            const uint32_t ctr[4] = {(uint32_t)rung / 4u, (uint32_t)round, (uint32_t)(round >> 32), 0x80000000u};
            uint32_t out[4];
            xwo_philox4x32_10(ctr, key, out);
            accept = (double)out[rung % 4] * 0x1p-32 < xwo_exp(x);
        }
        if (accept) {
            reps[a]->s.rung = rung + 1;
            reps[b]->s.rung = rung;
            reps[a]->s.temperature = ladder[rung + 1];
            reps[b]->s.temperature = ladder[rung];
            owner[rung] = b;
            owner[rung + 1] = a;
            ++swaps;
        }
    }
    return swaps;
}

/* row-only start from the init stream */
void xwo_row_start(int n, int w, uint32_t key0, uint32_t key1, uint32_t stream, int8_t* W) {
    memset(W, 0, (size_t)n * n);
    int perm[MAXN];
    for (int row = 0; row < n; ++row) {
        for (int c = 0; c < n; ++c) perm[c] = c;
        for (int i = 0; i < w; ++i) {
            const uint32_t ctr[4] = {(uint32_t)(i >> 2), (uint32_t)row, 0u, 0x40000000u | stream};
            const int j = i + (int)lemire_index(key0, key1, ctr, i & 3, (uint32_t)(n - i));
            const int t = perm[i]; perm[i] = perm[j]; perm[j] = t;
            const uint32_t sctr[4] = {32u + (uint32_t)(i >> 2), (uint32_t)row, 0u, 0x40000000u | stream};
            uint32_t out[4];
            const uint32_t key[2] = {key0, key1};
            xwo_philox4x32_10(sctr, key, out);
            W[(size_t)perm[i] * n + row] = out[i & 3] < 0x80000000u ? 1 : -1;
        }
    }
}

/* Evaluate (and optionally commit) one device-set move on W with the device
 * arithmetic; out = {score, conflicts, squared, parity} deltas.  For tests
 * that compare single moves with the reference's own evaluations. */
int xwo_move_eval(int n, int w, int8_t* W, int kind, int r1, int r2, int c1, int c2,
                  int v1, int v2, int commit, int64_t out[4]) {
    xwo_job job;
    memset(&job, 0, sizeof job);
    job.n = n; job.w = w; job.objective = 0;
    job.candidate_samples = 1; job.target_samples = 1;
    job.moves_per_cool = 1; job.stuck_threshold = 1; job.cooling = 0.5; job.t_min = 1.0;
    xwo_replica* r = xwo_rep_create(&job, 0, W, 1.0, 0);
    if (!r) return -1;
    dmove mv;
    memset(&mv, 0, sizeof mv);
    mv.kind = kind; mv.r1 = r1; mv.r2 = r2; mv.c1 = c1; mv.c2 = c2; mv.v1 = v1; mv.v2 = v2;
    if (kind == 1 || kind == 3) {
        /* minority positions of the moved entries */
        for (int p = 0; p < r->m; ++p) {
            if (kind == 1) {
                if (DMINO(r, r1, p) == (r->sparse ? c1 : c2)) mv.p1 = p;
                if (DMINO(r, r2, p) == (r->sparse ? c2 : c1)) mv.p2 = p;
            } else if (DMINO(r, r1, p) == (r->sparse ? c1 : c2)) {
                mv.p1 = p;
            }
        }
    }
    const deval e = d_evaluate(r, &mv);
    out[0] = e.ds; out[1] = e.dc; out[2] = e.dsq; out[3] = e.dpar;
    if (commit) {
        d_commit(r, &mv, &e);
        memcpy(W, r->W, (size_t)n * n);
    }
    const int bad = commit ? xwo_rep_check(r) : 0;
    free(r);
    return bad;
}

/* ======================================================================= */
/* Device elite-restart kicks (the batch engine's restart mode 1, which
 * replaces the reference's host kicks, cu:2089-2193, by a kernel with its
 * own Philox stream).  Draw k of the kick of replica `replica` in restart
 * round `round`: word k%4 of Philox({k/4, round_lo, round_hi,
 * 0x20000000 | replica}, key).  Indices in [0,count) by Lemire's
 * multiply-shift, a word in the rejection zone replaced by the next word
 * (at most 64 tries). */
typedef struct {
    uint32_t key[2], ctr[4];
    uint32_t k;
} kick_rng;

static uint32_t kick_word(kick_rng* g) {
    uint32_t ctr[4] = {g->k >> 2, g->ctr[1], g->ctr[2], g->ctr[3]}, out[4];
    xwo_philox4x32_10(ctr, g->key, out);
    return out[(g->k++) & 3];
}

static uint32_t kick_index(kick_rng* g, uint32_t count) {
    uint64_t prod = 0;
    for (int t = 0; t < 64; ++t) {
        prod = (uint64_t)kick_word(g) * count;
        const uint32_t low = (uint32_t)prod;
        if (low >= count || low >= (0u - count) % count) break;
    }
    return (uint32_t)(prod >> 32);
}

/* the k-th nonzero column of `row`, in column order */
static int kick_nonzero(const int8_t* K, int n, int row, int k) {
    for (int c = 0; c < n; ++c)
        if (K[(size_t)c * n + row] != 0 && k-- == 0) return c;
    return -1;
}

void xwo_kick(int n, int w, const int8_t* E, const int32_t* esc, uint32_t key0, uint32_t key1, uint64_t round,
              uint32_t replica, uint32_t index, int kick, uint64_t thr_sign, int8_t* K) {
    memcpy(K, E, (size_t)n * n);
#define KAT(r, c) K[(size_t)(c) * n + (r)]
    if (esc) {
        /* the escape switch: the nonzero at (r1,c1) moves to (r1,c2) with
         * sign new1, the one at (r2,c2) to (r2,c1) with sign new2 */
        KAT(esc[0], esc[2]) = 0;
        KAT(esc[1], esc[3]) = 0;
        KAT(esc[0], esc[3]) = (int8_t)esc[4];
        KAT(esc[1], esc[2]) = (int8_t)esc[5];
    }
    kick_rng g;
    g.key[0] = key0; g.key[1] = key1;
    g.ctr[0] = 0; g.ctr[1] = (uint32_t)round; g.ctr[2] = (uint32_t)(round >> 32); g.ctr[3] = 0x20000000u | replica;
    g.k = 0;
    const int mode = (int)((index + round) % 3);
    int steps = kick;
    uint64_t thr = thr_sign;
    if (mode == 0) {
        steps = 0;
    } else if (mode == 1 && kick > 0 && w >= 3) {
        /* row kicks: 2..max(2, w/2) distinct nonzeros of 1..4 random rows flip */
        int rows = 1 + kick / (w > 1 ? w : 1);
        if (rows > 4) rows = 4;
        const int maxf = w / 2 > 2 ? w / 2 : 2;
        int cols[MAXN];
        for (int rk = 0; rk < rows; ++rk) {
            const int row = (int)kick_index(&g, (uint32_t)n);
            int cnt = 0;
            for (int c = 0; c < n; ++c)
                if (KAT(row, c) != 0) cols[cnt++] = c;
            const int flips = 2 + (int)kick_index(&g, (uint32_t)(maxf - 1));
            for (int f = 0; f < flips && f < cnt; ++f) {
                const int j = f + (int)kick_index(&g, (uint32_t)(cnt - f));
                const int t = cols[f]; cols[f] = cols[j]; cols[j] = t;
                KAT(row, cols[f]) = (int8_t)-KAT(row, cols[f]);
            }
        }
        steps = kick / 4;
    } else if (mode == 2) {
        thr = 0;   /* support switches only */
    }
    /* random moves: a sign flip (u < thr, or no zeros at all) or a
     * value-preserving 2x2 support switch; `steps` moves within 8*steps
     * attempts */
    int applied = 0;
    for (int a = 0; a < 8 * steps && applied < steps; ++a) {
        const uint32_t u = kick_word(&g);
        if (w == n || (uint64_t)u < thr) {
            const int row = (int)kick_index(&g, (uint32_t)n);
            const int col = kick_nonzero(K, n, row, (int)kick_index(&g, (uint32_t)w));
            KAT(row, col) = (int8_t)-KAT(row, col);
            ++applied;
            continue;
        }
        if (n < 2) continue;
        const int r1 = (int)kick_index(&g, (uint32_t)n);
        int r2 = (int)kick_index(&g, (uint32_t)(n - 1));
        if (r2 >= r1) ++r2;
        const int c1 = kick_nonzero(K, n, r1, (int)kick_index(&g, (uint32_t)w));
        const int c2 = kick_nonzero(K, n, r2, (int)kick_index(&g, (uint32_t)w));
        if (c1 == c2 || KAT(r1, c2) != 0 || KAT(r2, c1) != 0) continue;
        const int8_t v1 = KAT(r1, c1), v2 = KAT(r2, c2);
        KAT(r1, c1) = 0;
        KAT(r2, c2) = 0;
        KAT(r1, c2) = v1;
        KAT(r2, c1) = v2;
        ++applied;
    }
#undef KAT
}
